// shim_harness.cpp -- TEST INFRASTRUCTURE ONLY.  Drives the drop-in shim
// (goodphotons_b200/shim/render_cuda_ftb.cpp) the way the reference's main.cpp does:
// a reference Scene and Camera in, renderForwardCuda(...) (render_cuda.h:79-82) called
// with the reference's own signature, a reference Film and EnergyReport out.  The Scene is
// built by ref_harness.cpp from the same POD description the tests use.
#include "render.h"
#include "render_cuda.h"

#include "../include/ftb200.h"

extern int g_ftbMaxBounce;
int ftbShimBakedSpectra(const Scene& scene, std::vector<ftb_spectrum>& spectra, std::vector<double>& table_w,
                        std::vector<double>& table_v);
extern "C" const void* ftr_scene(void* h);

extern "C" int ftshim_render(void* ref, const ftb_camera* cam, int64_t n, uint64_t seed_base, int max_bounce,
                             double* film_xyz, double* film_hits, double* energy) {
    const Scene& scene = *static_cast<const Scene*>(ftr_scene(ref));
    Camera c;
    c.eye = Vec3{cam->eye[0], cam->eye[1], cam->eye[2]};
    c.u = Vec3{cam->u[0], cam->u[1], cam->u[2]};
    c.v = Vec3{cam->v[0], cam->v[1], cam->v[2]};
    c.w = Vec3{cam->w[0], cam->w[1], cam->w[2]};
    c.tanHalfX = cam->tan_half_x; c.tanHalfY = cam->tan_half_y;
    c.film.resX = cam->res_x; c.film.resY = cam->res_y;
    if (!cudaAvailable() || !cudaForwardSupported(scene)) return -1;
    g_ftbMaxBounce = max_bounce;
    EnergyReport e;
    Film f = renderForwardCuda(scene, c, cam->res_x, cam->res_y, n, e, true, 'B', seed_base, false, 1);
    const size_t npix = (size_t)cam->res_x * cam->res_y;
    for (size_t i = 0; i < npix; ++i) {
        film_xyz[3 * i] = f.xyz[i].x; film_xyz[3 * i + 1] = f.xyz[i].y; film_xyz[3 * i + 2] = f.xyz[i].z;
        film_hits[i] = f.hits[i];
    }
    energy[0] = e.emitted; energy[1] = e.absorbed; energy[2] = e.sensor; energy[3] = e.escaped; energy[4] = e.residual;
    return 0;
}

// The shim's bake of the scene's spectra (no GPU needed): up to `cap` spectra and `tcap`
// table pairs; returns the number of spectra, or -1 if a buffer is too small.
extern "C" int ftshim_spectra(void* ref, ftb_spectrum* out, int cap, double* tw, double* tv, int tcap) {
    const Scene& scene = *static_cast<const Scene*>(ftr_scene(ref));
    std::vector<ftb_spectrum> sp;
    std::vector<double> w, v;
    ftbShimBakedSpectra(scene, sp, w, v);
    if ((int)sp.size() > cap || (int)w.size() > tcap) return -1;
    for (size_t i = 0; i < sp.size(); ++i) out[i] = sp[i];
    for (size_t i = 0; i < w.size(); ++i) { tw[i] = w[i]; tv[i] = v[i]; }
    return (int)sp.size();
}

// A resident session through the shim (sharedForwardGpuBegin/Batch/Download/End,
// render_cuda.h:121-143): n_cams cameras, two batches of n0 and n1 photons with the
// reference's cumulative seedBase convention, then the running totals of camera `which`.
extern "C" int ftshim_session(void* ref, const ftb_camera* cams, int n_cams, int64_t n0, int64_t n1, int max_bounce,
                              int hero_c, int which, double* film_xyz, double* film_hits, double* energy) {
    const Scene& scene = *static_cast<const Scene*>(ftr_scene(ref));
    std::vector<Camera> cs;
    std::vector<int> rx, ry;
    for (int i = 0; i < n_cams; ++i) {
        const ftb_camera* cam = cams + i;
        Camera c;
        c.eye = Vec3{cam->eye[0], cam->eye[1], cam->eye[2]};
        c.u = Vec3{cam->u[0], cam->u[1], cam->u[2]};
        c.v = Vec3{cam->v[0], cam->v[1], cam->v[2]};
        c.w = Vec3{cam->w[0], cam->w[1], cam->w[2]};
        c.tanHalfX = cam->tan_half_x; c.tanHalfY = cam->tan_half_y;
        c.film.resX = cam->res_x; c.film.resY = cam->res_y;
        cs.push_back(c);
        rx.push_back(cam->res_x);
        ry.push_back(cam->res_y);
    }
    g_ftbMaxBounce = max_bounce;
    SharedGpuSession* s = sharedForwardGpuBegin(scene, cs, rx, ry, 'B', false, hero_c, false, nullptr, nullptr);
    if (!s) return -1;
    sharedForwardGpuBatch(s, n0, 0, true);
    sharedForwardGpuBatch(s, n1, (unsigned long long)n0, true);
    std::vector<Film> films(cs.size());
    for (size_t i = 0; i < cs.size(); ++i) { films[i].resX = rx[i]; films[i].resY = ry[i]; films[i].alloc(); }
    EnergyReport e;
    sharedForwardGpuDownload(s, films, e);
    sharedForwardGpuEnd(s);
    const Film& f = films[which];
    const size_t npix = (size_t)f.resX * f.resY;
    for (size_t i = 0; i < npix; ++i) {
        film_xyz[3 * i] = f.xyz[i].x; film_xyz[3 * i + 1] = f.xyz[i].y; film_xyz[3 * i + 2] = f.xyz[i].z;
        film_hits[i] = f.hits[i];
    }
    energy[0] = e.emitted; energy[1] = e.absorbed; energy[2] = e.sensor; energy[3] = e.escaped; energy[4] = e.residual;
    return 0;
}
