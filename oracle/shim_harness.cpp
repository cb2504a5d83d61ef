// shim_harness.cpp -- TEST INFRASTRUCTURE ONLY.  Drives the drop-in shim
// (goodphotons_b200/shim/render_cuda_ftb.cpp) the way the reference's main.cpp does:
// a reference Scene and Camera in, renderForwardCuda(...) (render_cuda.h:79-82) called
// with the reference's own signature, a reference Film and EnergyReport out.  The Scene is
// built by ref_harness.cpp from the same POD description the tests use.
#include "render.h"
#include "render_cuda.h"

#include "../include/ftb200.h"

extern int g_ftbMaxBounce;
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
