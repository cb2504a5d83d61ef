// render_cuda_ftb.cpp -- drop-in implementation of the reference's forward GPU entry points
// (ftrace src/render_cuda.h:24-143) on top of the B200 C ABI (include/ftb200.h).
//
// Compile this file inside the reference tree (it includes the reference's scene.h,
// camera.h, render.h and render_cuda.h) and link libftb200.so; the reference's own
// definitions of the same functions in render_cuda.cu are then excluded (the build
// compiles this file in place of render_cuda.cu).  The signatures are the reference's; the behaviour differs only where
// the reference calls exit(): here a failed CUDA call prints the C ABI's error and returns
// an empty film, like the reference's "unsupported scene" path.
//
// Baking (the reference's buildUploadScene, render_cuda.cu:12692-13546, re-done for the
// C ABI):
//  - triangles, spheres and curve segments are copied verbatim (double precision);
//  - emitters pass their own EmissionSampler CDF and power, so wavelength sampling is
//    bit-identical to the CPU tracer;
//  - material / medium spectra arrive as std::function values.  A spectrum made by one of
//    the reference's closed-form builders -- cauchy, sellmeier, tabulatedSpectrum
//    (spectrum.h:128-175) -- is baked as that form with the builder's own parameters
//    (FTB_SPEC_CAUCHY / SELLMEIER / TABLE), so the device evaluates it with the same
//    arithmetic at every wavelength; a spectrum constant over [360, 830] nm becomes
//    FTB_SPEC_CONST.  Every such bake is checked against the original, bit for bit, at
//    ~3000 wavelengths before it is used.  Any other spectrum (or one whose check fails)
//    is tabulated at kTableStep nm and interpolated linearly, which is exact only for
//    piecewise-linear spectra with breakpoints on that grid.
//  - maxBounce: the reference's GPU path ignores -max-bounce and uses 32
//    (render_cuda.cu:13702); g_ftbMaxBounce keeps that default and can be set by the
//    caller to honour the CLI value like the CPU path does.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <typeinfo>
#include <utility>
#include <vector>

#include "render.h"
#include "render_cuda.h"

#include "ftb200.h"

int g_ftbMaxBounce = 32;

// Every renderForwardCuda call bakes its scene (the reference re-uploads per call too,
// render_cuda.cu:13712-13740).  The GPU-built tree bakes ~10x faster and renders a few
// percent slower, so it is used unless the photon budget dwarfs the scene: above
// g_ftbSahPhotonsPerPrim photons per primitive the host SAH tree pays for its bake.
long long g_ftbSahPhotonsPerPrim = 4096;

static int32_t pick_build(const ftb_scene_desc& d, long long n_photons) {
    const long long prims = d.n_tris + d.n_spheres + d.n_curves + d.n_instances;
    return n_photons > g_ftbSahPhotonsPerPrim * (prims > 0 ? prims : 1) ? FTB_BUILD_SAH : FTB_BUILD_DEVICE;
}

namespace {

constexpr double kTableStep = 0.5;   // nm

struct BakedBlas {
    std::vector<double> tri_v, tri_n;
    std::vector<int32_t> tri_mat;
};

struct Baked {
    std::vector<BakedBlas> blas;
    std::vector<ftb_blas_desc> blas_desc;
    std::vector<ftb_instance> instances;
    std::vector<double> tri_v, tri_n, sph, curve, table_w, table_v, cdf;
    std::vector<int32_t> tri_mat, sph_mat, curve_mat;
    std::vector<ftb_material> mats;
    std::vector<ftb_spectrum> spectra;
    std::vector<ftb_emitter> emitters;
    std::vector<ftb_medium> media;
    ftb_scene_desc desc{};
    bool supported = true;
    std::string why;
};

// ---- exact spectra -------------------------------------------------------------------
// The device's evaluation of each form (spec_eval in the kernels: the reference's own
// expressions, spectrum.h:128-175), restated here so a candidate can be checked on the host.
double eval_form(const ftb_spectrum& f, const std::vector<double>& tw, const std::vector<double>& tv, double w) {
    switch (f.kind) {
    case FTB_SPEC_CONST: return f.p[0];
    case FTB_SPEC_CAUCHY: { double um = w * 1e-3; return f.p[0] + f.p[1] / (um * um); }
    case FTB_SPEC_SELLMEIER: {
        double l2 = (w * 1e-3) * (w * 1e-3);
        double n2 = 1.0 + f.p[0] * l2 / (l2 - f.p[3]) + f.p[1] * l2 / (l2 - f.p[4]) + f.p[2] * l2 / (l2 - f.p[5]);
        return std::sqrt(n2 > 1.0 ? n2 : 1.0);
    }
    case FTB_SPEC_TABLE: {
        const double* x = tw.data() + f.offset;
        const double* y = tv.data() + f.offset;
        const int n = f.n;
        if (w <= x[0]) return y[0];
        if (w >= x[n - 1]) return y[n - 1];
        int lo = 0, hi = n - 1;
        while (lo + 1 < hi) { int mid = (lo + hi) / 2; if (x[mid] <= w) lo = mid; else hi = mid; }
        double w0 = x[lo], w1 = x[lo + 1], v0 = y[lo], v1 = y[lo + 1];
        double fr = (w1 > w0) ? (w - w0) / (w1 - w0) : 0.0;
        return v0 + (v1 - v0) * fr;
    }
    default: return 0.0;
    }
}

bool same_bits(double a, double b) {
    uint64_t x, y;
    std::memcpy(&x, &a, 8);
    std::memcpy(&y, &b, 8);
    return x == y || (a != a && b != b);
}

// Wavelengths a baked form is checked at: the 0.5 nm grid over [360, 830], 2048 seeded
// pseudo-random wavelengths in that band, and (tables) every breakpoint and its
// floating-point neighbours.
std::vector<double> check_wavelengths(const std::vector<double>& breaks) {
    std::vector<double> w;
    for (double x = LAMBDA_MIN; x <= LAMBDA_MAX + 1e-9; x += kTableStep) w.push_back(x);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < 2048; ++i) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        w.push_back(LAMBDA_MIN + (LAMBDA_MAX - LAMBDA_MIN) * ((double)(st >> 11) * 0x1.0p-53));
    }
    for (double x : breaks) {
        w.push_back(x);
        w.push_back(std::nextafter(x, -1e300));
        w.push_back(std::nextafter(x, 1e300));
    }
    return w;
}

bool form_matches(const Spectrum& s, const ftb_spectrum& f, const std::vector<double>& tw,
                  const std::vector<double>& tv, const std::vector<double>& ws) {
    for (double w : ws)
        if (!same_bits(eval_form(f, tw, tv, w), s(w))) return false;
    return true;
}

// The closure object inside a Spectrum made by a known builder (libstdc++ only): the
// target type identifies the builder -- every call of e.g. cauchy() yields the same closure
// type -- and libstdc++ keeps a closure of at most 16 trivially copyable bytes inside the
// function object itself, any other behind a pointer at its start.  Only closures whose
// type was matched are read, and only as the builder captured them: Cauchy 2 doubles
// (stored inside), Sellmeier 6 doubles and tabulatedSpectrum one vector of (w, v) pairs
// (both stored behind the pointer).  The order of the captured doubles is not fixed by
// the language, so every order is tried, and each candidate must pass form_matches.
#if defined(__GLIBCXX__)
static_assert(sizeof(Spectrum) == 32, "unexpected std::function layout");
const std::type_info& cauchy_type() { static const Spectrum p = cauchy(1.0, 1.0); return p.target_type(); }
const std::type_info& sellmeier_type() {
    static const Spectrum p = sellmeier(1.0, 1.0, 1.0, 1.0, 1.0, 1.0);
    return p.target_type();
}
const std::type_info& table_type() {
    static const Spectrum p = tabulatedSpectrum({{400.0, 0.0}, {500.0, 1.0}});
    return p.target_type();
}
const void* heap_closure(const Spectrum& s) {
    const void* p;
    std::memcpy(&p, &s, sizeof p);
    return p;
}
#endif

bool exact_form(Baked& b, const Spectrum& s, ftb_spectrum& out) {
#if defined(__GLIBCXX__)
    if (!s) return false;
    const std::type_info& t = s.target_type();
    if (t == cauchy_type()) {
        double c[2];
        std::memcpy(c, &s, sizeof c);
        static const std::vector<double> ws = check_wavelengths({});
        for (int order = 0; order < 2; ++order) {
            ftb_spectrum f{};
            f.kind = FTB_SPEC_CAUCHY;
            f.p[0] = c[order];
            f.p[1] = c[1 - order];
            if (form_matches(s, f, b.table_w, b.table_v, ws)) { out = f; return true; }
        }
        return false;
    }
    if (t == sellmeier_type()) {
        double c[6];
        std::memcpy(c, heap_closure(s), sizeof c);
        static const std::vector<double> ws = check_wavelengths({});
        int idx[6] = {0, 1, 2, 3, 4, 5};
        do {
            ftb_spectrum f{};
            f.kind = FTB_SPEC_SELLMEIER;
            for (int k = 0; k < 6; ++k) f.p[k] = c[idx[k]];
            if (form_matches(s, f, b.table_w, b.table_v, ws)) { out = f; return true; }
        } while (std::next_permutation(idx, idx + 6));
        return false;
    }
    if (t == table_type()) {
        const auto* pairs = static_cast<const std::vector<std::pair<double, double>>*>(heap_closure(s));
        if (pairs->empty()) return false;
        ftb_spectrum f{};
        f.kind = FTB_SPEC_TABLE;
        f.offset = (int64_t)b.table_w.size();
        f.n = (int32_t)pairs->size();
        std::vector<double> breaks;
        for (const auto& pr : *pairs) {
            b.table_w.push_back(pr.first);
            b.table_v.push_back(pr.second);
            breaks.push_back(pr.first);
        }
        bool distinct = true;
        for (size_t i = 1; i < breaks.size(); ++i) distinct = distinct && breaks[i] > breaks[i - 1];
        if (distinct && form_matches(s, f, b.table_w, b.table_v, check_wavelengths(breaks))) { out = f; return true; }
        b.table_w.resize((size_t)f.offset);   // not usable: drop the candidate's pairs
        b.table_v.resize((size_t)f.offset);
        return false;
    }
#else
    (void)b; (void)s; (void)out;
#endif
    return false;
}

int bake_spectrum(Baked& b, const Spectrum& s) {
    ftb_spectrum out{};
    double v0 = s(LAMBDA_MIN);
    bool constant = true;
    for (double w = LAMBDA_MIN; w <= LAMBDA_MAX; w += kTableStep)
        if (!same_bits(s(w), v0)) { constant = false; break; }
    if (constant) {
        out.kind = FTB_SPEC_CONST;
        out.p[0] = v0;
    } else if (!exact_form(b, s, out)) {
        out.kind = FTB_SPEC_TABLE;
        out.offset = (int64_t)b.table_w.size();
        int n = 0;
        for (double w = LAMBDA_MIN; w <= LAMBDA_MAX + 1e-9; w += kTableStep, ++n) {
            b.table_w.push_back(w);
            b.table_v.push_back(s(w));
        }
        out.n = n;
    }
    b.spectra.push_back(out);
    return (int)b.spectra.size() - 1;
}

void bake(const Scene& sc, Baked& b) {
    for (const Material& m : sc.mats) {
        ftb_material o{};
        o.type = (int32_t)m.type;
        o.priority = m.priority;
        o.roughness = m.roughness;
        o.reflect = bake_spectrum(b, m.reflect);
        o.ior = bake_spectrum(b, m.ior);
        o.absorb = bake_spectrum(b, m.absorb);
        o.transmit = bake_spectrum(b, m.transmit);
        if (m.reflectTex >= 0 || m.roughnessTex >= 0 || m.normalTex >= 0 || m.reflectPat >= 0 ||
            m.transmitPat >= 0 || m.roughnessPat >= 0) {
            b.supported = false;
            b.why = "textured / patterned materials are not on this path";
        }
        b.mats.push_back(o);
    }
    for (const Tri& t : sc.tris) {
        const Vec3 v[3] = {t.v0, t.v1, t.v2};
        const Vec3 n[3] = {t.n0, t.n1, t.n2};
        for (int k = 0; k < 3; ++k) {
            b.tri_v.insert(b.tri_v.end(), {v[k].x, v[k].y, v[k].z});
            b.tri_n.insert(b.tri_n.end(), {n[k].x, n[k].y, n[k].z});
        }
        b.tri_mat.push_back(t.matId);
    }
    for (const Sphere& s : sc.spheres) {
        b.sph.insert(b.sph.end(), {s.c.x, s.c.y, s.c.z, s.r});
        b.sph_mat.push_back(s.matId);
    }
    for (const CurveSeg& c : sc.curveSegs) {
        b.curve.insert(b.curve.end(), {c.p0.x, c.p0.y, c.p0.z, c.p1.x, c.p1.y, c.p1.z, c.r0, c.r1,
                                       (double)c.u0, (double)c.u1});
        b.curve_mat.push_back(c.matId);
    }
    // shared mesh assets and their placements (Scene::blasList / instances, scene.h:1089-1090)
    for (const Blas& bl : sc.blasList) {
        BakedBlas bb;
        for (const Tri& t : bl.tris) {
            const Vec3 v[3] = {t.v0, t.v1, t.v2};
            const Vec3 n[3] = {t.n0, t.n1, t.n2};
            for (int k = 0; k < 3; ++k) {
                bb.tri_v.insert(bb.tri_v.end(), {v[k].x, v[k].y, v[k].z});
                bb.tri_n.insert(bb.tri_n.end(), {n[k].x, n[k].y, n[k].z});
            }
            bb.tri_mat.push_back(t.matId);
        }
        b.blas.push_back(std::move(bb));
    }
    for (const MeshInstance& mi : sc.instances) {
        ftb_instance o{};
        o.blas = mi.blasId;
        o.mat_override = mi.matOverride;
        for (int k = 0; k < 9; ++k) o.to_world[k] = mi.toWorld.m[k];
        o.to_world[9] = mi.toWorld.t.x; o.to_world[10] = mi.toWorld.t.y; o.to_world[11] = mi.toWorld.t.z;
        b.instances.push_back(o);
    }
    // planar mirrors are on the path: the library groups the mirror triangles into planes
    // itself, as Scene::buildMirrorPlanes does (scene.h:1646-1720)
    if (!sc.implicits.empty() || !sc.emissiveVolumes.empty() || sc.envMap || !sc.dielSphereIdx.empty() ||
        !sc.mirrorSphereIdx.empty()) {
        b.supported = false;
        b.why = "implicits, emissive volumes, environment maps and the sphere connectors are not on this path";
    }
    for (const Emitter& e : sc.emitters) {
        ftb_emitter o{};
        if (e.shape == EmitterShape::Quad) o.shape = FTB_EMIT_QUAD;
        else if (e.shape == EmitterShape::Sphere) o.shape = FTB_EMIT_SPHERE;
        else { b.supported = false; b.why = "only quad and sphere emitters are on this path"; }
        if (e.emitPat >= 0) { b.supported = false; b.why = "emission patterns are not on this path"; }
        o.collimated = e.collimated ? 1 : 0;
        o.spd = -1;
        o.cdf_n = (int32_t)e.spd.cdf.size() - 1;
        o.cdf_offset = (int64_t)b.cdf.size();
        b.cdf.insert(b.cdf.end(), e.spd.cdf.begin(), e.spd.cdf.end());
        o.step = e.spd.step;
        o.power = e.power;
        const Vec3 src[5] = {e.origin, e.u, e.v, e.normal, e.beamDir};
        double* dst[5] = {o.origin, o.u, o.v, o.normal, o.beam};
        for (int k = 0; k < 5; ++k) { dst[k][0] = src[k].x; dst[k][1] = src[k].y; dst[k][2] = src[k].z; }
        o.area = e.area;
        o.radius = e.radius;
        b.emitters.push_back(o);
    }
    for (const Medium& m : sc.media) {
        if (m.heterogeneous() || m.rainbow() || m.emissive() || !m.ior.empty()) {
            b.supported = false;
            b.why = "only homogeneous Henyey-Greenstein media are on this path";
        }
        ftb_medium o{};
        o.sigma_a = bake_spectrum(b, m.sigma_a);
        o.sigma_s = bake_spectrum(b, m.sigma_s);
        o.g = m.g;
        o.bound = !m.bounded ? FTB_BOUND_NONE
                  : (m.boundShape == MediumBound::Sphere ? FTB_BOUND_SPHERE : FTB_BOUND_BOX);
        const Vec3 src[3] = {m.bmin, m.bmax, m.bcenter};
        double* dst[3] = {o.bmin, o.bmax, o.center};
        for (int k = 0; k < 3; ++k) { dst[k][0] = src[k].x; dst[k][1] = src[k].y; dst[k][2] = src[k].z; }
        o.radius = m.bradius;
        b.media.push_back(o);
    }
    ftb_scene_desc& d = b.desc;
    d.n_tris = (int64_t)sc.tris.size();
    d.tri_v = b.tri_v.data();
    d.tri_n = b.tri_n.data();
    d.tri_mat = b.tri_mat.data();
    d.n_spheres = (int64_t)sc.spheres.size();
    d.sph = b.sph.data();
    d.sph_mat = b.sph_mat.data();
    d.n_curves = (int64_t)sc.curveSegs.size();
    d.curve = b.curve.data();
    d.curve_mat = b.curve_mat.data();
    d.n_mats = (int32_t)b.mats.size();
    d.mats = b.mats.data();
    d.n_spectra = (int32_t)b.spectra.size();
    d.spectra = b.spectra.data();
    d.n_table = (int64_t)b.table_w.size();
    d.table_w = b.table_w.data();
    d.table_v = b.table_v.data();
    d.n_emitters = (int32_t)b.emitters.size();
    d.emitters = b.emitters.data();
    d.emitter_cdf = b.cdf.data();
    d.n_media = (int32_t)b.media.size();
    d.media = b.media.data();
    for (BakedBlas& bb : b.blas) {
        ftb_blas_desc o{};
        o.n_tris = (int64_t)bb.tri_mat.size();
        o.tri_v = bb.tri_v.data();
        o.tri_n = bb.tri_n.data();
        o.tri_mat = bb.tri_mat.data();
        b.blas_desc.push_back(o);
    }
    d.n_blas = (int32_t)b.blas_desc.size();
    d.blas = b.blas_desc.data();
    d.n_instances = (int64_t)b.instances.size();
    d.instances = b.instances.data();
}

ftb_camera bake_camera(const Camera& c, int resX, int resY) {
    ftb_camera o{};
    const Vec3 src[4] = {c.eye, c.u, c.v, c.w};
    double* dst[4] = {o.eye, o.u, o.v, o.w};
    for (int k = 0; k < 4; ++k) { dst[k][0] = src[k].x; dst[k][1] = src[k].y; dst[k][2] = src[k].z; }
    o.tan_half_x = c.tanHalfX;
    o.tan_half_y = c.tanHalfY;
    o.res_x = resX;
    o.res_y = resY;
    return o;
}

void to_film(const std::vector<int64_t>& fx, const ftb_film_info& info, Film& out) {
    const size_t npix = (size_t)out.resX * out.resY;
    for (size_t i = 0; i < npix; ++i) {
        out.xyz[i] = Vec3((double)fx[4 * i] * info.scale, (double)fx[4 * i + 1] * info.scale,
                          (double)fx[4 * i + 2] * info.scale);
        out.hits[i] = (double)fx[4 * i + 3];
    }
}

void add_energy(EnergyReport& e, const ftb_energy& en) {
    e.emitted += en.emitted; e.absorbed += en.absorbed; e.sensor += en.sensor;
    e.escaped += en.escaped; e.residual += en.residual;
}

bool report(ftb_status s, const char* what) {
    if (s == FTB_OK) return true;
    std::fprintf(stderr, "[ftb200] %s: %s\n", what, ftb_last_error());
    return false;
}

}  // namespace

// What the bake makes of a scene's material and medium spectra, in bake order (reflect,
// ior, absorb, transmit of each material, then sigma_a, sigma_s of each medium), with the
// table pairs the TABLE entries index: an integrator can check that the scene's spectra
// bake in closed form (CAUCHY, SELLMEIER, or TABLE with the authored breakpoints) and not
// as a 0.5 nm sampled table.  Not part of render_cuda.h.
int ftbShimBakedSpectra(const Scene& scene, std::vector<ftb_spectrum>& spectra, std::vector<double>& table_w,
                        std::vector<double>& table_v) {
    Baked b;
    bake(scene, b);
    spectra = b.spectra;
    table_w = b.table_w;
    table_v = b.table_v;
    return (int)spectra.size();
}

bool cudaAvailable() { return ftb_available() != 0; }

const char* cudaDeviceName() { return ftb_device_name(); }

bool cudaMemInfo(size_t* freeB, size_t* totalB) { return ftb_mem_info(freeB, totalB) == FTB_OK; }

bool cudaForwardSupported(const Scene& scene) {
    Baked b;
    bake(scene, b);
    return b.supported && ftb_forward_supported(&b.desc) == 1;
}

// camMode 'B' (pinhole), any heroC (bundles as tracePhotonHero), and the megakernel/wavefront
// choice folded into the one wavefront backend; other camera models are not on this path and
// return empty films.
Film renderForwardCuda(const Scene& scene, const Camera& cam, int resX, int resY, long long N,
                       EnergyReport& eOut, bool /*diffraction*/, char camMode,
                       unsigned long long seedBase, bool /*wavefront*/, int heroC) {
    Film out;
    out.resX = resX; out.resY = resY; out.alloc();
    if (camMode != 'B') return out;
    Baked b;
    bake(scene, b);
    if (!b.supported) return out;
    ftb_scene* s = nullptr;
    b.desc.build = pick_build(b.desc, N);
    if (!report(ftb_scene_create(&b.desc, 0, &s), "scene bake")) return out;
    ftb_camera c = bake_camera(cam, resX, resY);
    ftb_render_params p{N, seedBase, g_ftbMaxBounce, 0, heroC, 0};   // bundles when heroC > 1 (no media)
    std::vector<int64_t> fx((size_t)resX * resY * 4);
    ftb_film_info info{};
    ftb_energy en{};
    if (report(ftb_render_forward(s, &c, &p, fx.data(), &info, &en), "render")) {
        to_film(fx, info, out);
        add_energy(eOut, en);
    }
    ftb_scene_destroy(s);
    return out;
}

// ---- resident session (render_cuda.h:121-143) -------------------------------------------
struct SharedGpuSession {
    ftb_scene* scene = nullptr;
    ftb_session* session = nullptr;
    std::vector<int> resX, resY;
    std::vector<Film> seedFilms;
    EnergyReport seedEnergy;
};

SharedGpuSession* sharedForwardGpuBegin(const Scene& scene, const std::vector<Camera>& cams,
                                        const std::vector<int>& resX, const std::vector<int>& resY,
                                        char camMode, bool /*wavefront*/, int heroC, bool beamGather,
                                        const std::vector<Film>* seedFilms, const EnergyReport* seedEnergy) {
    if (camMode != 'B' || beamGather || cams.empty()) return nullptr;
    Baked b;
    bake(scene, b);
    if (!b.supported) return nullptr;
    auto* g = new SharedGpuSession();
    if (!report(ftb_scene_create(&b.desc, 0, &g->scene), "scene bake")) { delete g; return nullptr; }
    std::vector<ftb_camera> cs;
    for (size_t i = 0; i < cams.size(); ++i) cs.push_back(bake_camera(cams[i], resX[i], resY[i]));
    if (!report(ftb_session_begin(g->scene, cs.data(), (int32_t)cs.size(), g_ftbMaxBounce, 0, heroC,
                                  &g->session),
                "session")) {
        ftb_scene_destroy(g->scene);
        delete g;
        return nullptr;
    }
    g->resX = resX;
    g->resY = resY;
    // Resume: the device films start at zero and the seed is added on download, so that
    // download() keeps returning full running totals (render_cuda.cu:13801-13825).
    if (seedFilms) g->seedFilms = *seedFilms;
    if (seedEnergy) g->seedEnergy = *seedEnergy;
    return g;
}

void sharedForwardGpuBatch(SharedGpuSession* s, long long N, unsigned long long seedBase, bool) {
    if (s) report(ftb_session_batch(s->session, N, seedBase), "batch");
}

void sharedForwardGpuHits0(SharedGpuSession* s, std::vector<double>& hits) {
    if (!s) return;
    report(ftb_session_hits0(s->session, hits.data()), "hits");
    if (!s->seedFilms.empty())
        for (size_t i = 0; i < hits.size() && i < s->seedFilms[0].hits.size(); ++i) hits[i] += s->seedFilms[0].hits[i];
}

void sharedForwardGpuDownload(SharedGpuSession* s, std::vector<Film>& films, EnergyReport& e) {
    if (!s) return;
    ftb_energy en{};
    for (size_t c = 0; c < films.size() && c < s->resX.size(); ++c) {
        std::vector<int64_t> fx((size_t)s->resX[c] * s->resY[c] * 4);
        ftb_film_info info{};
        if (!report(ftb_session_download(s->session, (int32_t)c, fx.data(), &info, c == 0 ? &en : nullptr),
                    "download"))
            return;
        to_film(fx, info, films[c]);
        if (c < s->seedFilms.size()) films[c].merge(s->seedFilms[c]);
    }
    e = s->seedEnergy;
    add_energy(e, en);
}

void sharedForwardGpuEnd(SharedGpuSession* s) {
    if (!s) return;
    ftb_session_end(s->session);
    ftb_scene_destroy(s->scene);
    delete s;
}

std::vector<Film> renderForwardSharedCuda(const Scene& scene, const std::vector<Camera>& cams,
                                          const std::vector<int>& resX, const std::vector<int>& resY,
                                          long long N, EnergyReport& eOut, bool diffraction, char camMode,
                                          unsigned long long seedBase, bool wavefront, int heroC,
                                          bool beamGather) {
    std::vector<Film> out(cams.size());
    for (size_t c = 0; c < cams.size(); ++c) { out[c].resX = resX[c]; out[c].resY = resY[c]; out[c].alloc(); }
    SharedGpuSession* s = sharedForwardGpuBegin(scene, cams, resX, resY, camMode, wavefront, heroC,
                                                beamGather, nullptr, nullptr);
    if (!s) return out;
    sharedForwardGpuBatch(s, N, seedBase, diffraction);
    EnergyReport e;
    sharedForwardGpuDownload(s, out, e);
    eOut.emitted += e.emitted; eOut.absorbed += e.absorbed; eOut.sensor += e.sensor;
    eOut.escaped += e.escaped; eOut.residual += e.residual;
    sharedForwardGpuEnd(s);
    return out;
}
