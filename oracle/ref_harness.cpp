// ref_harness.cpp -- builds the REFERENCE's own CPU light tracer into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: tests/, the golden-vector script and bench.py's CPU
// baseline call it; the product never does.
//
// This file contains no reference code.  It is compiled against the reference's headers
// where they lie (oracle/Makefile passes -I <reference>/src) and drives the reference's
// public C++ API: it builds a `Scene` from the same POD description the C ABI takes
// (Tri / Sphere / CurveSeg / Blas / MeshInstance / Material / addAreaLight /
// addSphereLight / Medium, then Scene::build, scene.h:1907), bakes the `Camera` fields, and runs
// Renderer::tracePhoton (render.h:1811) photon by photon with the reference's per-photon
// seeding (seedUnit, main.cpp:11326) and std::thread banding (main.cpp:11305-11340).
#include "render.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "../include/ftb200.h"

namespace {

Spectrum make_spectrum(const ftb_scene_desc* d, int idx, double dflt) {
    if (idx < 0) return constantSpectrum(dflt);
    const ftb_spectrum& s = d->spectra[idx];
    switch (s.kind) {
    case FTB_SPEC_CONST: return constantSpectrum(s.p[0]);
    case FTB_SPEC_TABLE: {
        std::vector<std::pair<double, double>> pairs;
        for (int i = 0; i < s.n; ++i)
            pairs.push_back({d->table_w[s.offset + i], d->table_v[s.offset + i]});
        return tabulatedSpectrum(pairs);
    }
    case FTB_SPEC_CAUCHY: return cauchy(s.p[0], s.p[1]);
    case FTB_SPEC_SELLMEIER: return sellmeier(s.p[0], s.p[1], s.p[2], s.p[3], s.p[4], s.p[5]);
    case FTB_SPEC_BLACKBODY:
        if (s.p[1] == 1.0) return blackbody(s.p[0]);
        return scaledSpectrum(sharedSpectrum(blackbody(s.p[0])), s.p[1]);
    }
    return constantSpectrum(0.0);
}

Vec3 v3(const double* p) { return Vec3{p[0], p[1], p[2]}; }

struct Ref {
    Scene scene;
};

}  // namespace

extern "C" {

void* ftr_prepare(const ftb_scene_desc* d) {
    auto* r = new Ref();
    Scene& s = r->scene;
    for (int i = 0; i < d->n_mats; ++i) {
        const ftb_material& m = d->mats[i];
        Material mm;
        mm.type = (MatType)m.type;
        mm.reflect = make_spectrum(d, m.reflect, 0.5);
        mm.ior = m.ior >= 0 ? make_spectrum(d, m.ior, 1.5) : iorConstant(1.5);
        mm.absorb = make_spectrum(d, m.absorb, 0.0);
        mm.transmit = make_spectrum(d, m.transmit, 0.0);
        mm.roughness = m.roughness;
        mm.priority = m.priority;
        s.mats.push_back(mm);
    }
    for (int64_t i = 0; i < d->n_tris; ++i) {
        const double* v = d->tri_v + 9 * i;
        Tri t{v3(v), v3(v + 3), v3(v + 6), d->tri_mat[i], -1, {}};
        if (d->tri_n) {
            const double* n = d->tri_n + 9 * i;
            t.n0 = v3(n); t.n1 = v3(n + 3); t.n2 = v3(n + 6);
        }
        s.tris.push_back(t);
    }
    for (int64_t i = 0; i < d->n_spheres; ++i) {
        Sphere sp;
        sp.c = v3(d->sph + 4 * i); sp.r = d->sph[4 * i + 3]; sp.matId = d->sph_mat[i];
        s.spheres.push_back(sp);
    }
    for (int64_t i = 0; i < d->n_curves; ++i) {
        const double* c = d->curve + 10 * i;
        CurveSeg cs;
        cs.p0 = v3(c); cs.p1 = v3(c + 3); cs.r0 = c[6]; cs.r1 = c[7];
        cs.u0 = (float)c[8]; cs.u1 = (float)c[9]; cs.matId = d->curve_mat[i];
        s.curveSegs.push_back(cs);
    }
    // shared BLAS assets and their placements (scene.h:996-1063)
    for (int b = 0; b < d->n_blas; ++b) {
        const ftb_blas_desc& bd = d->blas[b];
        Blas bl;
        for (int64_t i = 0; i < bd.n_tris; ++i) {
            const double* v = bd.tri_v + 9 * i;
            Tri t{v3(v), v3(v + 3), v3(v + 6), bd.tri_mat[i], -1, {}};
            if (bd.tri_n) {
                const double* n = bd.tri_n + 9 * i;
                t.n0 = v3(n); t.n1 = v3(n + 3); t.n2 = v3(n + 6);
            }
            bl.tris.push_back(t);
        }
        s.blasList.push_back(std::move(bl));
    }
    for (int64_t k = 0; k < d->n_instances; ++k) {
        const ftb_instance& in = d->instances[k];
        MeshInstance mi;
        mi.blasId = in.blas;
        mi.matOverride = in.mat_override;
        Affine xf;
        for (int j = 0; j < 9; ++j) xf.m[j] = in.to_world[j];
        xf.t = Vec3{in.to_world[9], in.to_world[10], in.to_world[11]};
        mi.setToWorld(xf);
        s.instances.push_back(mi);
    }
    for (int i = 0; i < d->n_emitters; ++i) {
        const ftb_emitter& e = d->emitters[i];
        Spectrum spd = make_spectrum(d, e.spd, 0.0);
        if (e.shape == FTB_EMIT_SPHERE)
            s.addSphereLight(v3(e.origin), e.radius, spd, e.step);
        else
            s.addAreaLight(v3(e.origin), v3(e.u), v3(e.v), v3(e.normal), e.area, spd, e.step,
                           e.collimated != 0, v3(e.beam));
    }
    for (int i = 0; i < d->n_media; ++i) {
        const ftb_medium& m = d->media[i];
        Medium md;
        md.enabled = true;
        md.sigma_a = make_spectrum(d, m.sigma_a, 0.0);
        md.sigma_s = make_spectrum(d, m.sigma_s, 0.0);
        md.g = m.g;
        if (m.bound == FTB_BOUND_BOX) {
            md.bounded = true; md.boundShape = MediumBound::Box;
            md.bmin = v3(m.bmin); md.bmax = v3(m.bmax);
        } else if (m.bound == FTB_BOUND_SPHERE) {
            md.bounded = true; md.boundShape = MediumBound::Sphere;
            md.bcenter = v3(m.center); md.bradius = m.radius;
            md.bmin = v3(m.center) - Vec3{m.radius, m.radius, m.radius};
            md.bmax = v3(m.center) + Vec3{m.radius, m.radius, m.radius};
        }
        s.media.push_back(md);
    }
    s.build();
    return r;
}

void ftr_release(void* h) { delete static_cast<Ref*>(h); }

/* The first `count` uniforms of photon k's stream (seedUnit, rng.h:40; uniform, rng.h:22). */
void ftr_uniforms(uint64_t k, int count, double* out) {
    Pcg32 rng;
    seedUnit(rng, k, 0x9E3779B97F4A7C15ULL);
    for (int i = 0; i < count; ++i) out[i] = rng.uniform();
}

/* Camera::lookAt (camera.h:110) baked into the C ABI camera. */
void ftr_look_at(const double* eye, const double* target, const double* up, double fov, int rx, int ry,
                 ftb_camera* out) {
    Camera c;
    c.lookAt(v3(eye), v3(target), v3(up), fov, rx, ry);
    Vec3 src[4] = {c.eye, c.u, c.v, c.w};
    double* dst[4] = {out->eye, out->u, out->v, out->w};
    for (int k = 0; k < 4; ++k) { dst[k][0] = src[k].x; dst[k][1] = src[k].y; dst[k][2] = src[k].z; }
    out->tan_half_x = c.tanHalfX; out->tan_half_y = c.tanHalfY; out->res_x = rx; out->res_y = ry;
}

double ftr_total_power(void* h) { return static_cast<Ref*>(h)->scene.totalPower; }

/* The reference Scene behind a handle (for the drop-in shim test, oracle/shim_harness.cpp). */
const void* ftr_scene(void* h) { return &static_cast<Ref*>(h)->scene; }

/* emitter i: power, integral and its cdf (cap entries) */
int ftr_emitter(void* h, int i, double* power, double* integral, double* cdf, int cap) {
    const Scene& s = static_cast<Ref*>(h)->scene;
    if (i < 0 || i >= (int)s.emitters.size()) return -1;
    const Emitter& e = s.emitters[i];
    *power = e.power;
    *integral = e.spd.integral;
    int n = (int)e.spd.cdf.size();
    for (int k = 0; k < n && k < cap; ++k) cdf[k] = e.spd.cdf[k];
    return n;
}

int ftr_closest_hit(void* h, const double* o, const double* d, double* t_out, double* ng_out) {
    const Scene& s = static_cast<Ref*>(h)->scene;
    Hit hh = s.closestHit(Ray{v3(o), v3(d)});
    *t_out = hh.valid ? hh.t : -1.0;
    if (ng_out) { ng_out[0] = hh.ng.x; ng_out[1] = hh.ng.y; ng_out[2] = hh.ng.z; }
    return hh.valid ? hh.matId : -1;
}

int ftr_occluded(void* h, const double* o, const double* d, double max_dist) {
    const Scene& s = static_cast<Ref*>(h)->scene;
    return s.occluded(v3(o), v3(d), max_dist) ? 1 : 0;
}

/* Trace photons [seed_base, seed_base+n) like renderForward's CPU branch.  With logs
 * (threads must be 1) each photon gets its own EnergyReport so its fate and final beta
 * are exact: fate[i] = 0 absorbed, 1 escaped, 2 residual, 3 sensor, 4 nothing booked. */
int ftr_trace(void* h, const ftb_camera* cam, int64_t n, uint64_t seed_base, int max_bounce, int hero_c,
              int threads, double* film_xyz, double* film_hits, double* energy,
              int64_t* rays, int32_t* fate, double* beta) {
    const Scene& scene = static_cast<Ref*>(h)->scene;
    Camera c;
    c.eye = v3(cam->eye); c.u = v3(cam->u); c.v = v3(cam->v); c.w = v3(cam->w);
    c.tanHalfX = cam->tan_half_x; c.tanHalfY = cam->tan_half_y;
    c.projection = CAM_RECTILINEAR;
    c.film.resX = cam->res_x; c.film.resY = cam->res_y;
    const int rx = cam->res_x, ry = cam->res_y;
    if (threads < 1) threads = 1;
    if ((rays || fate || beta) && threads != 1) return -1;
    std::vector<Film> films(threads);
    std::vector<EnergyReport> reports(threads);
    for (auto& f : films) { f.resX = rx; f.resY = ry; f.alloc(); }
    auto worker = [&](int tid) {
        Renderer r;
        // hero sampling as renderForward sets it (main.cpp:11309-11315): -heroc clamped to
        // [1, kHeroMax], on only without media
        const int hc = hero_c < 1 ? 1 : (hero_c > hero::kHeroMax ? hero::kHeroMax : hero_c);
        r.useHero = hc > 1 && scene.media.empty(); r.heroC = hc; r.maxBounce = max_bounce;
        Pcg32 rng;
        long long lo = n * tid / threads, hi = n * (tid + 1) / threads;
        for (long long i = lo; i < hi; ++i) {
            seedUnit(rng, seed_base + (uint64_t)i, 0x9E3779B97F4A7C15ULL);
            if (rays || fate || beta) {
                unsigned long long r0 = raystats::tls;
                EnergyReport ep;
                r.tracePhoton(scene, &c, nullptr, &films[tid], rng, ep);
                if (rays) rays[i] = (int64_t)(raystats::tls - r0);
                int f = 4; double b = 0.0;
                if (ep.absorbed != 0.0) { f = 0; b = ep.absorbed; }
                else if (ep.escaped != 0.0) { f = 1; b = ep.escaped; }
                else if (ep.residual != 0.0) { f = 2; b = ep.residual; }
                else if (ep.sensor != 0.0) { f = 3; b = ep.sensor; }
                if (fate) fate[i] = f;
                if (beta) beta[i] = b;
                EnergyReport& e = reports[tid];
                e.emitted += ep.emitted; e.absorbed += ep.absorbed; e.sensor += ep.sensor;
                e.escaped += ep.escaped; e.residual += ep.residual;
            } else {
                r.tracePhoton(scene, &c, nullptr, &films[tid], rng, reports[tid]);
            }
        }
    };
    if (threads == 1) worker(0);
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker, t);
        for (auto& th : pool) th.join();
    }
    Film out; out.resX = rx; out.resY = ry; out.alloc();
    for (int t = 0; t < threads; ++t) out.merge(films[t]);
    const size_t npix = (size_t)rx * ry;
    for (size_t i = 0; i < npix; ++i) {
        film_xyz[3 * i] += out.xyz[i].x;
        film_xyz[3 * i + 1] += out.xyz[i].y;
        film_xyz[3 * i + 2] += out.xyz[i].z;
        film_hits[i] += out.hits[i];
    }
    for (auto& rp : reports) {
        energy[0] += rp.emitted; energy[1] += rp.absorbed; energy[2] += rp.sensor;
        energy[3] += rp.escaped; energy[4] += rp.residual;
    }
    return 0;
}

}  // extern "C"
