/*
 * ftoracle.h -- CPU ORACLE for parity tests.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, double-precision restatement of the reference's forward pinhole light
 * tracer (ftrace Renderer::tracePhoton, src/render.h:1811-2240, single wavelength,
 * model B).  It exists to check the CUDA path: tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py are its only callers.  The product library never links
 * or calls it.
 *
 * Parity pin: tests/test_oracle_pin.py checks this restatement against the reference
 * itself (compiled from its own headers into oracle/_ref/ by oracle/Makefile) and against
 * the committed golden vectors in tests/golden/: bit-identical film sums and energy
 * report, and identical per-photon ray-query counts.
 *
 * Input is the same POD scene description the C ABI takes (include/ftb200.h).
 */
#ifndef FTORACLE_H
#define FTORACLE_H

#include "../include/ftb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fto_ctx fto_ctx;

/* Copy the scene, finalize triangles (geometry.h:51-55), build emitter tables
 * (scene.h:1491-1518) and an acceleration structure.  NULL on invalid input. */
fto_ctx* fto_prepare(const ftb_scene_desc* desc);
void fto_release(fto_ctx* ctx);

/* Trace photons [seed_base, seed_base+n) with `threads` worker threads banded like the
 * reference's renderForward CPU branch (main.cpp:11305-11340): thread t takes
 * [n*t/T, n*(t+1)/T) and the per-thread films are merged in thread order, so a run is
 * bit-identical to the reference run with the same thread count.
 *   film_xyz: res_x*res_y*3 doubles (accumulated, += )
 *   film_hits: res_x*res_y doubles (accumulated)
 *   energy: 5 doubles emitted/absorbed/sensor/escaped/residual (accumulated)
 *   logs: optional, n records (see ftb_photon_log)
 *   rays: optional, n per-photon counts of closest-hit + occlusion queries
 *   hero_c: wavelengths per photon (Renderer::tracePhotonHero when > 1; clamped to 1..8;
 *           1 in scenes with media, as the reference gates it)
 * Returns 0, or -1 on invalid input (message in fto_last_error()). */
int fto_trace(const fto_ctx* ctx, const ftb_camera* cam, int64_t n, uint64_t seed_base,
              int max_bounce, int hero_c, int threads, double* film_xyz, double* film_hits,
              double* energy, ftb_photon_log* logs, int64_t* rays);

/* Total emitted power (Scene::totalPower, scene.h:1509-1511). */
double fto_total_power(const fto_ctx* ctx);

/* Wavelength policy of later fto_trace calls (ftb_lambda_mode; FTB_LAMBDA_SPD, the
 * reference's, by default).  Returns 0, or -1 on invalid input. */
int fto_set_lambda_mode(fto_ctx* ctx, int mode);

/* EmissionSampler::build (spectrum.h:357-369) for spectrum `spec` of the descriptor;
 * returns the bin count (cdf has count+1 entries) or -1. */
int fto_emission_cdf(const ftb_scene_desc* desc, int spec, double step, double* cdf,
                     int cap, double* integral);

/* Spectrum evaluation (spectrum.h builders). */
double fto_spectrum_eval(const ftb_scene_desc* desc, int spec, double lambda_nm);

/* Camera::lookAt (camera.h:110-125). */
void fto_camera_look_at(const double eye[3], const double target[3], const double up[3],
                        double fov_y_deg, int res_x, int res_y, ftb_camera* out);

/* The first `count` uniforms of photon k's stream (seedUnit rng.h:40, uniform rng.h:22). */
void fto_uniforms(uint64_t k, int count, double* out);

/* Scene::closestHit (scene.h:2194): returns the global primitive index or -1; sets t. */
int fto_closest_hit(const fto_ctx* ctx, const double o[3], const double d[3], double tmin,
                    double* t_out);
/* Scene::occluded (scene.h:2249) */
int fto_occluded(const fto_ctx* ctx, const double o[3], const double d[3], double max_dist,
                 double tmin);

/* The planar mirrors the tracer connects through (Scene::buildMirrorPlanes,
 * scene.h:1646-1720): writes up to `cap` planes as {n[3], d, lo[3], hi[3]} and returns their
 * number. */
int fto_mirror_planes(const fto_ctx* ctx, double* out, int cap);

const char* fto_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
