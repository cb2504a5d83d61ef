/*
 * ftb200.h -- C ABI of the B200-native forward pinhole light tracer.
 *
 * This is the drop-in boundary for the ftrace (inhahe/GoodPhotons) mode-B GPU path.
 * The reference exposes that path as a plain C++ API in src/render_cuda.h; every entry
 * point below names the reference interface it replaces.  Unlike the reference, nothing
 * here calls exit(): every function returns an ftb_status and the text of the last error
 * is available from ftb_last_error() (thread-local).
 *
 * Conventions
 *  - Plain pointers and sizes only; no C++ or torch types cross the boundary.
 *  - All geometry and spectral inputs are double precision, exactly as the reference's
 *    Scene holds them after FTSL load (scene.h), so a baked scene is bit-identical input.
 *  - Host pointers unless the parameter name says d_ (device pointer on the scene's GPU).
 *  - Films are 64-bit fixed point (see ftb_film_info): a pixel's sum does not depend on the
 *    order in which photons land, so renders are bit-reproducible across launches, stream
 *    counts and GPU counts.
 *  - Primitive indices are global, in the reference's order (scene.h:2194-2234):
 *    triangles, then spheres, then curve segments, then instances.
 */
#ifndef FTB200_H
#define FTB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FTB_ABI_VERSION 6

typedef enum ftb_status {
    FTB_OK = 0,
    FTB_ERR_INVALID = 1,      /* bad argument (null pointer, index out of range, ...) */
    FTB_ERR_NO_DEVICE = 2,    /* no usable CUDA device */
    FTB_ERR_UNSUPPORTED = 3,  /* scene uses a feature this path does not implement */
    FTB_ERR_CUDA = 4,         /* a CUDA runtime call failed */
    FTB_ERR_OOM = 5,          /* device allocation failed */
    FTB_ERR_DEVICE_LIMIT = 6, /* a bounded device loop gave up (stack/queue overflow) */
    FTB_ERR_TOO_LARGE = 7,    /* request exceeds a documented maximum */
    FTB_ERR_TIMEOUT = 8       /* a wait ran out of time (the work goes on) */
} ftb_status;

/* ---- spectra ------------------------------------------------------------------------
 * A spectrum is a function of wavelength in nm (reference: `Spectrum`, spectrum.h:15).
 * The kinds are the reference's closed-form builders, evaluated with the same arithmetic:
 *   CONST      p[0]                                      constantSpectrum  spectrum.h:179
 *   TABLE      piecewise linear over n (w,v) pairs        tabulatedSpectrum spectrum.h:264
 *              stored at table_w/table_v[offset..offset+n), sorted by w, distinct w
 *   CAUCHY     p[0] + p[1]/um^2                           cauchy            spectrum.h:243
 *   SELLMEIER  p[0..5] = B1 B2 B3 C1 C2 C3                sellmeier         spectrum.h:233
 *   BLACKBODY  Planck at p[0] kelvin, times p[1]          blackbody         spectrum.h:185
 *              (host-side only: emission CDFs; not allowed as a material slot) */
typedef enum ftb_spec_kind {
    FTB_SPEC_CONST = 0,
    FTB_SPEC_TABLE = 1,
    FTB_SPEC_CAUCHY = 2,
    FTB_SPEC_SELLMEIER = 3,
    FTB_SPEC_BLACKBODY = 4
} ftb_spec_kind;

typedef struct ftb_spectrum {
    int32_t kind;     /* ftb_spec_kind */
    int32_t n;        /* TABLE: number of pairs */
    int64_t offset;   /* TABLE: first pair in table_w/table_v */
    double p[6];
} ftb_spectrum;

/* ---- materials ----------------------------------------------------------------------
 * Type numbering equals the reference's MatType (scene.h:42) for the supported subset. */
typedef enum ftb_mat_type {
    FTB_MAT_DIFFUSE = 0,
    FTB_MAT_DIELECTRIC = 1,
    FTB_MAT_MIRROR = 2,
    FTB_MAT_HALF_MIRROR = 3,
    FTB_MAT_GLOSSY = 4,
    FTB_MAT_DIFFUSE_TRANSMIT = 11,
    FTB_MAT_FILTER = 12
} ftb_mat_type;

#define FTB_PRIORITY_UNSET INT32_MIN

typedef struct ftb_material {
    int32_t type;      /* ftb_mat_type */
    int32_t priority;  /* nested-dielectric priority, FTB_PRIORITY_UNSET if unset */
    int32_t reflect;   /* spectrum index: albedo / tint / reflect probability */
    int32_t ior;       /* spectrum index: dielectric IOR (-1: constant 1.5) */
    int32_t absorb;    /* spectrum index: interior sigma_a in 1/m (-1: none) */
    int32_t transmit;  /* spectrum index: DiffuseTransmit albedo / Filter T (-1: zero) */
    double roughness;  /* glossy lobe width; dielectric frosting when > 1e-3 */
} ftb_material;

/* ---- emitters -----------------------------------------------------------------------
 * Area emitters as registered by Scene::addAreaLight / addSphereLight (scene.h:1306-1327).
 * The wavelength CDF is the reference's EmissionSampler (spectrum.h:352-389): cdf_n+1
 * values over [360, 830] nm in bins of `step` nm, at emitter_cdf[cdf_offset..].  `power`
 * is emitIntegral*area*PI (scene.h:1509).  ftb_emission_cdf() computes both from an
 * ftb_spectrum with the reference's arithmetic. */
typedef enum ftb_emit_shape { FTB_EMIT_QUAD = 0, FTB_EMIT_SPHERE = 1 } ftb_emit_shape;

typedef struct ftb_emitter {
    int32_t shape;       /* ftb_emit_shape */
    int32_t collimated;  /* quad only: every photon fires along beam[] */
    int32_t cdf_n;       /* number of bins (cdf has cdf_n+1 entries) */
    int32_t spd;         /* spectrum index of the SPD the cdf was built from (-1: n/a) */
    int64_t cdf_offset;  /* into emitter_cdf */
    double step;         /* bin width in nm */
    double power;        /* selection weight and carried beta */
    double origin[3], u[3], v[3], normal[3];
    double area;
    double radius;       /* sphere */
    double beam[3];
} ftb_emitter;

/* ---- media --------------------------------------------------------------------------
 * Homogeneous Henyey-Greenstein media (scene.h:422-688), optionally bounded by an AABB or
 * a sphere.  sigma_a / sigma_s are spectrum indices in 1/m. */
typedef enum ftb_bound { FTB_BOUND_NONE = 0, FTB_BOUND_BOX = 1, FTB_BOUND_SPHERE = 2 } ftb_bound;

typedef struct ftb_medium {
    int32_t sigma_a, sigma_s;
    int32_t bound;       /* ftb_bound */
    int32_t pad0;
    double g;
    double bmin[3], bmax[3];
    double center[3];
    double radius;
} ftb_medium;

/* BVH builds (no counterpart in the reference, which builds with binned SAH on the host at
 * scene load, bvh.h:89-176).  Either tree gives the same hits: only culling efficiency
 * differs. */
typedef enum ftb_build {
    FTB_BUILD_SAH = 0,      /* binned SAH on the host: the tighter tree (default) */
    FTB_BUILD_DEVICE = 1    /* linear BVH on the GPU: a much faster bake, a looser tree */
} ftb_build;

/* ---- instanced meshes --------------------------------------------------------------
 * A BLAS is a triangle asset in its own (local) space; instances place it in the world by
 * an affine map, like the reference's Blas / MeshInstance (scene.h:996-1063).  A ray meets
 * an instance by being mapped into local space with the inverse map (toLocal, computed from
 * to_world with the reference's Affine::inverse, linalg.h:129-144); local t equals world t.
 * A BLAS may be baked once into a device-resident handle (ftb_blas_create) and shared by
 * many scenes, e.g. the frames of an animation, which then only build their small
 * top-level hierarchy. */
typedef struct ftb_blas ftb_blas;

typedef struct ftb_blas_desc {
    int64_t n_tris;
    const double* tri_v;    /* n_tris x 9, local space */
    const double* tri_n;    /* optional per-vertex shading normals, n_tris x 9 */
    const int32_t* tri_mat; /* indices into the scene's materials */
    ftb_blas* handle;       /* optional: a baked copy of this BLAS (ftb_blas_create); the
                               scene then shares it instead of baking its own, and the
                               arrays above are not read. */
} ftb_blas_desc;

typedef struct ftb_instance {
    int32_t blas;           /* index into ftb_scene_desc.blas */
    int32_t mat_override;   /* >= 0 replaces the BLAS triangles' material */
    double to_world[12];    /* 3x3 linear part row-major, then the translation */
} ftb_instance;

/* ---- scene --------------------------------------------------------------------------
 * tri_v:    n_tris x 9 doubles (v0 v1 v2), winding defines the geometric normal
 * tri_n:    optional n_tris x 9 doubles of per-vertex shading normals (NULL: flat);
 *           zero-length entries fall back to the geometric normal (geometry.h:51-55)
 * sph:      n_spheres x 4 doubles (cx cy cz r)
 * curve:    n_curves x 10 doubles (p0[3] p1[3] r0 r1 u0 u1): round cones (curve.h:85-92) */
typedef struct ftb_scene_desc {
    int64_t n_tris;
    const double* tri_v;
    const double* tri_n;
    const int32_t* tri_mat;
    int64_t n_spheres;
    const double* sph;
    const int32_t* sph_mat;
    int64_t n_curves;
    const double* curve;
    const int32_t* curve_mat;
    int32_t n_mats;
    int32_t n_spectra;
    const ftb_material* mats;
    const ftb_spectrum* spectra;
    int64_t n_table;
    const double* table_w;
    const double* table_v;
    int32_t n_emitters;
    int32_t n_media;
    const ftb_emitter* emitters;
    const double* emitter_cdf;
    const ftb_medium* media;
    int32_t n_blas;
    int32_t build;          /* ftb_build: how ftb_scene_create builds the scene's BVH */
    const ftb_blas_desc* blas;
    int64_t n_instances;
    const ftb_instance* instances;
} ftb_scene_desc;

/* ---- camera -------------------------------------------------------------------------
 * Rectilinear pinhole (camera.h:58-213).  ftb_camera_look_at fills it like
 * Camera::lookAt (camera.h:110). */
typedef struct ftb_camera {
    double eye[3], u[3], v[3], w[3];
    double tan_half_x, tan_half_y;
    int32_t res_x, res_y;
} ftb_camera;

/* ---- render parameters and outputs -------------------------------------------------- */
typedef struct ftb_render_params {
    int64_t n_photons;    /* photons traced by this call */
    uint64_t seed_base;   /* absolute index of the first photon (render_cuda.h:65-68) */
    int32_t max_bounce;   /* bounce cap (reference Renderer::maxBounce, render.h:301) */
    int32_t frac_bits;    /* film fixed-point fraction bits; <=0 picks a safe default */
    int32_t hero_c;       /* wavelengths per photon (-heroc, render_cuda.h:74-82): <= 1 one
                             wavelength; 2..8 hero bundles (Renderer::tracePhotonHero), used
                             only in scenes without media, as the reference does; larger
                             values are clamped to 8 */
    int32_t lambda_mode;  /* ftb_lambda_mode: how the photon's wavelength is drawn */
} ftb_render_params;

/* Wavelength policy of emission.  FTB_LAMBDA_SPD is the reference's: lambda drawn from the
 * emitter's SPD over 360-830 nm (EmissionSampler::sampleAt, spectrum.h:374-383), the photon
 * carrying the emitter's power.  FTB_LAMBDA_UNIFORM_380_780 has no counterpart in the
 * reference: lambda = 380 + 400 u from the same variate u, the photon's power times
 * pdf_SPD(lambda) / (1/400 nm) with the same binned SPD pdf, so the estimate of the light in
 * 380-780 nm is unbiased (light outside the band is not emitted); a photon whose bin has zero
 * SPD is not emitted, like a zero-pdf draw.  Hero bundles stratify u as before and weight
 * each wavelength the same way. */
typedef enum ftb_lambda_mode { FTB_LAMBDA_SPD = 0, FTB_LAMBDA_UNIFORM_380_780 = 1 } ftb_lambda_mode;

/* Energy report (reference EnergyReport, render.h:29-31).  Each tally is the sum of the
 * photons' carried beta, kept in 64-bit fixed point with 32 fraction bits relative to the
 * scene's total emitted power; the doubles are that sum converted back to absolute units. */
typedef struct ftb_energy {
    double emitted, absorbed, sensor, escaped, residual;
    int64_t fx[5];        /* fixed-point tallies, same order */
} ftb_energy;

/* Film layout: 4 int64 words per pixel, row-major (py*res_x+px): X, Y, Z in fixed point,
 * then the splat count (reference Film::hits).  The absolute XYZ sum of a pixel, as the
 * reference Film::xyz holds it, is word * scale. */
typedef struct ftb_film_info {
    int32_t frac_bits;
    int32_t pad0;
    double scale;         /* power_ref * 2^-frac_bits */
    double power_ref;     /* scene total emitted power */
} ftb_film_info;

typedef struct ftb_scene ftb_scene;       /* device-resident baked scene */
typedef struct ftb_session ftb_session;   /* resident film(s) + scene */

/* Memory estimate for admission control (the reference has only cudaMemInfo,
 * render_cuda.h:32, and cudaMegakernelLocalBytes, render_cuda.h:40). */
typedef struct ftb_footprint {
    uint64_t scene_bytes;     /* BVH + primitive records + tables */
    uint64_t film_bytes;      /* per camera film */
    uint64_t wave_bytes;      /* path state, queues and connection records of the device's
                                 two wave buffers at its current tuning (wave_slots) */
    uint64_t total_bytes;
} ftb_footprint;

/* ---- entry points ------------------------------------------------------------------- */

/* Last error message of this thread ("" if none). */
const char* ftb_last_error(void);
int ftb_abi_version(void);

/* replaces cudaAvailable() (render_cuda.h:24) */
int ftb_available(void);
/* replaces cudaDeviceName() (render_cuda.h:27) */
const char* ftb_device_name(void);
/* replaces cudaMemInfo() (render_cuda.h:32) */
ftb_status ftb_mem_info(size_t* free_bytes, size_t* total_bytes);
/* replaces cudaForwardSupported() (render_cuda.h:56): 1 if supported, 0 if not (reason in
 * ftb_last_error), negative on invalid input */
int ftb_forward_supported(const ftb_scene_desc* desc);

/* Camera::lookAt (camera.h:110) */
ftb_status ftb_camera_look_at(const double eye[3], const double target[3],
                              const double up[3], double fov_y_deg, int32_t res_x,
                              int32_t res_y, ftb_camera* out);
/* EmissionSampler::build (spectrum.h:357-369) over the reference band [360, 830] nm:
 * fills cdf[0..n] (n = (830-360)/step) and *integral; `out_cdf` must hold n+1 doubles. */
ftb_status ftb_emission_cdf(const ftb_spectrum* spd, const double* table_w,
                            const double* table_v, double step, double* out_cdf,
                            int32_t out_cap, int32_t* out_n, double* integral);

/* Bake + upload a scene to device `device` (replaces buildUploadScene,
 * render_cuda.cu:12692-13546).  The descriptor is only read during the call. */
ftb_status ftb_scene_create(const ftb_scene_desc* desc, int32_t device, ftb_scene** out);
ftb_status ftb_scene_destroy(ftb_scene* scene);

/* Bake a BLAS (its wide BVH and records) once, for sharing by scenes (no counterpart in
 * the reference, which rebuilds everything per scene load).  Triangle materials index the
 * material table of each scene that uses it.  ftb_blas_destroy releases the caller's
 * handle; scenes created on it hold their own reference, so the device copy lives until
 * the last of them is destroyed. */
ftb_status ftb_blas_create(const ftb_blas_desc* desc, int32_t device, ftb_blas** out);
ftb_status ftb_blas_destroy(ftb_blas* blas);

/* Move the scene's instances (TLAS refit; no counterpart in the reference): new to_world
 * maps (12 doubles each) for instances [0, n), same BLAS and materials.  The top-level
 * hierarchy keeps its topology and gets recomputed, re-quantized bounds, so a render after
 * the refit traces the same paths as a scene created with the new maps (up to exact ties
 * in t, which any two hierarchies may order differently).  No render of this scene may
 * be in flight during the call (synchronize the streams of stream-ordered renders). */
ftb_status ftb_scene_set_instance_transforms(ftb_scene* scene, const double* to_world,
                                             int64_t n);

/* A new scene that shares `src`'s device tables (geometry, materials, emitters, media,
 * BLAS assets) and has its own top-level hierarchy, refit for new maps of instances
 * [0, n) (no counterpart in the reference).  This is how the frames of an animation are
 * made: one scene per frame costs one small top-level copy, and the frames can be
 * rendered together in one ftb_render_batch.  Clones are destroyed with
 * ftb_scene_destroy, in any order relative to `src`. */
ftb_status ftb_scene_clone_instances(const ftb_scene* src, const double* to_world, int64_t n,
                                     ftb_scene** out);
ftb_status ftb_scene_footprint(const ftb_scene* scene, int32_t res_x, int32_t res_y,
                               ftb_footprint* out);

/* Device residency of a scene (no counterpart in the reference, which bakes and frees a
 * scene inside every renderForwardCuda call, render_cuda.cu:13712-13756).
 * ftb_scene_evict frees the scene's device tables (footprint.scene_bytes) and keeps a host
 * copy of them (made on the first eviction); ftb_scene_restore uploads that copy again, so
 * a scene library larger than the device can stay baked in host memory while a working set
 * stays on the device.  Renders of an evicted scene fail with FTB_ERR_INVALID.  Only a scene
 * that owns all its tables can leave the device -- no instances, not a clone and not the
 * source of live clones -- others return FTB_ERR_UNSUPPORTED.  ftb_scene_evict waits for
 * the device first (renders in flight finish).  A render server created with hbm_budget
 * manages the residency of the scenes its jobs use itself. */
ftb_status ftb_scene_evict(ftb_scene* scene);
ftb_status ftb_scene_restore(ftb_scene* scene);
int ftb_scene_resident(const ftb_scene* scene);   /* 1 on the device, 0 evicted */
/* Total emitted power the film and energy fixed point are relative to. */
double ftb_scene_power(const ftb_scene* scene);

/* One-shot render into a HOST film (replaces renderForwardCuda, render_cuda.h:79-82, with
 * camMode 'B' and heroC 1).  film: res_x*res_y*4 int64 (see ftb_film_info); the call
 * OVERWRITES it.  energy is ACCUMULATED (+=), like the reference's eOut. */
ftb_status ftb_render_forward(ftb_scene* scene, const ftb_camera* cam,
                              const ftb_render_params* params, int64_t* film,
                              ftb_film_info* info, ftb_energy* energy);

/* Same, accumulating into a DEVICE film the caller owns (res_x*res_y*4 int64 on the
 * scene's device, zero it first); frac_bits must match across accumulating calls.
 * Asynchronous on `stream` (a cudaStream_t, NULL for the legacy stream) unless
 * energy != NULL, which synchronizes. */
ftb_status ftb_render_forward_device(ftb_scene* scene, const ftb_camera* cam,
                                     const ftb_render_params* params, int64_t* d_film,
                                     ftb_film_info* info, ftb_energy* energy, void* stream);

/* Batched render (no counterpart in the reference, whose closest analogue is the
 * multi-camera shared pass renderForwardSharedCuda, render_cuda.h:94-101): many jobs -- each
 * with its own scene, camera, device film, photon range and bounce cap -- traced together in
 * shared waves, so small jobs and the short tails of long ones fill the GPU together.  All
 * scenes must live on one device.  A job's film and energy are bit-identical to rendering
 * that job alone with ftb_render_forward_device (same frac_bits): photons are keyed by
 * index and the film is fixed point.  Asynchronous on `stream` unless energies != NULL
 * (then it synchronizes, checks the device status word and ACCUMULATES into energies[j]). */
typedef struct ftb_job {
    ftb_scene* scene;
    ftb_camera cam;
    int64_t* d_film;       /* device film, res_x*res_y*4 int64, accumulated */
    int64_t n_photons;
    uint64_t seed_base;
    int32_t max_bounce;
    int32_t frac_bits;     /* <= 0: the default for n_photons */
    int32_t hero_c;        /* wavelengths per photon, as ftb_render_params.hero_c */
    int32_t lambda_mode;   /* as ftb_render_params.lambda_mode */
} ftb_job;

ftb_status ftb_render_batch(const ftb_job* jobs, int32_t n_jobs, ftb_film_info* infos,
                            ftb_energy* energies, void* stream);

/* Resident session (replaces sharedForwardGpuBegin/Batch/Hits0/Download/End,
 * render_cuda.h:121-143).  Films and energy stay on the device between batches.  Every
 * batch traces its photons once and connects each path vertex to every camera (the
 * multi-camera shared splat); hero_c is the wavelengths per photon, as in
 * ftb_render_params (the reference's session takes heroC too, render_cuda.h:122-128). */
ftb_status ftb_session_begin(ftb_scene* scene, const ftb_camera* cams, int32_t n_cams,
                             int32_t max_bounce, int32_t frac_bits, int32_t hero_c,
                             ftb_session** out);
ftb_status ftb_session_batch(ftb_session* s, int64_t n_photons, uint64_t seed_base);
/* hits of camera 0 as doubles (reference sharedForwardGpuHits0) */
ftb_status ftb_session_hits0(ftb_session* s, double* hits);
/* running totals; film_c (camera c) must hold res_x*res_y*4 int64.  Replaces energy. */
ftb_status ftb_session_download(ftb_session* s, int32_t cam, int64_t* film,
                                ftb_film_info* info, ftb_energy* energy);
ftb_status ftb_session_end(ftb_session* s);

/* ---- parity support (test instrumentation, not used on the timed path) --------------
 * Per-photon event record, filled by ftb_trace_log for photons
 * [seed_base, seed_base+n): the number of closest-hit queries (bounce iterations
 * entered), a 64-bit FNV-1a hash over the sequence of hit primitive indices (-1 for a
 * miss), the termination (0 absorbed, 1 escaped, 2 residual, 3 sensor, 4 dropped at
 * emission), the final beta, and the first 8 primitive indices. */
typedef struct ftb_photon_log {
    int32_t n_hits;
    int32_t fate;
    uint64_t prim_hash;
    double beta;
    int32_t prims[8];
} ftb_photon_log;

ftb_status ftb_trace_log(ftb_scene* scene, const ftb_camera* cam,
                         const ftb_render_params* params, ftb_photon_log* out);

/* ---- rendering without device allocation (no counterpart in the reference) ----------
 * For callers that cannot call cudaMalloc: hosts that own all device memory and forbid
 * allocation inside their render callbacks (engine / DCC plug-in hosts with their own
 * allocator), frame loops that must not allocate once running, and code for which a
 * cudaMalloc or cudaFree would synchronize the device mid-stream.  Create the scene once at
 * start-up (ftb_scene_create allocates); then this call only launches kernels on `stream`
 * (a staging kernel that takes the job as kernel arguments, then the wave's kernels),
 * accumulating into the caller's DEVICE film like ftb_render_forward_device.  Its scratch
 * (one wave of path state, queues, shadow records, tallies and status) is a fixed device
 * array of exactly FTB_NOALLOC_SCRATCH_BYTES in the library, held by every GPU that loads
 * the library until exit.
 *  - Limit: n_photons <= FTB_NOALLOC_MAX_PHOTONS per call; larger requests return
 *    FTB_ERR_TOO_LARGE.  Render more with calls of consecutive seed_base, all passing one
 *    explicit frac_bits (e.g. the default for the total photon count): with frac_bits <= 0
 *    each call picks the default for its own n_photons, and calls of different sizes would
 *    add to the film at different scales.
 *  - The first call on a device resolves the array's device address (cudaGetSymbolAddress)
 *    with that device current: make it before any stream capture.
 *  - All calls share the one array, which keeps the last call's contents (the call clears
 *    what must start at zero), so calls that overlap on the GPU (other streams, other
 *    threads) race; serialize them.
 *  - hero_c > 1 is refused (FTB_ERR_UNSUPPORTED) in scenes without media; in scenes with
 *    media every entry point traces one wavelength per photon and so does this one.
 *  - energy != NULL synchronizes `stream` and also checks the device status word. */
#define FTB_NOALLOC_MAX_PHOTONS 32768
#define FTB_NOALLOC_SCRATCH_BYTES 21062912
ftb_status ftb_render_forward_noalloc(ftb_scene* scene, const ftb_camera* cam,
                                      const ftb_render_params* params, int64_t* d_film,
                                      ftb_film_info* info, ftb_energy* energy, void* stream);

/* ---- profiling (measurement support; no counterpart in the reference, which times
 * whole renders by wall clock) ---------------------------------------------------------
 * mode 0: off.  mode 1: every kernel launch of this scene's renders is bracketed by CUDA
 * events on its own stream; ftb_scene_profile sums the durations per kernel.  mode 2:
 * additionally run the counting variants of the traversal kernels, which tally rays, BVH
 * node visits and primitive-record tests (slower: never time a mode-2 render). */
typedef struct ftb_kernel_profile {
    double ms[4];          /* summed launch durations: emit, extend, shade, shadow */
    int64_t launches[4];
    uint64_t counters[8];  /* mode 2: closest-hit rays, their node visits, their record
                              tests; any-hit rays, node visits, record tests; the record
                              tests that reached the exact fp64 test (closest, any) */
} ftb_kernel_profile;

ftb_status ftb_scene_set_profiling(ftb_scene* scene, int32_t mode);
/* Waits for the recorded events, returns the totals since the last reset. */
ftb_status ftb_scene_profile(ftb_scene* scene, ftb_kernel_profile* out, int32_t reset);

/* ---- launch tuning (no counterpart in the reference) ---------------------------------
 * How a device's renders are launched: photon slots per wave (path state is ~400 B per
 * slot, two waves in flight), blocks per SM of the queue-driven kernels, whether each
 * wave's bounce loop (about 5 launches per bounce) is replayed from a captured CUDA graph,
 * and whether closest-hit rays are bucketed by direction before traversal.
 * Renders on the device use the setting current when they start; results do not depend on
 * it (photons are keyed by index, films are fixed point). */
typedef struct ftb_tuning {
    int32_t wave_slots;   /* paths in flight per wave buffer, 1 .. 2^24 */
    int32_t grid_mult;    /* 1 .. 64 */
    int32_t use_graphs;   /* 0 / 1 */
    int32_t sort_rays;    /* 0 / 1: reorder closest-hit rays by direction within each block */
    int32_t regenerate;   /* 0 / 1: streaming passes -- a slot freed by a finished path is
                             refilled with the next photon at once, so the device stays full
                             until the last photons (1), or waves traced to their last bounce
                             one after another (0) */
} ftb_tuning;

ftb_status ftb_get_tuning(int32_t device, ftb_tuning* out);
ftb_status ftb_set_tuning(int32_t device, const ftb_tuning* t);
/* Autotuner: render n_photons of `scene` through `cam` (into a scratch film) under
 * candidate tunings -- grid sizes, wave sizes, graphs on and off, one knob at a time from the
 * current setting -- timing each with CUDA events after a warm-up, then keep the fastest
 * for the scene's device and return it.  n_photons of at least a few waves (>= 2^23) gives
 * stable timings. */
ftb_status ftb_autotune(ftb_scene* scene, const ftb_camera* cam, int64_t n_photons, int32_t max_bounce,
                        ftb_tuning* out);

/* ---- render server (continuous batching; no counterpart in the reference) ------------
 * A server owns two wave buffers and streams on one device, a scheduler thread and a
 * completion thread.  Jobs (a resident scene, a camera, a photon range) are submitted from
 * any thread and admitted in arrival order while their film fits the film budget and a
 * job slot is free.  The scheduler keeps packing the unscheduled photons of the admitted
 * jobs into passes of up to 4 x wave_slots photons (wave_slots paths in flight, freed paths
 * refilled at once; a wave of wave_slots photons when the device's tuning turns refill off)
 * -- the jobs of one kernel class per pass (bundles or not, media, spheres/curves,
 * instances: the class of the job with the least work left, a class that waited two passes
 * first), every job of the class at least a fair share, the rest shortest remaining work
 * first -- so a job that arrives while others are on the GPU joins the next pass and small
 * jobs are not queued behind large ones.  A job's film and energy are exactly those of
 * ftb_render_forward with the same arguments, whatever shares its passes (photons are
 * keyed by index and the film is fixed point).  The scenes referenced by
 * submitted jobs must stay alive until those jobs are done.
 *
 * Admission by device-memory footprint (hbm_budget > 0): the server then accounts its two
 * wave buffers, the films of the admitted jobs and the scenes its jobs use against
 * hbm_budget, and manages those scenes' residency -- a job is admitted when its film, plus
 * its scene's tables if the scene is not on the device, fits the budget; to make room the
 * server evicts scenes that no admitted job uses, least recently used first, and restores a
 * job's scene on admission (ftb_scene_evict / ftb_scene_restore, stream-ordered; a scene's
 * first eviction copies its tables to host memory and waits for the device, later ones only
 * free).  Jobs are admitted in arrival order, except that while the job at the head waits
 * for room, later jobs whose scene is on the device and whose film fits are admitted past
 * it, for two passes; then admission waits for the head.  Scenes that cannot leave the
 * device (instances, clones) count as resident.  The
 * server may evict or restore any scene its jobs have used until it is destroyed, so such
 * scenes must outlive the server, and while it runs they are rendered only through it; when
 * it is destroyed, scenes stay as they are (ftb_scene_resident tells). */
typedef struct ftb_server ftb_server;

typedef struct ftb_server_config {
    int32_t device;
    int32_t max_active;        /* jobs admitted at once, 1..256 (0: 64) */
    uint64_t film_budget;      /* bytes of device films admitted at once (0: a quarter of the
                                  free device memory) */
    int32_t wave_slots;        /* paths in flight per pass, 1..2^24 (0: the device's tuning,
                                  ftb_get_tuning) */
    int32_t hero_max;          /* largest hero_c a request may carry, 1..8 (0: 4); the wave
                                  buffers grow by ~260 B per slot at 4 */
    uint64_t hbm_budget;       /* bytes of wave buffers + admitted films + resident scenes the
                                  server may hold, with scene residency managed (0: films
                                  only, against film_budget; scenes stay where they are) */
} ftb_server_config;

typedef struct ftb_request {
    const ftb_scene* scene;
    ftb_camera cam;
    int64_t n_photons;
    uint64_t seed_base;
    int32_t max_bounce;
    int32_t frac_bits;         /* <= 0: the default for n_photons */
    int32_t hero_c;            /* wavelengths per photon, as ftb_render_params.hero_c */
    int32_t lambda_mode;       /* as ftb_render_params.lambda_mode */
    int64_t* host_film;        /* res_x*res_y*4 int64, written at completion (page-locked memory
                                  copies fastest); NULL: the film is dropped */
} ftb_request;

typedef struct ftb_job_result {
    ftb_status status;         /* of the render: FTB_OK or the error that failed it */
    int32_t pad;
    ftb_film_info info;
    ftb_energy energy;
    double submit_s, admit_s, finish_s;   /* server clock: seconds since ftb_server_create */
} ftb_job_result;

typedef struct ftb_server_stats {
    int64_t submitted, completed, failed, queued, active;
    int64_t photons_done;      /* photons of completed jobs */
    int64_t waves;             /* waves launched */
    double busy_s;             /* time with at least one wave in flight */
    uint64_t film_bytes;       /* device film bytes of admitted jobs now */
    uint64_t scene_bytes;      /* hbm_budget: device bytes of the resident scenes it counts */
    uint64_t wave_bytes;       /* device bytes of the two wave buffers */
    int64_t evictions, restores;   /* hbm_budget: scene evictions and restores so far */
} ftb_server_stats;

ftb_status ftb_server_create(const ftb_server_config* cfg, ftb_server** out);
/* Queue a job; never blocks on the GPU.  A job whose film alone exceeds the budget fails
 * here with FTB_ERR_TOO_LARGE. */
ftb_status ftb_server_submit(ftb_server* s, const ftb_request* req, uint64_t* job_id);
/* Wait for a job (timeout_s < 0: without limit).  FTB_OK: the job is finished, `out` holds
 * its result and the server forgets it (wait once per job); FTB_ERR_TIMEOUT: still running. */
ftb_status ftb_server_wait(ftb_server* s, uint64_t job_id, double timeout_s, ftb_job_result* out);
ftb_status ftb_server_get_stats(ftb_server* s, ftb_server_stats* out);
/* Finish every submitted job, then stop and release the server. */
ftb_status ftb_server_destroy(ftb_server* s);

#ifdef __cplusplus
}
#endif
#endif /* FTB200_H */
