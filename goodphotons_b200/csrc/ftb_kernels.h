// ftb_kernels.h -- host-callable launch API of the wavefront kernels (ftb_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ftb200.h"
#include "ftb_layout.h"

namespace ftb {

// Device status word bits (Frame::status); any nonzero value fails the render.
enum : int32_t {
    ST_STACK_OVERFLOW = 1,    // traversal stack exhausted
    ST_FILM_SATURATED = 2,    // a splat exceeded the fixed-point range
    ST_MEDIUM_STACK = 4,      // nested-dielectric stack deeper than kStkCap
    ST_QUEUE_OVERFLOW = 8,    // shadow queue capacity exceeded
    ST_LOOP_CAP = 16          // a streaming pass ran out of iterations with work left
};

constexpr int kStkCap = 4;
constexpr int kHeroMax = 8;      // wavelengths a hero bundle can carry (hero::kHeroMax)
constexpr int kWaveJobs = 256;   // jobs (frames / requests) one wave can carry

// A camera and its film (one view of a multi-camera job).
struct DevView {
    DevCam cam;
    int64_t* film;
};

// One job's share of a wave: its scene, camera(s) and film(s), and the slots
// [slot0, slot0+n) of the wave that trace its photons photon0, photon0+1, ...  In a
// streaming pass the table is a list of photon ranges instead: the pass hands out photons
// g = 0, 1, ... in order, and g in [g0, g0+n) is this job's photon photon0 + (g - g0).
struct DevJob {
    DevScene sc;
    DevCam cam;
    int64_t* film;             // 4 words per pixel
    const DevView* views;      // n_views > 1: every vertex connects to each view (shared splat)
    int32_t n_views;
    int32_t lambda_mode;       // ftb_lambda_mode of the job's photons
    unsigned long long* tally; // 5 fixed-point energy tallies
    double film_scale_inv;     // 2^frac / power_ref
    double tally_scale_inv;    // 2^32 / power_ref
    uint64_t photon0;
    int64_t g0;                // streaming pass: first stream index of this range
    int32_t slot0, n;
    int32_t max_bounce;
    int32_t hero_c;            // wavelengths per photon (1: the scalar tracer)
};

// Progress of a streaming pass (device memory, updated by k_stream_advance).
struct StreamCtl {
    long long next;            // photons of the pass handed out so far
    int32_t taken;             // paths the current refill appended
    int32_t half;              // half-iterations (extend / shade / refill / shadow) run
    int32_t more;              // work left after the last half-iteration (0 / 1)
    int32_t pad;
};

// The state of the paths in flight, compacted: path i of a queue of n lives at index i of
// every array (structure of arrays, W entries each), so every kernel reads and writes it
// with consecutive lanes on consecutive entries.  A wave holds two, and shading copies the
// surviving paths from one to the other.
struct PathState {
    uint64_t* rng_s; uint64_t* rng_i;
    double *ox, *oy, *oz, *dx, *dy, *dz, *lam, *beta;
    double* cie;               // [3][W] the CIE matching functions at the path's wavelength
    int32_t* stk_n;            // medium-stack depth
    int2* stk;                 // [kStkCap][W] (material, priority)
    int32_t* nbounce;          // bounces traced so far
    int32_t* job;              // job of each path (multi-job tables)
    // hero-wavelength bundles (null unless the buffer carries bundles)
    double* hlam;              // [hero][W] wavelengths, index 0 the hero
    double* hbeta;             // [hero][W] per-wavelength throughput
    int32_t* hlive;            // live wavelengths (hero_c, 1 after a dielectric)
    // parity instrumentation (null unless logging)
    uint64_t* pid;             // photon index
    uint64_t* lhash;
    int32_t* lnh;
    int32_t* lprims;           // [8][W]
};

// Per-wave path state, hits, queues and shadow-ray records (structure of arrays).
struct Wave {
    int32_t W;                 // paths
    int32_t S;                 // shadow-record capacity
    PathState ps[2];           // the paths to trace and the survivors of shading (ping-pong)
    double* hit_t;             // closest hit of path i (indexed like the queue being traced)
    int32_t* hit_rec;          // world record of the closest hit, or -1
    int32_t* hit_sub;          // BLAS record when hit_rec is an instance
    int32_t* perm;             // optional traversal order of a queue (bucketed by direction)
    int32_t* counts;           // [2a], [2a+1]: the two ends of the queue in ps[a]; [4] shadow records;
                               // [5..7] per-launch work counters
    int32_t* sjob;             // job of each shadow record
    DevJob* jobs;              // device job table, kWaveJobs entries
    int32_t* params;           // [0] jobs in the table, [1] paths in flight at most (written with
                               // the table); streaming pass: int64 [1] photons, [2] half-iteration cap
    StreamCtl* ctl;
    double *sox, *soy, *soz, *sdx, *sdy, *sdz, *smax, *sval, *slam;
    double* sxyz;              // [3][S] film increments (X, Y, Z) of one-wavelength connections
    int32_t* spix;
    int32_t* sview;            // view of each connection (multi-camera jobs)
    int32_t hero;              // wavelengths a path of this buffer can carry
    double* xlam;              // [hero-1][S] further wavelengths of a connection
    double* xval;              // [hero-1][S] and their contributions
    int32_t* snup;             // [S] wavelengths in each connection
    ftb_photon_log* logs;      // output, indexed by photon - log_base (null unless logging)
    int64_t log_base;
    void* block;               // the single allocation backing everything above
    size_t bytes;
};

struct Frame {
    unsigned long long* stats; // traversal counters (counting variant only, else null), 8:
                               // [0] closest-hit rays [1] their node visits [2] their record
                               // tests [3] any-hit rays [4] node visits [5] record tests
                               // [6] closest-hit / [7] any-hit exact (fp64) record tests
    int32_t* status;
};

// Queue counts of path buffer a (front and back end), the shadow-record count and the
// per-launch work counters of the closest-hit, shading and shadow kernels in Wave::counts
// ([4] .. [4 + kCountWords - 1] are cleared together after every connection launch).
constexpr int kShadowCount = 4;
constexpr int kFetchExtend = 5, kFetchShade = 6, kFetchShadow = 7;
constexpr int kCountWords = 4;
inline int32_t* queue_counts(const Wave& w, int a) { return w.counts + 2 * a; }

// Shadow records per path: a path queues at most 2 connections per view per bounce, and in
// a streaming pass a refilled path's emission adds one more in the same half-iteration.
constexpr int kShadowPerSlot = 3;

// Bytes of one wave of W paths: every array rounded up to 256 B, in the order wave_carve
// lays them out.  constexpr so a fixed device array can hold a wave (ftb_noalloc.cu).
constexpr size_t wave_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t path_state_bytes(size_t w, bool log, int32_t hero) {
    size_t b = 2 * wave_align(8 * w);                                   // rng
    b += 8 * wave_align(8 * w) + wave_align(24 * w);                    // ray + lam + beta + cie
    b += wave_align(4 * w) + wave_align(8 * w * kStkCap);               // medium stack
    b += 2 * wave_align(4 * w);                                         // bounces, job
    if (hero > 1) b += 2 * wave_align(8 * w * (size_t)hero) + wave_align(4 * w);
    if (log) b += 2 * wave_align(8 * w) + wave_align(4 * w) + wave_align(4 * w * 8);
    return b;
}
constexpr size_t wave_bytes(int32_t W, bool log, int32_t hero = 1) {
    size_t w = (size_t)W, s = kShadowPerSlot * (size_t)W;
    size_t b = 2 * path_state_bytes(w, log, hero);
    b += wave_align(8 * w) + 3 * wave_align(4 * w);                     // hit t, record, sub-record, perm
    b += wave_align(64) + wave_align(4 * s) + wave_align(sizeof(DevJob) * kWaveJobs);   // counts, sjob, table
    b += 2 * wave_align(64);                                            // table parameters, ctl
    b += 9 * wave_align(8 * s) + wave_align(24 * s) + 2 * wave_align(4 * s);   // shadow records
    if (hero > 1) b += 2 * wave_align(8 * s * (hero - 1)) + wave_align(4 * s);
    return b;
}
// Point the arrays of `w` into `block` (wave_bytes(W, log, hero) bytes, 256-B aligned).
void wave_carve(Wave& w, void* block, int32_t W, bool log, int32_t hero = 1);
cudaError_t wave_alloc(Wave& w, int32_t W, bool log, int32_t hero = 1);
void wave_free(Wave& w);

// Kernel ids for profiling.
enum { K_EMIT = 0, K_EXTEND = 1, K_SHADE = 2, K_SHADOW = 3, K_COUNT = 4 };

// Optional observer of kernel launches (profiling): called before and after every launch
// on the launching stream, so it can record CUDA events there.
struct LaunchSink {
    virtual void mark(int kernel, bool end, cudaStream_t stream) = 0;
    virtual ~LaunchSink() {}
};

// Launch shape chosen by the autotuner: blocks per SM of the queue-driven kernels, whether a
// wave is replayed from a captured CUDA graph, and whether closest-hit rays are reordered by
// direction within each block.
struct LaunchShape {
    int32_t grid_mult = 16;
    bool graph = true;
    bool sort_rays = false;   // reorder each block's closest-hit rays by direction first
    bool regenerate = true;   // streaming passes: freed slots are refilled with new photons
};

// Instantiated graphs of one wave buffer, by (bounce cap, grid, instance variant, status
// word): captured on first use, replayed after.
struct WaveGraphs;
WaveGraphs* wave_graphs_create();
void wave_graphs_destroy(WaveGraphs* g);

// Which kernel variants a wave needs, from the jobs of its table.
struct WaveKind {
    bool instances = false;   // some scene has instance records (two-level traversal)
    bool bundles = false;     // hero-wavelength jobs (every job of the table has hero_c > 1)
    bool media = false;       // some scene has participating media
    bool shapes = false;      // some scene has spheres or curves (not only triangles)
    bool mirrors = false;     // some scene has planar mirrors (mirror connections queued)
};
// Connection records one path vertex of job J can queue: a camera connection and one per
// planar mirror, for each of the job's views.  A wave or pass keeps its slots at most
// W / fanout so that the shadow queue (kShadowPerSlot records per slot) cannot overflow.
inline int conn_fanout(const DevJob& J) { return (J.n_views > 1 ? J.n_views : 1) * (1 + J.sc.n_planes); }
// Whether a scene's world records include spheres or curves.
inline bool scene_has_shapes(const DevScene& sc) { return (int64_t)sc.n_recs > sc.n_tris + sc.n_inst; }

// Trace one wave on `stream`.  The caller has written, stream-ordered before this call, the
// job table to w.jobs (slot ranges consecutive from 0) and w.params = {jobs, slots} (slots
// <= W); every slot runs through at most max_bounce bounces (the largest of its jobs).
// Bundles need a buffer allocated with hero >= the largest hero_c of the table.  With
// `graphs` and shape.graph the sequence is replayed from a CUDA graph; profiling (sink),
// counting (f.stats) and logging (w.logs) launches are issued directly.  A cache's graphs
// hold the addresses of its wave buffer and status word: destroy the cache when either
// changes.
cudaError_t launch_wave(Wave& w, int32_t max_bounce, const WaveKind& kind, const Frame& f, int32_t sms,
                        const LaunchShape& shape, cudaStream_t stream, LaunchSink* sink = nullptr,
                        WaveGraphs* graphs = nullptr);

// Trace a streaming pass on `stream`: the caller has written the table of photon ranges to
// w.jobs (g0 consecutive from 0) and w.params = {ranges, slots, photons (int64 at [1]),
// half-iteration cap (int64 at [2])}.  The pass keeps up to `slots` paths in flight: every
// half-iteration runs closest hit, shading (the survivors are compacted into the other
// path buffer), a refill that appends the next photons of the pass up to `slots` paths,
// and the queued connections, until every photon is done.  With `graphs` and shape.graph the loop is one
// graph launch (a conditional while node whose condition the device sets); otherwise the
// host issues half-iterations in groups and reads the progress word between groups.
cudaError_t launch_stream(Wave& w, const WaveKind& kind, const Frame& f, int32_t sms, const LaunchShape& shape,
                          cudaStream_t stream, LaunchSink* sink = nullptr, WaveGraphs* graphs = nullptr);

// Half-iterations a streaming pass of `photons` with `slots` paths in flight can need: a
// path ends within max_bounce half-iterations and its place is refilled in the one it ends
// in, so while photons remain every max_bounce + 1 half-iterations hand out >= slots.
inline int64_t stream_half_cap(int64_t photons, int64_t slots, int32_t max_bounce) {
    const int64_t per = slots > 0 ? (photons + slots - 1) / slots : 0;
    return (per + 2) * ((int64_t)(max_bounce > 0 ? max_bounce : 0) + 2) + 4;
}

}  // namespace ftb
