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
    ST_QUEUE_OVERFLOW = 8     // shadow queue capacity exceeded
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
// [slot0, slot0+n) of the wave that trace its photons photon0, photon0+1, ...
struct DevJob {
    DevScene sc;
    DevCam cam;
    int64_t* film;             // 4 words per pixel
    const DevView* views;      // n_views > 1: every vertex connects to each view (shared splat)
    int32_t n_views, pad;
    unsigned long long* tally; // 5 fixed-point energy tallies
    double film_scale_inv;     // 2^frac / power_ref
    double tally_scale_inv;    // 2^32 / power_ref
    uint64_t photon0;
    int32_t slot0, n;
    int32_t max_bounce;
    int32_t hero_c;            // wavelengths per photon (1: the scalar tracer)
};

// Per-wave path state, queues and shadow-ray records (structure of arrays, W slots).
struct Wave {
    int32_t W;                 // slots
    int32_t S;                 // shadow-record capacity
    uint64_t* rng_s; uint64_t* rng_i;
    double *ox, *oy, *oz, *dx, *dy, *dz, *lam, *beta;
    double* cie;               // [3][W] the CIE matching functions at the path's wavelength
    int32_t* stk_n;            // medium-stack depth per slot
    int2* stk;                 // [kStkCap][W] (material, priority)
    double* hit_t;
    int32_t* hit_rec;          // world record of the closest hit, or -1
    int32_t* hit_sub;          // BLAS record when hit_rec is an instance
    int32_t* qa;               // active slot lists (ping-pong)
    int32_t* qb;
    int32_t* counts;           // [0] qa count, [1] qb count, [2] shadow count
    int32_t* job;              // job of each slot (multi-job waves)
    int32_t* sjob;             // job of each shadow record
    DevJob* jobs;              // device job table, kWaveJobs entries
    int32_t* params;           // [0] jobs in the table, [1] slots in use (written with the table)
    double *sox, *soy, *soz, *sdx, *sdy, *sdz, *smax, *sval, *slam;
    double* sxyz;              // [3][S] film increments (X, Y, Z) of one-wavelength connections
    int32_t* spix;
    int32_t* sview;            // view of each connection (multi-camera jobs)
    // hero-wavelength bundles (hero > 1 only; null otherwise)
    int32_t hero;              // wavelengths a path of this buffer can carry
    double* hlam;              // [hero][W] wavelengths, index 0 the hero
    double* hbeta;             // [hero][W] per-wavelength throughput
    int32_t* hlive;            // [W] live wavelengths (hero_c, 1 after a dielectric)
    double* xlam;              // [hero-1][S] further wavelengths of a connection
    double* xval;              // [hero-1][S] and their contributions
    int32_t* snup;             // [S] wavelengths in each connection
    // parity instrumentation (null unless logging)
    uint64_t* lhash;
    int32_t* lnh;
    int32_t* lprims;           // [8][W]
    ftb_photon_log* logs;      // output, indexed by photon - log_base
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

// Bytes of one wave of W slots: every array rounded up to 256 B, in the order wave_carve
// lays them out.  constexpr so a fixed device array can hold a wave (ftb_noalloc.cu).
constexpr size_t wave_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t wave_bytes(int32_t W, bool log, int32_t hero = 1) {
    size_t w = (size_t)W, s = 2 * (size_t)W;
    size_t b = 0;
    b += 2 * wave_align(8 * w);                                     // rng
    b += 8 * wave_align(8 * w) + wave_align(24 * w);                // ray + lam + beta + cie
    b += wave_align(4 * w) + wave_align(8 * w * kStkCap);           // medium stack
    b += wave_align(8 * w) + 2 * wave_align(4 * w);                 // hit t, record, sub-record
    b += 2 * wave_align(4 * w) + wave_align(64);                    // queues + counts
    b += wave_align(4 * w) + wave_align(4 * s) + wave_align(sizeof(DevJob) * kWaveJobs);   // job ids + table
    b += wave_align(64);                                            // table parameters
    b += 9 * wave_align(8 * s) + wave_align(24 * s) + 2 * wave_align(4 * s);   // shadow records
    if (log) b += wave_align(8 * w) + wave_align(4 * w) + wave_align(4 * w * 8);
    if (hero > 1)                                                   // bundles
        b += 2 * wave_align(8 * w * hero) + wave_align(4 * w) + 2 * wave_align(8 * s * (hero - 1)) +
             wave_align(4 * s);
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
};

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

}  // namespace ftb
