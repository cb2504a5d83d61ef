// ftb_api.cpp -- host side of the C ABI declared in include/ftb200.h.
//
// Replaces the host half of the reference's forward GPU path: the scene bake
// (buildUploadScene, render_cuda.cu:12692-13546), the launch (launchForward /
// renderForwardCuda, render_cuda.cu:13683-13756) and the resident sessions
// (render_cuda.cu:13763-13871).  Every failure is reported through a status code and
// ftb_last_error(); nothing exits the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ftb200.h"
#include "bvh_build.h"
#include "ftb_internal.h"
#include "ftb_kernels.h"
#include "ftb_layout.h"

namespace {

thread_local std::string g_err;

ftb_status fail(ftb_status s, const std::string& m) {
    g_err = m;
    return s;
}
ftb_status cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? FTB_ERR_OOM : FTB_ERR_CUDA;
}
#define CK(call, what)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

constexpr double kLambdaMin = 360.0, kLambdaMax = 830.0;
constexpr double kPi = 3.141592653589793;

// ---- host restatements used at bake time ---------------------------------------------
double blackbody_radiance(double kelvin, double lambda_nm) {   // spectrum.h:185-190
    const double h = 6.62607015e-34, c = 2.99792458e8, kb = 1.380649e-23;
    double l = lambda_nm * 1e-9;
    double e = std::exp((h * c) / (l * kb * kelvin)) - 1.0;
    return (2.0 * h * c * c) / (std::pow(l, 5.0) * e);
}

bool spec_valid(const ftb_scene_desc* d, int idx, std::string& why) {
    if (idx < 0 || idx >= d->n_spectra || !d->spectra) { why = "spectrum index out of range"; return false; }
    const ftb_spectrum& s = d->spectra[idx];
    if (s.kind < FTB_SPEC_CONST || s.kind > FTB_SPEC_BLACKBODY) { why = "unknown spectrum kind"; return false; }
    if (s.kind == FTB_SPEC_TABLE) {
        if (s.n <= 0 || s.offset < 0 || s.offset + s.n > d->n_table || !d->table_w || !d->table_v) {
            why = "table spectrum out of range"; return false;
        }
        for (int i = 1; i < s.n; ++i)
            if (!(d->table_w[s.offset + i] > d->table_w[s.offset + i - 1])) {
                why = "table spectrum wavelengths must be strictly increasing"; return false;
            }
    }
    return true;
}

double spec_eval_host(const ftb_scene_desc* d, int idx, double w) {
    const ftb_spectrum& s = d->spectra[idx];
    switch (s.kind) {
    case FTB_SPEC_CONST: return s.p[0];
    case FTB_SPEC_TABLE: {   // tabulatedSpectrum (spectrum.h:264-281)
        const double* x = d->table_w + s.offset;
        const double* y = d->table_v + s.offset;
        int n = s.n;
        if (w <= x[0]) return y[0];
        if (w >= x[n - 1]) return y[n - 1];
        size_t lo = 0, hi = (size_t)n - 1;
        while (lo + 1 < hi) { size_t mid = (lo + hi) / 2; (x[mid] <= w ? lo : hi) = mid; }
        double w0 = x[lo], w1 = x[lo + 1], v0 = y[lo], v1 = y[lo + 1];
        double f = (w1 > w0) ? (w - w0) / (w1 - w0) : 0.0;
        return v0 + (v1 - v0) * f;
    }
    case FTB_SPEC_CAUCHY: { double um = w * 1e-3; return s.p[0] + s.p[1] / (um * um); }
    case FTB_SPEC_SELLMEIER: {
        double l2 = (w * 1e-3) * (w * 1e-3);
        double n2 = 1.0 + s.p[0] * l2 / (l2 - s.p[3]) + s.p[1] * l2 / (l2 - s.p[4]) + s.p[2] * l2 / (l2 - s.p[5]);
        return std::sqrt(n2 > 1.0 ? n2 : 1.0);
    }
    case FTB_SPEC_BLACKBODY: return blackbody_radiance(s.p[0], w) * s.p[1];
    }
    return 0.0;
}

struct V { double x, y, z; };
V vsub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V vcross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double vdot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V vnorm(V a) { double l = std::sqrt(vdot(a, a)); return {a.x / l, a.y / l, a.z / l}; }

}  // namespace

// ---- profiling sink -------------------------------------------------------------------
namespace {
struct ProfSink : ftb::LaunchSink {
    struct Rec { int kernel; cudaEvent_t a, b; };
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<Rec> pending;
    cudaEvent_t open[ftb::K_COUNT][2] = {};   // per kernel kind and stream slot
    double ms[ftb::K_COUNT] = {0, 0, 0, 0};
    int64_t launches[ftb::K_COUNT] = {0, 0, 0, 0};
    cudaEvent_t take() {
        if (used == pool.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            pool.push_back(e);
        }
        return pool[used++];
    }
    // launches on one stream are serialized, so the begin event of a kernel kind is
    // paired with the next end event of the same kind on the same stream
    std::vector<std::pair<cudaStream_t, cudaEvent_t>> begun[ftb::K_COUNT];
    void mark(int k, bool end, cudaStream_t st) override {
        cudaEvent_t e = take();
        if (!e) return;
        cudaEventRecord(e, st);
        if (!end) { begun[k].push_back({st, e}); return; }
        for (size_t i = 0; i < begun[k].size(); ++i)
            if (begun[k][i].first == st) {
                pending.push_back({k, begun[k][i].second, e});
                begun[k].erase(begun[k].begin() + (long)i);
                return;
            }
    }
    void resolve() {
        for (auto& r : pending) {
            float t = 0.f;
            cudaEventSynchronize(r.b);
            if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) { ms[r.kernel] += t; launches[r.kernel]++; }
        }
        pending.clear();
        used = 0;
        for (auto& b : begun) b.clear();
    }
    ~ProfSink() override { for (auto e : pool) cudaEventDestroy(e); }
};
}  // namespace

// ---- job-table staging ------------------------------------------------------------------
namespace {
// Pinned host ring from which a wave's job table is copied to the device on the wave's
// stream; an entry is reused only after its previous copy has completed.
struct JobStage {
    static constexpr int kRing = 4;
    ftb::DevJob* host = nullptr;
    cudaEvent_t ev[kRing] = {};
    int next = 0;
    cudaError_t init() {
        if (host) return cudaSuccess;
        cudaError_t e = cudaHostAlloc((void**)&host, sizeof(ftb::DevJob) * (ftb::kWaveJobs + 1) * kRing,
                                      cudaHostAllocDefault);
        if (e != cudaSuccess) { host = nullptr; return e; }
        for (auto& v : ev) {
            e = cudaEventCreateWithFlags(&v, cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // The table and its parameters {jobs, slots} into the wave (w.jobs, w.params); a
    // streaming pass adds its photon count and half-iteration cap (int64 at [1], [2]).
    cudaError_t push(const ftb::DevJob* jobs, int n, int32_t slots, ftb::Wave& w, cudaStream_t st,
                     int64_t photons = 0, int64_t half_cap = 0) {
        int e = next;
        next = (next + 1) % kRing;
        cudaError_t r = cudaEventSynchronize(ev[e]);
        if (r != cudaSuccess) return r;
        ftb::DevJob* h = host + (size_t)e * (ftb::kWaveJobs + 1);
        std::memcpy(h, jobs, sizeof(ftb::DevJob) * (size_t)n);
        int32_t* par = reinterpret_cast<int32_t*>(h + ftb::kWaveJobs);
        par[0] = n;
        par[1] = slots;
        reinterpret_cast<int64_t*>(par)[1] = photons;
        reinterpret_cast<int64_t*>(par)[2] = half_cap;
        r = cudaMemcpyAsync(w.jobs, h, sizeof(ftb::DevJob) * (size_t)n, cudaMemcpyHostToDevice, st);
        if (r == cudaSuccess) r = cudaMemcpyAsync(w.params, par, 6 * sizeof(int32_t), cudaMemcpyHostToDevice, st);
        if (r != cudaSuccess) return r;
        return cudaEventRecord(ev[e], st);
    }
    ~JobStage() {
        for (auto v : ev) if (v) cudaEventDestroy(v);
        if (host) cudaFreeHost(host);
    }
};
}  // namespace

// ---- device blocks and BLAS assets ----------------------------------------------------
namespace {
// Device allocations released together, on their device.  Shared (std::shared_ptr) by the
// objects that read them: a scene and its clones share their tables, scenes share a BLAS.
struct DevBlock {
    int device = 0;
    std::vector<void*> ptrs;
    uint64_t bytes = 0;
    // Residency (ftb_scene_evict / ftb_scene_restore): the size of each allocation, whether
    // it came from the stream-ordered allocator (a restore), and host copies of the arrays
    // (made on the first eviction and kept, so later evictions only free).  The copies are
    // pinned, so a restore's uploads are asynchronous: a render server restores scenes
    // without stalling the thread that launches its passes.
    std::vector<size_t> sizes;
    std::vector<char> pooled;
    std::vector<unsigned char*> saved;
    std::vector<void*> evicted;   // the allocations' addresses when they were freed
    bool resident = true;
    DevBlock() = default;
    DevBlock(const DevBlock&) = delete;
    DevBlock& operator=(const DevBlock&) = delete;
    ~DevBlock() {
        if (ptrs.empty()) return;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        if (resident)
            for (void* p : ptrs) cudaFree(p);   // waits for the device, pooled allocations too
        for (unsigned char* h : saved) if (h) cudaFreeHost(h);
        cudaSetDevice(cur);
    }
};

template <class T>
ftb_status upload(DevBlock& blk, const T* host, size_t n, const T** out, const char* what) {
    if (n == 0) { *out = nullptr; return FTB_OK; }
    void* p = nullptr;
    CK(cudaMalloc(&p, n * sizeof(T)), what);
    blk.ptrs.push_back(p);
    blk.sizes.push_back(n * sizeof(T));
    blk.pooled.push_back(0);
    blk.bytes += n * sizeof(T);
    CK(cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice), what);
    *out = (const T*)p;
    return FTB_OK;
}

// A baked BLAS (Blas, scene.h:996-1033): wide BVH and triangle records in local space.
struct BlasDev {
    DevBlock mem;
    const FNode* nodes = nullptr;
    const PrimRec* recs = nullptr;
    const double* tri_n = nullptr;
    int64_t n_tris = 0;
    int32_t max_mat = -1;
    double lo[3], hi[3];   // localBounds: union of the triangle boxes padded by 1e-6
};

// Host state kept for refitting the top-level hierarchy of a scene with instances.
struct TlasHost {
    ftb::WideBvh bvh;
    std::vector<ftb::Box> boxes;     // unmargined primitive boxes, global order
    double base_maxabs = 1.0;        // coordinate magnitude of everything but the instances
    int64_t first_inst = 0;          // global index of instance 0
    std::vector<int32_t> inst_blas;  // BLAS of each instance
    std::vector<DevInst> inst;       // host copy of the device instance table
};
}  // namespace

struct ftb_blas {
    std::shared_ptr<BlasDev> p;
};

// ---- per-device render engine ------------------------------------------------------------
namespace {
// The wave buffers, streams and scratch every render on one device uses.  Shared by all
// scenes of the device (a scene, its clones, the scenes of a batch), so their number does
// not multiply the ~300 B per wave slot; renders on a device serialize on `mu`.
struct Engine {
    int device = 0;
    std::mutex mu;
    cudaStream_t streams[2] = {nullptr, nullptr};
    ftb::Wave waves[2]{};
    JobStage stage[2];
    int32_t wave_W = 0;
    bool wave_log = false;
    int64_t* film = nullptr;          // film of the host-film entry points
    size_t film_words = 0;
    unsigned long long* tally = nullptr;
    int32_t* status = nullptr;
    unsigned long long* batch_tally = nullptr;   // 8 words per job of the last batch
    size_t batch_cap = 0;
    ftb::WaveGraphs* graphs[2] = {nullptr, nullptr};
    ftb::LaunchShape shape;                      // grid and graph choice (autotuned)
    int32_t wave_cap = 1 << 22;                  // largest wave (autotuned)
    ~Engine() {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        for (auto g : graphs) ftb::wave_graphs_destroy(g);
        for (auto& w : waves) ftb::wave_free(w);
        for (auto s : streams) if (s) cudaStreamDestroy(s);
        if (film) cudaFree(film);
        if (tally) cudaFree(tally);
        if (status) cudaFree(status);
        if (batch_tally) cudaFree(batch_tally);
        cudaSetDevice(cur);
    }
};

std::mutex g_engine_mu;
std::weak_ptr<Engine> g_engines[256];
ftb_tuning g_tuning[256];          // per device; a new engine starts from it
bool g_tuning_set[256] = {};

ftb_tuning default_tuning() { return ftb_tuning{1 << 22, 16, 1, 0, 1}; }

void apply_tuning(Engine& e, const ftb_tuning& t) {
    e.wave_cap = t.wave_slots;
    e.shape.grid_mult = t.grid_mult;
    e.shape.graph = t.use_graphs != 0;
    e.shape.sort_rays = t.sort_rays != 0;
    e.shape.regenerate = t.regenerate != 0;
}

// The device's engine, created on first use; it lives while any scene holds it.
std::shared_ptr<Engine> engine_for(int device) {
    std::lock_guard<std::mutex> lk(g_engine_mu);
    auto e = g_engines[device].lock();
    if (!e) {
        e = std::make_shared<Engine>();
        e->device = device;
        apply_tuning(*e, g_tuning_set[device] ? g_tuning[device] : default_tuning());
        g_engines[device] = e;
    }
    return e;
}
}  // namespace

// ---- scene object ----------------------------------------------------------------------
struct ftb_scene {
    int device = 0;
    int sms = 148;
    DevScene dev{};
    std::shared_ptr<DevBlock> tables;              // geometry, materials, emitters (shared with clones)
    std::vector<std::shared_ptr<BlasDev>> blas;    // BLAS assets the instances place
    std::unique_ptr<DevBlock> own;                 // this scene's TLAS nodes and instance table
    TlasHost tlas;                                 // for refits (scenes with instances)
    FNode* d_nodes = nullptr;                      // mutable TLAS nodes (in `own`)
    DevInst* d_inst = nullptr;
    double power = 0.0;
    uint64_t scene_bytes = 0;
    std::vector<int> field_alloc;                  // while evicted: the allocation of each device pointer of `dev`
    std::shared_ptr<Engine> eng;                   // render resources of the device
    int32_t prof_mode = 0;
    ProfSink* prof = nullptr;
    unsigned long long* stats = nullptr;   // device counters for profiling mode 2
    ~ftb_scene() {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        if (stats) cudaFree(stats);
        delete prof;
        cudaSetDevice(cur);
    }
};

struct ftb_session {
    ftb_scene* scene = nullptr;
    std::vector<ftb_camera> cams;
    std::vector<int64_t*> films;
    ftb::DevView* views = nullptr;   // device: every camera with its film (one shared pass)
    unsigned long long* tally = nullptr;
    int32_t max_bounce = 32;
    int32_t frac_bits = 0;
    int32_t hero_c = 1;              // wavelengths per photon (bundles of every camera's paths)
};

namespace {

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int dev) { cudaGetDevice(&prev); cudaSetDevice(dev); }
    ~DeviceGuard() { cudaSetDevice(prev); }
};

template <class T>
ftb_status upload(ftb_scene* s, const T* host, size_t n, const T** out, const char* what) {
    return upload(*s->tables, host, n, out, what);
}

bool mat_type_supported(int t) {
    return t == FTB_MAT_DIFFUSE || t == FTB_MAT_DIELECTRIC || t == FTB_MAT_GLOSSY ||
           t == FTB_MAT_DIFFUSE_TRANSMIT || t == FTB_MAT_FILTER || t == FTB_MAT_MIRROR ||
           t == FTB_MAT_HALF_MIRROR;
}

// isPlanarMirrorMat (scene.h:356-360)
bool planar_mirror(const ftb_material& m) {
    return m.type == FTB_MAT_MIRROR || m.type == FTB_MAT_HALF_MIRROR ||
           (m.type == FTB_MAT_GLOSSY && m.roughness <= 0.0);
}

constexpr int kMaxMirrorPlanes = 64;   // Scene::kMaxMirrorPlanes (scene.h:1641)

// Scene::buildMirrorPlanes (scene.h:1646-1720) over the world triangles: each planar-mirror
// triangle's unit normal (Tri::finalize's, normalized again), flipped so its largest
// component is positive, and offset d = dot(n, v0) form a key quantized to 1e-6 in
// direction and 10 um in offset; triangles with equal keys share a plane, planes numbered
// in first-seen order, each with the AABB of its vertices and its total area; the boxes are
// padded by 1e-6 (1 + diagonal).  More than 64 planes -- where the reference keeps the 64
// largest by an unstable sort -- is reported as unsupported.
ftb_status build_mirror_planes(const ftb_scene_desc* d, std::vector<DevPlane>& out) {
    out.clear();
    struct Acc { DevPlane p; long long key[4]; };
    std::vector<Acc> acc;
    std::unordered_map<std::string, int> by_key;
    for (int64_t i = 0; i < d->n_tris; ++i) {
        if (!planar_mirror(d->mats[d->tri_mat[i]])) continue;
        const double* v = d->tri_v + 9 * i;
        const double e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
        const double e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
        double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double cl = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        double n[3] = {c[0] / cl, c[1] / cl, c[2] / cl};   // Tri::finalize: normalize(cross)
        const double nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nl < 1e-12) continue;
        const double inv = 1.0 / nl;
        for (double& x : n) x = x * inv;
        const double sx = std::fabs(n[0]), sy = std::fabs(n[1]), sz = std::fabs(n[2]);
        const double lead = (sx >= sy && sx >= sz) ? n[0] : ((sy >= sz) ? n[1] : n[2]);
        if (lead < 0.0) for (double& x : n) x = -x;
        const double off = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
        const long long key[4] = {std::llround(n[0] * 1e6), std::llround(n[1] * 1e6), std::llround(n[2] * 1e6),
                                  std::llround(off * 1e5)};
        const std::string ks(reinterpret_cast<const char*>(key), sizeof key);
        auto it = by_key.find(ks);
        int idx;
        if (it == by_key.end()) {
            idx = (int)acc.size();
            by_key.emplace(ks, idx);
            Acc a;
            for (int k = 0; k < 3; ++k) { a.p.n[k] = n[k]; a.p.lo[k] = v[k]; a.p.hi[k] = v[k]; }
            a.p.d = off;
            std::memcpy(a.key, key, sizeof key);
            acc.push_back(a);
        } else {
            idx = it->second;
        }
        DevPlane& p = acc[(size_t)idx].p;
        for (int q = 0; q < 3; ++q)
            for (int k = 0; k < 3; ++k) {
                p.lo[k] = std::min(p.lo[k], v[3 * q + k]);
                p.hi[k] = std::max(p.hi[k], v[3 * q + k]);
            }
    }
    if ((int)acc.size() > kMaxMirrorPlanes)
        return fail(FTB_ERR_UNSUPPORTED, "more than 64 mirror planes (the reference keeps the 64 largest by an "
                    "unstable sort)");
    for (Acc& a : acc) {
        DevPlane& p = a.p;
        const double dx = p.hi[0] - p.lo[0], dy = p.hi[1] - p.lo[1], dz = p.hi[2] - p.lo[2];
        const double pad = 1e-6 * (1.0 + std::sqrt(dx * dx + dy * dy + dz * dz));
        for (int k = 0; k < 3; ++k) { p.lo[k] = p.lo[k] - pad; p.hi[k] = p.hi[k] + pad; }
        out.push_back(p);
    }
    return FTB_OK;
}

// Validation shared by ftb_forward_supported and ftb_scene_create.  Returns FTB_OK,
// FTB_ERR_INVALID (malformed) or FTB_ERR_UNSUPPORTED.
ftb_status check_desc(const ftb_scene_desc* d) {
    if (!d) return fail(FTB_ERR_INVALID, "null scene descriptor");
    if (d->n_tris < 0 || d->n_spheres < 0 || d->n_curves < 0 || d->n_mats < 0 || d->n_spectra < 0 ||
        d->n_emitters < 0 || d->n_media < 0 || d->n_table < 0)
        return fail(FTB_ERR_INVALID, "negative count in scene descriptor");
    if ((d->n_tris && (!d->tri_v || !d->tri_mat)) || (d->n_spheres && (!d->sph || !d->sph_mat)) ||
        (d->n_curves && (!d->curve || !d->curve_mat)) || (d->n_mats && !d->mats) ||
        (d->n_emitters && (!d->emitters || !d->emitter_cdf)) || (d->n_media && !d->media))
        return fail(FTB_ERR_INVALID, "null array for a nonzero count");
    if (d->n_blas < 0 || d->n_instances < 0) return fail(FTB_ERR_INVALID, "negative count in scene descriptor");
    if (d->build != FTB_BUILD_SAH && d->build != FTB_BUILD_DEVICE) return fail(FTB_ERR_INVALID, "unknown BVH build");
    if ((d->n_blas && !d->blas) || (d->n_instances && !d->instances))
        return fail(FTB_ERR_INVALID, "null array for a nonzero count");
    int64_t np = d->n_tris + d->n_spheres + d->n_curves + d->n_instances;
    if (np > ((int64_t)1 << 29)) return fail(FTB_ERR_TOO_LARGE, "too many primitives (max 2^29)");
    for (int b = 0; b < d->n_blas; ++b) {
        const ftb_blas_desc& bd = d->blas[b];
        if (bd.handle) {
            if (!bd.handle->p || bd.handle->p->max_mat >= d->n_mats)
                return fail(FTB_ERR_INVALID, "BLAS " + std::to_string(b) + ": material out of range for this scene");
            continue;
        }
        if (bd.n_tris < 1 || bd.n_tris > ((int64_t)1 << 29) || !bd.tri_v || !bd.tri_mat)
            return fail(FTB_ERR_INVALID, "BLAS " + std::to_string(b) + ": needs 1..2^29 triangles");
        for (int64_t i = 0; i < bd.n_tris; ++i)
            if (bd.tri_mat[i] < 0 || bd.tri_mat[i] >= d->n_mats)
                return fail(FTB_ERR_INVALID, "BLAS " + std::to_string(b) + ": triangle material out of range");
    }
    for (int64_t k = 0; k < d->n_instances; ++k) {
        const ftb_instance& in = d->instances[k];
        if (in.blas < 0 || in.blas >= d->n_blas) return fail(FTB_ERR_INVALID, "instance BLAS index out of range");
        if (in.mat_override < -1 || in.mat_override >= d->n_mats)
            return fail(FTB_ERR_INVALID, "instance material override out of range");
        for (int j = 0; j < 12; ++j)
            if (!std::isfinite(in.to_world[j])) return fail(FTB_ERR_INVALID, "instance transform not finite");
    }
    std::string why;
    for (int i = 0; i < d->n_spectra; ++i)
        if (!spec_valid(d, i, why)) return fail(FTB_ERR_INVALID, "spectrum " + std::to_string(i) + ": " + why);
    auto chk_slot = [&](int s) { return s >= -1 && s < d->n_spectra; };
    for (int i = 0; i < d->n_mats; ++i) {
        const ftb_material& m = d->mats[i];
        if (!chk_slot(m.reflect) || !chk_slot(m.ior) || !chk_slot(m.absorb) || !chk_slot(m.transmit))
            return fail(FTB_ERR_INVALID, "material " + std::to_string(i) + ": spectrum index out of range");
        if (!mat_type_supported(m.type))
            return fail(FTB_ERR_UNSUPPORTED, "material " + std::to_string(i) + ": type " + std::to_string(m.type) +
                        " is not on this path");
    }
    for (int64_t i = 0; i < d->n_tris; ++i)
        if (d->tri_mat[i] < 0 || d->tri_mat[i] >= d->n_mats) return fail(FTB_ERR_INVALID, "triangle material out of range");
    for (int64_t i = 0; i < d->n_spheres; ++i) {
        if (d->sph_mat[i] < 0 || d->sph_mat[i] >= d->n_mats) return fail(FTB_ERR_INVALID, "sphere material out of range");
        if (d->mats[d->sph_mat[i]].type == FTB_MAT_DIELECTRIC)
            return fail(FTB_ERR_UNSUPPORTED, "dielectric sphere: the reference splats it through its analytic "
                        "sphere connector, which is not on this path");
        if (planar_mirror(d->mats[d->sph_mat[i]]))
            return fail(FTB_ERR_UNSUPPORTED, "mirror sphere: the reference splats it through its spherical "
                        "mirror connector, which is not on this path");
    }
    for (int64_t i = 0; i < d->n_curves; ++i)
        if (d->curve_mat[i] < 0 || d->curve_mat[i] >= d->n_mats) return fail(FTB_ERR_INVALID, "curve material out of range");
    for (int i = 0; i < d->n_emitters; ++i) {
        const ftb_emitter& e = d->emitters[i];
        if (e.shape != FTB_EMIT_QUAD && e.shape != FTB_EMIT_SPHERE)
            return fail(FTB_ERR_UNSUPPORTED, "emitter shape not supported (quad and sphere only)");
        if (e.cdf_n < 1 || e.cdf_offset < 0 || !(e.step > 0.0))
            return fail(FTB_ERR_INVALID, "emitter wavelength CDF malformed");
    }
    for (int i = 0; i < d->n_media; ++i) {
        const ftb_medium& m = d->media[i];
        if (m.sigma_a < 0 || m.sigma_a >= d->n_spectra || m.sigma_s < 0 || m.sigma_s >= d->n_spectra)
            return fail(FTB_ERR_INVALID, "medium spectrum index out of range");
        if (m.bound < FTB_BOUND_NONE || m.bound > FTB_BOUND_SPHERE) return fail(FTB_ERR_INVALID, "bad medium bound");
    }
    std::vector<DevPlane> planes;
    return build_mirror_planes(d, planes);
}

// Affine::inverse (linalg.h:129-144): 3x3 row-major then t; identity when singular.
void affine_inverse(const double* x, double* r) {
    for (int j = 0; j < 12; ++j) r[j] = 0.0;
    r[0] = r[4] = r[8] = 1.0;
    double a = x[0], b = x[1], c = x[2];
    double d = x[3], e = x[4], f = x[5];
    double g = x[6], h = x[7], i = x[8];
    double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    if (std::fabs(det) < 1e-30) return;
    double id = 1.0 / det;
    r[0] = (e * i - f * h) * id; r[1] = (c * h - b * i) * id; r[2] = (b * f - c * e) * id;
    r[3] = (f * g - d * i) * id; r[4] = (a * i - c * g) * id; r[5] = (c * d - a * f) * id;
    r[6] = (d * h - e * g) * id; r[7] = (b * g - a * h) * id; r[8] = (a * e - b * d) * id;
    const double* t = x + 9;
    r[9] = -(r[0] * t[0] + r[1] * t[1] + r[2] * t[2]);
    r[10] = -(r[3] * t[0] + r[4] * t[1] + r[5] * t[2]);
    r[11] = -(r[6] * t[0] + r[7] * t[1] + r[8] * t[2]);
}

// World box of an instance: the 8 corners of its BLAS's local bounds mapped by to_world
// (Scene::collectPrimBoxes, scene.h:2030-2041).
ftb::Box instance_box(const BlasDev& b, const double* xf) {
    ftb::Box w;
    for (int c = 0; c < 8; ++c) {
        double q[3] = {(c & 1) ? b.hi[0] : b.lo[0], (c & 2) ? b.hi[1] : b.lo[1], (c & 4) ? b.hi[2] : b.lo[2]};
        double p[3];
        for (int r = 0; r < 3; ++r) p[r] = xf[3 * r] * q[0] + xf[3 * r + 1] * q[1] + xf[3 * r + 2] * q[2] + xf[9 + r];
        w.grow_point(p);
    }
    return w;
}

double box_maxabs(const ftb::Box& b, double m) {
    for (int a = 0; a < 3; ++a) m = std::max(m, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
    return m;
}

// Bake one BLAS on `device` (current): triangle boxes, wide BVH with a margin from the
// local coordinate magnitude, records in leaf order (prim = the triangle's BLAS index).
ftb_status bake_blas(const ftb_blas_desc& d, int device, ftb::BuildMethod method, std::shared_ptr<BlasDev>& out) {
    auto b = std::make_shared<BlasDev>();
    b->mem.device = device;
    b->n_tris = d.n_tris;
    const int64_t nt = d.n_tris;
    std::vector<ftb::Box> boxes((size_t)nt);
    double maxabs = 1.0;
    const double pad = 1e-6;
    for (int a = 0; a < 3; ++a) { b->lo[a] = DBL_MAX; b->hi[a] = -DBL_MAX; }
    for (int64_t i = 0; i < nt; ++i) {
        const double* v = d.tri_v + 9 * i;
        ftb::Box x;
        for (int k = 0; k < 3; ++k) x.grow_point(v + 3 * k);
        boxes[(size_t)i] = x;
        maxabs = box_maxabs(x, maxabs);
        for (int a = 0; a < 3; ++a) {
            b->lo[a] = std::min(b->lo[a], x.lo[a] - pad);
            b->hi[a] = std::max(b->hi[a], x.hi[a] + pad);
        }
        b->max_mat = std::max(b->max_mat, d.tri_mat[i]);
    }
    ftb::WideBvh bvh;
    std::string err;
    if (!ftb::build_wide_bvh(boxes, std::ldexp(maxabs, -18), bvh, err, method, device))
        return fail(FTB_ERR_INVALID, err);
    if (!ftb::validate_wide_bvh(bvh, (int)nt, err)) return fail(FTB_ERR_INVALID, "BLAS BVH check: " + err);
    std::vector<PrimRec> recs(bvh.order.size());
    bool any_smooth = false;
    for (size_t r = 0; r < bvh.order.size(); ++r) {
        int p = bvh.order[r];
        PrimRec& R = recs[r];
        std::memset(&R, 0, sizeof R);
        std::memcpy(R.d, d.tri_v + 9 * (size_t)p, 9 * sizeof(double));
        R.prim = p;
        int smooth = 0;
        if (d.tri_n)
            for (int k = 0; k < 9; ++k) if (d.tri_n[9 * (size_t)p + k] != 0.0) smooth = 1;
        any_smooth |= smooth != 0;
        R.info = d.tri_mat[p] | (REC_TRI << 24) | (smooth << 30);
    }
    const std::vector<FNode> fn = ftb::widen_nodes(bvh);
    ftb_status st = upload(b->mem, fn.data(), fn.size(), &b->nodes, "upload BLAS nodes");
    if (st == FTB_OK) st = upload(b->mem, recs.data(), recs.size(), &b->recs, "upload BLAS records");
    if (st == FTB_OK && any_smooth) st = upload(b->mem, d.tri_n, (size_t)nt * 9, &b->tri_n, "upload BLAS normals");
    if (st != FTB_OK) return st;
    out = std::move(b);
    return FTB_OK;
}

int default_frac_bits(int64_t n) {
    int lg = 0;
    while (lg < 62 && ((int64_t)1 << lg) < n) ++lg;
    int f = 62 - lg - 20;
    return std::max(4, std::min(40, f));
}

DevCam dev_cam(const ftb_camera* c) {
    DevCam d;
    for (int i = 0; i < 3; ++i) { d.eye[i] = c->eye[i]; d.u[i] = c->u[i]; d.v[i] = c->v[i]; d.w[i] = c->w[i]; }
    d.thx = c->tan_half_x; d.thy = c->tan_half_y; d.rx = c->res_x; d.ry = c->res_y;
    return d;
}

ftb_status ensure_waves(ftb_scene* s, int32_t W, bool log, int32_t hero = 1) {
    if (s->eng->wave_W >= W && s->eng->wave_log == log && s->eng->waves[0].block && s->eng->waves[0].hero >= hero)
        return FTB_OK;
    hero = std::max(hero, s->eng->waves[0].block ? s->eng->waves[0].hero : 1);   // keep the bundle room
    if (s->eng->wave_log == log) W = std::max(W, s->eng->wave_W);
    for (auto& w : s->eng->waves) ftb::wave_free(w);
    for (auto& g : s->eng->graphs) {   // captured graphs hold the old buffers' addresses
        ftb::wave_graphs_destroy(g);
        g = ftb::wave_graphs_create();
    }
    s->eng->wave_W = 0;
    for (auto& w : s->eng->waves) {
        cudaError_t e = ftb::wave_alloc(w, W, log, hero);
        if (e != cudaSuccess) return cuda_fail(e, "wave allocation");
    }
    for (auto& st : s->eng->streams)
        if (!st) CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream create");
    for (auto& sg : s->eng->stage) CK(sg.init(), "job staging");
    s->eng->wave_W = W;
    s->eng->wave_log = log;
    return FTB_OK;
}

ftb_status ensure_frame(ftb_scene* s, size_t words) {
    if (!s->eng->tally) CK(cudaMalloc(&s->eng->tally, 8 * sizeof(unsigned long long)), "tally alloc");
    if (!s->eng->status) CK(cudaMalloc(&s->eng->status, 64), "status alloc");
    if (s->eng->film_words < words) {
        if (s->eng->film) cudaFree(s->eng->film);
        s->eng->film = nullptr;
        s->eng->film_words = 0;
        CK(cudaMalloc(&s->eng->film, words * sizeof(int64_t)), "film alloc");
        s->eng->film_words = words;
    }
    return FTB_OK;
}

int32_t pick_wave(int64_t n, int32_t cap) {
    int64_t W = std::min<int64_t>(n, (int64_t)cap);
    return (int32_t)std::max<int64_t>(W, 1);
}

// Wavelengths a photon of this scene carries for a requested -heroc: clamped to
// [1, kHeroMax], and 1 in scenes with media (main.cpp:11309-11312, hero.h:81-86).
int32_t effective_hero(const ftb_scene* s, int32_t hero_c) {
    if (hero_c <= 1 || s->dev.n_med > 0) return 1;
    return hero_c > ftb::kHeroMax ? ftb::kHeroMax : hero_c;
}

ftb::DevJob make_job(const ftb_scene* s, const ftb_camera* cam, int64_t* d_film, unsigned long long* d_tally,
                     int32_t frac_bits, int32_t max_bounce, int32_t hero_c = 1, int32_t lambda_mode = 0) {
    ftb::DevJob J;
    std::memset(&J, 0, sizeof J);
    J.sc = s->dev;
    J.cam = dev_cam(cam);
    J.film = d_film;
    J.tally = d_tally;
    J.film_scale_inv = std::ldexp(1.0, frac_bits) / s->power;
    J.tally_scale_inv = std::ldexp(1.0, 32) / s->power;
    J.max_bounce = max_bounce;
    J.hero_c = effective_hero(s, hero_c);
    J.lambda_mode = lambda_mode;
    return J;
}

// A piece of a job placed in one wave.
struct Segment { int job; int64_t first; int32_t n; };

// Pack jobs' photon ranges into waves of at most W slots and kWaveJobs segments, launch
// them alternately on the scene's two streams (handing off from and back to `user_stream`).
// `base[j]` is job j's DevJob template; each segment gets its photon0 / slot range.
ftb_status run_jobs(ftb_scene* s, const std::vector<ftb::DevJob>& base, const std::vector<int64_t>& count,
                    const std::vector<uint64_t>& seed, bool log, ftb_photon_log* d_logs, int64_t log_base,
                    cudaStream_t user_stream) {
    int64_t total = 0;
    int32_t hero = 1;
    for (size_t i = 0; i < count.size(); ++i) {
        total += count[i];
        hero = std::max(hero, base[i].hero_c);
    }
    int32_t W = pick_wave(total, s->eng->wave_cap);
    ftb_status st = ensure_waves(s, W, log, hero);   // may keep larger buffers; waves use W slots
    if (st != FTB_OK) return st;
    ftb::Frame f;
    f.stats = s->prof_mode == 2 ? s->stats : nullptr;
    f.status = s->eng->status;
    cudaEvent_t ready = nullptr;
    CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
    CK(cudaEventRecord(ready, user_stream), "event record");
    for (auto st2 : s->eng->streams) CK(cudaStreamWaitEvent(st2, ready, 0), "stream wait");
    size_t j = 0;
    int64_t done_in_job = 0;
    int k = 0;
    std::vector<ftb::DevJob> table;
    // Streaming passes: up to kWaveJobs photon ranges of one class (bundles or not) and one
    // view count, traced with every freed slot refilled, so the device stays full until the
    // pass's last photons.
    while (s->eng->shape.regenerate && j < base.size()) {
        table.clear();
        int64_t g = 0;
        int32_t max_bounce = 0, slots = W;
        bool inst = false, media = false, shapes = false, mirrors = false;
        int bundles = -1, views = -1;
        while (j < base.size() && (int)table.size() < ftb::kWaveJobs) {
            const int64_t left = count[j] - done_in_job;
            if (left <= 0) { ++j; done_in_job = 0; continue; }
            const int is_bundle = base[j].hero_c > 1 ? 1 : 0;
            const int nv = ftb::conn_fanout(base[j]);
            if ((bundles >= 0 && is_bundle != bundles) || (views >= 0 && nv != views)) break;
            bundles = is_bundle;
            views = nv;
            // a path queues at most 2 connections per view (and per mirror) per bounce and a
            // refilled slot one more; the shadow queue holds 3W records, so a fan-out of F
            // connections per vertex gets W / F slots
            slots = std::max(1, W / nv);
            const int64_t m = std::min<int64_t>(left, (int64_t)1 << 30);
            ftb::DevJob J = base[j];
            J.photon0 = seed[j] + (uint64_t)done_in_job;
            J.g0 = g;
            J.slot0 = 0;
            J.n = (int32_t)m;
            table.push_back(J);
            max_bounce = std::max(max_bounce, J.max_bounce);
            inst |= J.sc.n_inst > 0;
            media |= J.sc.n_med > 0;
            shapes |= ftb::scene_has_shapes(J.sc);
            mirrors |= J.sc.n_planes > 0;
            g += m;
            done_in_job += m;
            if (done_in_job >= count[j]) { ++j; done_in_job = 0; }
        }
        if (table.empty()) break;
        slots = (int32_t)std::min<int64_t>(slots, std::max<int64_t>(1, g));
        ftb::Wave& w = s->eng->waves[k & 1];
        cudaStream_t ws = s->eng->streams[k & 1];
        w.logs = d_logs;
        w.log_base = log_base;
        cudaError_t e = s->eng->stage[k & 1].push(table.data(), (int)table.size(), slots, w, ws, g,
                                                  ftb::stream_half_cap(g, slots, max_bounce));
        if (e != cudaSuccess) return cuda_fail(e, "job table upload");
        ftb::WaveKind kind;
        kind.instances = inst;
        kind.bundles = bundles == 1;
        kind.media = media;
        kind.shapes = shapes;
        kind.mirrors = mirrors;
        e = ftb::launch_stream(w, kind, f, s->sms, s->eng->shape, ws, s->prof_mode ? s->prof : nullptr,
                               s->eng->graphs[k & 1]);
        if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
        ++k;
    }
    while (j < base.size()) {
        table.clear();
        int32_t slots = 0, max_bounce = 0;
        bool inst = false, media = false, shapes = false, mirrors = false;
        int bundles = -1;   // a wave holds either one-wavelength jobs or bundles, not both
        // A path queues at most 2 connections per view (and per mirror) per bounce, so a wave
        // of jobs with a fan-out of F connections per vertex carries W / F slots.
        int32_t cap = W;
        while (j < base.size() && slots < cap && (int)table.size() < ftb::kWaveJobs) {
            int64_t left = count[j] - done_in_job;
            if (left <= 0) { ++j; done_in_job = 0; continue; }
            const int is_bundle = base[j].hero_c > 1 ? 1 : 0;
            if (bundles >= 0 && is_bundle != bundles) break;
            const int32_t jcap = std::max(1, W / ftb::conn_fanout(base[j]));
            if (jcap < cap && slots >= jcap) break;   // this job needs a roomier wave of its own
            cap = std::min(cap, jcap);
            bundles = is_bundle;
            int32_t m = (int32_t)std::min<int64_t>(left, (int64_t)(cap - slots));
            ftb::DevJob J = base[j];
            J.photon0 = seed[j] + (uint64_t)done_in_job;
            J.slot0 = slots;
            J.n = m;
            table.push_back(J);
            max_bounce = std::max(max_bounce, J.max_bounce);
            inst |= J.sc.n_inst > 0;
            media |= J.sc.n_med > 0;
            shapes |= ftb::scene_has_shapes(J.sc);
            mirrors |= J.sc.n_planes > 0;
            slots += m;
            done_in_job += m;
            if (done_in_job >= count[j]) { ++j; done_in_job = 0; }
        }
        if (table.empty()) break;
        ftb::Wave& w = s->eng->waves[k & 1];
        cudaStream_t ws = s->eng->streams[k & 1];
        w.logs = d_logs;
        w.log_base = log_base;
        cudaError_t e = s->eng->stage[k & 1].push(table.data(), (int)table.size(), slots, w, ws);
        if (e != cudaSuccess) return cuda_fail(e, "job table upload");
        ftb::WaveKind kind;
        kind.instances = inst;
        kind.bundles = bundles == 1;
        kind.media = media;
        kind.shapes = shapes;
        kind.mirrors = mirrors;
        e = ftb::launch_wave(w, max_bounce, kind, f, s->sms, s->eng->shape, ws, s->prof_mode ? s->prof : nullptr,
                             s->eng->graphs[k & 1]);
        if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
        ++k;
    }
    for (auto st2 : s->eng->streams) {
        CK(cudaEventRecord(ready, st2), "event record");
        CK(cudaStreamWaitEvent(user_stream, ready, 0), "stream wait");
    }
    cudaEventDestroy(ready);
    return FTB_OK;
}

// Trace n photons from seed_base into d_film / tally, on the scene's streams.
ftb_status run_photons(ftb_scene* s, const ftb_camera* cam, int64_t n, uint64_t seed_base, int32_t max_bounce,
                       int32_t frac_bits, int64_t* d_film, unsigned long long* d_tally, ftb_photon_log* d_logs,
                       cudaStream_t user_stream, int32_t hero_c = 1, int32_t lambda_mode = 0) {
    std::vector<ftb::DevJob> base{make_job(s, cam, d_film, d_tally, frac_bits, max_bounce, hero_c, lambda_mode)};
    return run_jobs(s, base, {n}, {seed_base}, d_logs != nullptr, d_logs, (int64_t)seed_base, user_stream);
}

ftb_status read_status(ftb_scene* s) {
    int32_t stv = 0;
    CK(cudaMemcpy(&stv, s->eng->status, 4, cudaMemcpyDeviceToHost), "status readback");
    if (stv) {
        std::string m = "device reported:";
        if (stv & ftb::ST_STACK_OVERFLOW) m += " traversal stack overflow;";
        if (stv & ftb::ST_FILM_SATURATED) m += " film fixed-point saturation (lower frac_bits);";
        if (stv & ftb::ST_MEDIUM_STACK) m += " nested dielectrics deeper than 4;";
        if (stv & ftb::ST_QUEUE_OVERFLOW) m += " shadow queue overflow;";
        if (stv & ftb::ST_LOOP_CAP) m += " streaming pass iteration cap reached with work left;";
        return fail(FTB_ERR_DEVICE_LIMIT, m);
    }
    return FTB_OK;
}

void tally_to_energy(const unsigned long long* fx, double power, ftb_energy* e, bool accumulate) {
    double k = power * std::ldexp(1.0, -32);
    double v[5];
    for (int i = 0; i < 5; ++i) v[i] = (double)(long long)fx[i] * k;
    if (accumulate) {
        e->emitted += v[0]; e->absorbed += v[1]; e->sensor += v[2]; e->escaped += v[3]; e->residual += v[4];
        for (int i = 0; i < 5; ++i) e->fx[i] += (int64_t)fx[i];
    } else {
        e->emitted = v[0]; e->absorbed = v[1]; e->sensor = v[2]; e->escaped = v[3]; e->residual = v[4];
        for (int i = 0; i < 5; ++i) e->fx[i] = (int64_t)fx[i];
    }
}

ftb_status check_params(const ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p) {
    if (!s || !cam || !p) return fail(FTB_ERR_INVALID, "null argument");
    if (cam->res_x <= 0 || cam->res_y <= 0 || (int64_t)cam->res_x * cam->res_y > ((int64_t)1 << 28))
        return fail(FTB_ERR_INVALID, "camera resolution out of range");
    if (p->n_photons < 0) return fail(FTB_ERR_INVALID, "negative photon count");
    if (p->max_bounce < 0 || p->max_bounce > 1024) return fail(FTB_ERR_INVALID, "max_bounce out of range [0, 1024]");
    if (p->frac_bits > 56) return fail(FTB_ERR_INVALID, "frac_bits too large");
    if (p->lambda_mode != FTB_LAMBDA_SPD && p->lambda_mode != FTB_LAMBDA_UNIFORM_380_780)
        return fail(FTB_ERR_INVALID, "unknown lambda_mode");
    if (!(s->power > 0.0)) return fail(FTB_ERR_UNSUPPORTED, "scene emits no power");
    if (s->tables && !s->tables->resident) return fail(FTB_ERR_INVALID, "scene is evicted from the device");
    return FTB_OK;
}

// ---- device residency -------------------------------------------------------------------
// The device pointers of a scene's view, in a fixed order.
constexpr int kDevPtrFields = 12;
void dev_ptr_fields(DevScene& d, const void** (&f)[kDevPtrFields]) {
    f[0] = (const void**)&d.nodes; f[1] = (const void**)&d.recs; f[2] = (const void**)&d.tri_n;
    f[3] = (const void**)&d.spec; f[4] = (const void**)&d.tw; f[5] = (const void**)&d.tv;
    f[6] = (const void**)&d.mats; f[7] = (const void**)&d.emit; f[8] = (const void**)&d.emit_cdf;
    f[9] = (const void**)&d.med; f[10] = (const void**)&d.inst; f[11] = (const void**)&d.planes;
}
// A scene can leave the device when its view reads only its own tables: no instances (their
// TLAS and BLAS assets live elsewhere) and no clones sharing the tables.
bool evictable(const ftb_scene* s) {
    return s->tables && !s->own && s->blas.empty() && s->tables.use_count() == 1 && s->dev.n_inst == 0;
}

// Frees the scene's device tables (host copies are made on the first eviction).  The caller
// guarantees that no render of the scene is in flight.  stream: where pooled allocations are
// freed (stream-ordered); allocations of the scene's bake are freed with cudaFree, which waits
// for the device.  eng->mu held.
ftb_status evict_locked(ftb_scene* s, cudaStream_t stream) {
    DevBlock& b = *s->tables;
    if (!b.resident) return FTB_OK;
    if (!evictable(s)) return fail(FTB_ERR_UNSUPPORTED, "only a scene without instances or clones can be evicted");
    const void** f[kDevPtrFields];
    dev_ptr_fields(s->dev, f);
    std::vector<int> fa(kDevPtrFields, -1);
    for (int i = 0; i < kDevPtrFields; ++i) {
        if (!*f[i]) continue;
        for (size_t k = 0; k < b.ptrs.size(); ++k)
            if (b.ptrs[k] == *f[i]) fa[i] = (int)k;
        if (fa[i] < 0) return fail(FTB_ERR_UNSUPPORTED, "scene view points inside an allocation");
    }
    DeviceGuard guard(s->device);
    if (b.saved.size() != b.ptrs.size()) {
        std::vector<unsigned char*> host(b.ptrs.size(), nullptr);
        cudaError_t e = cudaSuccess;
        for (size_t k = 0; k < b.ptrs.size() && e == cudaSuccess; ++k) {
            e = cudaHostAlloc((void**)&host[k], b.sizes[k], cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaMemcpy(host[k], b.ptrs[k], b.sizes[k], cudaMemcpyDeviceToHost);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (unsigned char* h : host) if (h) cudaFreeHost(h);
            return fail(e == cudaErrorMemoryAllocation ? FTB_ERR_OOM : FTB_ERR_CUDA,
                        std::string("evict copy: ") + cudaGetErrorString(e));
        }
        b.saved = std::move(host);
    }
    b.evicted = b.ptrs;
    for (size_t k = 0; k < b.ptrs.size(); ++k) {
        CK(b.pooled[k] ? cudaFreeAsync(b.ptrs[k], stream) : cudaFree(b.ptrs[k]), "evict free");
        b.ptrs[k] = nullptr;
    }
    for (int i = 0; i < kDevPtrFields; ++i) *f[i] = nullptr;
    s->field_alloc = fa;
    b.resident = false;
    return FTB_OK;
}

// Uploads the tables again (stream-ordered allocations and copies on `stream`; work issued
// to the same stream afterwards, or ordered after it, sees them).  eng->mu held.
ftb_status restore_locked(ftb_scene* s, cudaStream_t stream) {
    DevBlock& b = *s->tables;
    if (b.resident) return FTB_OK;
    DeviceGuard guard(s->device);
    // The emitter table holds device pointers itself (each emitter's wavelength CDF, an
    // allocation of this block): its host copy is re-pointed at the new allocations as they
    // are made, before it is uploaded (allocations are restored in upload order, and the
    // CDFs were uploaded before the table).
    const int emit_alloc = s->field_alloc[7];
    for (size_t k = 0; k < b.ptrs.size(); ++k) {
        if ((int)k == emit_alloc) {
            DevEmit* em = reinterpret_cast<DevEmit*>(b.saved[k]);
            const size_t ne = b.sizes[k] / sizeof(DevEmit);
            for (size_t e = 0; e < ne; ++e)
                for (size_t q = 0; q < k; ++q)
                    if (em[e].cdf && (const void*)em[e].cdf == b.evicted[q]) { em[e].cdf = (const double*)b.ptrs[q]; break; }
        }
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, b.sizes[k], stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(p, b.saved[k], b.sizes[k], cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (p) cudaFreeAsync(p, stream);
            for (size_t q = 0; q < k; ++q) { cudaFreeAsync(b.ptrs[q], stream); b.ptrs[q] = nullptr; }
            return fail(e == cudaErrorMemoryAllocation ? FTB_ERR_OOM : FTB_ERR_CUDA,
                        std::string("restore: ") + cudaGetErrorString(e));
        }
        b.ptrs[k] = p;
        b.pooled[k] = 1;
    }
    const void** f[kDevPtrFields];
    dev_ptr_fields(s->dev, f);
    for (int i = 0; i < kDevPtrFields; ++i)
        if (s->field_alloc[i] >= 0) *f[i] = b.ptrs[(size_t)s->field_alloc[i]];
    b.resident = true;
    return FTB_OK;
}

}  // namespace

// ---- internal accessors (ftb_internal.h) ------------------------------------------------
namespace ftb {
void set_last_error(const std::string& m) { g_err = m; }
int default_frac_bits(int64_t n) { return ::default_frac_bits(n); }
DevCam camera_to_dev(const ftb_camera* c) { return dev_cam(c); }
void energy_from_tally(const unsigned long long* fx, double power, ftb_energy* e) {
    tally_to_energy(fx, power, e, false);
}

ftb_status check_render_params(const ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p) {
    return check_params(s, cam, p);
}
std::mutex& scene_mutex(const ftb_scene* s) { return s->eng->mu; }

ftb_status scene_evict(const ftb_scene* cs, cudaStream_t stream) {
    ftb_scene* s = const_cast<ftb_scene*>(cs);
    std::lock_guard<std::mutex> lk(s->eng->mu);
    return evict_locked(s, stream);
}
ftb_status scene_restore(const ftb_scene* cs, cudaStream_t stream) {
    ftb_scene* s = const_cast<ftb_scene*>(cs);
    std::lock_guard<std::mutex> lk(s->eng->mu);
    return restore_locked(s, stream);
}
bool scene_resident(const ftb_scene* s) {
    std::lock_guard<std::mutex> lk(s->eng->mu);
    return !s->tables || s->tables->resident;
}
bool scene_evictable(const ftb_scene* s) {
    std::lock_guard<std::mutex> lk(s->eng->mu);
    return evictable(s);
}
uint64_t scene_device_bytes(const ftb_scene* s) { return s->scene_bytes; }

bool scene_internals(const ftb_scene* s, DevScene* dev, int* device, int* sms, double* power) {
    if (!s) return false;
    *dev = s->dev;
    *device = s->device;
    *sms = s->sms;
    *power = s->power;
    return true;
}
}  // namespace ftb

// ---- entry points ----------------------------------------------------------------------
extern "C" {

const char* ftb_last_error(void) { return g_err.c_str(); }
int ftb_abi_version(void) { return FTB_ABI_VERSION; }

int ftb_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n > 0 ? 1 : 0;
}

const char* ftb_device_name(void) {
    static char name[256] = "none";
    int n = 0;
    if (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, 0) == cudaSuccess) std::snprintf(name, sizeof name, "%s", p.name);
    } else {
        cudaGetLastError();
    }
    return name;
}

ftb_status ftb_mem_info(size_t* free_b, size_t* total_b) {
    if (!free_b || !total_b) return fail(FTB_ERR_INVALID, "null argument");
    if (!ftb_available()) return fail(FTB_ERR_NO_DEVICE, "no CUDA device");
    CK(cudaMemGetInfo(free_b, total_b), "cudaMemGetInfo");
    return FTB_OK;
}

int ftb_forward_supported(const ftb_scene_desc* desc) {
    ftb_status s = check_desc(desc);
    if (s == FTB_OK) return 1;
    if (s == FTB_ERR_UNSUPPORTED) return 0;
    return -1;
}

ftb_status ftb_camera_look_at(const double eye[3], const double target[3], const double up[3], double fov,
                              int32_t rx, int32_t ry, ftb_camera* out) {
    if (!eye || !target || !up || !out || rx <= 0 || ry <= 0) return fail(FTB_ERR_INVALID, "bad camera arguments");
    // Camera::lookAt (camera.h:110-125)
    V e{eye[0], eye[1], eye[2]};
    V w = vnorm(vsub(V{target[0], target[1], target[2]}, e));
    V u = vnorm(vcross(w, V{up[0], up[1], up[2]}));
    V v = vcross(u, w);
    double thy = std::tan(0.5 * fov * 3.141592653589793 / 180.0);
    double thx = thy * (double)rx / (double)ry;
    std::memset(out, 0, sizeof *out);
    double* dst[4] = {out->eye, out->u, out->v, out->w};
    V src[4] = {e, u, v, w};
    for (int k = 0; k < 4; ++k) { dst[k][0] = src[k].x; dst[k][1] = src[k].y; dst[k][2] = src[k].z; }
    out->tan_half_x = thx;
    out->tan_half_y = thy;
    out->res_x = rx;
    out->res_y = ry;
    return FTB_OK;
}

ftb_status ftb_emission_cdf(const ftb_spectrum* spd, const double* table_w, const double* table_v, double step,
                            double* out_cdf, int32_t out_cap, int32_t* out_n, double* integral) {
    if (!spd || !out_cdf || !out_n || !integral || !(step > 0.0)) return fail(FTB_ERR_INVALID, "bad arguments");
    ftb_scene_desc d{};
    ftb_spectrum one = *spd;
    if (one.kind == FTB_SPEC_TABLE) {
        d.table_w = table_w;
        d.table_v = table_v;
        d.n_table = one.offset + one.n;
    }
    d.spectra = &one;
    d.n_spectra = 1;
    std::string why;
    if (!spec_valid(&d, 0, why)) return fail(FTB_ERR_INVALID, why);
    // EmissionSampler::build (spectrum.h:357-369)
    int n = (int)((kLambdaMax - kLambdaMin) / step);
    if (n < 1 || n + 1 > out_cap) return fail(FTB_ERR_INVALID, "cdf buffer too small");
    for (int i = 0; i <= n; ++i) out_cdf[i] = 0.0;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        double w = kLambdaMin + (i + 0.5) * step;
        double v = spec_eval_host(&d, 0, w);
        acc += std::max(0.0, v) * step;
        out_cdf[i + 1] = acc;
    }
    *integral = acc;
    if (acc > 0) for (int i = 0; i <= n; ++i) out_cdf[i] /= acc;
    *out_n = n;
    return FTB_OK;
}

ftb_status ftb_scene_create(const ftb_scene_desc* d, int32_t device, ftb_scene** out) {
    if (!out) return fail(FTB_ERR_INVALID, "null output");
    *out = nullptr;
    ftb_status st = check_desc(d);
    if (st != FTB_OK) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return fail(FTB_ERR_NO_DEVICE, "no CUDA device"); }
    if (device < 0 || device >= ndev) return fail(FTB_ERR_INVALID, "device index out of range");
    DeviceGuard guard(device);
    auto s = new ftb_scene();
    s->device = device;
    s->tables = std::make_shared<DevBlock>();
    s->tables->device = device;
    s->eng = engine_for(device);
    {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, device) == cudaSuccess) s->sms = p.multiProcessorCount;
    }
    // BLAS assets: shared handles or baked here
    for (int b = 0; b < d->n_blas; ++b) {
        std::shared_ptr<BlasDev> bp;
        if (d->blas[b].handle) {
            bp = d->blas[b].handle->p;
            if (bp->mem.device != device) { delete s; return fail(FTB_ERR_INVALID, "BLAS handle lives on another device"); }
        } else {
            ftb_status bs = bake_blas(d->blas[b], device,
                                      d->build == FTB_BUILD_DEVICE ? ftb::BuildMethod::kDeviceLbvh
                                                                   : ftb::BuildMethod::kHostSah, bp);
            if (bs != FTB_OK) { delete s; return bs; }
        }
        s->blas.push_back(std::move(bp));
    }
    const int64_t nt = d->n_tris, ns = d->n_spheres, nc = d->n_curves, ni = d->n_instances;
    const int64_t np = nt + ns + nc + ni;
    // primitive boxes and the scene's coordinate magnitude (for the traversal margin)
    std::vector<ftb::Box> boxes((size_t)np);
    double maxabs = 1.0;
    auto see = [&](double v) { double a = std::fabs(v); if (a > maxabs) maxabs = a; };
    for (int64_t i = 0; i < nt; ++i) {
        const double* v = d->tri_v + 9 * i;
        ftb::Box b;
        for (int k = 0; k < 3; ++k) { b.grow_point(v + 3 * k); see(v[3 * k]); see(v[3 * k + 1]); see(v[3 * k + 2]); }
        boxes[(size_t)i] = b;
    }
    for (int64_t i = 0; i < ns; ++i) {
        const double* sp = d->sph + 4 * i;
        ftb::Box b;
        for (int a = 0; a < 3; ++a) { b.lo[a] = sp[a] - sp[3]; b.hi[a] = sp[a] + sp[3]; see(b.lo[a]); see(b.hi[a]); }
        boxes[(size_t)(nt + i)] = b;
    }
    for (int64_t i = 0; i < nc; ++i) {
        const double* c = d->curve + 10 * i;
        ftb::Box b;   // curveSegBounds (curve.h:99-104)
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = std::min(c[a] - c[6], c[3 + a] - c[7]);
            b.hi[a] = std::max(c[a] + c[6], c[3 + a] + c[7]);
            see(b.lo[a]); see(b.hi[a]);
        }
        boxes[(size_t)(nt + ns + i)] = b;
    }
    for (int i = 0; i < d->n_emitters; ++i) {
        const ftb_emitter& e = d->emitters[i];
        for (int a = 0; a < 3; ++a) { see(e.origin[a] + std::fabs(e.u[a]) + std::fabs(e.v[a]) + e.radius); }
    }
    // instances: world boxes, world -> local maps (MeshInstance::setToWorld, scene.h:1052-1062)
    TlasHost& T = s->tlas;
    T.base_maxabs = maxabs;
    T.first_inst = nt + ns + nc;
    for (int64_t k = 0; k < ni; ++k) {
        const ftb_instance& in = d->instances[k];
        const BlasDev& B = *s->blas[(size_t)in.blas];
        ftb::Box b = instance_box(B, in.to_world);
        boxes[(size_t)(nt + ns + nc + k)] = b;
        maxabs = box_maxabs(b, maxabs);
        DevInst I;
        std::memset(&I, 0, sizeof I);
        affine_inverse(in.to_world, I.xl);
        I.nodes = B.nodes; I.recs = B.recs; I.tri_n = B.tri_n;
        I.mat_override = in.mat_override;
        T.inst.push_back(I);
        T.inst_blas.push_back(in.blas);
    }
    double margin = std::ldexp(maxabs, -18);
    ftb::WideBvh bvh;
    std::string err;
    const ftb::BuildMethod method = d->build == FTB_BUILD_DEVICE ? ftb::BuildMethod::kDeviceLbvh
                                                                 : ftb::BuildMethod::kHostSah;
    // Scenes with both curves and other primitives (and no instances) get two hierarchies,
    // one over the curves and one over the rest, stored one after the other; a closest-hit
    // or occlusion walk covers both with the shared t bound, so each walk tests one kind of
    // record and the lanes of a warp stay on one code path.
    const int64_t n_other = nt + ns;
    const bool split = nc > 0 && n_other > 0 && ni == 0;
    int32_t root2 = -1;
    if (split) {
        ftb::WideBvh a, b;
        std::vector<ftb::Box> ba(boxes.begin(), boxes.begin() + n_other), bb(boxes.begin() + n_other, boxes.end());
        if (!ftb::build_wide_bvh(ba, margin, a, err, method, device) ||
            !ftb::build_wide_bvh(bb, margin, b, err, method, device)) {
            delete s;
            return fail(FTB_ERR_INVALID, err);
        }
        if (!ftb::validate_wide_bvh(a, (int)n_other, err) || !ftb::validate_wide_bvh(b, (int)nc, err)) {
            delete s;
            return fail(FTB_ERR_INVALID, "BVH check: " + err);
        }
        const uint32_t node_shift = (uint32_t)a.nodes.size(), rec_shift = (uint32_t)a.order.size();
        root2 = (int32_t)node_shift;
        bvh.nodes = std::move(a.nodes);
        bvh.order = std::move(a.order);
        for (WNode nd : b.nodes) {   // child and record indices of the second tree move up
            nd.child_base += node_shift;
            nd.prim_base += rec_shift;
            bvh.nodes.push_back(nd);
        }
        if (a.planes.size() == node_shift * FTB_PLANES && b.planes.size() == b.nodes.size() * FTB_PLANES) {
            bvh.planes = std::move(a.planes);
            bvh.planes.insert(bvh.planes.end(), b.planes.begin(), b.planes.end());
        }
        for (int p : b.order) bvh.order.push_back(p + (int)n_other);
        // Occlusion walks take both trees in one walk: three nodes appended after them, a top
        // node whose two children are copies of the roots (children of a node are
        // consecutive).  Closest-hit walks keep the two separate walks, which measured faster
        // for them; occlusion walks measured faster over the top node.
        if (bvh.planes.size() != bvh.nodes.size() * FTB_PLANES) {   // planes from the decoded bytes
            const std::vector<FNode> dec = ftb::widen_nodes(bvh);
            bvh.planes.resize(dec.size() * FTB_PLANES);
            for (size_t i = 0; i < dec.size(); ++i) {
                std::memcpy(&bvh.planes[i * FTB_PLANES], dec[i].lo, 24 * sizeof(float));
                std::memcpy(&bvh.planes[i * FTB_PLANES + 24], dec[i].hi, 24 * sizeof(float));
            }
        }
        const size_t top = bvh.nodes.size();
        WNode t;
        std::memset(&t, 0, sizeof t);
        t.child_base = (uint32_t)top + 1;
        t.meta[0] = (uint8_t)((1 << 5) | 0);
        t.meta[1] = (uint8_t)((1 << 5) | 1);
        t.imask = 3;
        const WNode ra = bvh.nodes[0], rb = bvh.nodes[node_shift];
        bvh.nodes.push_back(t);
        bvh.nodes.push_back(ra);
        bvh.nodes.push_back(rb);
        std::vector<float> tp(FTB_PLANES);
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 8; ++k) { tp[8 * a + k] = INFINITY; tp[24 + 8 * a + k] = -INFINITY; }
        const size_t roots[2] = {0, node_shift};
        for (int c = 0; c < 2; ++c)
            for (int a = 0; a < 3; ++a)
                for (int k = 0; k < 8; ++k) {   // the root's box: the union of its children's (empty: +inf / -inf)
                    tp[8 * a + c] = std::min(tp[8 * a + c], bvh.planes[roots[c] * FTB_PLANES + 8 * a + k]);
                    tp[24 + 8 * a + c] = std::max(tp[24 + 8 * a + c], bvh.planes[roots[c] * FTB_PLANES + 24 + 8 * a + k]);
                }
        bvh.planes.insert(bvh.planes.end(), tp.begin(), tp.end());
        for (int c = 0; c < 2; ++c) {
            const std::vector<float> copy(bvh.planes.begin() + (ptrdiff_t)(roots[c] * FTB_PLANES),
                                          bvh.planes.begin() + (ptrdiff_t)((roots[c] + 1) * FTB_PLANES));
            bvh.planes.insert(bvh.planes.end(), copy.begin(), copy.end());
        }
    } else {
        if (np > 0 && !ftb::build_wide_bvh(boxes, margin, bvh, err, method, device)) {
            delete s;
            return fail(FTB_ERR_INVALID, err);
        }
        if (np > 0 && !ftb::validate_wide_bvh(bvh, (int)np, err)) { delete s; return fail(FTB_ERR_INVALID, "BVH check: " + err); }
    }
    if (np == 0) {   // an empty root with no children
        bvh.nodes.resize(1);
        bvh.planes.clear();
        std::memset(&bvh.nodes[0], 0, sizeof(WNode));
    }
    // records in leaf order
    std::vector<PrimRec> recs(bvh.order.size());
    bool any_smooth = false;
    for (size_t r = 0; r < bvh.order.size(); ++r) {
        int p = bvh.order[r];
        PrimRec& R = recs[r];
        std::memset(&R, 0, sizeof R);
        R.prim = p;
        int ty, mat, smooth = 0;
        if (p < nt) {
            std::memcpy(R.d, d->tri_v + 9 * (size_t)p, 9 * sizeof(double));
            ty = REC_TRI; mat = d->tri_mat[p];
            if (d->tri_n) {
                const double* n = d->tri_n + 9 * (size_t)p;
                for (int k = 0; k < 9; ++k) if (n[k] != 0.0) smooth = 1;
            }
        } else if (p < nt + ns) {
            std::memcpy(R.d, d->sph + 4 * (size_t)(p - nt), 4 * sizeof(double));
            ty = REC_SPHERE; mat = d->sph_mat[p - nt];
        } else if (p < nt + ns + nc) {
            std::memcpy(R.d, d->curve + 10 * (size_t)(p - nt - ns), 8 * sizeof(double));
            ty = REC_CURVE; mat = d->curve_mat[p - nt - ns];
        } else {
            int64_t k = p - nt - ns - nc;
            std::memcpy(&R.d[0], &k, sizeof k);
            ty = REC_INST; mat = 0;
        }
        any_smooth |= smooth != 0;
        R.info = mat | (ty << 24) | (smooth << 30);
    }
    std::vector<DevSpec> spec((size_t)d->n_spectra);
    for (int i = 0; i < d->n_spectra; ++i) {
        spec[i].kind = d->spectra[i].kind; spec[i].n = d->spectra[i].n; spec[i].offset = d->spectra[i].offset;
        for (int k = 0; k < 6; ++k) spec[i].p[k] = d->spectra[i].p[k];
    }
    std::vector<DevMat> mats((size_t)d->n_mats);
    for (int i = 0; i < d->n_mats; ++i) {
        const ftb_material& m = d->mats[i];
        mats[i] = DevMat{m.type, m.priority, m.reflect, m.ior, m.absorb, m.transmit, m.roughness};
    }
    DevScene& D = s->dev;
    const FNode* dn; const PrimRec* dr;
    const std::vector<FNode> fn = ftb::widen_nodes(bvh);
#define UP(host, n, out, what) do { ftb_status u_ = upload(s, host, n, out, what); if (u_ != FTB_OK) { delete s; return u_; } } while (0)
    UP(recs.data(), recs.size(), &dr, "upload records");
    if (ni > 0) {   // the nodes and the instance table are this scene's own: refits rewrite them
        s->own.reset(new DevBlock());
        s->own->device = device;
        const DevInst* di = nullptr;
        ftb_status us = upload(*s->own, fn.data(), fn.size(), &dn, "upload nodes");
        if (us == FTB_OK) us = upload(*s->own, T.inst.data(), T.inst.size(), &di, "upload instances");
        if (us != FTB_OK) { delete s; return us; }
        s->d_nodes = const_cast<FNode*>(dn);
        s->d_inst = const_cast<DevInst*>(di);
        D.inst = di;
        D.n_inst = ni;
        T.bvh = bvh;
        T.boxes = std::move(boxes);
    } else {
        UP(fn.data(), fn.size(), &dn, "upload nodes");
    }
    D.nodes = dn; D.recs = dr;
    D.root2 = root2;
    if (any_smooth) UP(d->tri_n, (size_t)nt * 9, &D.tri_n, "upload normals");
    UP(spec.data(), spec.size(), &D.spec, "upload spectra");
    UP(d->table_w, (size_t)d->n_table, &D.tw, "upload tables");
    UP(d->table_v, (size_t)d->n_table, &D.tv, "upload tables");
    UP(mats.data(), mats.size(), &D.mats, "upload materials");
    // emitters: wavelength CDFs, then the power CDF (Scene::finalizeEmitters, scene.h:1499-1513)
    std::vector<DevEmit> em((size_t)d->n_emitters);
    std::vector<double> sel((size_t)d->n_emitters);
    double tp = 0.0;
    for (int i = 0; i < d->n_emitters; ++i) {
        const ftb_emitter& e = d->emitters[i];
        const double* cdf_dev = nullptr;
        UP(d->emitter_cdf + e.cdf_offset, (size_t)e.cdf_n + 1, &cdf_dev, "upload emitter cdf");
        DevEmit& o = em[i];
        o.shape = e.shape; o.collimated = e.collimated; o.n = e.cdf_n; o.pad = 0;
        o.step = e.step; o.power = e.power; o.radius = e.radius;
        for (int a = 0; a < 3; ++a) {
            o.origin[a] = e.origin[a]; o.u[a] = e.u[a]; o.v[a] = e.v[a]; o.normal[a] = e.normal[a]; o.beam[a] = e.beam[a];
        }
        o.cdf = cdf_dev;
        tp += e.power;
        sel[i] = tp;
    }
    if (tp > 0) for (auto& c : sel) c /= tp;
    UP(em.data(), em.size(), &D.emit, "upload emitters");
    UP(sel.data(), sel.size(), &D.emit_cdf, "upload emitter cdf");
    std::vector<DevMed> med((size_t)d->n_media);
    for (int i = 0; i < d->n_media; ++i) {
        const ftb_medium& m = d->media[i];
        DevMed& o = med[i];
        o.sa = m.sigma_a; o.ss = m.sigma_s; o.bound = m.bound; o.pad = 0; o.g = m.g; o.radius = m.radius;
        for (int a = 0; a < 3; ++a) { o.bmin[a] = m.bmin[a]; o.bmax[a] = m.bmax[a]; o.center[a] = m.center[a]; }
    }
    UP(med.data(), med.size(), &D.med, "upload media");
    {   // planar mirrors the camera connections reflect in (already validated by check_desc)
        std::vector<DevPlane> planes;
        build_mirror_planes(d, planes);
        UP(planes.data(), planes.size(), &D.planes, "upload mirror planes");
        D.n_planes = (int32_t)planes.size();
    }
#undef UP
    D.n_nodes = (int32_t)bvh.nodes.size();
    D.n_recs = (int32_t)recs.size();
    D.n_mats = d->n_mats;
    D.n_emit = d->n_emitters;
    D.n_med = d->n_media;
    D.n_spec = d->n_spectra;
    D.n_tris = nt;
    D.total_power = tp;
    s->power = tp;
    s->scene_bytes = s->tables->bytes + (s->own ? s->own->bytes : 0);
    for (auto& b : s->blas) s->scene_bytes += b->mem.bytes;
    *out = s;
    return FTB_OK;
}

ftb_status ftb_scene_destroy(ftb_scene* s) {
    delete s;
    return FTB_OK;
}

ftb_status ftb_scene_evict(ftb_scene* s) {
    if (!s) return fail(FTB_ERR_INVALID, "null scene");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    if (!s->tables || !s->tables->resident) return FTB_OK;
    if (!evictable(s)) return fail(FTB_ERR_UNSUPPORTED, "only a scene without instances or clones can be evicted");
    DeviceGuard guard(s->device);
    CK(cudaDeviceSynchronize(), "evict: wait for the device");   // renders of the scene still in flight
    return evict_locked(s, nullptr);
}

ftb_status ftb_scene_restore(ftb_scene* s) {
    if (!s) return fail(FTB_ERR_INVALID, "null scene");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    ftb_status st = restore_locked(s, nullptr);
    if (st != FTB_OK) return st;
    CK(cudaStreamSynchronize(nullptr), "restore");
    return FTB_OK;
}

int ftb_scene_resident(const ftb_scene* s) {
    if (!s) return 0;
    return ftb::scene_resident(s) ? 1 : 0;
}

ftb_status ftb_blas_create(const ftb_blas_desc* d, int32_t device, ftb_blas** out) {
    if (!out || !d) return fail(FTB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->handle) return fail(FTB_ERR_INVALID, "descriptor already names a baked BLAS");
    if (d->n_tris < 1 || d->n_tris > ((int64_t)1 << 29) || !d->tri_v || !d->tri_mat)
        return fail(FTB_ERR_INVALID, "a BLAS needs 1..2^29 triangles");
    for (int64_t i = 0; i < d->n_tris; ++i)
        if (d->tri_mat[i] < 0) return fail(FTB_ERR_INVALID, "negative triangle material");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return fail(FTB_ERR_NO_DEVICE, "no CUDA device"); }
    if (device < 0 || device >= ndev) return fail(FTB_ERR_INVALID, "device index out of range");
    DeviceGuard guard(device);
    std::shared_ptr<BlasDev> b;
    ftb_status st = bake_blas(*d, device, ftb::BuildMethod::kHostSah, b);
    if (st != FTB_OK) return st;
    *out = new ftb_blas{std::move(b)};
    return FTB_OK;
}

ftb_status ftb_blas_destroy(ftb_blas* b) {
    delete b;   // scenes built on it keep their own reference
    return FTB_OK;
}

namespace {
// New world maps for instances [0, n): instance table, boxes, refit of the top level.
ftb_status set_transforms(ftb_scene* s, const double* to_world, int64_t n) {
    TlasHost& T = s->tlas;
    for (int64_t k = 0; k < n; ++k) {
        const double* xf = to_world + 12 * k;
        for (int j = 0; j < 12; ++j)
            if (!std::isfinite(xf[j])) return fail(FTB_ERR_INVALID, "instance transform not finite");
    }
    for (int64_t k = 0; k < n; ++k) {
        const double* xf = to_world + 12 * k;
        affine_inverse(xf, T.inst[(size_t)k].xl);
        T.boxes[(size_t)(T.first_inst + k)] = instance_box(*s->blas[(size_t)T.inst_blas[(size_t)k]], xf);
    }
    double maxabs = T.base_maxabs;
    for (size_t k = 0; k < T.inst.size(); ++k) maxabs = box_maxabs(T.boxes[(size_t)T.first_inst + k], maxabs);
    std::string err;
    if (!ftb::refit_wide_bvh(T.bvh, T.boxes, std::ldexp(maxabs, -18), err)) return fail(FTB_ERR_INVALID, err);
    DeviceGuard guard(s->device);
    const std::vector<FNode> fn = ftb::widen_nodes(T.bvh);
    CK(cudaMemcpy(s->d_nodes, fn.data(), fn.size() * sizeof(FNode), cudaMemcpyHostToDevice), "upload refit nodes");
    CK(cudaMemcpy(s->d_inst, T.inst.data(), T.inst.size() * sizeof(DevInst), cudaMemcpyHostToDevice),
       "upload instances");
    return FTB_OK;
}
}  // namespace

ftb_status ftb_scene_set_instance_transforms(ftb_scene* s, const double* to_world, int64_t n) {
    if (!s) return fail(FTB_ERR_INVALID, "null scene");
    if (n < 0 || n > s->dev.n_inst || (n > 0 && !to_world)) return fail(FTB_ERR_INVALID, "bad instance range");
    if (n == 0) return FTB_OK;
    std::lock_guard<std::mutex> lk(s->eng->mu);
    return set_transforms(s, to_world, n);
}

ftb_status ftb_scene_clone_instances(const ftb_scene* src, const double* to_world, int64_t n, ftb_scene** out) {
    if (!src || !out) return fail(FTB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n < 0 || n > src->dev.n_inst || (n > 0 && !to_world)) return fail(FTB_ERR_INVALID, "bad instance range");
    DeviceGuard guard(src->device);
    auto c = new ftb_scene();
    c->device = src->device;
    c->sms = src->sms;
    c->dev = src->dev;
    c->tables = src->tables;
    c->eng = src->eng;
    c->blas = src->blas;
    c->tlas = src->tlas;
    c->power = src->power;
    if (src->dev.n_inst > 0) {
        c->own.reset(new DevBlock());
        c->own->device = c->device;
        const FNode* dn = nullptr;
        const DevInst* di = nullptr;
        const std::vector<FNode> fn = ftb::widen_nodes(c->tlas.bvh);
        ftb_status st = upload(*c->own, fn.data(), fn.size(), &dn, "upload nodes");
        if (st == FTB_OK) st = upload(*c->own, c->tlas.inst.data(), c->tlas.inst.size(), &di, "upload instances");
        if (st != FTB_OK) { delete c; return st; }
        c->d_nodes = const_cast<FNode*>(dn);
        c->d_inst = const_cast<DevInst*>(di);
        c->dev.nodes = dn;
        c->dev.inst = di;
        if (n > 0) {
            st = set_transforms(c, to_world, n);
            if (st != FTB_OK) { delete c; return st; }
        }
    }
    c->scene_bytes = src->scene_bytes;
    *out = c;
    return FTB_OK;
}

double ftb_scene_power(const ftb_scene* s) { return s ? s->power : 0.0; }

ftb_status ftb_scene_footprint(const ftb_scene* s, int32_t rx, int32_t ry, ftb_footprint* out) {
    if (!s || !out || rx <= 0 || ry <= 0) return fail(FTB_ERR_INVALID, "bad arguments");
    out->scene_bytes = s->scene_bytes;
    out->film_bytes = (uint64_t)rx * (uint64_t)ry * 4 * sizeof(int64_t);
    int32_t W = 1 << 22;
    {
        std::lock_guard<std::mutex> lk(s->eng->mu);
        W = s->eng->wave_cap;   // the device's current tuning
    }
    out->wave_bytes = 2 * (uint64_t)ftb::wave_bytes(W, false);
    out->total_bytes = out->scene_bytes + out->film_bytes + out->wave_bytes;
    return FTB_OK;
}

ftb_status ftb_render_forward_device(ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p,
                                     int64_t* d_film, ftb_film_info* info, ftb_energy* energy, void* stream) {
    ftb_status st = check_params(s, cam, p);
    if (st != FTB_OK) return st;
    if (!d_film) return fail(FTB_ERR_INVALID, "null film");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    int frac = p->frac_bits > 0 ? p->frac_bits : default_frac_bits(p->n_photons);
    st = ensure_frame(s, 0);
    if (st != FTB_OK) return st;
    cudaStream_t us = (cudaStream_t)stream;
    CK(cudaMemsetAsync(s->eng->tally, 0, 8 * sizeof(unsigned long long), us), "memset");
    CK(cudaMemsetAsync(s->eng->status, 0, 64, us), "memset");
    st = run_photons(s, cam, p->n_photons, p->seed_base, p->max_bounce, frac, d_film, s->eng->tally, nullptr, us,
                     p->hero_c, p->lambda_mode);
    if (st != FTB_OK) return st;
    if (info) { info->frac_bits = frac; info->scale = s->power * std::ldexp(1.0, -frac); info->power_ref = s->power; }
    if (energy) {
        CK(cudaStreamSynchronize(us), "sync");
        st = read_status(s);
        if (st != FTB_OK) return st;
        unsigned long long fx[5];
        CK(cudaMemcpy(fx, s->eng->tally, sizeof fx, cudaMemcpyDeviceToHost), "tally readback");
        tally_to_energy(fx, s->power, energy, true);
    }
    return FTB_OK;
}

ftb_status ftb_render_forward(ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p, int64_t* film,
                              ftb_film_info* info, ftb_energy* energy) {
    ftb_status st = check_params(s, cam, p);
    if (st != FTB_OK) return st;
    if (!film) return fail(FTB_ERR_INVALID, "null film");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    size_t words = (size_t)cam->res_x * cam->res_y * 4;
    int frac = p->frac_bits > 0 ? p->frac_bits : default_frac_bits(p->n_photons);
    st = ensure_frame(s, words);
    if (st != FTB_OK) return st;
    CK(cudaMemset(s->eng->film, 0, words * sizeof(int64_t)), "memset film");
    CK(cudaMemset(s->eng->tally, 0, 8 * sizeof(unsigned long long)), "memset tally");
    CK(cudaMemset(s->eng->status, 0, 64), "memset status");
    st = run_photons(s, cam, p->n_photons, p->seed_base, p->max_bounce, frac, s->eng->film, s->eng->tally, nullptr,
                     nullptr, p->hero_c, p->lambda_mode);
    if (st != FTB_OK) return st;
    CK(cudaDeviceSynchronize(), "render");
    st = read_status(s);
    if (st != FTB_OK) return st;
    CK(cudaMemcpy(film, s->eng->film, words * sizeof(int64_t), cudaMemcpyDeviceToHost), "film download");
    if (info) { info->frac_bits = frac; info->scale = s->power * std::ldexp(1.0, -frac); info->power_ref = s->power; }
    if (energy) {
        unsigned long long fx[5];
        CK(cudaMemcpy(fx, s->eng->tally, sizeof fx, cudaMemcpyDeviceToHost), "tally readback");
        tally_to_energy(fx, s->power, energy, true);
    }
    return FTB_OK;
}

ftb_status ftb_render_batch(const ftb_job* jobs, int32_t n, ftb_film_info* infos, ftb_energy* energies,
                            void* stream) {
    if (!jobs || n < 1) return fail(FTB_ERR_INVALID, "empty batch");
    ftb_scene* s = jobs[0].scene;
    if (!s) return fail(FTB_ERR_INVALID, "job 0: null scene");
    for (int j = 0; j < n; ++j) {
        const ftb_job& b = jobs[j];
        if (!b.scene || !b.d_film) return fail(FTB_ERR_INVALID, "job " + std::to_string(j) + ": null scene or film");
        if (b.scene->device != s->device) return fail(FTB_ERR_INVALID, "batch jobs must share one device");
        ftb_render_params p{b.n_photons, b.seed_base, b.max_bounce, b.frac_bits, b.hero_c, b.lambda_mode};
        ftb_status st = check_params(b.scene, &b.cam, &p);
        if (st != FTB_OK) return fail(st, "job " + std::to_string(j) + ": " + g_err);
    }
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    ftb_status st = ensure_frame(s, 0);
    if (st != FTB_OK) return st;
    if (s->eng->batch_cap < (size_t)n) {
        if (s->eng->batch_tally) cudaFree(s->eng->batch_tally);
        s->eng->batch_tally = nullptr;
        s->eng->batch_cap = 0;
        CK(cudaMalloc(&s->eng->batch_tally, sizeof(unsigned long long) * 8 * (size_t)n), "batch tallies");
        s->eng->batch_cap = (size_t)n;
    }
    cudaStream_t us = (cudaStream_t)stream;
    CK(cudaMemsetAsync(s->eng->batch_tally, 0, sizeof(unsigned long long) * 8 * (size_t)n, us), "memset");
    CK(cudaMemsetAsync(s->eng->status, 0, 64, us), "memset");
    std::vector<ftb::DevJob> base;
    std::vector<int64_t> count;
    std::vector<uint64_t> seed;
    for (int j = 0; j < n; ++j) {
        const ftb_job& b = jobs[j];
        int frac = b.frac_bits > 0 ? b.frac_bits : default_frac_bits(b.n_photons);
        base.push_back(make_job(b.scene, &b.cam, b.d_film, s->eng->batch_tally + 8 * (size_t)j, frac, b.max_bounce,
                                b.hero_c, b.lambda_mode));
        count.push_back(b.n_photons);
        seed.push_back(b.seed_base);
        if (infos) {
            infos[j].frac_bits = frac;
            infos[j].scale = b.scene->power * std::ldexp(1.0, -frac);
            infos[j].power_ref = b.scene->power;
        }
    }
    st = run_jobs(s, base, count, seed, false, nullptr, 0, us);
    if (st != FTB_OK) return st;
    if (energies) {
        CK(cudaStreamSynchronize(us), "sync");
        st = read_status(s);
        if (st != FTB_OK) return st;
        std::vector<unsigned long long> fx(8 * (size_t)n);
        CK(cudaMemcpy(fx.data(), s->eng->batch_tally, fx.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
           "tally readback");
        for (int j = 0; j < n; ++j) tally_to_energy(&fx[8 * (size_t)j], jobs[j].scene->power, &energies[j], true);
    }
    return FTB_OK;
}

ftb_status ftb_trace_log(ftb_scene* s, const ftb_camera* cam, const ftb_render_params* p, ftb_photon_log* out) {
    ftb_status st = check_params(s, cam, p);
    if (st != FTB_OK) return st;
    if (!out) return fail(FTB_ERR_INVALID, "null log buffer");
    if (p->n_photons > ((int64_t)1 << 24)) return fail(FTB_ERR_TOO_LARGE, "ftb_trace_log: at most 2^24 photons per call");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    size_t words = (size_t)cam->res_x * cam->res_y * 4;
    int frac = p->frac_bits > 0 ? p->frac_bits : default_frac_bits(p->n_photons);
    st = ensure_frame(s, words);
    if (st != FTB_OK) return st;
    ftb_photon_log* d_logs = nullptr;
    size_t lb = (size_t)std::max<int64_t>(p->n_photons, 1) * sizeof(ftb_photon_log);
    CK(cudaMalloc(&d_logs, lb), "log alloc");
    cudaMemset(s->eng->film, 0, words * sizeof(int64_t));
    cudaMemset(s->eng->tally, 0, 8 * sizeof(unsigned long long));
    cudaMemset(s->eng->status, 0, 64);
    st = run_photons(s, cam, p->n_photons, p->seed_base, p->max_bounce, frac, s->eng->film, s->eng->tally, d_logs,
                     nullptr, p->hero_c, p->lambda_mode);
    if (st == FTB_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) st = cuda_fail(e, "trace_log");
    }
    if (st == FTB_OK) st = read_status(s);
    if (st == FTB_OK) {
        cudaError_t e = cudaMemcpy(out, d_logs, (size_t)p->n_photons * sizeof(ftb_photon_log), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "log download");
    }
    cudaFree(d_logs);
    return st;
}

ftb_status ftb_scene_set_profiling(ftb_scene* s, int32_t mode) {
    if (!s || mode < 0 || mode > 2) return fail(FTB_ERR_INVALID, "bad profiling arguments");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    if (mode && !s->prof) s->prof = new ProfSink();
    if (mode == 2 && !s->stats) {
        CK(cudaMalloc(&s->stats, 8 * sizeof(unsigned long long)), "stats alloc");
        CK(cudaMemset(s->stats, 0, 8 * sizeof(unsigned long long)), "stats memset");
    }
    s->prof_mode = mode;
    return FTB_OK;
}

ftb_status ftb_scene_profile(ftb_scene* s, ftb_kernel_profile* out, int32_t reset) {
    if (!s || !out) return fail(FTB_ERR_INVALID, "bad arguments");
    std::lock_guard<std::mutex> lk(s->eng->mu);
    DeviceGuard guard(s->device);
    std::memset(out, 0, sizeof *out);
    if (s->prof) {
        s->prof->resolve();
        for (int k = 0; k < 4; ++k) { out->ms[k] = s->prof->ms[k]; out->launches[k] = s->prof->launches[k]; }
        if (reset) for (int k = 0; k < 4; ++k) { s->prof->ms[k] = 0; s->prof->launches[k] = 0; }
    }
    if (s->stats) {
        CK(cudaDeviceSynchronize(), "sync");
        unsigned long long c[8];
        CK(cudaMemcpy(c, s->stats, sizeof c, cudaMemcpyDeviceToHost), "stats readback");
        for (int k = 0; k < 8; ++k) out->counters[k] = c[k];
        if (reset) CK(cudaMemset(s->stats, 0, sizeof c), "stats reset");
    }
    return FTB_OK;
}

// ---- sessions ---------------------------------------------------------------------------
ftb_status ftb_get_tuning(int32_t device, ftb_tuning* out) {
    if (!out || device < 0 || device >= 256) return fail(FTB_ERR_INVALID, "bad arguments");
    std::lock_guard<std::mutex> lk(g_engine_mu);
    *out = g_tuning_set[device] ? g_tuning[device] : default_tuning();
    return FTB_OK;
}

ftb_status ftb_set_tuning(int32_t device, const ftb_tuning* t) {
    if (!t || device < 0 || device >= 256) return fail(FTB_ERR_INVALID, "bad arguments");
    if (t->wave_slots < 1 || t->wave_slots > (1 << 24) || t->grid_mult < 1 || t->grid_mult > 64)
        return fail(FTB_ERR_INVALID, "tuning out of range");
    std::shared_ptr<Engine> e;
    {
        std::lock_guard<std::mutex> lk(g_engine_mu);
        g_tuning[device] = *t;
        g_tuning_set[device] = true;
        e = g_engines[device].lock();
    }
    if (e) {
        std::lock_guard<std::mutex> lk(e->mu);
        apply_tuning(*e, *t);
    }
    return FTB_OK;
}

ftb_status ftb_autotune(ftb_scene* s, const ftb_camera* cam, int64_t n, int32_t max_bounce, ftb_tuning* out) {
    ftb_render_params p{n, (uint64_t)1 << 60, max_bounce, 0};
    ftb_status st = check_params(s, cam, &p);
    if (st != FTB_OK) return st;
    if (n < 1) return fail(FTB_ERR_INVALID, "autotune needs photons");
    DeviceGuard guard(s->device);
    int64_t* film = nullptr;
    const size_t words = (size_t)cam->res_x * cam->res_y * 4;
    CK(cudaMalloc(&film, words * sizeof(int64_t)), "autotune film");
    cudaStream_t us = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreate(&a);
    if (ce == cudaSuccess) ce = cudaEventCreate(&b);
    ftb_tuning best;
    ftb_get_tuning(s->device, &best);
    double best_ms = 1e300;
    auto trial = [&](const ftb_tuning& t, double& ms) -> ftb_status {
        ftb_status r = ftb_set_tuning(s->device, &t);
        if (r != FTB_OK) return r;
        float v = 0.f;
        for (int rep = 0; rep < 2; ++rep) {   // the first run warms (allocations, graph capture)
            if (cudaMemsetAsync(film, 0, words * sizeof(int64_t), us) != cudaSuccess) return fail(FTB_ERR_CUDA, "memset");
            if (cudaEventRecord(a, us) != cudaSuccess) return fail(FTB_ERR_CUDA, "event");
            r = ftb_render_forward_device(s, cam, &p, film, nullptr, nullptr, us);
            if (r != FTB_OK) return r;
            if (cudaEventRecord(b, us) != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess)
                return fail(FTB_ERR_CUDA, "event");
            cudaEventElapsedTime(&v, a, b);
        }
        r = read_status(s);
        ms = v;
        return r;
    };
    if (ce == cudaSuccess) {
        // one knob at a time from the current setting: slot refill, grid, wave size, graphs,
        // ray reordering
        const int grids[] = {4, 8, 16, 32};
        const int waves[] = {1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24};
        for (int pass = 0; pass < 5 && st == FTB_OK; ++pass) {
            std::vector<ftb_tuning> cand;
            if (pass == 0) for (int u = 0; u < 2; ++u) { ftb_tuning t = best; t.regenerate = u; cand.push_back(t); }
            if (pass == 1) for (int g : grids) { ftb_tuning t = best; t.grid_mult = g; cand.push_back(t); }
            if (pass == 2) for (int w : waves) { ftb_tuning t = best; t.wave_slots = w; cand.push_back(t); }
            if (pass == 3) for (int u = 0; u < 2; ++u) { ftb_tuning t = best; t.use_graphs = u; cand.push_back(t); }
            if (pass == 4) for (int u = 0; u < 2; ++u) { ftb_tuning t = best; t.sort_rays = u; cand.push_back(t); }
            for (const ftb_tuning& t : cand) {
                double ms = 0;
                st = trial(t, ms);
                if (st != FTB_OK) break;
                if (ms < best_ms) { best_ms = ms; best = t; }
            }
        }
    } else {
        st = cuda_fail(ce, "autotune setup");
    }
    ftb_set_tuning(s->device, &best);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (us) cudaStreamDestroy(us);
    cudaFree(film);
    if (st == FTB_OK && out) *out = best;
    return st;
}

ftb_status ftb_session_begin(ftb_scene* s, const ftb_camera* cams, int32_t n_cams, int32_t max_bounce,
                             int32_t frac_bits, int32_t hero_c, ftb_session** out) {
    if (!s || !cams || n_cams < 1 || n_cams > 65535 || !out) return fail(FTB_ERR_INVALID, "bad session arguments");
    if (max_bounce < 0 || max_bounce > 1024) return fail(FTB_ERR_INVALID, "max_bounce out of range");
    DeviceGuard guard(s->device);
    auto ss = new ftb_session();
    ss->scene = s;
    ss->max_bounce = max_bounce;
    ss->frac_bits = frac_bits > 0 ? frac_bits : default_frac_bits((int64_t)1 << 36);
    ss->hero_c = effective_hero(s, hero_c);
    for (int c = 0; c < n_cams; ++c) {
        if (cams[c].res_x <= 0 || cams[c].res_y <= 0) { delete ss; return fail(FTB_ERR_INVALID, "bad camera"); }
        ss->cams.push_back(cams[c]);
        int64_t* f = nullptr;
        size_t words = (size_t)cams[c].res_x * cams[c].res_y * 4;
        cudaError_t e = cudaMalloc(&f, words * sizeof(int64_t));
        if (e == cudaSuccess) e = cudaMemset(f, 0, words * sizeof(int64_t));
        if (e != cudaSuccess) { for (auto p : ss->films) cudaFree(p); delete ss; return cuda_fail(e, "session film"); }
        ss->films.push_back(f);
    }
    std::vector<ftb::DevView> hv((size_t)n_cams);
    for (int c = 0; c < n_cams; ++c) { hv[c].cam = dev_cam(&cams[c]); hv[c].film = ss->films[c]; }
    cudaError_t e = cudaMalloc(&ss->tally, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(ss->tally, 0, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&ss->views, sizeof(ftb::DevView) * hv.size());
    if (e == cudaSuccess) e = cudaMemcpy(ss->views, hv.data(), sizeof(ftb::DevView) * hv.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        for (auto p : ss->films) cudaFree(p);
        if (ss->tally) cudaFree(ss->tally);
        if (ss->views) cudaFree(ss->views);
        delete ss;
        return cuda_fail(e, "session setup");
    }
    *out = ss;
    return FTB_OK;
}

ftb_status ftb_session_batch(ftb_session* ss, int64_t n, uint64_t seed_base) {
    if (!ss || n < 0) return fail(FTB_ERR_INVALID, "bad batch arguments");
    ftb_scene* s = ss->scene;
    std::lock_guard<std::mutex> lk(s->eng->mu);
    if (s->tables && !s->tables->resident) return fail(FTB_ERR_INVALID, "scene is evicted from the device");
    DeviceGuard guard(s->device);
    ftb_status st = ensure_frame(s, 0);
    if (st != FTB_OK) return st;
    CK(cudaMemset(s->eng->status, 0, 64), "memset status");
    // One shared pass (the multi-camera shared splat, render_cuda.cu:13873-13895): every
    // path vertex connects to each camera; the paths are traced once.
    ftb::DevJob J = make_job(s, &ss->cams[0], ss->films[0], ss->tally, ss->frac_bits, ss->max_bounce, ss->hero_c);
    J.views = ss->views;
    J.n_views = (int32_t)ss->cams.size();
    st = run_jobs(s, {J}, {n}, {seed_base}, false, nullptr, 0, nullptr);
    if (st != FTB_OK) return st;
    CK(cudaDeviceSynchronize(), "session batch");
    return read_status(s);
}

ftb_status ftb_session_hits0(ftb_session* ss, double* hits) {
    if (!ss || !hits) return fail(FTB_ERR_INVALID, "bad arguments");
    DeviceGuard guard(ss->scene->device);
    const ftb_camera& c = ss->cams[0];
    size_t npix = (size_t)c.res_x * c.res_y;
    std::vector<int64_t> buf(npix * 4);
    CK(cudaMemcpy(buf.data(), ss->films[0], buf.size() * sizeof(int64_t), cudaMemcpyDeviceToHost), "hits");
    for (size_t i = 0; i < npix; ++i) hits[i] = (double)buf[4 * i + 3];
    return FTB_OK;
}

ftb_status ftb_session_download(ftb_session* ss, int32_t cam, int64_t* film, ftb_film_info* info, ftb_energy* energy) {
    if (!ss || cam < 0 || cam >= (int32_t)ss->cams.size()) return fail(FTB_ERR_INVALID, "bad arguments");
    DeviceGuard guard(ss->scene->device);
    const ftb_camera& c = ss->cams[cam];
    size_t words = (size_t)c.res_x * c.res_y * 4;
    if (film) CK(cudaMemcpy(film, ss->films[cam], words * sizeof(int64_t), cudaMemcpyDeviceToHost), "download");
    if (info) {
        info->frac_bits = ss->frac_bits;
        info->scale = ss->scene->power * std::ldexp(1.0, -ss->frac_bits);
        info->power_ref = ss->scene->power;
    }
    if (energy) {
        unsigned long long fx[5];
        CK(cudaMemcpy(fx, ss->tally, sizeof fx, cudaMemcpyDeviceToHost), "tally");
        tally_to_energy(fx, ss->scene->power, energy, false);
    }
    return FTB_OK;
}

ftb_status ftb_session_end(ftb_session* ss) {
    if (!ss) return FTB_OK;
    DeviceGuard guard(ss->scene->device);
    for (auto p : ss->films) cudaFree(p);
    if (ss->tally) cudaFree(ss->tally);
    if (ss->views) cudaFree(ss->views);
    delete ss;
    return FTB_OK;
}

}  // extern "C"
