// ftb_server.cpp -- resident render server with continuous batching (ftb_server_*, declared
// in include/ftb200.h).
//
// The reference's closest analogue is the resident SharedGpuSession (render_cuda.cu:
// 13763-13871, driven by main.cpp:19036-19236): one scene, fixed cameras, batches submitted
// by one caller.  Here many jobs on many resident scenes share the device:
//
//   submit (any thread) -> queue -> admission (FIFO; film budget and job slots) -> active
//   scheduler thread: packs unscheduled photons of the active jobs of one kernel class into
//                     a streaming pass of up to 4 W photons (W paths in flight; or a wave of
//                     W slots when the device's tuning turns slot refill off) and launches the
//                     passes alternately on two streams / wave buffers; before a buffer is
//                     reused, its previous pass is retired (event sync, status)
//   completion thread: copies a finished job's film and tallies out, frees its film
//
// With an HBM budget the server also owns the residency of its jobs' scenes: admission
// counts the two wave buffers, the admitted films and the resident scenes against the
// budget, evicts idle scenes (least recently used first) to make room and restores a job's
// scene when the job is admitted -- the "scene BVHs kept resident across jobs" of a serving
// loop whose scene library is larger than the device.
//
// Photons are keyed by index (seed_base + i) and the film is int64 fixed point, so how a
// job's photons are split over waves and mixed with other jobs cannot change its result.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ftb200.h"
#include "ftb_internal.h"
#include "ftb_kernels.h"
#include "ftb_layout.h"

namespace {

using Clock = std::chrono::steady_clock;

ftb_status fail(ftb_status s, const std::string& m) {
    ftb::set_last_error(m);
    return s;
}

enum JobState { kQueued = 0, kActive = 1, kFinishing = 2, kDone = 3 };

struct Job {
    uint64_t id = 0;
    ftb_request req{};
    DevScene sc{};              // the scene's device view, read again at admission
    double power = 0.0;
    int frac = 0;
    int hero = 1;               // wavelengths per photon (1 or a bundle)
    int klass = 0;              // kernel variant class: bundles, media, spheres/curves, instances, mirrors
    uint64_t film_bytes = 0;
    int64_t next = 0;           // photons handed to waves so far
    int32_t pending = 0;        // launched waves holding this job's photons, not yet retired
    int64_t* d_film = nullptr;
    int slot = -1;              // tally slot
    JobState state = kQueued;
    ftb_status error = FTB_OK;
    double t_submit = 0, t_admit = 0, t_finish = 0;
    ftb_energy energy{};
};

// A scene used by the server's jobs (HBM budget mode).
struct SceneUse {
    uint64_t bytes = 0;         // device bytes of its tables
    int users = 0;              // admitted jobs that use it
    uint64_t last = 0;          // admission clock of its latest job
    bool evictable = false;
    bool counted = false;       // resident and counted in scene_bytes
};

struct WaveSlot {
    ftb::Wave wave{};
    ftb::WaveGraphs* graphs = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    ftb::DevJob* table = nullptr;   // pinned staging of this buffer's job table
    std::vector<Job*> jobs;         // jobs with photons in the wave in flight
    bool busy = false;
};

}  // namespace

struct ftb_server {
    int device = 0;
    int sms = 148;
    int max_active = 64;
    int32_t W = 1 << 22;
    int32_t hero_max = 4;              // largest bundle the wave buffers hold
    ftb::LaunchShape shape;
    uint64_t budget = 0;               // film budget (no HBM budget)
    uint64_t hbm = 0;                  // HBM budget: waves + films + resident scenes (0: off)
    uint64_t wave_bytes = 0;
    uint64_t scene_bytes = 0;          // resident scenes counted against hbm
    uint64_t use_clock = 0;
    std::map<const ftb_scene*, SceneUse> scenes;
    uint64_t blocked = 0;              // id of the queue's head while it waits for room
    int64_t blocked_wave = 0;          // passes launched when it started waiting
    Clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_fin;
    bool stopping = false;
    bool sched_exited = false;
    std::deque<Job*> queue;
    std::vector<Job*> active;          // admitted, photons left to schedule or in flight
    std::deque<Job*> finishing;        // every wave retired; film and tallies to copy out
    std::map<uint64_t, Job*> jobs;     // live jobs by id
    uint64_t next_id = 1;
    uint64_t film_bytes = 0;
    std::vector<int> free_slots;
    int skipped[32] = {};              // passes since each kernel class was last served
    ftb_server_stats st{};
    int inflight = 0;
    Clock::time_point busy_since;

    WaveSlot ws[2];
    cudaStream_t admit_stream = nullptr, copy_stream = nullptr;
    cudaEvent_t admit_ev = nullptr;
    bool admitted_since_launch = false;
    cudaMemPool_t pool = nullptr;
    unsigned long long* d_tally = nullptr;   // 8 words per slot
    unsigned long long* h_tally = nullptr;   // pinned mirror
    int32_t* d_status = nullptr;             // 16 words per wave buffer
    std::thread sched, completer;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void set_device(ftb_server* s) { cudaSetDevice(s->device); }

// HBM budget mode: make room for job j (its film, and its scene's tables if the scene is
// not on the device) by evicting scenes no admitted job uses, least recently used first;
// then restore j's scene.  false: it does not fit yet (mu held).
// An admitted job takes its scene's device view (re-read at admission: a restore moves the
// tables) and counts as one of the scene's users.
void use_scene_locked(ftb_server* s, Job* j) {
    SceneUse& u = s->scenes[j->req.scene];
    int dev = 0, sms = 0;
    double power = 0.0;
    ftb::scene_internals(j->req.scene, &j->sc, &dev, &sms, &power);
    u.users++;
    u.last = ++s->use_clock;
}

bool fit_locked(ftb_server* s, Job* j) {
    SceneUse& u = s->scenes[j->req.scene];
    const bool resident = ftb::scene_resident(j->req.scene);
    const uint64_t need = j->film_bytes + (resident ? 0 : u.bytes);
    while (s->wave_bytes + s->film_bytes + s->scene_bytes + need > s->hbm) {
        const ftb_scene* victim = nullptr;
        uint64_t oldest = UINT64_MAX;
        for (auto& kv : s->scenes)
            if (kv.first != j->req.scene && kv.second.counted && kv.second.evictable && kv.second.users == 0 &&
                kv.second.last < oldest) {
                victim = kv.first;
                oldest = kv.second.last;
            }
        if (!victim) return false;
        // every job of the victim has retired (users == 0), so the free can be stream-ordered
        if (ftb::scene_evict(victim, s->admit_stream) != FTB_OK) { s->scenes[victim].evictable = false; continue; }
        s->scenes[victim].counted = false;
        s->scene_bytes -= s->scenes[victim].bytes;
        s->st.evictions++;
    }
    if (!resident) {
        if (ftb::scene_restore(j->req.scene, s->admit_stream) != FTB_OK) {
            j->error = FTB_ERR_OOM;
        } else {
            u.counted = true;
            s->scene_bytes += u.bytes;
            s->st.restores++;
            s->admitted_since_launch = true;   // passes wait for the restore (admit_ev)
        }
    }
    use_scene_locked(s, j);
    return true;
}

// Admit queued jobs in arrival order while a slot is free and the film (HBM budget: the
// job's footprint) fits (mu held).
void start_job_locked(ftb_server* s, Job* j);

// With an HBM budget, a job waiting at the head of the queue for room holds back the jobs
// behind it.  Those whose scene is on the device and whose film fits the room left -- no
// eviction, no restore -- are admitted past it, during the two passes after the head began
// to wait; then admission waits for the head, so it is not starved.
void backfill_locked(ftb_server* s) {
    const uint64_t head = s->queue.front()->id;
    if (s->blocked != head) { s->blocked = head; s->blocked_wave = s->st.waves; }
    if (s->st.waves - s->blocked_wave >= 2) return;
    int scanned = 0;
    for (auto it = std::next(s->queue.begin()); it != s->queue.end() && !s->free_slots.empty() && scanned < 256;
         ++scanned) {
        Job* j = *it;
        auto u = s->scenes.find(j->req.scene);
        if (u != s->scenes.end() && u->second.counted &&
            s->wave_bytes + s->film_bytes + s->scene_bytes + j->film_bytes <= s->hbm) {
            it = s->queue.erase(it);
            use_scene_locked(s, j);
            start_job_locked(s, j);
        } else {
            ++it;
        }
    }
}

void admit_locked(ftb_server* s) {
    while (!s->queue.empty() && !s->free_slots.empty()) {
        Job* j = s->queue.front();
        if (s->hbm) {
            if (!fit_locked(s, j)) { backfill_locked(s); break; }
        } else if (s->film_bytes + j->film_bytes > s->budget) {
            break;
        }
        s->queue.pop_front();
        start_job_locked(s, j);
    }
    if (s->admitted_since_launch) cudaEventRecord(s->admit_ev, s->admit_stream);
}

// An admitted job: a slot, a zeroed device film and tallies (stream-ordered on the admission
// stream), and a place among the active jobs.
void start_job_locked(ftb_server* s, Job* j) {
    j->slot = s->free_slots.back();
    s->free_slots.pop_back();
    cudaError_t e = cudaSuccess;
    if (j->req.n_photons > 0 && j->error == FTB_OK) {   // an empty job needs no device film
        void* p = nullptr;
        e = cudaMallocFromPoolAsync(&p, j->film_bytes, s->pool, s->admit_stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, j->film_bytes, s->admit_stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(s->d_tally + 8 * (size_t)j->slot, 0, 8 * sizeof(unsigned long long),
                                s->admit_stream);
        j->d_film = (int64_t*)p;
        s->admitted_since_launch = true;
    }
    j->t_admit = s->now();
    s->film_bytes += j->film_bytes;
    s->st.queued--;
    s->st.active++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (j->d_film) cudaFreeAsync(j->d_film, s->admit_stream);
        j->d_film = nullptr;
        j->error = e == cudaErrorMemoryAllocation ? FTB_ERR_OOM : FTB_ERR_CUDA;
    }
    if (j->error != FTB_OK) j->next = j->req.n_photons;   // nothing to trace
    j->state = kActive;
    if (j->next >= j->req.n_photons) {   // empty or failed: straight to completion
        j->state = kFinishing;
        s->finishing.push_back(j);
        s->cv_fin.notify_one();
    } else {
        s->active.push_back(j);
    }
}

// The table of the next pass (or wave).  Its jobs share one kernel class -- bundles or not,
// media, spheres/curves, instances -- so the pass runs the leanest kernel variants that
// serve them: the class of the job with the least work left, unless another class has
// waited two passes (then the longest-waiting one).  Within the class every job with
// photons left gets min(left, cap / (4 * jobs)) photons, then the remaining capacity goes
// to the jobs with the least work left.  cap = the pass's photon budget (4 W in a
// streaming pass, W in a wave).  One entry per job (mu held).
int64_t build_table_locked(ftb_server* s, std::vector<ftb::DevJob>& table, std::vector<Job*>& members,
                           int32_t& max_bounce, ftb::WaveKind& kind, int& fanout) {
    std::vector<Job*> c;
    for (Job* j : s->active)
        if (j->next < j->req.n_photons) c.push_back(j);
    if (c.empty()) return 0;
    std::stable_sort(c.begin(), c.end(), [](const Job* a, const Job* b) {
        return a->req.n_photons - a->next < b->req.n_photons - b->next;
    });
    bool present[32] = {};
    for (Job* j : c) present[j->klass] = true;
    int klass = c[0]->klass;
    for (int k = 0; k < 32; ++k)
        if (present[k] && s->skipped[k] >= 2 && (klass == c[0]->klass || s->skipped[k] > s->skipped[klass])) klass = k;
    for (int k = 0; k < 32; ++k) s->skipped[k] = (present[k] && k != klass) ? s->skipped[k] + 1 : 0;
    c.erase(std::remove_if(c.begin(), c.end(), [&](const Job* j) { return j->klass != klass; }), c.end());
    if ((int)c.size() > ftb::kWaveJobs) c.resize(ftb::kWaveJobs);
    std::vector<int64_t> give(c.size(), 0);
    const int64_t budget = s->shape.regenerate ? 4 * (int64_t)s->W : (int64_t)s->W;
    int64_t cap = budget;
    const int64_t fair = std::max<int64_t>(1, budget / (4 * (int64_t)c.size()));
    for (size_t i = 0; i < c.size() && cap > 0; ++i) {
        give[i] = std::min<int64_t>({c[i]->req.n_photons - c[i]->next, fair, cap});
        cap -= give[i];
    }
    for (size_t i = 0; i < c.size() && cap > 0; ++i) {
        int64_t more = std::min<int64_t>(c[i]->req.n_photons - c[i]->next - give[i], cap);
        give[i] += more;
        cap -= more;
    }
    int64_t photons = 0;
    max_bounce = 0;
    fanout = 1;
    kind = ftb::WaveKind{};
    for (size_t i = 0; i < c.size(); ++i) {
        if (give[i] <= 0) continue;
        Job* j = c[i];
        ftb::DevJob J;
        std::memset(&J, 0, sizeof J);
        J.sc = j->sc;
        J.cam = ftb::camera_to_dev(&j->req.cam);
        J.film = j->d_film;
        J.tally = s->d_tally + 8 * (size_t)j->slot;
        J.film_scale_inv = std::ldexp(1.0, j->frac) / j->power;
        J.tally_scale_inv = std::ldexp(1.0, 32) / j->power;
        J.photon0 = j->req.seed_base + (uint64_t)j->next;
        J.g0 = photons;                // stream index of a streaming pass
        J.slot0 = (int32_t)photons;    // first slot of a wave
        J.n = (int32_t)give[i];
        J.max_bounce = j->req.max_bounce;
        J.hero_c = j->hero;
        J.lambda_mode = j->req.lambda_mode;
        table.push_back(J);
        members.push_back(j);
        j->next += give[i];
        j->pending++;
        photons += give[i];
        max_bounce = std::max(max_bounce, J.max_bounce);
        kind.bundles |= j->hero > 1;
        kind.instances |= J.sc.n_inst > 0;
        kind.media |= J.sc.n_med > 0;
        kind.shapes |= ftb::scene_has_shapes(J.sc);
        kind.mirrors |= J.sc.n_planes > 0;
        fanout = std::max(fanout, ftb::conn_fanout(J));
    }
    return photons;
}

// Wait for buffer b's wave, read its status word, release its jobs.
void retire(ftb_server* s, int b) {
    WaveSlot& w = s->ws[b];
    if (!w.busy) return;
    cudaError_t e = cudaEventSynchronize(w.done);
    int32_t status = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&status, s->d_status + 16 * b, sizeof status, cudaMemcpyDeviceToHost);
    std::lock_guard<std::mutex> lk(s->mu);
    for (Job* j : w.jobs) {
        if (e != cudaSuccess) j->error = FTB_ERR_CUDA;
        else if (status != 0 && j->error == FTB_OK) j->error = FTB_ERR_DEVICE_LIMIT;
        if (--j->pending == 0 && j->next >= j->req.n_photons) {
            s->active.erase(std::find(s->active.begin(), s->active.end(), j));
            j->state = kFinishing;
            s->finishing.push_back(j);
            s->cv_fin.notify_one();
        }
    }
    w.jobs.clear();
    w.busy = false;
    if (--s->inflight == 0) s->st.busy_s += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
}

void scheduler(ftb_server* s) {
    set_device(s);
    int k = 0;
    std::vector<ftb::DevJob> table;
    std::vector<Job*> members;
    for (;;) {
        table.clear();
        members.clear();
        int64_t photons = 0;
        int32_t mb = 0;
        int fanout = 1;
        ftb::WaveKind kind;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            admit_locked(s);
            photons = build_table_locked(s, table, members, mb, kind, fanout);
            if (photons == 0) {
                bool busy = s->ws[0].busy || s->ws[1].busy;
                if (!busy) {
                    if (s->stopping && s->queue.empty() && s->active.empty()) break;
                    s->cv_sched.wait(lk);
                    continue;
                }
            }
        }
        const int b = k & 1;
        if (photons == 0) {   // nothing new to launch: retire the older wave in flight
            retire(s, s->ws[b].busy ? b : 1 - b);
            continue;
        }
        retire(s, b);   // the buffer's previous wave
        WaveSlot& w = s->ws[b];
        std::memcpy(w.table, table.data(), sizeof(ftb::DevJob) * table.size());
        // streaming pass: {ranges, paths in flight, photons (int64), half-iteration cap (int64)};
        // wave: {jobs, slots}
        const bool stream = s->shape.regenerate;
        // the pass's connection fan-out (planar mirrors) bounds its paths in flight
        const int32_t slots = (int32_t)std::min<int64_t>(photons, std::max(1, s->W / fanout));
        int32_t* par = reinterpret_cast<int32_t*>(w.table + ftb::kWaveJobs);
        par[0] = (int32_t)table.size();
        par[1] = slots;
        reinterpret_cast<int64_t*>(par)[1] = photons;
        reinterpret_cast<int64_t*>(par)[2] = ftb::stream_half_cap(photons, slots, mb);
        cudaError_t e = cudaMemcpyAsync(w.wave.jobs, w.table, sizeof(ftb::DevJob) * table.size(),
                                        cudaMemcpyHostToDevice, w.stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(w.wave.params, par, 6 * sizeof(int32_t), cudaMemcpyHostToDevice, w.stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_status + 16 * b, 0, 64, w.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(w.stream, s->admit_ev, 0);
        ftb::Frame f;
        f.stats = nullptr;
        f.status = s->d_status + 16 * b;
        if (e == cudaSuccess)
            e = stream ? ftb::launch_stream(w.wave, kind, f, s->sms, s->shape, w.stream, nullptr, w.graphs)
                       : ftb::launch_wave(w.wave, mb, kind, f, s->sms, s->shape, w.stream, nullptr, w.graphs);
        if (e == cudaSuccess) e = cudaEventRecord(w.done, w.stream);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->admitted_since_launch = false;
            w.jobs = members;
            w.busy = true;
            if (s->inflight++ == 0) s->busy_since = Clock::now();
            s->st.waves++;
            if (e != cudaSuccess)
                for (Job* j : members) j->error = FTB_ERR_CUDA;
        }
        ++k;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->sched_exited = true;
    s->cv_fin.notify_all();
}

void completer(ftb_server* s) {
    set_device(s);
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_fin.wait(lk, [&] { return !s->finishing.empty() || s->sched_exited; });
            if (s->finishing.empty()) break;
            j = s->finishing.front();
            s->finishing.pop_front();
        }
        cudaError_t e = cudaSuccess;
        const unsigned long long* ht = s->h_tally + 8 * (size_t)j->slot;
        if (j->d_film) {
            if (j->req.host_film && j->error == FTB_OK)
                e = cudaMemcpyAsync(j->req.host_film, j->d_film, j->film_bytes, cudaMemcpyDeviceToHost, s->copy_stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->h_tally + 8 * (size_t)j->slot, s->d_tally + 8 * (size_t)j->slot,
                                    8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->copy_stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
            cudaFreeAsync(j->d_film, s->copy_stream);
            if (e != cudaSuccess && j->error == FTB_OK) j->error = FTB_ERR_CUDA;
        } else if (j->req.host_film && j->error == FTB_OK) {   // empty job: a zero film
            std::memset(j->req.host_film, 0, j->film_bytes);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (j->d_film && j->error == FTB_OK) ftb::energy_from_tally(ht, j->power, &j->energy);
            j->d_film = nullptr;
            s->free_slots.push_back(j->slot);
            s->film_bytes -= j->film_bytes;
            if (s->hbm) s->scenes[j->req.scene].users--;
            s->st.active--;
            if (j->error == FTB_OK) { s->st.completed++; s->st.photons_done += j->req.n_photons; }
            else s->st.failed++;
            j->t_finish = s->now();
            j->state = kDone;
            s->cv_done.notify_all();
            s->cv_sched.notify_one();   // a slot and film budget came free
        }
    }
}

void release(ftb_server* s) {
    set_device(s);
    for (auto& w : s->ws) {
        ftb::wave_graphs_destroy(w.graphs);
        ftb::wave_free(w.wave);
        if (w.stream) cudaStreamDestroy(w.stream);
        if (w.done) cudaEventDestroy(w.done);
        if (w.table) cudaFreeHost(w.table);
    }
    if (s->admit_stream) cudaStreamDestroy(s->admit_stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->admit_ev) cudaEventDestroy(s->admit_ev);
    if (s->d_tally) cudaFree(s->d_tally);
    if (s->h_tally) cudaFreeHost(s->h_tally);
    if (s->d_status) cudaFree(s->d_status);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    for (auto& kv : s->jobs) delete kv.second;
    delete s;
}

}  // namespace

extern "C" {

ftb_status ftb_server_create(const ftb_server_config* cfg, ftb_server** out) {
    if (!cfg || !out) return fail(FTB_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return fail(FTB_ERR_NO_DEVICE, "no CUDA device"); }
    if (cfg->device < 0 || cfg->device >= ndev) return fail(FTB_ERR_INVALID, "device index out of range");
    if (cfg->max_active < 0 || cfg->max_active > ftb::kWaveJobs) return fail(FTB_ERR_INVALID, "max_active out of range");
    if (cfg->wave_slots < 0 || cfg->wave_slots > (1 << 24)) return fail(FTB_ERR_INVALID, "wave_slots out of range");
    int prev = 0;
    cudaGetDevice(&prev);
    auto s = new ftb_server();
    s->device = cfg->device;
    s->max_active = cfg->max_active ? cfg->max_active : 64;
    s->W = cfg->wave_slots ? cfg->wave_slots : (1 << 22);
    s->hero_max = cfg->hero_max > 0 ? (cfg->hero_max > ftb::kHeroMax ? ftb::kHeroMax : cfg->hero_max) : 4;
    {   // launch shape: the device's current tuning (ftb_set_tuning / ftb_autotune)
        ftb_tuning t;
        if (ftb_get_tuning(cfg->device, &t) == FTB_OK) {
            if (!cfg->wave_slots) s->W = t.wave_slots;
            s->shape.grid_mult = t.grid_mult;
            s->shape.graph = t.use_graphs != 0;
            s->shape.sort_rays = t.sort_rays != 0;
            s->shape.regenerate = t.regenerate != 0;
        }
    }
    s->t0 = Clock::now();
    set_device(s);
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, s->device) == cudaSuccess) s->sms = p.multiProcessorCount;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = cfg->film_budget ? cfg->film_budget : free_b / 4;
    s->hbm = cfg->hbm_budget;
    s->wave_bytes = 2 * (uint64_t)ftb::wave_bytes(s->W, false, s->hero_max);
    if (s->hbm && s->wave_bytes >= s->hbm) {
        delete s;
        cudaSetDevice(prev);
        return fail(FTB_ERR_TOO_LARGE, "hbm_budget does not cover the wave buffers");
    }
    auto bad = [&](cudaError_t e, const char* what) {
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        release(s);
        cudaSetDevice(prev);
        return fail(e == cudaErrorMemoryAllocation ? FTB_ERR_OOM : FTB_ERR_CUDA, m);
    };
    cudaError_t e;
    for (auto& w : s->ws) {
        if ((e = ftb::wave_alloc(w.wave, s->W, false, s->hero_max)) != cudaSuccess) return bad(e, "wave allocation");
        if ((e = cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(e, "stream");
        if ((e = cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming)) != cudaSuccess) return bad(e, "event");
        if ((e = cudaHostAlloc((void**)&w.table, sizeof(ftb::DevJob) * (ftb::kWaveJobs + 1), cudaHostAllocDefault)) !=
            cudaSuccess)
            return bad(e, "job table staging");
        w.graphs = ftb::wave_graphs_create();
    }
    if ((e = cudaStreamCreateWithFlags(&s->admit_stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(e, "stream");
    if ((e = cudaEventCreateWithFlags(&s->admit_ev, cudaEventDisableTiming)) != cudaSuccess) return bad(e, "event");
    if ((e = cudaMalloc(&s->d_tally, 8 * sizeof(unsigned long long) * (size_t)s->max_active)) != cudaSuccess)
        return bad(e, "tallies");
    if ((e = cudaHostAlloc((void**)&s->h_tally, 8 * sizeof(unsigned long long) * (size_t)s->max_active,
                           cudaHostAllocDefault)) != cudaSuccess)
        return bad(e, "tallies");
    if ((e = cudaMalloc(&s->d_status, 2 * 64)) != cudaSuccess) return bad(e, "status");
    if ((e = cudaMemset(s->d_status, 0, 2 * 64)) != cudaSuccess) return bad(e, "status");
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof pp);
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = s->device;
    if ((e = cudaMemPoolCreate(&s->pool, &pp)) != cudaSuccess) return bad(e, "film pool");
    // films are recycled without returning memory to the driver (up to what may be admitted)
    uint64_t keep = s->hbm ? std::min<uint64_t>(s->budget, s->hbm - s->wave_bytes) : s->budget;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if ((e = cudaEventRecord(s->admit_ev, s->admit_stream)) != cudaSuccess) return bad(e, "event");
    for (int i = s->max_active - 1; i >= 0; --i) s->free_slots.push_back(i);
    s->sched = std::thread(scheduler, s);
    s->completer = std::thread(completer, s);
    cudaSetDevice(prev);
    *out = s;
    return FTB_OK;
}

ftb_status ftb_server_submit(ftb_server* s, const ftb_request* r, uint64_t* job_id) {
    if (!s || !r || !job_id) return fail(FTB_ERR_INVALID, "null argument");
    auto j = new Job();
    int dev = 0, sms = 0;
    if (!ftb::scene_internals(r->scene, &j->sc, &dev, &sms, &j->power)) { delete j; return fail(FTB_ERR_INVALID, "null scene"); }
    if (dev != s->device) { delete j; return fail(FTB_ERR_INVALID, "scene lives on another device"); }
    const ftb_camera& c = r->cam;
    if (c.res_x <= 0 || c.res_y <= 0 || (int64_t)c.res_x * c.res_y > ((int64_t)1 << 28) || r->n_photons < 0 ||
        r->max_bounce < 0 || r->max_bounce > 1024 || r->frac_bits > 56 ||
        (r->lambda_mode != FTB_LAMBDA_SPD && r->lambda_mode != FTB_LAMBDA_UNIFORM_380_780)) {
        delete j;
        return fail(FTB_ERR_INVALID, "bad request");
    }
    if (!(j->power > 0.0)) { delete j; return fail(FTB_ERR_UNSUPPORTED, "scene emits no power"); }
    j->req = *r;
    j->frac = r->frac_bits > 0 ? r->frac_bits : ftb::default_frac_bits(r->n_photons);
    // bundles as the reference gates them: clamped to kHeroMax, none in scenes with media
    j->hero = (r->hero_c <= 1 || j->sc.n_med > 0) ? 1 : (r->hero_c > ftb::kHeroMax ? ftb::kHeroMax : r->hero_c);
    j->klass = (j->hero > 1 ? 1 : 0) | (j->sc.n_med > 0 ? 2 : 0) | (ftb::scene_has_shapes(j->sc) ? 4 : 0) |
               (j->sc.n_inst > 0 ? 8 : 0) | (j->sc.n_planes > 0 ? 16 : 0);
    if (j->hero > s->hero_max) {
        delete j;
        return fail(FTB_ERR_TOO_LARGE, "bundle larger than the server's hero_max");
    }
    j->film_bytes = (uint64_t)c.res_x * (uint64_t)c.res_y * 4 * sizeof(int64_t);
    if (!s->hbm && j->film_bytes > s->budget) {
        delete j;
        return fail(FTB_ERR_TOO_LARGE, "film exceeds the server's film budget");
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) { delete j; return fail(FTB_ERR_INVALID, "server is stopping"); }
    if (s->hbm) {   // the footprint: waves + film + the scene's tables
        auto it = s->scenes.find(r->scene);
        const uint64_t sb = it != s->scenes.end() ? it->second.bytes : ftb::scene_device_bytes(r->scene);
        if (s->wave_bytes + j->film_bytes + sb > s->hbm) {
            delete j;
            return fail(FTB_ERR_TOO_LARGE, "job footprint (waves + film + scene) exceeds the server's hbm_budget");
        }
        if (it == s->scenes.end()) {
            SceneUse u;
            u.bytes = sb;
            u.evictable = ftb::scene_evictable(r->scene);
            u.counted = ftb::scene_resident(r->scene);
            if (u.counted) s->scene_bytes += sb;
            s->scenes[r->scene] = u;
        }
    }
    j->id = s->next_id++;
    j->t_submit = s->now();
    s->jobs[j->id] = j;
    s->queue.push_back(j);
    s->st.submitted++;
    s->st.queued++;
    s->cv_sched.notify_one();
    *job_id = j->id;
    return FTB_OK;
}

ftb_status ftb_server_wait(ftb_server* s, uint64_t id, double timeout_s, ftb_job_result* out) {
    if (!s || !out) return fail(FTB_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(FTB_ERR_INVALID, "unknown job id");
    Job* j = it->second;
    auto done = [&] { return j->state == kDone; };
    if (timeout_s < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
        return fail(FTB_ERR_TIMEOUT, "job still running");
    std::memset(out, 0, sizeof *out);
    out->status = j->error;
    out->info.frac_bits = j->frac;
    out->info.scale = j->power * std::ldexp(1.0, -j->frac);
    out->info.power_ref = j->power;
    out->energy = j->energy;
    out->submit_s = j->t_submit;
    out->admit_s = j->t_admit;
    out->finish_s = j->t_finish;
    s->jobs.erase(it);
    delete j;
    return FTB_OK;
}

ftb_status ftb_server_get_stats(ftb_server* s, ftb_server_stats* out) {
    if (!s || !out) return fail(FTB_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->film_bytes = s->film_bytes;
    out->scene_bytes = s->scene_bytes;
    out->wave_bytes = s->wave_bytes;
    if (s->inflight > 0) out->busy_s += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
    return FTB_OK;
}

ftb_status ftb_server_destroy(ftb_server* s) {
    if (!s) return FTB_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_sched.notify_all();
    }
    s->sched.join();
    s->completer.join();
    release(s);
    return FTB_OK;
}

}  // extern "C"
