// ftb_noalloc.cu -- ftb_render_forward_noalloc: a render entry point that allocates no
// device memory.
//
// Who needs it: hosts that own every byte of device memory and forbid allocation inside
// their render callbacks (engine and DCC plug-in hosts with their own allocator), frame
// loops that must not allocate once they are running, and callers for which a cudaMalloc /
// cudaFree would synchronize the device in the middle of their own stream work.  Such a
// caller creates the scene once at start-up and then renders with this entry point, which
// only launches kernels and issues async memsets on the caller's stream.
//
// Its scratch -- the path state, queues and shadow records of one wave of photons, plus the
// energy tallies and the status word -- lives in one file-scope __device__ array of exactly
// FTB_NOALLOC_SCRATCH_BYTES (21,062,912 B, 20.1 MiB, for FTB_NOALLOC_MAX_PHOTONS = 32768
// slots), which every GPU that loads the library holds until the process exits.  Host code
// cannot use the array's name as a device address (it is a host-side stand-in), so the
// first call on each device, with that device current, resolves it with
// cudaGetSymbolAddress; make that first call before any stream capture.
//
// A call issues one staging kernel (the job table, launch parameters, zeroed tallies and
// status word, all passed as kernel arguments) and the wave's kernels on the caller's
// stream; it copies nothing from host memory.  Every call shares the one array and leaves
// its contents behind, so the staging kernel clears what must start at zero, and calls that
// overlap on the GPU race.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ftb200.h"
#include "ftb_internal.h"
#include "ftb_kernels.h"
#include "ftb_layout.h"


namespace {

constexpr int32_t kNoAllocPhotons = 1 << 15;

constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr size_t kWaveBytes = ftb::wave_bytes(kNoAllocPhotons, false);
constexpr size_t kNoAllocBytes = kWaveBytes + al(8 * sizeof(unsigned long long)) + al(64);
static_assert(kNoAllocPhotons == FTB_NOALLOC_MAX_PHOTONS, "photon limit out of step with ftb200.h");
static_assert(kNoAllocBytes == FTB_NOALLOC_SCRATCH_BYTES, "scratch size out of step with ftb200.h");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[256] = {};   // per device, resolved once

ftb_status na_fail(ftb_status s, const std::string& m) {
    ftb::set_last_error(m);
    return s;
}

// Stream-ordered staging of one call: the one-job table and the wave parameters {jobs,
// slots} arrive as kernel arguments (no host memory is read), the five energy tallies and
// the status word are cleared.  One block of 32 threads.
__global__ void k_noalloc_stage(ftb::DevJob job, ftb::DevJob* jobs, int32_t* params, unsigned long long* tally,
                                int32_t* status) {
    const int t = threadIdx.x;
    if (t == 0) {
        jobs[0] = job;
        params[0] = 1;
        params[1] = job.n;
    }
    if (t < 8) tally[t] = 0;
    if (t < 16) status[t] = 0;
}


}  // namespace

extern "C" ftb_status ftb_render_forward_noalloc(ftb_scene* scene, const ftb_camera* cam,
                                                 const ftb_render_params* p, int64_t* d_film,
                                                 ftb_film_info* info, ftb_energy* energy,
                                                 void* stream) {
    DevScene dev;
    int device = 0, sms = 0;
    double power = 0.0;
    if (!d_film) return na_fail(FTB_ERR_INVALID, "null film");
    ftb_status chk = ftb::check_render_params(scene, cam, p);   // the same checks as every render call
    if (chk != FTB_OK) return chk;
    if (!ftb::scene_internals(scene, &dev, &device, &sms, &power)) return na_fail(FTB_ERR_INVALID, "bad scene");
    // Bundles: the scratch holds one wavelength per path, so hero_c > 1 is refused -- except
    // in scenes with media, where every render path traces one wavelength per photon
    // whatever hero_c says (the reference's tracer ignores -heroc there too), so the call
    // goes ahead as hero_c = 1.
    if (p->hero_c > 1 && dev.n_med == 0)
        return na_fail(FTB_ERR_UNSUPPORTED, "ftb_render_forward_noalloc traces one wavelength per photon "
                                            "(its scratch holds no bundles); use hero_c <= 1");
    if (p->n_photons > kNoAllocPhotons)
        return na_fail(FTB_ERR_TOO_LARGE, "ftb_render_forward_noalloc: at most " + std::to_string(kNoAllocPhotons) +
                                              " photons per call (its scratch is a fixed device array); "
                                              "split the render into calls with consecutive seed_base and one "
                                              "explicit frac_bits");
    // a vertex queues one connection per planar mirror besides the camera's: the one wave's
    // connection records fit only if the photons times that fan-out stay within the limit
    if (dev.n_planes > 0 && p->n_photons * (1 + (int64_t)dev.n_planes) > kNoAllocPhotons)
        return na_fail(FTB_ERR_TOO_LARGE, "ftb_render_forward_noalloc: a scene with " + std::to_string(dev.n_planes) +
                                              " mirror planes takes at most " +
                                              std::to_string(kNoAllocPhotons / (1 + dev.n_planes)) +
                                              " photons per call");
    if (device < 0 || device >= 256) return na_fail(FTB_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> scene_lock(ftb::scene_mutex(scene));
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[device]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) {
                if (prev != device) cudaSetDevice(prev);
                return na_fail(FTB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
            g_scratch_addr[device] = ptr;
        }
        base = (char*)g_scratch_addr[device];
    }
    cudaStream_t st = (cudaStream_t)stream;
    ftb::Wave w;
    ftb::wave_carve(w, base, kNoAllocPhotons, false);
    unsigned long long* tally = (unsigned long long*)(base + kWaveBytes);
    int32_t* status = (int32_t*)(base + kWaveBytes + al(8 * sizeof(unsigned long long)));
    const int frac = p->frac_bits > 0 ? p->frac_bits : ftb::default_frac_bits(p->n_photons);
    ftb::Frame f;
    f.stats = nullptr;
    f.status = status;
    ftb::DevJob J;   // the one-job table, passed to the staging kernel by value
    std::memset(&J, 0, sizeof J);
    J.sc = dev;
    for (int i = 0; i < 3; ++i) {
        J.cam.eye[i] = cam->eye[i]; J.cam.u[i] = cam->u[i]; J.cam.v[i] = cam->v[i]; J.cam.w[i] = cam->w[i];
    }
    J.cam.thx = cam->tan_half_x; J.cam.thy = cam->tan_half_y; J.cam.rx = cam->res_x; J.cam.ry = cam->res_y;
    J.film = d_film;
    J.tally = tally;
    J.film_scale_inv = std::ldexp(1.0, frac) / power;
    J.tally_scale_inv = std::ldexp(1.0, 32) / power;
    J.photon0 = p->seed_base;
    J.slot0 = 0;
    J.n = (int32_t)p->n_photons;
    J.max_bounce = p->max_bounce;
    J.lambda_mode = p->lambda_mode;
    ftb_status out = FTB_OK;
    k_noalloc_stage<<<1, 32, 0, st>>>(J, w.jobs, w.params, tally, status);
    cudaError_t e = cudaGetLastError();
    ftb::LaunchShape shape;
    shape.graph = false;
    ftb::WaveKind kind;
    kind.instances = dev.n_inst > 0;
    kind.media = dev.n_med > 0;
    kind.shapes = ftb::scene_has_shapes(dev);
    kind.mirrors = dev.n_planes > 0;
    if (e == cudaSuccess && p->n_photons > 0) e = ftb::launch_wave(w, p->max_bounce, kind, f, sms, shape, st);
    if (e != cudaSuccess) out = na_fail(FTB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (out == FTB_OK && info) {
        info->frac_bits = frac;
        info->scale = power * std::ldexp(1.0, -frac);
        info->power_ref = power;
    }
    if (out == FTB_OK && energy) {
        unsigned long long fx[5] = {0, 0, 0, 0, 0};
        int32_t stv = 0;
        e = cudaMemcpyAsync(fx, tally, sizeof fx, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&stv, status, sizeof stv, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) out = na_fail(FTB_ERR_CUDA, std::string("readback: ") + cudaGetErrorString(e));
        else if (stv) out = na_fail(FTB_ERR_DEVICE_LIMIT, "device reported status " + std::to_string(stv));
        else {
            double k = power * std::ldexp(1.0, -32);
            double v[5];
            for (int i = 0; i < 5; ++i) v[i] = (double)(long long)fx[i] * k;
            energy->emitted += v[0]; energy->absorbed += v[1]; energy->sensor += v[2];
            energy->escaped += v[3]; energy->residual += v[4];
            for (int i = 0; i < 5; ++i) energy->fx[i] += (int64_t)fx[i];
        }
    }
    if (prev != device) cudaSetDevice(prev);
    return out;
}
