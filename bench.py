"""Benchmark: photon paths/s of the forward pinhole light tracer on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload glass|cornell|fog_strands] [--level 7]

Workload (default): the dispersive-caustics configuration -- the Cornell box holding a
level-7 noise-displaced icosphere (327,680 triangles) of Cauchy glass n = 1.5 + 0.0042/um^2,
1024x1024 film, 2^28 photons per frame, at most 16 bounces; seeded synthetic scene.
A step is one frame: 2^28 photons traced from emission to termination on each GPU
(weak scaling), plus, with N > 1, the frame-end NCCL sum of the int64 films.

Reported (one JSON line on rank 0):
  value        photons / s over the timed steps, device-resident inputs, max over ranks
  e2e          the same through the C ABI call a user makes (ftb_render_forward): host
               film in pinned memory, film download inside every step
  roofline     the dominant kernel's algorithmic bytes / its CUDA-event duration, against
               the measured HBM copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline the reference's own CPU tracer (oracle/_ref, "reference") or the oracle port
               on this host's cores, over a bounded sample of the same workload
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (res, photons per frame, max bounce)
    "glass": (1024, 1 << 28, 16),
    "cornell": (256, 1 << 24, 8),
    "fog_strands": (512, 1 << 26, 32),
}
METRIC = "photon paths/s on 1 B200"
NODE_BYTES = 80     # a node in its compressed form (WNode, 8-bit child planes): the algorithmic
                    # unit, although the device reads the 208-byte widened form (FNode)
NODE_READ_BYTES = 208   # FNode, the node as the kernels read it (the secondary figure)
REC_BYTES = 80      # PrimRec
RAY_IO_BYTES = 64   # extend: queue index 4 + ray 48 read, hit t 8 + record 4 written
SHADOW_IO_BYTES = 140   # shadow: record read (origin 24, direction 24, max 8, XYZ 24, pixel, job,
                        # view 12) + 4 film words of 8 B updated (read + write)


def make_scene(name, level, lib_):
    from goodphotons_b200 import scenes
    if name == "glass":
        return scenes.make_glass(lib_, level=level)
    if name == "cornell":
        return scenes.make_cornell(lib_)
    return scenes.make_fog_strands(lib_)


def lambda_mode(args):
    from goodphotons_b200 import abi
    band = args.lambda_policy == "band" or (args.lambda_policy == "auto" and args.workload == "cornell")
    return abi.LAMBDA_UNIFORM_380_780 if band else abi.LAMBDA_SPD


def workload_config(args):
    res, n, mb = WORKLOADS[args.workload]
    lam = ("uniform over 380-780 nm, power weighted by the SPD pdf (FTB_LAMBDA_UNIFORM_380_780)"
           if lambda_mode(args) else "sampled from the emitter SPD over 360-830 nm")
    cfg = {"workload": args.workload, "film": f"{res}x{res}", "photons_per_frame": n,
           "max_bounce": mb, "seed": 0, "lambda": lam}
    if args.workload == "glass":
        cfg.update(mesh=f"level-{args.level} icosphere r=0.4 m, 3-octave value noise 0.05 m",
                   triangles=20 * 4 ** args.level, ior="Cauchy 1.5 + 0.0042/um^2")
    return cfg, res, n, mb


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if self.index < 0:   # sampling off
            return self
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_ray(workload):
    """dram bytes per closest-hit ray of the extend kernel, from the committed ncu summary
    (profiles/k_extend_<workload>.md, line `dram_bytes_per_ray: <x>`), or None."""
    p = os.path.join(ROOT, "profiles", f"k_extend_{workload}.md")
    try:
        for line in open(p):
            if line.strip().startswith("dram_bytes_per_ray:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def calibrate(run, target_s):
    """Photon count that takes about target_s: double a probe until it runs >= 1 s (so
    thread start-up and film merge costs are amortized), then scale."""
    n = 1 << 13
    while True:
        t = run(n, 1 << 40)
        if t >= 1.0 or n >= (1 << 24):
            return int(max(1 << 13, min(1 << 26, n * target_s / max(t, 1e-3))))
        n *= 2


def cpu_baseline(desc, cam, mb, target_s=12.0):
    """The reference CPU tracer (oracle/_ref) on all host threads, else the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import Oracle, Reference
    threads = os.cpu_count() or 1
    if Reference.available():
        impl, kind = Reference(), "reference"
    else:
        impl, kind = Oracle(), "port"
    ctx = impl.prepare(desc)
    try:
        def run(n, seed):
            t = time.perf_counter()
            impl.trace(desc, cam, n, seed_base=seed, max_bounce=mb, threads=threads, ctx=ctx)
            return time.perf_counter() - t
        n = calibrate(run, target_s)
        t = run(n, 1 << 41)
    finally:
        (impl.L.ftr_release if kind == "reference" else impl.L.fto_release)(ctx)
    return {"value": n / t, "unit": "photon paths/s", "cores": threads, "kind": kind,
            "sample": f"{n} photons of the same scene and film, seed_base 2^41, {t:.1f} s on {threads} threads"}


def run_reference_arm(args):
    """`--impl reference`: the reference's CPU implementation of the path on this host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from goodphotons_b200 import lib, scenes
    cfg, res, _, mb = workload_config(args)
    if lambda_mode(args):   # the reference can only draw from the SPD
        cfg["lambda"] = "sampled from the emitter SPD over 360-830 nm (the reference has no uniform-band policy)"
    L = lib.load()
    desc = make_scene(args.workload, args.level, L)
    cam = scenes.default_camera(L, res)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_bind import Oracle, Reference
    threads = os.cpu_count() or 1
    impl, kind = (Reference(), "reference") if Reference.available() else (Oracle(), "port")
    ctx = impl.prepare(desc)

    def run(count, seed):
        t = time.perf_counter()
        impl.trace(desc, cam, count, seed_base=seed, max_bounce=mb, threads=threads, ctx=ctx)
        return time.perf_counter() - t
    per_step = calibrate(run, 8.0)
    for w in range(args.warmup):
        impl.trace(desc, cam, 1 << 13, seed_base=(1 << 45) + w * (1 << 13), max_bounce=mb, threads=threads, ctx=ctx)
    times = []
    for k in range(args.steps):
        t = time.perf_counter()
        impl.trace(desc, cam, per_step, seed_base=k * per_step, max_bounce=mb, threads=threads, ctx=ctx)
        times.append(time.perf_counter() - t)
    (impl.L.ftr_release if kind == "reference" else impl.L.fto_release)(ctx)
    total = sum(times)
    value = per_step * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "photon paths/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generator)",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "photon paths/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} photons per step (bounded sample of the {cfg['photons_per_frame']}-photon frame)"},
        "e2e": {"value": value, "unit": "photon paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def animation_batch(n_frames, level, warmup, steps, baseline_frames, budget_log2, local, L):
    """Batched animation: frames of the glass scene (one shared BLAS, a refit clone per
    frame) rendered in one ftb_render_batch, against rendering the same frames one at a
    time -- resident clones, and the plain path that bakes every frame as a scene load with
    the build the drop-in shim picks.  Returns the record."""
    import torch
    from goodphotons_b200 import abi, lib, scenes, workloads

    dev = torch.device("cuda", local)
    frames = workloads.animation_frames(n_frames, seed=0, budget_log2=budget_log2)
    blob = scenes.blob_tris(level)
    t = time.perf_counter()
    d0 = scenes.make_glass_instanced(L, level, to_world=frames[0].to_world)
    mat = int(d0.blas_arrays[0][2][0])
    blas = lib.Blas(blob, mat, device=local, lib=L)
    base = lib.Scene(scenes.make_glass_instanced(L, level, handle=blas), local, L)
    blas_ms = 1e3 * (time.perf_counter() - t)
    t = time.perf_counter()
    clones = [base.clone_instances([f.to_world]) for f in frames]
    clone_ms = 1e3 * (time.perf_counter() - t)
    cams = {r: scenes.default_camera(L, r) for r in {f.res for f in frames}}
    films = [torch.zeros((f.res, f.res, 4), dtype=torch.int64, device=dev) for f in frames]
    hosts = [torch.empty((f.res, f.res, 4), dtype=torch.int64, pin_memory=True) for f in frames]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    total = sum(f.photons for f in frames)

    def jobs(scale=1):
        return [dict(scene=c, cam=cams[f.res], d_film=fl.data_ptr(), n=max(1, f.photons // scale),
                     seed_base=f.seed_base, max_bounce=16, frac_bits=0) for c, f, fl in zip(clones, frames, films)]

    t = time.perf_counter()   # autotuner on frame 0 (untimed)
    tuning = L.autotune(clones[0], cams[frames[0].res], 1 << 23, 16)
    tune_s = time.perf_counter() - t
    for w in range(warmup):   # warm-up at 1/16 of every budget (same wave sizes)
        L.render_batch(jobs(16), stream=stream.cuda_stream, want_energy=False)
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local) as clocks:
        for k in range(steps):
            for fl in films:
                fl.zero_()
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            L.render_batch(jobs(), stream=stream.cuda_stream, want_energy=False)
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
    batch_s = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    value = total * steps / batch_s
    # launches of one batch, counted by the profiler on an untimed copy of it (direct
    # launches, the same sequence a graph replay makes; progress kernels as in main())
    clones[0].set_profiling(1)
    clones[0].profile(reset=True)
    L.render_batch(jobs(), stream=stream.cuda_stream, want_energy=False)
    torch.cuda.synchronize(dev)
    pl = clones[0].profile(reset=True).launches
    clones[0].set_profiling(0)
    launches = int(sum(pl)) + (int(pl[1]) + 2 if tuning.regenerate else 0)

    # end to end: per-frame TLAS refit + the batch + every film to pinned host memory
    t = time.perf_counter()
    for c, f in zip(clones, frames):
        c.set_instance_transforms([f.to_world])
    infos, _ = L.render_batch(jobs(), stream=stream.cuda_stream, want_energy=False)
    for fl, h in zip(films, hosts):
        h.copy_(fl, non_blocking=True)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t
    film_bytes = sum(f.res * f.res * 32 for f in frames)

    # one frame at a time on resident clones (device films, CUDA events)
    seq_ev = []
    for c, f, fl in zip(clones, frames, films):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        c.render_device(cams[f.res], f.photons, fl.data_ptr(), seed_base=f.seed_base, max_bounce=16,
                        stream=stream.cuda_stream)
        b.record(stream)
        seq_ev.append((a, b))
    torch.cuda.synchronize(dev)
    seq_s = sum(a.elapsed_time(b) for a, b in seq_ev) / 1e3

    # the plain path: every frame baked from world-space triangles (the shim's build: device
    # LBVH unless the budget exceeds 4096 photons per primitive), rendered, released
    nb = min(baseline_frames, len(frames))
    plain_s, plain_ph = 0.0, 0
    for f in frames[:nb]:
        d = workloads.make_glass_world(L, level, f.to_world, blob=blob)
        host = np.zeros((f.res, f.res, 4), dtype=np.int64)
        t = time.perf_counter()
        sc = lib.Scene(d, local, L, build=abi.BUILD_SAH if f.photons > 4096 * d.n_prims else abi.BUILD_DEVICE)
        sc.render(cams[f.res], f.photons, seed_base=f.seed_base, max_bounce=16, out=host)
        sc.close()
        plain_s += time.perf_counter() - t
        plain_ph += f.photons

    cfg = {"workload": "animation", "frames": len(frames), "mesh": f"level-{level} glass icosphere "
           f"({20 * 4 ** level} triangles) as one shared BLAS, one refit TLAS clone per frame",
           "resolutions": sorted({f.res for f in frames}), "photons_total": total,
           "photon_budgets": f"log-uniform 2^{budget_log2[0]:g}-2^{budget_log2[1]:g} per frame", "max_bounce": 16,
           "transforms": "seeded rotation about a random axis 0-360 deg, translation +-0.2 m",
           "warmup": f"{warmup} batches at 1/16 of every budget",
           "l2": "flushed between timed steps (256 MiB write)", "blas_bake_ms": round(blas_ms, 1),
           "clone_refit_ms_per_frame": round(clone_ms / len(frames), 3),
           "tuning": {"wave_slots": tuning.wave_slots, "grid_blocks_per_sm": tuning.grid_mult,
                      "graph_replay": bool(tuning.use_graphs), "regenerate": bool(tuning.regenerate),
                      "autotune_s": round(tune_s, 2)}}
    line = {
        "metric": "photon paths/s on 1 B200 (batched animation)", "value": value, "unit": "photon paths/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * batch_s / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded scene and transforms)", "config": cfg,
        "e2e": {"value": total / e2e_s, "unit": "photon paths/s",
                "h2d_bytes_per_step": len(frames) * (96 + C.sizeof(abi.Job)),
                "d2h_bytes_per_step": film_bytes,
                "call": "64 x ftb_scene_set_instance_transforms + ftb_render_batch, films to pinned host"},
        "one_at_a_time": {
            "resident_clones": {"value": total / seq_s, "unit": "photon paths/s",
                                "call": "ftb_render_forward_device per frame"},
            "plain_bake_per_frame": {"value": plain_ph / plain_s, "unit": "photon paths/s", "frames": nb,
                                     "call": "ftb_scene_create (the shim's build choice) + "
                                             "ftb_render_forward + destroy per frame"},
        },
        "speedup_e2e_vs_plain": round((total / e2e_s) / (plain_ph / plain_s), 3),
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    for c in clones:
        c.close()
    base.close()
    blas.close()
    return line


def run_animation(args):
    import torch
    from goodphotons_b200 import lib

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    line = animation_batch(args.frames, args.level, args.warmup, args.steps, args.baseline_frames, (22.0, 27.0),
                           local, lib.load())
    print(json.dumps(line), flush=True)


def serve_stream(n_jobs, budget_hi, sizes, library_build, scene_mb, film_mb, max_active, plain_sample, local, L):
    """Served stream on resident scenes through the render server (continuous batching) with
    admission by HBM footprint: the scene library is baked once and held in host memory, the
    server keeps a working set of it on the device within its HBM budget (wave buffers +
    film_mb + scene_mb, films and scenes sharing the last two), evicting idle scenes least
    recently used first.  Poisson
    arrivals at 80% of the capacity the server measured on the same mix.  Against it: every
    job of the same stream rendered one at a time on resident scenes (service times measured,
    latencies of a one-job-at-a-time FIFO server over the same arrivals), and the plain path
    -- bake the job's scene with the build the drop-in shim picks, render, free -- on a
    sample of the jobs.  Returns the record."""
    import torch
    from goodphotons_b200 import abi, lib, scenes, workloads

    probe = workloads.served_jobs(n_jobs, 1.0, seed=0, budget_log2=(20.0, budget_hi), sizes=sizes)
    keys = sorted({(j.family, j.size) for j in probe})
    descs, cache = {}, {}
    t = time.perf_counter()
    for key in keys:
        descs[key] = workloads.job_scene(L, *key)
        cache[key] = lib.Scene(descs[key], local, L, build=library_build)
    library_s = time.perf_counter() - t
    checkpoint("baking the scene library")
    library_bytes = sum(sc.footprint(1, 1).scene_bytes for sc in cache.values())
    cams = {}

    def cam(res):
        if res not in cams:
            cams[res] = scenes.default_camera(L, res)
        return cams[res]

    # deployment step: autotune the device's launch shape on a mid-size glass scene of the mix
    glass = sorted(k for k in keys if k[0] == "glass") or keys
    t = time.perf_counter()
    tuning = L.autotune(cache[glass[len(glass) // 2]], cam(1024), 1 << 26, 16)
    tune_s = time.perf_counter() - t
    checkpoint("the serve autotune")
    film_room = film_mb << 20

    def hbm_budget(srv_waves):
        return srv_waves + film_room + (scene_mb << 20)

    def evict_all():
        for sc in cache.values():
            if sc.resident:
                sc.evict()

    probe_srv = lib.Server(device=local, max_active=max_active, lib=L)
    waves = probe_srv.stats().wave_bytes   # the server's two wave buffers at the device's tuning
    probe_srv.close()
    checkpoint("the probe server")

    def serve(jobs, paced):
        srv = lib.Server(device=local, max_active=max_active, hbm_budget=hbm_budget(waves), lib=L)
        ids, films = [None] * len(jobs), [None] * len(jobs)
        t0 = time.perf_counter()

        def client():
            for i, j in enumerate(jobs):
                if paced:
                    dt = j.arrival_s - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                films[i] = np.empty((j.res, j.res, 4), dtype=np.int64)
                ids[i] = srv.submit(cache[(j.family, j.size)], cam(j.res), j.photons, seed_base=j.seed_base,
                                    max_bounce=j.max_bounce, host_film=films[i])
        th = threading.Thread(target=client)
        th.start()
        res = []
        for i in range(len(jobs)):
            while ids[i] is None:
                time.sleep(0.0005)
            res.append(srv.wait(ids[i]))
            films[i] = None
        th.join()
        st = srv.stats()
        srv.close()
        bad = sum(1 for r in res if r.status != 0)
        makespan = max(r.finish_s for r in res) - min(r.submit_s for r in res)
        lat = np.array([r.finish_s - r.submit_s for r in res])
        return {"res": res, "makespan": makespan, "lat": lat, "stats": st, "failed": bad,
                "budget": hbm_budget(waves), "waves": waves}

    # warm-up, then capacity: the whole mix submitted at once (closed loop); the library
    # starts in host memory each time
    evict_all()
    serve(probe[: min(8, len(probe))], paced=False)
    evict_all()
    cap = serve(probe, paced=False)
    photons = sum(j.photons for j in probe)
    cap_jobs_s = len(probe) / cap["makespan"]
    rate = 0.8 * cap_jobs_s
    jobs = workloads.served_jobs(n_jobs, rate, seed=0, budget_log2=(20.0, budget_hi), sizes=sizes)
    evict_all()
    with ClockSampler(local) as clocks:
        run = serve(jobs, paced=True)
    lat = run["lat"]

    # one job at a time over the same stream, every scene resident: service time of each job
    for sc in cache.values():
        sc.restore()
    service = np.empty(len(jobs))
    for i, j in enumerate(jobs):
        t = time.perf_counter()
        cache[(j.family, j.size)].render(cam(j.res), j.photons, seed_base=j.seed_base, max_bounce=j.max_bounce)
        service[i] = time.perf_counter() - t
    seq_lat = workloads.fifo_latencies([j.arrival_s for j in jobs], service)

    # the plain path on a sample: the drop-in shim's per-call bake (device build unless the
    # budget exceeds 4096 photons per primitive), render, free
    def shim_build(j):
        return abi.BUILD_SAH if j.photons > 4096 * descs[(j.family, j.size)].n_prims else abi.BUILD_DEVICE

    sample = jobs[: min(plain_sample, len(jobs))]
    plain_s = 0.0
    for j in sample:
        t = time.perf_counter()
        sc = lib.Scene(descs[(j.family, j.size)], local, L, build=shim_build(j))
        sc.render(cam(j.res), j.photons, seed_base=j.seed_base, max_bounce=j.max_bounce)
        sc.close()
        plain_s += time.perf_counter() - t
    sample_ph = sum(j.photons for j in sample)
    seq_sample_s = float(service[: len(sample)].sum())
    total_ph = sum(j.photons for j in jobs)
    served_ph_s = total_ph / run["makespan"]
    cap_ph_s = photons / cap["makespan"]
    seq_ph_s = total_ph / float(service.sum())
    plain_ph_s = sample_ph / plain_s
    for s_ in cache.values():
        s_.close()
    st = run["stats"]
    return {
        "value": served_ph_s, "makespan_s": run["makespan"],
        "config": {"jobs": len(jobs), "arrivals": f"Poisson at {rate:.2f} jobs/s (80% of the measured capacity "
                   "on the same mix)",
                   "mix": "scene family uniform over cornell / glass / fog_strands; mesh 1k-2M triangles "
                          f"log-uniform, from a library of {sizes} log-spaced sizes per family (glass: geodesic "
                          "icospheres of 20 f^2 triangles; fog: strands of 4 segments); resolution 128^2-1024^2 "
                          f"and photons 2^20-2^{budget_hi:g} log-uniform",
                   "library": {"scenes": len(cache), "device_bytes": int(library_bytes),
                               "build": "host SAH" if library_build == abi.BUILD_SAH else "device LBVH",
                               "bake_s": round(library_s, 2), "held": "host memory; the server restores and "
                               "evicts scenes on the device within its HBM budget"},
                   "hbm_budget": {"bytes": int(run["budget"]), "wave_buffers": int(run["waves"]),
                                  "films_and_scenes": film_room + (scene_mb << 20)},
                   "max_active": max_active,
                   "tuning": {"wave_slots": tuning.wave_slots, "grid_blocks_per_sm": tuning.grid_mult,
                              "graph_replay": bool(tuning.use_graphs), "sort_rays": bool(tuning.sort_rays),
                              "regenerate": bool(tuning.regenerate), "autotune_s": round(tune_s, 2),
                              "on": f"glass freq {glass[len(glass) // 2][1]}"}},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "mean": float(lat.mean()), "max": float(lat.max())},
        "utilization": round(st.busy_s / run["makespan"], 4),
        "failed_jobs": run["failed"],
        "scene_residency": {"evictions": int(st.evictions), "restores": int(st.restores)},
        "capacity": {"value": cap_ph_s, "unit": "photon paths/s", "jobs_per_s": cap_jobs_s,
                     "how": f"the {len(probe)}-job mix submitted at once"},
        "one_at_a_time": {
            "resident": {"value": seq_ph_s, "unit": "photon paths/s", "jobs": len(jobs),
                         "call": "ftb_render_forward per job, every scene resident",
                         "latency_s": {"p50": float(np.percentile(seq_lat, 50)),
                                       "p99": float(np.percentile(seq_lat, 99)), "max": float(seq_lat.max()),
                                       "how": "FIFO one-job server over the same arrivals, measured service times"}},
            "plain_bake_per_job": {"value": plain_ph_s, "unit": "photon paths/s", "sample_jobs": len(sample),
                                   "resident_same_sample": sample_ph / seq_sample_s,
                                   "call": "ftb_scene_create (the shim's build choice) + ftb_render_forward + "
                                           "destroy per job"},
        },
        "capacity_vs_plain": round(cap_ph_s / plain_ph_s, 3),
        "capacity_vs_resident_one_at_a_time": round(cap_ph_s / seq_ph_s, 3),
        "e2e": {"value": served_ph_s, "unit": "photon paths/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(j.res * j.res * 32 for j in jobs)),
                "call": "ftb_server_submit / ftb_server_wait, films to host"},
        "clocks": clocks.summary(),
    }


def run_serve(args):
    import torch
    from goodphotons_b200 import abi, lib

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    L = lib.load()
    r = serve_stream(args.jobs, float(args.serve_budget_log2), args.serve_sizes, abi.BUILD_SAH, args.serve_scene_mb,
                     args.serve_film_mb, args.max_active, args.serve_sample, local, L)
    cfg = dict(workload="serve", **r.pop("config"))
    line = {"metric": "photon paths/s on 1 B200 (served stream)", "value": r.pop("value"), "unit": "photon paths/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": 1e3 * r.pop("makespan_s"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded job stream and scenes)",
            "config": cfg, "gpu_launches": None, **r}
    print(json.dumps(line), flush=True)


def plain_config(desc, res, n, mb, lam, steps, local, L):
    """One configuration of the plain path (one scene, one film, one frame per step) on a
    resident scene: device-timed frames (CUDA events, L2 flushed between them) and one frame
    end to end through ftb_render_forward with a pinned host film."""
    import torch
    from goodphotons_b200 import lib, scenes

    t = time.perf_counter()
    sc = lib.Scene(desc, local, L)
    bake_ms = 1e3 * (time.perf_counter() - t)
    cam = scenes.default_camera(L, res)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    film = torch.zeros((res, res, 4), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    sc.render_device(cam, n, film.data_ptr(), seed_base=1 << 40, max_bounce=mb, stream=stream.cuda_stream,
                     lambda_mode=lam)   # warm-up
    torch.cuda.synchronize(dev)
    ms = []
    for k in range(steps):
        film.zero_()
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sc.render_device(cam, n, film.data_ptr(), seed_base=k * n, max_bounce=mb, stream=stream.cuda_stream,
                         lambda_mode=lam)
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    host = torch.empty((res, res, 4), dtype=torch.int64, pin_memory=True)
    sc.render(cam, 1 << 20, seed_base=1 << 42, max_bounce=mb, out=host.numpy(), lambda_mode=lam)   # warm-up
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    sc.render(cam, n, seed_base=1 << 41, max_bounce=mb, out=host.numpy(), lambda_mode=lam)
    e2e_s = time.perf_counter() - t
    fp = sc.footprint(res, res)
    sc.close()
    return {"value": n * steps / (sum(ms) / 1e3), "unit": "photon paths/s", "steps": steps,
            "ms_per_step": sum(ms) / steps, "e2e": {"value": n / e2e_s, "unit": "photon paths/s",
                                                     "call": "ftb_render_forward (resident scene, host film)"},
            "bake_ms": round(bake_ms, 1), "scene_bytes": int(fp.scene_bytes)}


def checkpoint(what):
    """A checked device-wide wait between untimed phases: a device fault is reported with the
    phase it followed, not at some later call."""
    import torch
    try:
        torch.cuda.synchronize()
    except RuntimeError as e:
        raise RuntimeError(f"device error after {what}: {e}") from e


def config_records(args, local, L):
    """Compact records of the other configurations, measured after the headline: the
    >= 1M-triangle glass mesh, the Cornell box, fog + strands, a reduced animation batch and a
    reduced served stream (their full forms: --level 8, --workload cornell | fog_strands |
    animation | serve)."""
    from goodphotons_b200 import abi, lib, scenes

    out = {}
    # first use of the device builder loads its kernels (untimed, as in a long-running host)
    lib.Scene(scenes.make_cornell(L), local, L, build=abi.BUILD_DEVICE).close()
    t = time.perf_counter()
    r = plain_config(scenes.make_glass(L, level=8), 1024, 1 << 28, 16, abi.LAMBDA_SPD, 2, local, L)
    r["config"] = {"workload": "glass", "mesh": "level-8 icosphere", "triangles": 20 * 4 ** 8, "film": "1024x1024",
                   "photons_per_frame": 1 << 28, "max_bounce": 16, "lambda": "emitter SPD"}
    out["glass_level8"] = r
    checkpoint("the level-8 glass record")
    r = plain_config(scenes.make_cornell(L), 256, 1 << 24, 8, abi.LAMBDA_UNIFORM_380_780, 3, local, L)
    r["config"] = {"workload": "cornell", "film": "256x256", "photons_per_frame": 1 << 24, "max_bounce": 8,
                   "lambda": "uniform 380-780 nm (FTB_LAMBDA_UNIFORM_380_780)"}
    out["cornell"] = r
    checkpoint("the Cornell record")
    r = plain_config(scenes.make_fog_strands(L), 512, 1 << 26, 32, abi.LAMBDA_SPD, 3, local, L)
    r["config"] = {"workload": "fog_strands", "strands": 250_000, "segments": 1_000_000, "film": "512x512",
                   "photons_per_frame": 1 << 26, "max_bounce": 32, "lambda": "emitter SPD"}
    out["fog_strands"] = r
    checkpoint("the fog + strands record")
    a = animation_batch(16, 7, 3, 2, 16, (22.0, 25.0), local, L)
    out["animation"] = {"value": a["value"], "unit": a["unit"], "ms_per_step": a["ms_per_step"],
                        "e2e": a["e2e"], "one_at_a_time": a["one_at_a_time"],
                        "speedup_e2e_vs_plain": a["speedup_e2e_vs_plain"],
                        "config": {k: a["config"][k] for k in ("frames", "mesh", "resolutions", "photons_total",
                                                               "photon_budgets")},
                        "reduced": "16 frames, budgets 2^22-2^25 (full: --workload animation)"}
    checkpoint("the animation record")
    sv = serve_stream(150, 25.0, 8, abi.BUILD_DEVICE, 512, 512, 64, 20, local, L)
    out["serve"] = {"value": sv["value"], "unit": "photon paths/s", "latency_s": sv["latency_s"],
                    "capacity": sv["capacity"], "one_at_a_time": sv["one_at_a_time"],
                    "capacity_vs_plain": sv["capacity_vs_plain"],
                    "capacity_vs_resident_one_at_a_time": sv["capacity_vs_resident_one_at_a_time"],
                    "scene_residency": sv["scene_residency"], "failed_jobs": sv["failed_jobs"],
                    "config": sv["config"],
                    "reduced": "150 jobs, budgets 2^20-2^25, a library of 8 sizes per family on the device build "
                               "(full: --workload serve)"}
    out["seconds"] = round(time.perf_counter() - t, 1)
    return out


def config_records_child(local, tuning, timeout_s=900):
    """config_records in a child process (its own CUDA context, `--configs-only`, the
    headline's launch tuning), so that a failure there is reported in the record instead of
    ending the headline's run."""
    t = ",".join(str(int(x)) for x in (tuning.wave_slots, tuning.grid_mult, tuning.use_graphs, tuning.sort_rays,
                                       tuning.regenerate))
    cmd = [sys.executable, os.path.abspath(__file__), "--configs-only", "--tuning", t]
    env = dict(os.environ, LOCAL_RANK=str(local))
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, env=env)
    except subprocess.TimeoutExpired:
        return {"error": f"the configuration records did not finish within {timeout_s} s"}
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr or r.stdout).strip().splitlines()[-3:]
        return {"error": f"exit {r.returncode}: " + " | ".join(tail)}
    return json.loads(lines[-1])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="glass", choices=sorted(WORKLOADS) + ["animation", "serve"])
    ap.add_argument("--jobs", type=int, default=2000, help="serve: jobs in the stream")
    ap.add_argument("--serve-budget-log2", type=float, default=28.0, help="serve: largest photon budget, log2")
    ap.add_argument("--serve-sample", type=int, default=40, help="serve: jobs of the plain (bake per job) sample")
    ap.add_argument("--serve-sizes", type=int, default=24, help="serve: library mesh sizes per family")
    ap.add_argument("--serve-scene-mb", type=int, default=512, help="serve: device MiB for resident scenes")
    ap.add_argument("--serve-film-mb", type=int, default=1024, help="serve: device MiB for admitted films")
    ap.add_argument("--max-active", type=int, default=64, help="serve: jobs admitted at once")
    ap.add_argument("--frames", type=int, default=64, help="animation: frames")
    ap.add_argument("--baseline-frames", type=int, default=64, help="animation: frames of the plain baseline")
    ap.add_argument("--level", type=int, default=7)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' records")
    ap.add_argument("--configs-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--photons", type=int, default=0, help="photons per step (default: the workload's frame)")
    ap.add_argument("--tuning", default="",
                    help="wave_slots,blocks_per_sm,graphs[,sort_rays[,regenerate]] instead of the autotuner")
    ap.add_argument("--hero", type=int, default=1, help="wavelengths per photon (hero bundles when > 1)")
    ap.add_argument("--lambda-policy", default="auto", choices=["auto", "spd", "band"],
                    help="wavelength draw: the emitter SPD (the reference's), uniform 380-780 nm, or auto "
                         "(uniform for the Cornell configuration, which specifies it; SPD otherwise)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.configs_only:   # the child of config_records_child
        import torch
        from goodphotons_b200 import lib
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        L = lib.load()
        if args.tuning:
            v = [int(x) for x in args.tuning.split(",")]
            L.set_tuning(local, wave_slots=v[0], grid_mult=v[1], use_graphs=v[2], sort_rays=v[3], regenerate=v[4])
        print(json.dumps(config_records(args, local, L)), flush=True)
        return
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.workload == "animation":
        run_animation(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return

    import torch
    from goodphotons_b200 import abi, lib, multigpu, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    cfg, res, n, mb = workload_config(args)
    if args.photons > 0:
        n = args.photons
        cfg["photons_per_frame"] = n
    cfg["parallelism"] = f"photon-index shards x{world} (weak), NCCL int64 film sum at frame end" if world > 1 else "single GPU"
    if args.hero > 1:
        cfg["wavelengths_per_photon"] = f"{args.hero} (hero bundles)"
    cfg["l2"] = "flushed between timed steps (256 MiB write)"
    L = lib.load()
    desc = make_scene(args.workload, args.level, L)
    lib.Scene(desc, local, L, build=abi.BUILD_DEVICE).close()   # first use loads the builder's kernels
    t = time.perf_counter()
    sc_fast = lib.Scene(desc, local, L, build=abi.BUILD_DEVICE)   # the GPU-built BVH, for comparison
    bake_fast_ms = 1e3 * (time.perf_counter() - t)
    t = time.perf_counter()
    sc = lib.Scene(desc, local, L)
    bake_ms = 1e3 * (time.perf_counter() - t)
    cam = scenes.default_camera(L, res)
    dev = torch.device("cuda", local)
    film = torch.zeros((res, res, 4), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    frac = 0  # default: sized for the photon count

    # counting pass (untimed): traversal work per closest-hit ray and per photon
    sc.set_profiling(2)
    n_count = min(n, 1 << 22)
    lam = lambda_mode(args)
    sc.render_device(cam, n_count, film.data_ptr(), seed_base=1 << 50, max_bounce=mb,
                     stream=stream.cuda_stream, hero_c=args.hero, lambda_mode=lam)
    torch.cuda.synchronize(dev)
    cp = sc.profile(reset=True)
    rays_c, nodes_c, recs_c = cp.counters[0], cp.counters[1], cp.counters[2]
    bytes_per_ray = (nodes_c * NODE_BYTES + recs_c * REC_BYTES) / max(1, rays_c) + RAY_IO_BYTES
    rays_per_photon = rays_c / n_count
    sc.set_profiling(0)

    def step(k):
        film.zero_()
        if dist is None:
            sc.render_device(cam, n, film.data_ptr(), seed_base=k * n, max_bounce=mb, frac_bits=frac,
                             stream=stream.cuda_stream, hero_c=args.hero, lambda_mode=lam)
        else:   # the frame is n photons per rank; each rank traces its index shard
            multigpu.render_sharded(sc, cam, n * world, film, seed_base=k * n * world, max_bounce=mb,
                                    hero_c=args.hero, lambda_mode=lam, dst=0, stream=stream.cuda_stream)

    # autotuner (untimed): grid size, wave size and graph replay for this workload
    t = time.perf_counter()
    if args.tuning:   # a fixed setting instead (reproducible launch sequences for profiling)
        v = [int(x) for x in args.tuning.split(",")]
        v += [0, 1][len(v) - 3:]
        tuning = L.set_tuning(local, wave_slots=v[0], grid_mult=v[1], use_graphs=v[2], sort_rays=v[3],
                              regenerate=v[4])
    else:
        tuning = L.autotune(sc, cam, min(n, 1 << 26), mb)   # (one wavelength per photon)
    cfg["tuning"] = {"wave_slots": tuning.wave_slots, "grid_blocks_per_sm": tuning.grid_mult,
                     "graph_replay": bool(tuning.use_graphs), "sort_rays": bool(tuning.sort_rays),
                     "regenerate": bool(tuning.regenerate),
                     "autotune_s": round(time.perf_counter() - t, 2)}

    for w in range(args.warmup):
        step(1000 + w)
    torch.cuda.synchronize(dev)

    def timed(first_step, clocks_on):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        with ClockSampler(local if clocks_on else -1) as clk:
            torch.cuda.nvtx.range_push("timed")   # ncu --nvtx --nvtx-include "timed/" selects these steps
            for k in range(args.steps):
                flush.fill_(k & 0xff)
                ev[k][0].record(stream)
                step(first_step + k)
                ev[k][1].record(stream)
            torch.cuda.synchronize(dev)
            torch.cuda.nvtx.range_pop()
        if dist is not None:
            dist.barrier()
        return [a.elapsed_time(b) for a, b in ev], clk

    # the timed steps: the product's own launch path (graph replay when tuned so)
    step_ms, clocks = timed(0, True)
    # the same steps again with per-kernel CUDA events (direct launches), for the roofline
    sc.set_profiling(1)
    sc.profile(reset=True)
    prof_ms, _ = timed(args.steps, False)
    prof = sc.profile(reset=True)
    sc.set_profiling(0)
    total_s = sum(step_ms) / 1e3
    if dist is not None:
        tt = torch.tensor([total_s], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_s = float(tt.item())
    photons = n * args.steps * world
    value = photons / total_s

    # roofline of the dominant traversal kernel: closest hit, or the shadow rays' any-hit walk
    # where that takes more of the frame (the Cornell and fog workloads)
    names = ["k_emit", "k_extend", "k_shade", "k_shadow"]
    kms = list(prof.ms)
    dom = int(np.argmax(kms))
    peak, peak_kind = measured_peak()
    traffic_ray = None
    if kms[3] > kms[1]:
        ki, kname = 3, "k_shadow (any-hit traversal of the camera connections + splat)"
        srays_c = max(1, cp.counters[3])
        unit_bytes = (cp.counters[4] * NODE_BYTES + cp.counters[5] * REC_BYTES) / srays_c + SHADOW_IO_BYTES
        read_bytes = unit_bytes + cp.counters[4] * (NODE_READ_BYTES - NODE_BYTES) / srays_c
        units_timed = cp.counters[3] / n_count * n * args.steps
    else:
        ki, kname = 1, "k_extend (closest-hit traversal)"
        unit_bytes = bytes_per_ray
        read_bytes = unit_bytes + nodes_c * (NODE_READ_BYTES - NODE_BYTES) / max(1, rays_c)
        units_timed = rays_per_photon * n * args.steps   # of the profiled steps
        traffic_ray = ncu_traffic_per_ray(args.workload)
    launches_k = max(1, prof.launches[ki])
    bytes_launch = units_timed * unit_bytes / launches_k
    avg_launch_s = kms[ki] / 1e3 / launches_k
    achieved = bytes_launch / avg_launch_s / 1e9
    roofline = {
        "bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
        "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
        "traffic": (round(traffic_ray * units_timed / launches_k) if traffic_ray else None),
        "traffic_source": (f"transcribed, not measured in this run: ncu dram bytes per ray from "
                           f"profiles/k_extend_{args.workload}.md (a smaller capture of the same kernel) "
                           f"x this run's rays per launch" if traffic_ray else None),
        "peak_source": f"{peak_kind} hbm_gbs (copy)",
        "algorithmic_bytes_per_unit": round(unit_bytes, 1),
        "algorithmic_bytes_per_ray": round(bytes_per_ray, 1),
        "node_bytes_counted": f"{NODE_BYTES} per visit (the compressed node; the kernel reads the "
                              f"{NODE_READ_BYTES}-byte widened node, which this figure does not credit)",
        "as_read": {"bytes_per_unit": round(read_bytes, 1),
                    "achieved": round(achieved * read_bytes / unit_bytes, 1),
                    "frac": round(achieved * read_bytes / unit_bytes / peak, 4),
                    "note": f"the same launches with each node visit counted at the {NODE_READ_BYTES} B "
                            "the kernel reads (nodes as laid out on the device); a wider layout raises "
                            "this figure without moving more useful data, so `frac` above is the one "
                            "to compare across layouts"},
        "node_visits_per_ray": round(nodes_c / max(1, rays_c), 3),
        "record_tests_per_ray": round(recs_c / max(1, rays_c), 3),
        "closest_hit_rays_per_photon": round(rays_per_photon, 4),
        "shadow_rays_per_photon": round(cp.counters[3] / n_count, 4),
        "kernel_share": {nm: round(x / max(1e-9, sum(kms)), 4) for nm, x in zip(names, kms)},
        "dominant_kernel": names[dom],
        "kernel_times": "CUDA events on the launching streams over a second set of the same timed steps "
                        f"(direct launches, {sum(prof_ms) / len(prof_ms):.2f} ms per step)",
    }
    # kernels the profiled steps launched: the four traced kernels (counted by the profiler),
    # plus, in streaming passes, the progress kernel after every half-iteration (one per
    # closest-hit launch) and a pass's set-up and first progress launch, and the queue sort
    gpu_launches = int(sum(prof.launches))
    if tuning.regenerate:
        gpu_launches += int(prof.launches[1]) + 2 * args.steps
    if tuning.sort_rays:
        gpu_launches += int(prof.launches[1])

    # the same frame on the GPU-built BVH (device LBVH: faster bake, looser tree)
    fa, fb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    film.zero_()
    fa.record(stream)
    sc_fast.render_device(cam, n, film.data_ptr(), seed_base=(1 << 51), max_bounce=mb, stream=stream.cuda_stream,
                          hero_c=args.hero, lambda_mode=lam)
    fb.record(stream)
    torch.cuda.synchronize(dev)
    device_build = {"bake_ms": round(bake_fast_ms, 1), "bake_ms_host_sah": round(bake_ms, 1),
                    "photons_per_s": n / (fa.elapsed_time(fb) / 1e3)}
    sc_fast.close()

    # end to end through the C ABI call with a pinned host film
    e2e = None
    host = torch.empty((res, res, 4), dtype=torch.int64, pin_memory=True)
    e2e_steps = 0 if args.no_e2e else max(2, min(args.steps, 3))
    host_np = host.numpy()
    if e2e_steps:
        sc.render(cam, 1 << 20, seed_base=1 << 52, max_bounce=mb, out=host_np, lambda_mode=lam)
    torch.cuda.synchronize(dev)
    e_times = []
    for k in range(e2e_steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        sc.render(cam, n, seed_base=(1 << 53) + (k * world + rank) * n, max_bounce=mb, out=host_np, hero_c=args.hero,
                  lambda_mode=lam)
        e_times.append(time.perf_counter() - t)
    e_total = sum(e_times)
    if dist is not None:
        tt = torch.tensor([e_total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e_total = float(tt.item())
    e2e = None if not e2e_steps else {"value": n * e2e_steps * world / e_total, "unit": "photon paths/s",
           "h2d_bytes_per_step": C.sizeof(abi.Camera) + C.sizeof(abi.RenderParams),
           "d2h_bytes_per_step": res * res * 4 * 8 + C.sizeof(abi.Energy),
           "call": "ftb_render_forward (resident scene, host film)", "bake_ms": round(bake_ms, 1)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(desc, cam, mb)
        if cpu and lam:
            cpu["lambda"] = "drawn from the emitter SPD: the reference has no uniform-band policy"

    configs = None
    if rank == 0 and world == 1 and not args.no_configs and args.workload == "glass" and args.hero == 1:
        configs = config_records_child(local, tuning)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "photon paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded scene generator; no dataset)", "config": cfg,
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": gpu_launches,
            "device_bvh_build": device_build,
            "clocks": clocks.summary(),
            "configs": configs,
            "notes": "fp64 path arithmetic (reference order), fp32 conservative BVH culling, int64 fixed-point film",
        }
        print(json.dumps(line), flush=True)
    sc.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
