"""Loader and thin Python wrappers over the C ABI (libftb200.so).

The native library is the product; this module only binds it.  `load()` raises if the
library is missing -- there is no Python or CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libftb200.so")
_lib = None


class FtbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _sig(L, name, res, *args):
    f = getattr(L, name)
    f.restype = res
    f.argtypes = list(args)


def load(path=None):
    """Load libftb200.so (build it with `python -m goodphotons_b200.build`)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or _LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is missing: run `python -m goodphotons_b200.build` first")
    L = C.CDLL(p)
    st = C.c_int
    PS = C.c_void_p
    _sig(L, "ftb_last_error", C.c_char_p)
    _sig(L, "ftb_abi_version", C.c_int)
    _sig(L, "ftb_available", C.c_int)
    _sig(L, "ftb_device_name", C.c_char_p)
    _sig(L, "ftb_mem_info", st, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t))
    _sig(L, "ftb_forward_supported", C.c_int, C.POINTER(abi.SceneDesc))
    _sig(L, "ftb_camera_look_at", st, C.POINTER(C.c_double), C.POINTER(C.c_double),
         C.POINTER(C.c_double), C.c_double, C.c_int32, C.c_int32, C.POINTER(abi.Camera))
    _sig(L, "ftb_emission_cdf", st, C.POINTER(abi.Spectrum), C.POINTER(C.c_double),
         C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_int32,
         C.POINTER(C.c_int32), C.POINTER(C.c_double))
    _sig(L, "ftb_scene_create", st, C.POINTER(abi.SceneDesc), C.c_int32, C.POINTER(PS))
    _sig(L, "ftb_scene_destroy", st, PS)
    _sig(L, "ftb_scene_footprint", st, PS, C.c_int32, C.c_int32, C.POINTER(abi.Footprint))
    _sig(L, "ftb_scene_power", C.c_double, PS)
    _sig(L, "ftb_scene_evict", st, PS)
    _sig(L, "ftb_scene_restore", st, PS)
    _sig(L, "ftb_scene_resident", C.c_int, PS)
    _sig(L, "ftb_render_forward", st, PS, C.POINTER(abi.Camera), C.POINTER(abi.RenderParams),
         C.POINTER(C.c_int64), C.POINTER(abi.FilmInfo), C.POINTER(abi.Energy))
    _sig(L, "ftb_render_forward_device", st, PS, C.POINTER(abi.Camera),
         C.POINTER(abi.RenderParams), C.c_void_p, C.POINTER(abi.FilmInfo),
         C.POINTER(abi.Energy), C.c_void_p)
    _sig(L, "ftb_session_begin", st, PS, C.POINTER(abi.Camera), C.c_int32, C.c_int32,
         C.c_int32, C.c_int32, C.POINTER(PS))
    _sig(L, "ftb_session_batch", st, PS, C.c_int64, C.c_uint64)
    _sig(L, "ftb_session_hits0", st, PS, C.POINTER(C.c_double))
    _sig(L, "ftb_session_download", st, PS, C.c_int32, C.POINTER(C.c_int64),
         C.POINTER(abi.FilmInfo), C.POINTER(abi.Energy))
    _sig(L, "ftb_session_end", st, PS)
    _sig(L, "ftb_trace_log", st, PS, C.POINTER(abi.Camera), C.POINTER(abi.RenderParams),
         C.POINTER(abi.PhotonLog))
    _sig(L, "ftb_render_forward_noalloc", st, PS, C.POINTER(abi.Camera),
         C.POINTER(abi.RenderParams), C.c_void_p, C.POINTER(abi.FilmInfo),
         C.POINTER(abi.Energy), C.c_void_p)
    _sig(L, "ftb_render_batch", st, C.POINTER(abi.Job), C.c_int32, C.POINTER(abi.FilmInfo),
         C.POINTER(abi.Energy), C.c_void_p)
    _sig(L, "ftb_blas_create", st, C.POINTER(abi.BlasDesc), C.c_int32, C.POINTER(PS))
    _sig(L, "ftb_blas_destroy", st, PS)
    _sig(L, "ftb_scene_set_instance_transforms", st, PS, C.POINTER(C.c_double), C.c_int64)
    _sig(L, "ftb_scene_clone_instances", st, PS, C.POINTER(C.c_double), C.c_int64, C.POINTER(PS))
    _sig(L, "ftb_get_tuning", st, C.c_int32, C.POINTER(abi.Tuning))
    _sig(L, "ftb_set_tuning", st, C.c_int32, C.POINTER(abi.Tuning))
    _sig(L, "ftb_autotune", st, PS, C.POINTER(abi.Camera), C.c_int64, C.c_int32, C.POINTER(abi.Tuning))
    _sig(L, "ftb_server_create", st, C.POINTER(abi.ServerConfig), C.POINTER(PS))
    _sig(L, "ftb_server_submit", st, PS, C.POINTER(abi.Request), C.POINTER(C.c_uint64))
    _sig(L, "ftb_server_wait", st, PS, C.c_uint64, C.c_double, C.POINTER(abi.JobResult))
    _sig(L, "ftb_server_get_stats", st, PS, C.POINTER(abi.ServerStats))
    _sig(L, "ftb_server_destroy", st, PS)
    _sig(L, "ftb_scene_set_profiling", st, PS, C.c_int32)
    _sig(L, "ftb_scene_profile", st, PS, C.POINTER(abi.KernelProfile), C.c_int32)
    w = _Lib(L)
    if path is None:
        _lib = w
    return w


class _Lib:
    """Pythonic view of the entry points (raises FtbError on a nonzero status)."""

    def __init__(self, L):
        self.L = L

    def check(self, status):
        if status != 0:
            raise FtbError(status, self.L.ftb_last_error().decode())

    def available(self):
        return bool(self.L.ftb_available())

    def device_name(self):
        return self.L.ftb_device_name().decode()

    def look_at(self, eye, target, up, fov, rx, ry):
        cam = abi.Camera()
        a = lambda v: (C.c_double * 3)(*v)
        self.check(self.L.ftb_camera_look_at(a(eye), a(target), a(up), float(fov), rx, ry,
                                             C.byref(cam)))
        return cam

    def emission_cdf(self, desc, spec, step):
        s = desc.spectra[spec]
        cap = int((830.0 - 360.0) / step) + 2
        out = np.zeros(cap, dtype=np.float64)
        n = C.c_int32()
        integral = C.c_double()
        tw = desc.table_w.ctypes.data_as(C.POINTER(C.c_double)) if len(desc.table_w) else None
        tv = desc.table_v.ctypes.data_as(C.POINTER(C.c_double)) if len(desc.table_v) else None
        self.check(self.L.ftb_emission_cdf(C.byref(s), tw, tv, float(step),
                                           out.ctypes.data_as(C.POINTER(C.c_double)), cap,
                                           C.byref(n), C.byref(integral)))
        return out[: n.value + 1].copy(), integral.value

    def render_batch(self, jobs, stream=None, want_energy=True):
        """jobs: list of dicts(scene=Scene, cam=Camera, d_film=int ptr, n=..., seed_base=...,
        max_bounce=..., frac_bits=0).  Returns (infos, energies or None)."""
        n = len(jobs)
        arr = (abi.Job * n)()
        for i, j in enumerate(jobs):
            arr[i].scene = j["scene"].h.value if hasattr(j["scene"].h, "value") else j["scene"].h
            arr[i].cam = j["cam"]
            arr[i].d_film = j["d_film"]
            arr[i].n_photons = j["n"]
            arr[i].seed_base = j.get("seed_base", 0)
            arr[i].max_bounce = j.get("max_bounce", 8)
            arr[i].frac_bits = j.get("frac_bits", 0)
            arr[i].hero_c = j.get("hero_c", 1)
            arr[i].lambda_mode = j.get("lambda_mode", abi.LAMBDA_SPD)
        infos = (abi.FilmInfo * n)()
        ens = (abi.Energy * n)() if want_energy else None
        self.check(self.L.ftb_render_batch(arr, n, infos, ens, C.c_void_p(stream or 0)))
        return infos, ens

    def get_tuning(self, device=0):
        t = abi.Tuning()
        self.check(self.L.ftb_get_tuning(device, C.byref(t)))
        return t

    def set_tuning(self, device=0, wave_slots=None, grid_mult=None, use_graphs=None, sort_rays=None,
                   regenerate=None):
        t = self.get_tuning(device)
        if sort_rays is not None:
            t.sort_rays = int(bool(sort_rays))
        if regenerate is not None:
            t.regenerate = int(bool(regenerate))
        if wave_slots is not None:
            t.wave_slots = wave_slots
        if grid_mult is not None:
            t.grid_mult = grid_mult
        if use_graphs is not None:
            t.use_graphs = int(bool(use_graphs))
        self.check(self.L.ftb_set_tuning(device, C.byref(t)))
        return t

    def autotune(self, scene, cam, n, max_bounce):
        t = abi.Tuning()
        self.check(self.L.ftb_autotune(scene.h, C.byref(cam), n, max_bounce, C.byref(t)))
        return t

    def supported(self, desc):
        r = self.L.ftb_forward_supported(desc.ref())
        return r, self.L.ftb_last_error().decode()


class Blas:
    """A baked, device-resident triangle asset (ftb_blas_create) that scenes can share:
    pass it as `handle` to SceneBuilder.blas."""

    def __init__(self, tri_v, tri_mat, normals=None, device=0, lib=None):
        self.lib = lib or load()
        self.tri_v = np.ascontiguousarray(tri_v, dtype=np.float64).reshape(-1, 9)
        self.tri_mat = np.ascontiguousarray(np.broadcast_to(tri_mat, (len(self.tri_v),)), dtype=np.int32)
        self.tri_n = None if normals is None else np.ascontiguousarray(normals, np.float64).reshape(-1, 9)
        d = abi.BlasDesc()
        d.n_tris = len(self.tri_v)
        d.tri_v = self.tri_v.ctypes.data_as(C.POINTER(C.c_double))
        d.tri_n = self.tri_n.ctypes.data_as(C.POINTER(C.c_double)) if self.tri_n is not None else None
        d.tri_mat = self.tri_mat.ctypes.data_as(C.POINTER(C.c_int32))
        h = C.c_void_p()
        self.lib.check(self.lib.L.ftb_blas_create(C.byref(d), device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.L.ftb_blas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _xf_array(to_world):
    a = np.ascontiguousarray(to_world, dtype=np.float64).reshape(-1, 12)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class Scene:
    """A baked, device-resident scene (ftb_scene_create)."""

    def __init__(self, desc, device=0, lib=None, _handle=None, build=abi.BUILD_SAH):
        """build: abi.BUILD_SAH (host binned SAH) or abi.BUILD_DEVICE (GPU linear BVH)."""
        self.lib = lib or load()
        self.desc = desc
        if _handle is not None:
            self.h = _handle
            return
        h = C.c_void_p()
        desc.desc.build = build
        try:
            self.lib.check(self.lib.L.ftb_scene_create(desc.ref(), device, C.byref(h)))
        finally:
            desc.desc.build = abi.BUILD_SAH
        self.h = h

    def set_instance_transforms(self, to_world):
        """Refit: new to_world maps (n x 12: 3x3 row-major, then translation) for
        instances 0..n-1."""
        a, ptr = _xf_array(to_world)
        self.lib.check(self.lib.L.ftb_scene_set_instance_transforms(self.h, ptr, len(a)))

    def clone_instances(self, to_world):
        """A scene sharing this one's device tables, with its own refit top level."""
        a, ptr = _xf_array(to_world)
        h = C.c_void_p()
        self.lib.check(self.lib.L.ftb_scene_clone_instances(self.h, ptr, len(a), C.byref(h)))
        return Scene(self.desc, lib=self.lib, _handle=h)

    def close(self):
        if self.h:
            self.lib.L.ftb_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def power(self):
        return self.lib.L.ftb_scene_power(self.h)

    def footprint(self, rx, ry):
        fp = abi.Footprint()
        self.lib.check(self.lib.L.ftb_scene_footprint(self.h, rx, ry, C.byref(fp)))
        return fp

    def evict(self):
        """Free the device tables, keeping a host copy (ftb_scene_evict)."""
        self.lib.check(self.lib.L.ftb_scene_evict(self.h))

    def restore(self):
        """Upload the tables again (ftb_scene_restore)."""
        self.lib.check(self.lib.L.ftb_scene_restore(self.h))

    @property
    def resident(self):
        return bool(self.lib.L.ftb_scene_resident(self.h))

    def render(self, cam, n, seed_base=0, max_bounce=8, frac_bits=0, out=None, hero_c=1, lambda_mode=0):
        """One-shot render into a host film: returns (film int64 [ry, rx, 4], info, energy).
        `out` may be a preallocated (e.g. pinned) int64 array of that shape."""
        film = out if out is not None else np.zeros((cam.res_y, cam.res_x, 4), dtype=np.int64)
        assert film.dtype == np.int64 and film.shape == (cam.res_y, cam.res_x, 4) and film.flags.c_contiguous
        p = abi.RenderParams(n, seed_base, max_bounce, frac_bits, hero_c, lambda_mode)
        info, en = abi.FilmInfo(), abi.Energy()
        self.lib.check(self.lib.L.ftb_render_forward(
            self.h, C.byref(cam), C.byref(p), film.ctypes.data_as(C.POINTER(C.c_int64)),
            C.byref(info), C.byref(en)))
        return film, info, en

    def render_device(self, cam, n, d_film_ptr, seed_base=0, max_bounce=8, frac_bits=0,
                      stream=None, want_energy=False, hero_c=1, lambda_mode=0):
        p = abi.RenderParams(n, seed_base, max_bounce, frac_bits, hero_c, lambda_mode)
        info = abi.FilmInfo()
        en = abi.Energy() if want_energy else None
        self.lib.check(self.lib.L.ftb_render_forward_device(
            self.h, C.byref(cam), C.byref(p), C.c_void_p(d_film_ptr), C.byref(info),
            C.byref(en) if en is not None else None, C.c_void_p(stream or 0)))
        return info, en

    def set_profiling(self, mode):
        self.lib.check(self.lib.L.ftb_scene_set_profiling(self.h, mode))

    def profile(self, reset=True):
        kp = abi.KernelProfile()
        self.lib.check(self.lib.L.ftb_scene_profile(self.h, C.byref(kp), 1 if reset else 0))
        return kp

    def trace_log(self, cam, n, seed_base=0, max_bounce=8, hero_c=1, lambda_mode=0):
        logs = (abi.PhotonLog * max(1, n))()
        p = abi.RenderParams(n, seed_base, max_bounce, 0, hero_c, lambda_mode)
        self.lib.check(self.lib.L.ftb_trace_log(self.h, C.byref(cam), C.byref(p), logs))
        return logs_to_numpy(logs, n)


class Server:
    """Resident render server with continuous batching (ftb_server_*)."""

    def __init__(self, device=0, max_active=64, film_budget=0, wave_slots=0, hero_max=0, hbm_budget=0, lib=None):
        self.lib = lib or load()
        cfg = abi.ServerConfig(device, max_active, film_budget, wave_slots, hero_max, hbm_budget)
        h = C.c_void_p()
        self.lib.check(self.lib.L.ftb_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._films = {}

    def submit(self, scene, cam, n, seed_base=0, max_bounce=8, frac_bits=0, host_film=None, hero_c=1,
               lambda_mode=0):
        """Queue a job; host_film (int64 [res_y, res_x, 4], C-contiguous) receives the film."""
        if host_film is not None:
            assert host_film.dtype == np.int64 and host_film.flags.c_contiguous
            assert host_film.size == cam.res_x * cam.res_y * 4
        r = abi.Request(scene.h.value if hasattr(scene.h, "value") else scene.h, cam, n, seed_base, max_bounce,
                        frac_bits, hero_c, lambda_mode,
                        host_film.ctypes.data_as(C.POINTER(C.c_int64)) if host_film is not None else None)
        jid = C.c_uint64()
        self.lib.check(self.lib.L.ftb_server_submit(self.h, C.byref(r), C.byref(jid)))
        self._films[jid.value] = host_film   # keep the buffer alive until the job is waited on
        return jid.value

    def wait(self, job_id, timeout=-1.0):
        res = abi.JobResult()
        self.lib.check(self.lib.L.ftb_server_wait(self.h, job_id, float(timeout), C.byref(res)))
        self._films.pop(job_id, None)
        return res

    def stats(self):
        st = abi.ServerStats()
        self.lib.check(self.lib.L.ftb_server_get_stats(self.h, C.byref(st)))
        return st

    def close(self):
        if self.h:
            self.lib.L.ftb_server_destroy(self.h)
            self.h = None
            self._films.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def logs_to_numpy(logs, n):
    raw = np.ctypeslib.as_array(C.cast(logs, C.POINTER(C.c_uint8)), shape=(n * C.sizeof(abi.PhotonLog),))
    dt = np.dtype([("n_hits", "<i4"), ("fate", "<i4"), ("prim_hash", "<u8"), ("beta", "<f8"),
                   ("prims", "<i4", (8,))])
    assert dt.itemsize == C.sizeof(abi.PhotonLog)
    return np.frombuffer(raw.tobytes(), dtype=dt).copy()


def film_to_xyz(film, info):
    """int64 fixed-point film -> absolute XYZ sums (reference Film::xyz) and hits."""
    xyz = film[..., :3].astype(np.float64) * info.scale
    hits = film[..., 3].astype(np.float64)
    return xyz, hits
