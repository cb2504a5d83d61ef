"""ctypes bindings of the CPU checkers under oracle/ (test infrastructure only).

  Oracle     -- oracle/libftoracle.so, the plain-C restatement of the reference tracer
  Reference  -- oracle/_ref/libftref.so, the reference's own tracer built from its
                headers (present only where the reference sources were available at build
                time; it travels with the repository snapshot)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from goodphotons_b200 import abi
from goodphotons_b200.lib import logs_to_numpy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libftoracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libftref.so")

_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)


def _ptr(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        L.fto_prepare.restype = C.c_void_p
        L.fto_prepare.argtypes = [C.POINTER(abi.SceneDesc)]
        L.fto_release.argtypes = [C.c_void_p]
        L.fto_trace.restype = C.c_int
        L.fto_trace.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int64, C.c_uint64, C.c_int,
                                C.c_int, C.c_int, _PD, _PD, _PD, C.POINTER(abi.PhotonLog), _PI64]
        L.fto_total_power.restype = C.c_double
        L.fto_total_power.argtypes = [C.c_void_p]
        L.fto_set_lambda_mode.restype = C.c_int
        L.fto_set_lambda_mode.argtypes = [C.c_void_p, C.c_int]
        L.fto_emission_cdf.restype = C.c_int
        L.fto_emission_cdf.argtypes = [C.POINTER(abi.SceneDesc), C.c_int, C.c_double, _PD, C.c_int, _PD]
        L.fto_spectrum_eval.restype = C.c_double
        L.fto_spectrum_eval.argtypes = [C.POINTER(abi.SceneDesc), C.c_int, C.c_double]
        L.fto_camera_look_at.argtypes = [_PD, _PD, _PD, C.c_double, C.c_int, C.c_int, C.POINTER(abi.Camera)]
        L.fto_uniforms.argtypes = [C.c_uint64, C.c_int, _PD]
        L.fto_closest_hit.restype = C.c_int
        L.fto_closest_hit.argtypes = [C.c_void_p, _PD, _PD, C.c_double, _PD]
        L.fto_occluded.restype = C.c_int
        L.fto_occluded.argtypes = [C.c_void_p, _PD, _PD, C.c_double, C.c_double]
        L.fto_last_error.restype = C.c_char_p
        self.L = L

    def prepare(self, desc):
        h = self.L.fto_prepare(desc.ref())
        if not h:
            raise RuntimeError(self.L.fto_last_error().decode())
        return h

    def trace(self, desc, cam, n, seed_base=0, max_bounce=8, threads=1, logs=False, rays=False, ctx=None,
              hero_c=1, lambda_mode=0):
        h = ctx or self.prepare(desc)
        if self.L.fto_set_lambda_mode(h, lambda_mode) != 0:
            raise RuntimeError(self.L.fto_last_error().decode())
        npix = cam.res_x * cam.res_y
        xyz = np.zeros((npix, 3))
        hits = np.zeros(npix)
        en = np.zeros(5)
        lg = (abi.PhotonLog * max(1, n))() if logs else None
        ry = np.zeros(max(1, n), dtype=np.int64) if rays else None
        try:
            r = self.L.fto_trace(h, C.byref(cam), n, seed_base, max_bounce, hero_c, threads, _ptr(xyz), _ptr(hits),
                                 _ptr(en), lg, _ptr(ry, C.c_int64) if rays else None)
            if r != 0:
                raise RuntimeError(self.L.fto_last_error().decode())
        finally:
            if ctx is None:
                self.L.fto_release(h)
        out = {"xyz": xyz.reshape(cam.res_y, cam.res_x, 3), "hits": hits.reshape(cam.res_y, cam.res_x),
               "energy": en}
        if logs:
            out["logs"] = logs_to_numpy(lg, n)
        if rays:
            out["rays"] = ry[:n]
        return out

    def uniforms(self, k, count):
        out = np.zeros(count)
        self.L.fto_uniforms(k, count, _ptr(out))
        return out

    def emission_cdf(self, desc, spec, step=1.0):
        out = np.zeros(int(470 / step) + 2)
        integ = C.c_double()
        n = self.L.fto_emission_cdf(desc.ref(), spec, step, _ptr(out), len(out), C.byref(integ))
        return out[: n + 1], integ.value

    def look_at(self, eye, target, up, fov, rx, ry):
        cam = abi.Camera()
        a = lambda v: (C.c_double * 3)(*v)
        self.L.fto_camera_look_at(a(eye), a(target), a(up), fov, rx, ry, C.byref(cam))
        return cam


class Reference:
    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (built by `make -C oracle` where the reference is present)")
        L = C.CDLL(path)
        L.ftr_prepare.restype = C.c_void_p
        L.ftr_prepare.argtypes = [C.POINTER(abi.SceneDesc)]
        L.ftr_release.argtypes = [C.c_void_p]
        L.ftr_total_power.restype = C.c_double
        L.ftr_total_power.argtypes = [C.c_void_p]
        L.ftr_emitter.restype = C.c_int
        L.ftr_emitter.argtypes = [C.c_void_p, C.c_int, _PD, _PD, _PD, C.c_int]
        L.ftr_closest_hit.restype = C.c_int
        L.ftr_closest_hit.argtypes = [C.c_void_p, _PD, _PD, _PD, _PD]
        L.ftr_occluded.restype = C.c_int
        L.ftr_occluded.argtypes = [C.c_void_p, _PD, _PD, C.c_double]
        L.ftr_uniforms.argtypes = [C.c_uint64, C.c_int, _PD]
        L.ftr_look_at.argtypes = [_PD, _PD, _PD, C.c_double, C.c_int, C.c_int, C.POINTER(abi.Camera)]
        L.ftr_trace.restype = C.c_int
        L.ftr_trace.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int64, C.c_uint64, C.c_int, C.c_int,
                                C.c_int, _PD, _PD, _PD, _PI64, C.POINTER(C.c_int32), _PD]
        self.L = L

    @staticmethod
    def available():
        return os.path.exists(REF_SO)

    def prepare(self, desc):
        return self.L.ftr_prepare(desc.ref())

    def trace(self, desc, cam, n, seed_base=0, max_bounce=8, threads=1, per_photon=False, ctx=None, hero_c=1):
        h = ctx or self.prepare(desc)
        npix = cam.res_x * cam.res_y
        xyz = np.zeros((npix, 3))
        hits = np.zeros(npix)
        en = np.zeros(5)
        rays = fate = beta = None
        if per_photon:
            rays = np.zeros(max(1, n), dtype=np.int64)
            fate = np.zeros(max(1, n), dtype=np.int32)
            beta = np.zeros(max(1, n))
        try:
            r = self.L.ftr_trace(h, C.byref(cam), n, seed_base, max_bounce, hero_c, threads, _ptr(xyz), _ptr(hits),
                                 _ptr(en), _ptr(rays, C.c_int64) if per_photon else None,
                                 _ptr(fate, C.c_int32) if per_photon else None,
                                 _ptr(beta) if per_photon else None)
            assert r == 0
        finally:
            if ctx is None:
                self.L.ftr_release(h)
        out = {"xyz": xyz.reshape(cam.res_y, cam.res_x, 3), "hits": hits.reshape(cam.res_y, cam.res_x),
               "energy": en}
        if per_photon:
            out.update(rays=rays[:n], fate=fate[:n], beta=beta[:n])
        return out

    def uniforms(self, k, count):
        out = np.zeros(count)
        self.L.ftr_uniforms(k, count, _ptr(out))
        return out

    def look_at(self, eye, target, up, fov, rx, ry):
        cam = abi.Camera()
        a = lambda v: (C.c_double * 3)(*v)
        self.L.ftr_look_at(a(eye), a(target), a(up), fov, rx, ry, C.byref(cam))
        return cam

    def closest_hit(self, ctx, o, d):
        t = C.c_double()
        ng = np.zeros(3)
        m = self.L.ftr_closest_hit(ctx, _ptr(np.asarray(o, float)), _ptr(np.asarray(d, float)), C.byref(t), _ptr(ng))
        return m, t.value

    def emitter(self, desc, i, ctx=None):
        h = ctx or self.prepare(desc)
        p, integ = C.c_double(), C.c_double()
        cdf = np.zeros(2000)
        n = self.L.ftr_emitter(h, i, C.byref(p), C.byref(integ), _ptr(cdf), len(cdf))
        if ctx is None:
            self.L.ftr_release(h)
        return p.value, integ.value, cdf[:n]
