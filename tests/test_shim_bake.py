"""The drop-in shim's scene bake (goodphotons_b200/shim/render_cuda_ftb.cpp), on the CPU.

The reference hands the shim its material and medium spectra as std::function values.
The shim recovers the closed form of spectra made by the reference's builders -- cauchy,
sellmeier, tabulatedSpectrum (spectrum.h:128-175) -- and bakes them with the builder's own
parameters, so the device evaluates them with the reference's arithmetic at every
wavelength; anything else falls back to a 0.5 nm sampled table.  Here a reference Scene is
built (oracle/_ref, from the same descriptor the tests render) and the shim's bake of it
must give back each spectrum's original form and parameters, bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "libftshim_test.so")


@pytest.fixture(scope="module")
def shim():
    if not os.path.exists(SHIM):
        pytest.skip("shim test library not built (needs the reference headers at build time)")
    L = C.CDLL(SHIM)
    L.ftr_prepare.restype = C.c_void_p
    L.ftr_prepare.argtypes = [C.POINTER(abi.SceneDesc)]
    L.ftr_release.argtypes = [C.c_void_p]
    PD = C.POINTER(C.c_double)
    L.ftshim_spectra.restype = C.c_int
    L.ftshim_spectra.argtypes = [C.c_void_p, C.POINTER(abi.Spectrum), C.c_int, PD, PD, C.c_int]
    return L


def baked(shim, d):
    ref = shim.ftr_prepare(d.ref())
    try:
        out = (abi.Spectrum * 512)()
        tw, tv = np.zeros(1 << 16), np.zeros(1 << 16)
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        n = shim.ftshim_spectra(ref, out, 512, P(tw), P(tv), len(tw))
        assert n >= 0
    finally:
        shim.ftr_release(ref)
    return [out[i] for i in range(n)], tw, tv


def original(d, idx, dflt):
    """(kind, params or pairs) of a descriptor spectrum slot as the reference Scene holds it."""
    if idx < 0:
        return abi.SPEC_CONST, (dflt,)
    s = d.spectra[idx]
    if s.kind == abi.SPEC_TABLE:
        w = d.table_w[s.offset:s.offset + s.n]
        v = d.table_v[s.offset:s.offset + s.n]
        if np.all(v == v[0]):
            return abi.SPEC_CONST, (float(v[0]),)
        return abi.SPEC_TABLE, (tuple(w), tuple(v))
    if s.kind == abi.SPEC_CONST:
        return abi.SPEC_CONST, (s.p[0],)
    if s.kind == abi.SPEC_CAUCHY:
        return abi.SPEC_CAUCHY, tuple(s.p[:2])
    return abi.SPEC_SELLMEIER, tuple(s.p[:6])


def as_tuple(s, tw, tv):
    if s.kind == abi.SPEC_TABLE:
        return abi.SPEC_TABLE, (tuple(tw[s.offset:s.offset + s.n]), tuple(tv[s.offset:s.offset + s.n]))
    if s.kind == abi.SPEC_CONST:
        return abi.SPEC_CONST, (s.p[0],)
    if s.kind == abi.SPEC_CAUCHY:
        return abi.SPEC_CAUCHY, tuple(s.p[:2])
    return abi.SPEC_SELLMEIER, tuple(s.p[:6])


@pytest.mark.parametrize("name", ["materials", "instances", "fog_strands"])
def test_shim_bakes_builder_spectra_in_closed_form(name, shim, L):
    d = cases.CASES[name][0](L)
    got, tw, tv = baked(shim, d)
    want = []
    for i in range(d.n_mats):
        m = d.mats[i]
        want += [original(d, m.reflect, 0.5), original(d, m.ior, 1.5), original(d, m.absorb, 0.0),
                 original(d, m.transmit, 0.0)]
    for i in range(d.n_media):
        want += [original(d, d.media[i].sigma_a, 0.0), original(d, d.media[i].sigma_s, 0.0)]
    assert len(got) == len(want)
    kinds = set()
    for k, (g, w) in enumerate(zip(got, want)):
        assert as_tuple(g, tw, tv) == w, f"spectrum {k}: baked {as_tuple(g, tw, tv)}, authored {w}"
        kinds.add(w[0])
    if name == "materials":   # every closed form occurs in this scene
        assert kinds == {abi.SPEC_CONST, abi.SPEC_TABLE, abi.SPEC_CAUCHY, abi.SPEC_SELLMEIER}


def test_shim_bakes_config_glass_exactly(shim, L):
    """The benchmarked glass: its Cauchy IOR n = 1.5 + 0.0042/um^2 and the walls' step tables
    (breakpoints off the 0.5 nm grid) bake exactly."""
    d = scenes.make_glass(L, level=1)
    got, tw, tv = baked(shim, d)
    cauchy = [as_tuple(g, tw, tv) for g in got if g.kind == abi.SPEC_CAUCHY]
    assert cauchy == [(abi.SPEC_CAUCHY, (1.5, 0.0042))]
    tables = [as_tuple(g, tw, tv) for g in got if g.kind == abi.SPEC_TABLE]
    assert len(tables) == 2 and all(len(t[1][0]) < 20 for t in tables)
