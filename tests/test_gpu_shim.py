"""The drop-in shim (goodphotons_b200/shim/render_cuda_ftb.cpp) driven like the reference's
main.cpp: a reference Scene and Camera in, renderForwardCuda(...) with the reference's own
signature (render_cuda.h:79-82), a reference Film out.

The shim bakes spectra made by the reference's builders (Cauchy, Sellmeier, tables) in
closed form, so the film through the shim must equal, bit for bit, the film through the C
ABI directly -- and match the reference CPU tracer on the same photons within the parity
tolerances of test_gpu_parity.py -- on the benchmarked dispersive glass (Cauchy IOR, step
spectra with breakpoints off any sampling grid) and on every material branch.  The
resident session (sharedForwardGpu*) is driven the same way, with one wavelength per
photon and with hero bundles (the reference CLI's default heroC is 4).
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "libftshim_test.so")


@pytest.fixture(scope="module")
def shim(gpu):
    if not os.path.exists(SHIM):
        pytest.skip("shim test library not built (needs the reference headers at build time)")
    L = C.CDLL(SHIM)
    L.ftr_prepare.restype = C.c_void_p
    L.ftr_prepare.argtypes = [C.POINTER(abi.SceneDesc)]
    L.ftr_release.argtypes = [C.c_void_p]
    PD = C.POINTER(C.c_double)
    L.ftshim_render.restype = C.c_int
    L.ftshim_render.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int64, C.c_uint64, C.c_int, PD, PD, PD]
    L.ftshim_session.restype = C.c_int
    L.ftshim_session.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int, C.c_int64, C.c_int64, C.c_int,
                                 C.c_int, C.c_int, PD, PD, PD]
    L.ftr_trace.restype = C.c_int
    L.ftr_trace.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int64, C.c_uint64, C.c_int, C.c_int, C.c_int,
                            PD, PD, PD, C.POINTER(C.c_int64), C.POINTER(C.c_int32), PD]
    return L


def cornell_on_grid(gpu):
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=True, ramp=0.5)
    return sb.build(gpu)


SHIM_SCENES = {
    "cornell": (cornell_on_grid, 8),
    "glass": (lambda L: scenes.make_glass(L, level=3), 16),
    "materials": (cases.make_materials, 16),
    "instances": (cases.make_instances, 16),
    "mirrors": (cases.make_mirrors, 16),
}


@pytest.mark.parametrize("scene", sorted(SHIM_SCENES))
def test_render_forward_cuda_through_shim(shim, gpu, scene):
    """`glass`: the benchmarked material (Cauchy IOR; wall steps with 0.01 nm ramps);
    `materials`: Sellmeier, nested priorities, filters, glossy; `instances`: the reference
    Scene's blasList / MeshInstances go through the shim's bake; `mirrors`: the reference
    Scene's mirror planes (Scene::build) and the plane connector."""
    mk, mb = SHIM_SCENES[scene]
    d = mk(gpu)
    cam = scenes.default_camera(gpu, 48)
    n, seed = 60_000, 77
    ref = shim.ftr_prepare(d.ref())
    try:
        npix = 48 * 48
        xyz, hits, en = np.zeros(npix * 3), np.zeros(npix), np.zeros(5)
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        assert shim.ftshim_render(ref, C.byref(cam), n, seed, mb, P(xyz), P(hits), P(en)) == 0
        cx, ch, ce = np.zeros(npix * 3), np.zeros(npix), np.zeros(5)
        assert shim.ftr_trace(ref, C.byref(cam), n, seed, mb, 1, 1, P(cx), P(ch), P(ce), None, None, None) == 0
    finally:
        shim.ftr_release(ref)
    # the shim bakes per call with the GPU-built tree unless the budget exceeds 4096 photons per
    # primitive; the direct render uses the same tree, so hits (ties included) are the same
    build = abi.BUILD_SAH if n > 4096 * d.n_prims else abi.BUILD_DEVICE
    sc = lib.Scene(d, 0, gpu, build=build)
    film, info, e2 = sc.render(cam, n, seed_base=seed, max_bounce=mb)
    sc.close()
    dx, dh = lib.film_to_xyz(film, info)
    np.testing.assert_array_equal(xyz.reshape(48, 48, 3), dx)
    np.testing.assert_array_equal(hits.reshape(48, 48), dh)
    np.testing.assert_array_equal(en, e2.as_list())
    # against the reference CPU tracer on the same photons
    np.testing.assert_array_equal(hits, ch)
    tol = ch[:, None] * info.scale + 1e-10 * np.abs(cx.reshape(-1, 3))
    assert (np.abs(xyz.reshape(-1, 3) - cx.reshape(-1, 3)) <= tol).all()
    np.testing.assert_allclose(en, ce, rtol=1e-9)


@pytest.mark.parametrize("scene,hero", [("glass", 1), ("glass", 4), ("cornell", 4), ("mirrors", 4)])
def test_shared_session_through_shim(shim, gpu, oracle, scene, hero):
    """sharedForwardGpuBegin with two cameras and heroC, two batches with the cumulative
    seedBase: camera 0's running total equals the reference CPU tracer's film of the same
    photons through that camera alone (the shared splat draws no random numbers)."""
    mk, mb = SHIM_SCENES[scene]
    d = mk(gpu)
    cams = (abi.Camera * 2)(scenes.default_camera(gpu, 40),
                            gpu.look_at((1.3, 1.2, 4.8), (1.0, 0.9, 1.0), (0, 1, 0), 38.0, 32, 24))
    n0, n1 = 30_000, 45_000
    ref = shim.ftr_prepare(d.ref())
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    try:
        npix = 40 * 40
        xyz, hits, en = np.zeros(npix * 3), np.zeros(npix), np.zeros(5)
        assert shim.ftshim_session(ref, cams, 2, n0, n1, mb, hero, 0, P(xyz), P(hits), P(en)) == 0
        cx, ch, ce = np.zeros(npix * 3), np.zeros(npix), np.zeros(5)
        assert shim.ftr_trace(ref, C.byref(cams[0]), n0 + n1, 0, mb, hero, 4, P(cx), P(ch), P(ce),
                              None, None, None) == 0
    finally:
        shim.ftr_release(ref)
    assert hits.sum() > 0
    np.testing.assert_array_equal(hits, ch)
    # the session's film format: the default for 2^36 photons (ftb_session_begin, frac_bits 0)
    sc = lib.Scene(d, 0, gpu)
    q = sc.power * 2.0 ** -(62 - 36 - 20)
    sc.close()
    tol = ch[:, None] * q + 1e-10 * np.abs(cx.reshape(-1, 3))
    assert (np.abs(xyz.reshape(-1, 3) - cx.reshape(-1, 3)) <= tol).all()
    np.testing.assert_allclose(en, ce, rtol=1e-9)
