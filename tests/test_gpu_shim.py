"""The drop-in shim (goodphotons_b200/shim/render_cuda_ftb.cpp) driven like the reference's
main.cpp: a reference Scene and Camera in, renderForwardCuda(...) with the reference's own
signature (render_cuda.h:79-82), a reference Film out.

The scene's step spectra have their breakpoints on the shim's 0.5 nm sampling grid, so the
shim's baked tables equal the originals and the film through the shim must equal, bit for
bit, the film through the C ABI directly -- and match the reference CPU tracer on the same
photons within the parity tolerances of test_gpu_parity.py.
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
    L.ftr_trace.restype = C.c_int
    L.ftr_trace.argtypes = [C.c_void_p, C.POINTER(abi.Camera), C.c_int64, C.c_uint64, C.c_int, C.c_int, C.c_int,
                            PD, PD, PD, C.POINTER(C.c_int64), C.POINTER(C.c_int32), PD]
    return L


def cornell_on_grid(gpu):
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=True, ramp=0.5)
    return sb.build(gpu)


@pytest.mark.parametrize("scene", ["cornell", "instances"])
def test_render_forward_cuda_through_shim(shim, gpu, scene):
    """`instances`: the reference Scene's blasList / MeshInstances go through the shim's bake
    (with a constant IOR: the shim tabulates non-constant spectra every 0.5 nm, exact only for
    piecewise-linear ones)."""
    d = cornell_on_grid(gpu) if scene == "cornell" else cases.make_instances(gpu, ramp=0.5, cauchy=False)
    cam = scenes.default_camera(gpu, 48)
    n, mb, seed = 60_000, (8 if scene == "cornell" else 16), 77
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
