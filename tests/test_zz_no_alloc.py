"""ftb_render_forward_noalloc: rendering without allocating device memory.

Some callers cannot call cudaMalloc while they render: hosts that own every byte of device
memory and forbid allocation inside their render callbacks (engine and DCC plug-in hosts
with their own allocator), frame loops that must not allocate once running, and code for
which a cudaMalloc / cudaFree would synchronize the device in the middle of its own stream
work.  For them the library keeps the scratch of one wave of photons in a fixed device
array of FTB_NOALLOC_SCRATCH_BYTES (at most FTB_NOALLOC_MAX_PHOTONS photons per call).

These tests call that entry point through the C ABI twice in a row (consecutive photon
ranges, so the second call runs on the scratch the first one left behind) and check each
film and energy report against the regular device-film entry point
(ftb_render_forward_device) on the same photons: the int64 film and the fixed-point energy
tallies must be identical, the tolerance every other film test here implies for equal
photon paths.  The scenes cover every kernel variant the call can pick: triangles only
(glass), media with curves in their own hierarchy (fog + strands), and instanced meshes.
They also check that the second call leaves the device's free memory unchanged, that an
oversized request is refused with a clear error, and that in a scene with media a request
for hero bundles traces one wavelength per photon, like every other entry point.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu

RES = 48


def _free_bytes(L):
    free, total = C.c_size_t(), C.c_size_t()
    L.check(L.L.ftb_mem_info(C.byref(free), C.byref(total)))
    return free.value


def _noalloc(L, sc, cam, film, n, seed, mb, hero_c=1, stream=0):
    p = abi.RenderParams(n, seed, mb, 30, hero_c, 0)
    info, en = abi.FilmInfo(), abi.Energy()
    L.check(L.L.ftb_render_forward_noalloc(sc.h, C.byref(cam), C.byref(p), C.c_void_p(film.data_ptr()),
                                           C.byref(info), C.byref(en), C.c_void_p(stream)))
    return info, en


SCENES = {
    "glass": (lambda L: scenes.make_glass(L, level=3), 16),
    "fog_strands": (lambda L: scenes.make_fog_strands(L, n_strands=2000), 32),
    "instances": (cases.make_instances, 16),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_noalloc_entry_matches_device_entry_on_two_calls(name, gpu):
    torch = pytest.importorskip("torch")
    L = gpu
    mk, mb = SCENES[name]
    sc = lib.Scene(mk(L), 0, L)
    cam = scenes.default_camera(L, RES)
    n = abi.NOALLOC_MAX_PHOTONS
    stream = torch.cuda.current_stream()
    films = [torch.zeros((RES, RES, 4), dtype=torch.int64, device="cuda:0") for _ in range(4)]
    torch.cuda.synchronize()
    try:
        for call, seed in enumerate((0, n)):
            if call == 1:
                torch.cuda.synchronize()
                free_before_second = _free_bytes(L)
            info, en = _noalloc(L, sc, cam, films[2 * call], n, seed, mb, stream=stream.cuda_stream)
            torch.cuda.synchronize()
            if call == 1:
                assert _free_bytes(L) == free_before_second
            ref_info, ref_en = sc.render_device(cam, n, films[2 * call + 1].data_ptr(), seed_base=seed,
                                                max_bounce=mb, frac_bits=30, stream=stream.cuda_stream,
                                                want_energy=True)
            torch.cuda.synchronize()
            a = films[2 * call].cpu().numpy()
            b = films[2 * call + 1].cpu().numpy()
            assert a[..., 3].sum() > 0
            np.testing.assert_array_equal(a, b)
            assert list(en.fx) == list(ref_en.fx)
            assert info.frac_bits == ref_info.frac_bits and info.scale == ref_info.scale
        # an oversized request is refused, not truncated
        p = abi.RenderParams(n + 1, 0, mb, 30)
        st = L.L.ftb_render_forward_noalloc(sc.h, C.byref(cam), C.byref(p), C.c_void_p(films[0].data_ptr()),
                                            None, None, C.c_void_p(stream.cuda_stream))
        assert st == 7  # FTB_ERR_TOO_LARGE
        assert str(n) in L.L.ftb_last_error().decode()
    finally:
        sc.close()


def test_noalloc_hero_request_in_media_traces_one_wavelength(gpu):
    torch = pytest.importorskip("torch")
    L = gpu
    sc = lib.Scene(scenes.make_fog_strands(L, n_strands=2000), 0, L)
    cam = scenes.default_camera(L, RES)
    stream = torch.cuda.current_stream()
    a = torch.zeros((RES, RES, 4), dtype=torch.int64, device="cuda:0")
    b = torch.zeros_like(a)
    try:
        _, ea = _noalloc(L, sc, cam, a, 20_000, 5, 32, hero_c=4, stream=stream.cuda_stream)
        _, eb = sc.render_device(cam, 20_000, b.data_ptr(), seed_base=5, max_bounce=32, frac_bits=30,
                                 stream=stream.cuda_stream, want_energy=True, hero_c=1)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
        assert list(ea.fx) == list(eb.fx)
    finally:
        sc.close()
