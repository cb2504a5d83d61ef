"""ftb_render_forward_noalloc: rendering without allocating device memory.

Some callers cannot call cudaMalloc while they render: hosts that own every byte of device
memory and forbid allocation inside their render callbacks (engine and DCC plug-in hosts
with their own allocator), frame loops that must not allocate once running, and code for
which a cudaMalloc / cudaFree would synchronize the device in the middle of its own stream
work.  For them the library keeps the scratch of one wave of photons in a fixed device
array (at most FTB_NOALLOC_MAX_PHOTONS photons per call).

This test calls that entry point through the C ABI twice in a row (consecutive photon
ranges, so the second call runs on the scratch the first one left behind) and checks each
film and energy report against the regular device-film entry point
(ftb_render_forward_device) on the same photons: the int64 film and the fixed-point energy
tallies must be identical, the tolerance every other film test here implies for equal
photon paths.  It also checks that the second call leaves the device's free memory
unchanged and that an oversized request is refused with a clear error.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from goodphotons_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu


def _free_bytes(L):
    free, total = C.c_size_t(), C.c_size_t()
    L.check(L.L.ftb_mem_info(C.byref(free), C.byref(total)))
    return free.value


def test_noalloc_entry_matches_device_entry_on_two_calls(gpu):
    torch = pytest.importorskip("torch")
    L = gpu
    desc = scenes.make_glass(L, level=3)
    sc = lib.Scene(desc, 0, L)
    cam = scenes.default_camera(L, 48)
    n = abi.NOALLOC_MAX_PHOTONS
    stream = torch.cuda.current_stream()
    films = [torch.zeros((48, 48, 4), dtype=torch.int64, device="cuda:0") for _ in range(4)]
    torch.cuda.synchronize()
    free_before_second = None
    try:
        for call, seed in enumerate((0, n)):
            p = abi.RenderParams(n, seed, 16, 30)
            info, en = abi.FilmInfo(), abi.Energy()
            if call == 1:
                torch.cuda.synchronize()
                free_before_second = _free_bytes(L)
            L.check(L.L.ftb_render_forward_noalloc(sc.h, C.byref(cam), C.byref(p),
                                                   C.c_void_p(films[2 * call].data_ptr()), C.byref(info),
                                                   C.byref(en), C.c_void_p(stream.cuda_stream)))
            torch.cuda.synchronize()
            if call == 1:
                assert _free_bytes(L) == free_before_second
            ref_info, ref_en = sc.render_device(cam, n, films[2 * call + 1].data_ptr(), seed_base=seed,
                                                max_bounce=16, frac_bits=30, stream=stream.cuda_stream,
                                                want_energy=True)
            torch.cuda.synchronize()
            a = films[2 * call].cpu().numpy()
            b = films[2 * call + 1].cpu().numpy()
            assert a[..., 3].sum() > 0
            np.testing.assert_array_equal(a, b)
            assert list(en.fx) == list(ref_en.fx)
            assert info.frac_bits == ref_info.frac_bits and info.scale == ref_info.scale
        # an oversized request is refused, not truncated
        p = abi.RenderParams(n + 1, 0, 16, 30)
        st = L.L.ftb_render_forward_noalloc(sc.h, C.byref(cam), C.byref(p), C.c_void_p(films[0].data_ptr()),
                                            None, None, C.c_void_p(stream.cuda_stream))
        assert st == 7  # FTB_ERR_TOO_LARGE
        assert str(n) in L.L.ftb_last_error().decode()
    finally:
        sc.close()
