"""Batched rendering (ftb_render_batch): jobs with different scenes, cameras, resolutions,
photon ranges and bounce caps share waves.  Each job's film and energy report must be
bit-identical to rendering that job alone -- photons are keyed by index and the film is
fixed point, so the mix cannot change a result."""
import ctypes as C

import numpy as np
import pytest

import cases
from goodphotons_b200 import lib, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[1, 0], ids=["streaming", "waves"])
def launch_mode(request, gpu):
    """Streaming passes (freed slots refilled at once) or waves traced to their last bounce."""
    saved = gpu.get_tuning(0)
    gpu.set_tuning(0, regenerate=request.param)
    yield request.param
    gpu.L.ftb_set_tuning(0, C.byref(saved))


def test_batch_results_equal_solo_renders(gpu, launch_mode):
    torch = pytest.importorskip("torch")
    L = gpu
    sc_c = lib.Scene(scenes.make_cornell(L), 0, L)
    sc_g = lib.Scene(scenes.make_glass(L, level=3), 0, L)
    sc_m = lib.Scene(cases.make_materials(L), 0, L)
    sc_f = lib.Scene(scenes.make_fog_strands(L, n_strands=300), 0, L)
    specs = [  # scene, res, photons, seed, max bounce
        (sc_c, 64, 3_000_000, 0, 8),        # spans the first wave
        (sc_g, 48, 2_500_000, 10**9, 16),   # split across waves
        (sc_m, 40, 70_000, 5, 12),
        (sc_f, 32, 50_000, 77, 32),
        (sc_c, 24, 1, 3, 8),                # a one-photon job
        (sc_g, 56, 300_000, 123, 0),        # no bounces: emission splat + residual only
    ]
    jobs, films = [], []
    for sc, res, n, seed, mb in specs:
        cam = scenes.default_camera(L, res)
        film = torch.zeros((res, res, 4), dtype=torch.int64, device="cuda:0")
        films.append(film)
        jobs.append(dict(scene=sc, cam=cam, d_film=film.data_ptr(), n=n, seed_base=seed, max_bounce=mb,
                         frac_bits=28))
    stream = torch.cuda.current_stream().cuda_stream
    infos, ens = L.render_batch(jobs, stream=stream)
    torch.cuda.synchronize()
    for i, ((sc, res, n, seed, mb), film) in enumerate(zip(specs, films)):
        solo = torch.zeros_like(film)
        _, en = sc.render_device(jobs[i]["cam"], n, solo.data_ptr(), seed_base=seed, max_bounce=mb,
                                 frac_bits=28, stream=stream, want_energy=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(film.cpu().numpy(), solo.cpu().numpy(), err_msg=f"job {i}")
        assert list(ens[i].fx) == list(en.fx), f"job {i} energy"
        assert infos[i].frac_bits == 28
    for sc in (sc_c, sc_g, sc_m, sc_f):
        sc.close()


def test_tuning_and_graph_replay_do_not_change_results(gpu):
    """Slot refill, wave size, grid size and graph replay change only how paths are launched:
    films and energy tallies stay bit-identical; the autotuner returns a setting in range."""
    L = gpu
    sc = lib.Scene(scenes.make_glass(L, level=3), 0, L)
    cam = scenes.default_camera(L, 40)
    saved = L.get_tuning(0)
    try:
        ref = None
        for slots, grid, graphs, srt, regen in [(1 << 22, 16, 0, 0, 0), (1 << 20, 4, 1, 1, 0),
                                                (1 << 19, 32, 1, 0, 1), (3 << 18, 8, 0, 1, 1),
                                                (1 << 22, 16, 1, 1, 1), (1 << 22, 16, 1, 0, 0),
                                                (40_000, 16, 1, 0, 1), (1_000, 4, 0, 0, 1),
                                                (1 << 23, 8, 1, 1, 1)]:
            L.set_tuning(0, wave_slots=slots, grid_mult=grid, use_graphs=graphs, sort_rays=srt, regenerate=regen)
            for _ in range(2):   # the second render replays a captured graph
                film, _, en = sc.render(cam, 1_500_000, seed_base=42, max_bounce=16, frac_bits=30)
                if ref is None:
                    ref = (film, list(en.fx))
                np.testing.assert_array_equal(film, ref[0], err_msg=f"{slots} {grid} {graphs} {srt} {regen}")
                assert list(en.fx) == ref[1]
        t = L.autotune(sc, cam, 1 << 21, 16)
        assert 1 <= t.wave_slots <= 1 << 24 and 1 <= t.grid_mult <= 64 and t.use_graphs in (0, 1)
        assert t.sort_rays in (0, 1) and t.regenerate in (0, 1)
        film, _, _ = sc.render(cam, 1_500_000, seed_base=42, max_bounce=16, frac_bits=30)
        np.testing.assert_array_equal(film, ref[0])
    finally:
        L.L.ftb_set_tuning(0, C.byref(saved))
        sc.close()


def test_bundles_and_single_wavelength_jobs_in_one_batch(gpu):
    """A batch mixing hero bundles (C = 4, 3) with one-wavelength jobs: waves hold one kind,
    and every job equals its solo render."""
    torch = pytest.importorskip("torch")
    L = gpu
    sc_g = lib.Scene(scenes.make_glass(L, level=3), 0, L)
    sc_c = lib.Scene(scenes.make_cornell(L), 0, L)
    specs = [(sc_g, 40, 700_000, 4), (sc_c, 32, 300_000, 1), (sc_c, 24, 900_000, 3), (sc_g, 48, 200_000, 1)]
    jobs, films = [], []
    for k, (sc, res, n, hero) in enumerate(specs):
        film = torch.zeros((res, res, 4), dtype=torch.int64, device="cuda:0")
        films.append(film)
        jobs.append(dict(scene=sc, cam=scenes.default_camera(L, res), d_film=film.data_ptr(), n=n,
                         seed_base=10_000 * k, max_bounce=16, frac_bits=30, hero_c=hero))
    stream = torch.cuda.current_stream().cuda_stream
    _, ens = L.render_batch(jobs, stream=stream)
    torch.cuda.synchronize()
    for k, (j, film) in enumerate(zip(jobs, films)):
        solo, _, en = j["scene"].render(j["cam"], j["n"], seed_base=j["seed_base"], max_bounce=16, frac_bits=30,
                                        hero_c=j["hero_c"])
        np.testing.assert_array_equal(film.cpu().numpy(), solo, err_msg=f"job {k}")
        assert list(ens[k].fx) == list(en.fx)
    sc_g.close()
    sc_c.close()
