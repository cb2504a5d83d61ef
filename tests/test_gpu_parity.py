"""GPU parity: the CUDA path (through the C ABI) against the oracle and the reference's
golden vectors.

Tolerances, stated here because the film is fixed point and the oracle is double:
  * per-photon hit-primitive sequence (count + 64-bit hash) and termination: identical for
    all but at most max(1, 1e-5 * n) photons (grazing / exact-tie allowance);
  * per-photon final beta: relative 1e-12 (CUDA's exp/log/sin/cos may differ from glibc in
    the last bit);
  * film: hits identical; XYZ within (hits * quantum + 1e-10 * |value|) per pixel, where the
    quantum is the film's fixed-point step (ftb_film_info.scale);
  * energy report: relative 1e-9 (32-bit fraction fixed point per photon).
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="module")
def scenes_cache(gpu):
    out = {}
    for name, (mk, res, n, mb, seed, hero) in cases.CASES.items():
        d = mk(gpu)
        out[name] = (d, lib.Scene(d, 0, gpu))
    yield out
    for _, s in out.values():
        s.close()


def assert_film_close(film, info, xyz_ref, hits_ref):
    xyz, hits = lib.film_to_xyz(film, info)
    np.testing.assert_array_equal(hits, hits_ref)
    tol = hits_ref[..., None] * info.scale + 1e-10 * np.abs(xyz_ref)
    bad = np.abs(xyz - xyz_ref) > tol
    assert not bad.any(), f"{bad.sum()} film values differ; max |d| {np.abs(xyz - xyz_ref).max()}"


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_film_and_energy_match_reference_golden(name, scenes_cache, gpu):
    mk, res, n, mb, seed, hero = cases.CASES[name]
    d, sc = scenes_cache[name]
    g = golden(f"trace_{name}.npz")
    assert cases.scene_hash(d) == str(g["scene_hash"])
    cam = cases.camera(gpu, res)
    film, info, en = sc.render(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
    assert_film_close(film, info, g["xyz"], g["hits"])
    np.testing.assert_allclose(en.as_list(), g["energy"], rtol=1e-9, atol=0)


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_per_photon_paths_match_oracle(name, scenes_cache, gpu, oracle):
    mk, res, _, mb, seed, hero = cases.CASES[name]
    d, sc = scenes_cache[name]
    n = 1 << 15
    cam = cases.camera(gpu, res)
    gl = sc.trace_log(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
    ol = oracle.trace(d, cam, n, seed_base=seed, max_bounce=mb, logs=True, threads=4, hero_c=hero)["logs"]
    # multi-threaded oracle logs are per photon, so order is by photon index either way
    same = (gl["n_hits"] == ol["n_hits"]) & (gl["prim_hash"] == ol["prim_hash"]) & (gl["fate"] == ol["fate"])
    allowed = max(1, int(1e-5 * n))
    assert (~same).sum() <= allowed, f"{(~same).sum()} of {n} photon paths differ; first {np.nonzero(~same)[0][:5]}"
    # Sampled directions carry last-bit differences of CUDA's sin / cos / pow against the
    # C library's.  On flat surfaces they never reach the throughput; at a smooth-shaded
    # diffuse vertex the shading-normal adjoint correction (a ratio of dot products with those
    # directions) multiplies them into beta, and they compound over the bounces.
    rtol = 1e-10 if name.startswith("smooth") else 1e-12
    np.testing.assert_allclose(gl["beta"][same], ol["beta"][same], rtol=rtol, atol=0)
    np.testing.assert_array_equal(gl["prims"][same], ol["prims"][same])


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_device_build_paths_match_oracle(name, gpu, oracle):
    """The GPU-built linear BVH culls differently but must find the same hits: per-photon
    paths equal the oracle's under the same allowance as the host-built tree."""
    mk, res, _, mb, seed, hero = cases.CASES[name]
    d = mk(gpu)
    sc = lib.Scene(d, 0, gpu, build=abi.BUILD_DEVICE)
    n = 1 << 14
    cam = cases.camera(gpu, res)
    gl = sc.trace_log(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
    sc.close()
    ol = oracle.trace(d, cam, n, seed_base=seed, max_bounce=mb, logs=True, threads=4, hero_c=hero)["logs"]
    same = (gl["n_hits"] == ol["n_hits"]) & (gl["prim_hash"] == ol["prim_hash"]) & (gl["fate"] == ol["fate"])
    assert (~same).sum() <= max(1, int(1e-5 * n)), f"{(~same).sum()} of {n} photon paths differ"


def test_film_is_order_independent_and_linear(scenes_cache, gpu):
    d, sc = scenes_cache["glass"]
    cam = cases.camera(gpu, 64)
    n = 300_000
    a, info, ea = sc.render(cam, n, seed_base=11, max_bounce=16, frac_bits=30)
    b, _, eb = sc.render(cam, n, seed_base=11, max_bounce=16, frac_bits=30)
    np.testing.assert_array_equal(a, b)
    assert list(ea.fx) == list(eb.fx)
    p1, _, e1 = sc.render(cam, 123_457, seed_base=11, max_bounce=16, frac_bits=30)
    p2, _, e2 = sc.render(cam, n - 123_457, seed_base=11 + 123_457, max_bounce=16, frac_bits=30)
    np.testing.assert_array_equal(p1 + p2, a)
    assert [x + y for x, y in zip(e1.fx, e2.fx)] == list(ea.fx)


@pytest.mark.parametrize("name,mb,hero", [("cornell", 8, 1), ("glass", 16, 4)])
def test_session_accumulates_like_one_render(name, mb, hero, scenes_cache, gpu):
    """Two cameras in one session (the shared splat), two batches: each camera's film equals
    a one-shot render of all the photons through that camera alone, with one wavelength per
    photon and with hero bundles."""
    d, sc = scenes_cache[name]
    cams = [cases.camera(gpu, 48), gpu.look_at((1.2, 1.1, 5.0), (1.0, 1.0, 1.0), (0, 1, 0), 35.0, 40, 32)]
    arr = (type(cams[0]) * 2)(*cams)
    h = C.c_void_p()
    gpu.check(gpu.L.ftb_session_begin(sc.h, arr, 2, mb, 28, hero, C.byref(h)))
    try:
        gpu.check(gpu.L.ftb_session_batch(h, 50_000, 0))
        gpu.check(gpu.L.ftb_session_batch(h, 70_000, 50_000))
        films = []
        for c, cam in enumerate(cams):
            film = np.zeros((cam.res_y, cam.res_x, 4), dtype=np.int64)
            gpu.check(gpu.L.ftb_session_download(h, c, film.ctypes.data_as(C.POINTER(C.c_int64)), None, None))
            whole, _, _ = sc.render(cam, 120_000, seed_base=0, max_bounce=mb, frac_bits=28, hero_c=hero)
            np.testing.assert_array_equal(film, whole)
            films.append(film)
        hits = np.zeros(48 * 48)
        gpu.check(gpu.L.ftb_session_hits0(h, hits.ctypes.data_as(C.POINTER(C.c_double))))
        np.testing.assert_array_equal(hits.reshape(48, 48), films[0][..., 3].astype(np.float64))
    finally:
        gpu.L.ftb_session_end(h)


def test_device_film_entry_point(scenes_cache, gpu):
    torch = pytest.importorskip("torch")
    d, sc = scenes_cache["materials"]
    cam = cases.camera(gpu, 40)
    film = torch.zeros((40, 40, 4), dtype=torch.int64, device="cuda:0")
    info, en = sc.render_device(cam, 40_000, film.data_ptr(), seed_base=3, max_bounce=16, frac_bits=30,
                                stream=torch.cuda.current_stream().cuda_stream, want_energy=True)
    torch.cuda.synchronize()
    host, _, en2 = sc.render(cam, 40_000, seed_base=3, max_bounce=16, frac_bits=30)
    np.testing.assert_array_equal(film.cpu().numpy(), host)
    assert list(en.fx) == list(en2.fx)


def test_energy_conservation_full_size_cornell(gpu):
    """Config-size run (2^24 photons, 256^2, 8 bounces): every photon's beta is booked once,
    so emitted == absorbed + escaped + residual to within one fixed-point step per photon
    (flat triangles: the shading-normal correction is 1 up to rounding)."""
    d = scenes.make_cornell(gpu)
    sc = lib.Scene(d, 0, gpu)
    cam = scenes.default_camera(gpu, 256)
    n = 1 << 24
    film, info, en = sc.render(cam, n, max_bounce=8)
    fx = list(en.fx)
    assert fx[0] == n * (1 << 32)
    assert abs(fx[0] - (fx[1] + fx[2] + fx[3] + fx[4])) <= n
    assert film[..., 3].sum() > 0
    sc.close()


@pytest.mark.parametrize("name,level", [("cornell", 0), ("glass", 5)])
def test_film_statistics_independent_photons(name, level, gpu, oracle):
    """The statistical film criterion with independent photons: the GPU renders indices
    [0, N), the oracle [N, 2N), each as K = 32 batches.  Per pixel, the two batch means of Y
    are compared in units of their combined standard error; the number of lit pixels beyond
    3 sigma must be consistent with chance (binomial tail 1e-4 at the Student-t rate for
    K - 1 degrees of freedom), and the mean luminance of the two films must agree within
    0.5%.  A systematic error shows up as many pixels beyond 3 sigma."""
    stats = pytest.importorskip("scipy.stats")
    d = scenes.make_cornell(gpu) if name == "cornell" else scenes.make_glass(gpu, level=level)
    mb = 8 if name == "cornell" else 16
    res, K, per = 32, 32, (1 << 16 if name == "cornell" else 1 << 18)
    cam = scenes.default_camera(gpu, res)
    sc = lib.Scene(d, 0, gpu)
    ctx = oracle.prepare(d)
    g, c = [], []
    try:
        for k in range(K):
            film, info, _ = sc.render(cam, per, seed_base=k * per, max_bounce=mb)
            g.append(lib.film_to_xyz(film, info)[0][..., 1])
            o = oracle.trace(d, cam, per, seed_base=(K + k) * per, max_bounce=mb, threads=os.cpu_count() or 4,
                             ctx=ctx)
            c.append(o["xyz"][..., 1])
    finally:
        oracle.L.fto_release(ctx)
        sc.close()
    g, c = np.array(g), np.array(c)
    mg, mc = g.mean(0), c.mean(0)
    se = np.sqrt(g.var(0, ddof=1) / K + c.var(0, ddof=1) / K)
    lit = se > 0
    bad = int((np.abs(mg - mc)[lit] > 3.0 * se[lit]).sum())
    p = 2.0 * stats.t.sf(3.0, K - 1)
    limit = stats.binom.isf(1e-4, int(lit.sum()), p)
    assert bad <= limit, f"{bad} of {lit.sum()} pixels beyond 3 sigma (chance allows {limit:.0f})"
    rel = mg.sum() / mc.sum() - 1.0
    assert abs(rel) < 0.005, f"mean luminance differs by {rel:.4%}"


@pytest.mark.parametrize("name,hero", [("cornell", 1), ("glass", 4), ("fog_strands", 1), ("instances", 1)])
def test_uniform_band_policy_matches_oracle(name, hero, scenes_cache, gpu, oracle):
    """FTB_LAMBDA_UNIFORM_380_780 (the build's uniform-band wavelength policy) against the
    oracle's restatement of it: per-photon paths, then film and energy."""
    mk, res, _, mb, seed, _ = cases.CASES[name]
    d, sc = scenes_cache[name]
    n = 1 << 14
    band = abi.LAMBDA_UNIFORM_380_780
    cam = cases.camera(gpu, res)
    gl = sc.trace_log(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero, lambda_mode=band)
    ol = oracle.trace(d, cam, n, seed_base=seed, max_bounce=mb, logs=True, threads=4, hero_c=hero,
                      lambda_mode=band)["logs"]
    same = (gl["n_hits"] == ol["n_hits"]) & (gl["prim_hash"] == ol["prim_hash"]) & (gl["fate"] == ol["fate"])
    assert (~same).sum() <= max(1, int(1e-5 * n)), f"{(~same).sum()} of {n} photon paths differ"
    np.testing.assert_allclose(gl["beta"][same], ol["beta"][same], rtol=1e-12, atol=0)
    film, info, en = sc.render(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero, lambda_mode=band)
    o = oracle.trace(d, cam, n, seed_base=seed, max_bounce=mb, threads=1, hero_c=hero, lambda_mode=band)
    assert_film_close(film, info, o["xyz"], o["hits"])
    np.testing.assert_allclose(en.as_list(), o["energy"], rtol=1e-9, atol=0)
    # the policy changes the film: the SPD-sampled render of the same photons differs
    film_spd, _, _ = sc.render(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
    assert not np.array_equal(film_spd, film)


@pytest.mark.parametrize("rx,ry,n,mb", [(37, 23, 20_000, 8), (1, 1, 5_000, 8), (64, 48, 20_000, 0),
                                        (24, 24, 1, 8), (24, 24, 0, 8)])
def test_ragged_and_tiny_renders_match_oracle(rx, ry, n, mb, scenes_cache, gpu, oracle):
    """Odd, non-square and one-pixel films, a one-photon and an empty render, and no
    bounces (emission splats only): film and energy equal the oracle's."""
    d, sc = scenes_cache["cornell"]
    cam = gpu.look_at((1.0, 1.0, 5.4), (1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 40.0, rx, ry)
    film, info, en = sc.render(cam, n, seed_base=4242, max_bounce=mb)
    o = oracle.trace(d, cam, n, seed_base=4242, max_bounce=mb, threads=1)
    assert film.shape == (ry, rx, 4)
    assert_film_close(film, info, o["xyz"], o["hits"])
    np.testing.assert_allclose(en.as_list(), o["energy"], rtol=1e-9, atol=0)
    if n == 0:
        assert not film.any() and not any(en.as_list())
