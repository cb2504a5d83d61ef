"""GPU parity at the benchmark configurations' own size.

The small cases of test_gpu_parity.py exercise every branch on 32^2 films and scenes of a
few hundred primitives.  The benchmarked scenes are much larger -- level-7 and level-8
glass (327,680 and 1,310,720 triangles) at 1024^2, fog with 250k strands (1M round cones)
at 512^2 and 32 bounces, the Cornell box at 256^2 -- and that is where the fp32 culling
margins (grown with the scene's largest coordinate), the quantized child planes and the
traversal stack depth are stressed.  So here, at those sizes:

  * films and energy reports equal the reference's own golden vectors (made by its CPU
    tracer from these exact scenes, tests/golden/make_golden.py);
  * every photon's hit-primitive sequence, bounce count and termination equal the oracle's
    on 2^15 photons, with the host-built and the GPU-built hierarchies, allowing
    max(1, 1e-5 n) mismatches (grazing hits) and 1e-12 relative on the final beta.  Among
    the strands, a ray can meet the joint of two consecutive segments of a strand, where
    both round cones pass through the same point and their distances agree to ~1e-16 m; a
    last-bit difference in the ray (CUDA's sin/cos/log against glibc's) can then decide
    which segment is reported, with the same path afterwards.  Those photons are counted
    apart (cases.joint_ties) and bounded by 1e-4 n; measured: 4 of 131072 photons of the
    fog + 250k strands configuration, none elsewhere;
  * the statistical film criterion on the configurations' full films: independent photons
    on each side (GPU indices [0, N), oracle [N, 2N)), K = 32 batches, per-pixel means of Y
    compared in units of their combined standard error -- the count of lit pixels beyond
    3 sigma must stay within chance (binomial tail 1e-4 at the Student-t rate), and the
    mean luminance must agree within 0.5 %.
"""
import os

import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="module")
def config_scenes(gpu):
    out = {}
    for name, (mk, *_rest) in cases.CONFIG_CASES.items():
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


def same_paths(gl, ol):
    return (gl["n_hits"] == ol["n_hits"]) & (gl["prim_hash"] == ol["prim_hash"]) & (gl["fate"] == ol["fate"])


@pytest.mark.parametrize("name", sorted(cases.CONFIG_CASES))
def test_config_film_and_energy_match_reference_golden(name, config_scenes, gpu):
    mk, res, n, mb, seed, hero = cases.CONFIG_CASES[name]
    d, sc = config_scenes[name]
    g = golden(f"trace_{name}.npz")
    assert cases.scene_hash(d) == str(g["scene_hash"])
    cam = cases.camera(gpu, res)
    film, info, en = sc.render(cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
    assert_film_close(film, info, g["xyz"], g["hits"])
    np.testing.assert_allclose(en.as_list(), g["energy"], rtol=1e-9, atol=0)


@pytest.mark.parametrize("build", ["host_sah", "device"])
@pytest.mark.parametrize("name", sorted(cases.CONFIG_CASES))
def test_config_per_photon_paths_match_oracle(name, build, config_scenes, gpu, oracle):
    mk, res, _, mb, seed, hero = cases.CONFIG_CASES[name]
    d, sc = config_scenes[name]
    own = None
    if build == "device":
        own = sc = lib.Scene(d, 0, gpu, build=abi.BUILD_DEVICE)
    n = 1 << 15
    cam = cases.camera(gpu, res)
    try:
        gl = sc.trace_log(cam, n, seed_base=seed + 12345, max_bounce=mb, hero_c=hero)
    finally:
        if own is not None:
            own.close()
    ol = oracle.trace(d, cam, n, seed_base=seed + 12345, max_bounce=mb, logs=True, threads=os.cpu_count() or 4,
                      hero_c=hero)["logs"]
    same = same_paths(gl, ol)
    bad = np.nonzero(~same)[0]
    ties = cases.joint_ties(d, gl, ol, bad)
    other = [int(i) for i in bad if int(i) not in set(ties)]
    allowed = max(1, int(1e-5 * n))
    assert len(other) <= allowed, f"{len(other)} of {n} photon paths differ (besides joint ties); first {other[:5]}"
    assert len(ties) <= max(1, int(1e-4 * n)), f"{len(ties)} strand-joint ties of {n}"
    np.testing.assert_allclose(gl["beta"][same], ol["beta"][same], rtol=1e-12, atol=0)
    np.testing.assert_array_equal(gl["prims"][same], ol["prims"][same])
    assert gl["n_hits"].mean() > 1.0   # the photons do bounce in these scenes


@pytest.mark.parametrize("name", ["cfg_glass_l7", "cfg_fog_strands"])
def test_config_film_statistics_full_film(name, config_scenes, gpu, oracle):
    stats = pytest.importorskip("scipy.stats")
    mk, res, _, mb, _, _ = cases.CONFIG_CASES[name]
    d, sc = config_scenes[name]
    K, per = 32, 1 << 19
    cam = cases.camera(gpu, res)
    ctx = oracle.prepare(d)
    g, c = [], []
    try:
        for k in range(K):
            film, info, _ = sc.render(cam, per, seed_base=k * per, max_bounce=mb)
            g.append(lib.film_to_xyz(film, info)[0][..., 1].astype(np.float32))
            o = oracle.trace(d, cam, per, seed_base=(K + k) * per, max_bounce=mb, threads=os.cpu_count() or 4,
                             ctx=ctx)
            c.append(o["xyz"][..., 1].astype(np.float32))
    finally:
        oracle.L.fto_release(ctx)
    g = np.array(g, dtype=np.float64)
    c = np.array(c, dtype=np.float64)
    mg, mc = g.mean(0), c.mean(0)
    se = np.sqrt(g.var(0, ddof=1) / K + c.var(0, ddof=1) / K)
    lit = se > 0
    assert lit.sum() > 0.25 * res * res   # most of the film is lit
    bad = int((np.abs(mg - mc)[lit] > 3.0 * se[lit]).sum())
    p = 2.0 * stats.t.sf(3.0, K - 1)
    limit = stats.binom.isf(1e-4, int(lit.sum()), p)
    assert bad <= limit, f"{bad} of {lit.sum()} pixels beyond 3 sigma (chance allows {limit:.0f})"
    rel = mg.sum() / mc.sum() - 1.0
    assert abs(rel) < 0.005, f"mean luminance differs by {rel:.4%}"
