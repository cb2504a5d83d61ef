"""Pin the CPU oracle (oracle/ftoracle.c) to the reference.

1. Against the golden vectors in tests/golden/, produced by the reference's own tracer
   (tests/golden/make_golden.py): bit-identical film, energy report and per-photon ray
   counts / termination / final beta.
2. Against the reference built in oracle/_ref (when present): the same, live, with other
   photon ranges and with 4 threads (per-thread films merged in thread order).
The product's host-side bake (ftb_camera_look_at, ftb_emission_cdf and the emitter power)
is checked against the same golden values.
"""
import os

import numpy as np
import pytest

import cases
from goodphotons_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def test_rng_streams(oracle):
    g = golden("streams.npz")
    for k, u in zip(g["photon"], g["uniforms"]):
        np.testing.assert_array_equal(oracle.uniforms(int(k), 16), u)


def test_camera_bake(oracle, L):
    g = golden("streams.npz")["camera"]
    for cam in (oracle.look_at((1.0, 1.0, 5.4), (1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 40.0, 256, 192),
                L.look_at((1.0, 1.0, 5.4), (1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 40.0, 256, 192)):
        v = np.array(list(cam.eye) + list(cam.u) + list(cam.v) + list(cam.w) + [cam.tan_half_x, cam.tan_half_y])
        np.testing.assert_array_equal(v, g)


def test_emission_cdf_and_power(oracle, L):
    g = golden("streams.npz")
    d = scenes.make_cornell(L)
    e = d.emitters[0]
    cdf = d.emitter_cdf[e.cdf_offset:e.cdf_offset + e.cdf_n + 1]
    np.testing.assert_array_equal(cdf, g["bb_cdf"])
    assert e.power == float(g["bb_power"])
    ocdf, ointeg = oracle.emission_cdf(d, e.spd)
    np.testing.assert_array_equal(ocdf, g["bb_cdf"])
    assert ointeg == float(g["bb_integral"])


ALL_CASES = {**cases.CASES, **cases.CONFIG_CASES}


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_trace_matches_golden(name, oracle, L):
    """Small cases and the benchmark configurations at their own scene and film size."""
    mk, res, n, mb, seed, hero = ALL_CASES[name]
    g = golden(f"trace_{name}.npz")
    d = mk(L)
    assert cases.scene_hash(d) == str(g["scene_hash"]), "scene generator drifted from the golden scene"
    cam = cases.camera(L, res)
    o = oracle.trace(d, cam, n, seed_base=seed, max_bounce=mb, logs=True, rays=True, hero_c=hero)
    np.testing.assert_array_equal(o["energy"], g["energy"])
    np.testing.assert_array_equal(o["xyz"], g["xyz"])
    np.testing.assert_array_equal(o["hits"], g["hits"])
    np.testing.assert_array_equal(o["rays"], g["rays"])
    if hero == 1:   # with a bundle, absorption is booked along the way: no single fate
        np.testing.assert_array_equal(o["logs"]["fate"], g["fate"])
        np.testing.assert_array_equal(o["logs"]["beta"], g["beta"])


@pytest.mark.parametrize("name,hero", [("cornell", 1), ("materials", 1), ("fog_strands", 1), ("materials", 4),
                                       ("instances", 8), ("fog_strands", 4), ("smooth", 1)])
def test_trace_matches_reference_live(name, hero, oracle, reference, L):
    mk, res, n, mb, _, _ = cases.CASES[name]
    d = mk(L)
    cam = cases.camera(L, 48)
    for seed, threads, count in ((555, 1, 6000), (10**9, 4, 20000)):
        o = oracle.trace(d, cam, count, seed_base=seed, max_bounce=mb, threads=threads, hero_c=hero)
        r = reference.trace(d, cam, count, seed_base=seed, max_bounce=mb, threads=threads, hero_c=hero)
        np.testing.assert_array_equal(o["energy"], r["energy"])
        np.testing.assert_array_equal(o["xyz"], r["xyz"])
        np.testing.assert_array_equal(o["hits"], r["hits"])


def test_closest_hit_known_answers(oracle, reference, L):
    """Modelled on the reference's -checkbvh (main.cpp:448-473): random rays, the
    closest hit's distance and material must agree."""
    d = scenes.make_glass(L, level=3)
    octx = oracle.prepare(d)
    rctx = reference.prepare(d)
    rng = np.random.default_rng(5)
    try:
        for _ in range(3000):
            o = rng.uniform(0.05, 1.95, 3)
            dv = rng.normal(size=3)
            dv /= np.linalg.norm(dv)
            m, t = reference.closest_hit(rctx, o, dv)
            to = np.zeros(1)
            import ctypes as C
            p = oracle.L.fto_closest_hit(octx, o.ctypes.data_as(C.POINTER(C.c_double)),
                                         dv.ctypes.data_as(C.POINTER(C.c_double)), 1e-6,
                                         to.ctypes.data_as(C.POINTER(C.c_double)))
            if m < 0:
                assert p < 0
            else:
                assert to[0] == t
                assert d.tri_mat[p] == m
    finally:
        oracle.L.fto_release(octx)
        reference.L.ftr_release(rctx)


def test_curve_and_occlusion_known_answers(oracle, reference, L):
    """Modelled on the reference's -checkcurve (main.cpp:565-903) and -checkfog
    (main.cpp:2730): rays aimed into the strand ball of the fog + strands scene (round cones
    among the box's triangles); the closest hit's distance and material, and occlusion of
    random segments, must agree with the reference's own Scene::closestHit / occluded."""
    import ctypes as C
    d = scenes.make_fog_strands(L, n_strands=3000)
    nt, ns = len(d.tri_mat), len(d.sph_mat)

    def mat_of(p):
        if p < nt:
            return int(d.tri_mat[p])
        if p < nt + ns:
            return int(d.sph_mat[p - nt])
        return int(d.curve_mat[p - nt - ns])

    octx = oracle.prepare(d)
    rctx = reference.prepare(d)
    rng = np.random.default_rng(11)
    roots = d.curve[:, :3]
    curve_hits = 0
    try:
        for i in range(2000):
            o = rng.uniform(0.05, 1.95, 3)
            target = roots[rng.integers(len(roots))] + rng.normal(scale=0.002, size=3)
            dv = target - o
            dv /= np.linalg.norm(dv)
            m, t = reference.closest_hit(rctx, o, dv)
            to = np.zeros(1)
            p = oracle.L.fto_closest_hit(octx, o.ctypes.data_as(C.POINTER(C.c_double)),
                                         dv.ctypes.data_as(C.POINTER(C.c_double)), 1e-6,
                                         to.ctypes.data_as(C.POINTER(C.c_double)))
            if m < 0:
                assert p < 0
                continue
            assert to[0] == t, (i, to[0], t)
            assert mat_of(p) == m
            curve_hits += p >= nt + ns
            # occlusion of the segment up to just before / after the hit
            for frac, expect in ((0.5, 0), (1.5, 1)):
                dist = t * frac
                occ_ref = reference.L.ftr_occluded(rctx, o.ctypes.data_as(C.POINTER(C.c_double)),
                                                   dv.ctypes.data_as(C.POINTER(C.c_double)), dist)
                occ_or = oracle.L.fto_occluded(octx, o.ctypes.data_as(C.POINTER(C.c_double)),
                                               dv.ctypes.data_as(C.POINTER(C.c_double)), dist, 1e-6)
                assert occ_ref == occ_or == expect, (i, frac, occ_ref, occ_or)
        assert curve_hits > 300
    finally:
        oracle.L.fto_release(octx)
        reference.L.ftr_release(rctx)
