"""The seeded job lists behind bench.py's animation and serve records (CPU).

The serve record measures the server's capacity on a job list drawn at one arrival rate and
then paces a list drawn at 80 % of that capacity; the two must be the same jobs, only with
their arrival times scaled, or capacity, paced service and one-at-a-time rendering would be
measured on different work.  Also: the scene library's sizes, the photon streams' disjoint
seeds, and the one-job FIFO latency model."""
import math

import numpy as np

from goodphotons_b200 import workloads


def _key(j):
    return (j.family, j.size, j.res, j.photons, j.max_bounce, j.seed_base)


def test_served_jobs_are_the_same_jobs_at_any_rate():
    a = workloads.served_jobs(300, 1.0, seed=0, budget_log2=(20.0, 25.0), sizes=8)
    b = workloads.served_jobs(300, 7.5, seed=0, budget_log2=(20.0, 25.0), sizes=8)
    assert [_key(j) for j in a] == [_key(j) for j in b]
    ta = np.array([j.arrival_s for j in a])
    tb = np.array([j.arrival_s for j in b])
    np.testing.assert_allclose(tb, ta / 7.5, rtol=1e-12)
    assert np.all(np.diff(ta) > 0)


def test_served_jobs_draw_within_their_ranges_and_from_the_library():
    lib_sizes = workloads.scene_library(24)
    jobs = workloads.served_jobs(2000, 5.0, seed=3)
    fams = {j.family for j in jobs}
    assert fams == {"cornell", "glass", "fog_strands"}
    for j in jobs:
        assert j.size in lib_sizes[j.family]
        assert 128 <= j.res <= 1024
        assert 2 ** 20 <= j.photons <= 2 ** 28
    # photon ranges of consecutive jobs follow one another: no two jobs share a photon
    starts = np.array([j.seed_base for j in jobs])
    counts = np.array([j.photons for j in jobs])
    np.testing.assert_array_equal(starts[1:], starts[:-1] + counts[:-1])


def test_scene_library_spans_the_mesh_range():
    lib_sizes = workloads.scene_library(24, (1e3, 2e6))
    for fam in ("glass", "fog_strands"):
        tris = [workloads.mesh_tris(fam, z) for z in lib_sizes[fam]]
        assert tris == sorted(tris) and len(set(tris)) == len(tris)
        assert tris[0] <= 1.5e3 and tris[-1] >= 1.8e6
        # log-spaced: neighbouring entries differ by a bounded factor
        assert max(b / a for a, b in zip(tris, tris[1:])) < 2.0
    assert lib_sizes["cornell"] == [0]


def test_fifo_latencies():
    arr = [0.0, 0.5, 0.6, 5.0]
    svc = [1.0, 1.0, 0.2, 0.5]
    lat = workloads.fifo_latencies(arr, svc)
    # job 0 runs 0-1; job 1 waits, runs 1-2; job 2 runs 2-2.2; job 3 arrives to an idle server
    np.testing.assert_allclose(lat, [1.0, 1.5, 1.6, 0.5])


def test_animation_frames_are_seeded_and_bounded():
    a = workloads.animation_frames(64, seed=0)
    b = workloads.animation_frames(64, seed=0)
    assert len(a) == 64
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.to_world, y.to_world)
        assert (x.res, x.photons, x.seed_base) == (y.res, y.photons, y.seed_base)
        assert x.res in (256, 512, 768, 1024)
        assert 2 ** 22 <= x.photons <= 2 ** 27
        m = np.asarray(x.to_world[:9]).reshape(3, 3)
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-12)   # a rigid rotation
        assert math.isclose(np.linalg.det(m), 1.0, rel_tol=1e-12)
