"""Multi-rank host logic on CPU (gloo, world size 2): photon-index shards cover the frame
once, every rank uses the frame's fixed-point format, and the frame-end sum of int64 films
and tallies is exactly the single-process film.  The render itself is a stand-in that adds
a deterministic fixed-point contribution per photon index (no GPU here)."""
import os
import socket
import types

import numpy as np
import pytest

from goodphotons_b200 import multigpu

RES = 16
N = 100_003


def contributions(first, count, frac):
    """Stand-in splats: photon k lands on pixel hash(k) with a value depending on k and frac."""
    k = np.arange(first, first + count, dtype=np.int64)
    pix = (k * 2654435761) % (RES * RES)
    val = ((k * 40503) % 9973 + 1) << (frac - 20)
    film = np.zeros((RES * RES, 4), dtype=np.int64)
    for c in range(3):
        np.add.at(film[:, c], pix, val * (c + 1))
    np.add.at(film[:, 3], pix, 1)
    return film.reshape(RES, RES, 4)


class FakeScene:
    """Records the call and writes the stand-in splats into the film tensor it was given."""

    def __init__(self, film):
        self.film = film
        self.calls = []

    def render_device(self, cam, n, d_film_ptr, seed_base=0, max_bounce=8, frac_bits=0, stream=None,
                      want_energy=False, hero_c=1, lambda_mode=0):
        import torch
        assert d_film_ptr == self.film.data_ptr()
        self.calls.append((n, seed_base, frac_bits))
        self.film += torch.from_numpy(contributions(seed_base, n, frac_bits))
        fx = [n << 32, 3 * n, 0, 5 * n, 7]
        return None, types.SimpleNamespace(fx=fx)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        film = torch.zeros((RES, RES, 4), dtype=torch.int64)
        sc = FakeScene(film)
        tally = multigpu.render_sharded(sc, None, N, film, seed_base=1000, max_bounce=8)
        q.put((rank, sc.calls, film.numpy().copy(), tally.numpy().copy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shards_partition_the_frame():
    for n in (0, 1, 7, 100_003, 1 << 28):
        for world in (1, 2, 3, 8):
            parts = [multigpu.shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0
            assert sum(c for _, c in parts) == n
            for (f0, c0), (f1, _) in zip(parts, parts[1:]):
                assert f0 + c0 == f1


def test_default_frac_bits_formula():
    assert multigpu.default_frac_bits(1 << 28) == 62 - 28 - 20
    assert multigpu.default_frac_bits((1 << 24) + 1) == 62 - 25 - 20
    assert multigpu.default_frac_bits(1) == 40
    assert multigpu.default_frac_bits(1 << 60) == 4


def test_two_rank_reduce_equals_one_process():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(2):
        rank, calls, film, tally = q.get(timeout=120)
        out[rank] = (calls, film, tally)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    frac = multigpu.default_frac_bits(N)
    (c0, f0, t0), (c1, f1, t1) = out[0], out[1]
    assert c0 == [(N // 2, 1000, frac)]
    assert c1 == [(N - N // 2, 1000 + N // 2, frac)]
    whole = contributions(1000, N, frac)
    np.testing.assert_array_equal(f0, whole)
    np.testing.assert_array_equal(f1, whole)
    np.testing.assert_array_equal(t0, [N << 32, 3 * N, 0, 5 * N, 14])
    np.testing.assert_array_equal(t0, t1)
