"""Photon-index sharding across GPUs (one process per GPU, torch.distributed for plumbing).

Photons are independent and keyed by their absolute index, so a frame of N photons splits
into contiguous index ranges, one per rank: rank g traces [g*N/G, (g+1)*N/G) with the same
per-photon seeding, and the realisation is identical to a single-GPU render of all N.
The only exchange is one sum of the int64 fixed-point films (and of the five energy
tallies) at frame end; integer addition is exact and order-free, so the reduced film is
bit-identical to the single-GPU film.  All ranks must use the same fixed-point format,
sized for the whole frame (default_frac_bits(N)), not for their shard.
"""
from __future__ import annotations


def default_frac_bits(n):
    """The library's default film format for an n-photon frame: 62 - ceil(log2 n) - 20,
    clamped to [4, 40] (ftb_render_params.frac_bits = 0)."""
    lg = 0
    while lg < 62 and (1 << lg) < n:
        lg += 1
    return max(4, min(40, 62 - lg - 20))


def shard(n, rank, world):
    """(first photon, count) of rank's contiguous share of an n-photon frame."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    first = rank * n // world
    return first, (rank + 1) * n // world - first


def reduce_film(film, tally=None, dst=None, group=None):
    """Sum the int64 films (and the int64 energy tallies) of all ranks: into every rank
    (dst None, all-reduce) or into rank dst."""
    import torch
    import torch.distributed as dist
    if film.dtype != torch.int64:
        raise TypeError("films are int64 fixed point")
    ts = [film] + ([tally] if tally is not None else [])
    for t in ts:
        if dst is None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        else:
            dist.reduce(t, dst=dst, op=dist.ReduceOp.SUM, group=group)


def render_sharded(scene, cam, n, film, seed_base=0, max_bounce=8, frac_bits=0, dst=None,
                   group=None, stream=None, hero_c=1, lambda_mode=0):
    """This rank's share of an n-photon frame into the device film `film` (int64 tensor of
    shape [res_y, res_x, 4]), then the frame-end sum over ranks.  Returns the frame's
    energy tallies (int64 tensor of 5, fixed point with 32 fraction bits per unit of the
    scene's power) after the same reduction."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    first, count = shard(n, rank, world)
    frac = frac_bits or default_frac_bits(n)
    _, en = scene.render_device(cam, count, film.data_ptr(), seed_base=seed_base + first,
                                max_bounce=max_bounce, frac_bits=frac, stream=stream, want_energy=True,
                                hero_c=hero_c, lambda_mode=lambda_mode)
    tally = torch.tensor([int(x) - (1 << 64) if x >= (1 << 63) else int(x) for x in en.fx],
                         dtype=torch.int64, device=film.device)
    reduce_film(film, tally, dst=dst, group=group)
    return tally
