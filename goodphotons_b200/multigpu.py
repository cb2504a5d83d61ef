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


class ServerPool:
    """Serving on several GPUs of one node: one render server per device (replicas of the
    scene library), each job sent whole to one device -- the one with the least photons
    queued or running -- so jobs never span GPUs and no collective is involved (a job's film
    is its server's, exactly what one GPU renders for it).

    `scene_of(key, device)` returns the resident scene of library entry `key` on `device`
    (it is asked once per pair and the result kept); `server_cfg` goes to every server
    (max_active, hbm_budget, ...).  `make_server(device, **cfg)` builds a server (the
    library's lib.Server by default)."""

    def __init__(self, devices, scene_of, lib=None, make_server=None, **server_cfg):
        if not devices:
            raise ValueError("no devices")
        if make_server is None:
            from . import lib as lib_mod
            L = lib or lib_mod.load()

            def make_server(device, **cfg):
                return lib_mod.Server(device=device, lib=L, **cfg)
        self.devices = list(devices)
        self.servers = {d: make_server(d, **server_cfg) for d in self.devices}
        self.scene_of = scene_of
        self.scenes = {}
        self.load = {d: 0 for d in self.devices}   # photons submitted and not yet waited on
        self.jobs = {}                              # handle -> (device, server job id, photons)
        self.next_handle = 1

    def pick(self):
        """The device with the least outstanding photons (ties to the first listed)."""
        return min(self.devices, key=lambda d: (self.load[d], self.devices.index(d)))

    def submit(self, key, cam, n, **kw):
        d = self.pick()
        if (key, d) not in self.scenes:
            self.scenes[(key, d)] = self.scene_of(key, d)
        jid = self.servers[d].submit(self.scenes[(key, d)], cam, n, **kw)
        h = self.next_handle
        self.next_handle += 1
        self.jobs[h] = (d, jid, n)
        self.load[d] += n
        return h

    def device_of(self, handle):
        return self.jobs[handle][0]

    def wait(self, handle, timeout=-1.0):
        d, jid, n = self.jobs[handle]
        r = self.servers[d].wait(jid, timeout)
        del self.jobs[handle]
        self.load[d] -= n
        return r

    def close(self):
        for s in self.servers.values():
            s.close()
        self.servers = {}
