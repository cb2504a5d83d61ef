"""Seeded job lists of the batched and served workloads (no dataset behind them).

Batched animation: 64 frames of the dispersive-glass scene.  Per frame the glass mesh takes
a rigid rotation about a random axis (0-360 deg) and a translation of +-0.2 m from its
rest position; one BLAS is shared by all frames and each frame's top level is a refit
clone.  Frame resolutions are drawn uniformly from {256, 512, 768, 1024}^2 and photon
budgets log-uniformly from 2^22-2^27.

Served stream: jobs arrive as a Poisson process.  Each picks a scene family (Cornell,
glass, fog + strands) with a mesh size of 1k-2M triangles (log-uniform), a resolution of
128^2-1024^2 and a photon budget of 2^20-2^28 (both log-uniform).  Mesh sizes come from a
scene library of `sizes` log-spaced entries per family (a service renders the scenes it
holds, not a fresh mesh per request): glass meshes are geodesic icospheres of 20 f^2
triangles, fog + strands scenes hold n strands of 4 segments, each drawn size goes to the
nearest library entry in log scale.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import scenes


@dataclass
class Frame:
    to_world: np.ndarray   # 12 doubles
    res: int
    photons: int
    seed_base: int


def animation_frames(n_frames=64, seed=0, budget_log2=(22.0, 27.0), res_choices=(256, 512, 768, 1024),
                     max_shift=0.2):
    rng = np.random.default_rng(seed)
    out = []
    seed_base = 0
    for _ in range(n_frames):
        axis = rng.normal(size=3)
        angle = rng.uniform(0.0, 360.0)
        shift = rng.uniform(-max_shift, max_shift, size=3)
        xf = scenes.affine(axis, angle, np.asarray(scenes.GLASS_CENTER) + shift)
        res = int(rng.choice(res_choices))
        n = int(2.0 ** rng.uniform(*budget_log2))
        out.append(Frame(xf, res, n, seed_base))
        seed_base += n
    return out


def transform_tris(tv, xf):
    """World-space copy of local triangles (n x 9) under a 12-double to_world map, for the
    one-at-a-time comparison that bakes every frame like a scene load."""
    m = np.asarray(xf[:9]).reshape(3, 3)
    t = np.asarray(xf[9:12])
    p = np.asarray(tv).reshape(-1, 3)
    return (p @ m.T + t).reshape(-1, 9)


def make_glass_world(lib, level, xf, blob=None, seed=0):
    """The glass scene with the blob's triangles transformed into the world (no instance)."""
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    mat = scenes.glass_material(sb)
    tv = scenes.blob_tris(level, seed=seed) if blob is None else blob
    sb.tris(transform_tris(tv, xf), mat)
    sb.meta.update(name="glass_world", level=level)
    return sb.build(lib)


# ---- served stream --------------------------------------------------------------------
@dataclass
class Job:
    arrival_s: float
    family: str        # "cornell" | "glass" | "fog_strands"
    size: int          # glass: geodesic frequency (20 f^2 triangles); fog_strands: strand count; cornell: 0
    res: int
    photons: int
    max_bounce: int
    seed_base: int


def scene_library(sizes=24, tris_range=(1e3, 2e6)):
    """The library's mesh sizes per family: `sizes` triangle (segment) counts log-spaced over
    tris_range, as glass geodesic frequencies and fog strand counts (duplicates dropped)."""
    t = np.exp(np.linspace(math.log(tris_range[0]), math.log(tris_range[1]), sizes))
    glass = sorted({max(7, int(round(math.sqrt(x / 20.0)))) for x in t})
    fog = sorted({max(250, int(round(x / 4.0))) for x in t})
    return {"glass": glass, "fog_strands": fog, "cornell": [0]}


def mesh_tris(family, size):
    return 20 * size * size if family == "glass" else (4 * size if family == "fog_strands" else 36)


def served_jobs(n_jobs, rate_hz, seed=0, tris_range=(1e3, 2e6), res_log2=(7.0, 10.0),
                budget_log2=(20.0, 28.0), sizes=24):
    rng = np.random.default_rng(seed)
    lib_sizes = scene_library(sizes, tris_range)
    t = 0.0
    out = []
    seed_base = 0
    for _ in range(n_jobs):
        t += rng.exponential(1.0 / rate_hz)
        fam = ("cornell", "glass", "fog_strands")[int(rng.integers(0, 3))]
        tris = math.exp(rng.uniform(math.log(tris_range[0]), math.log(tris_range[1])))
        if fam == "cornell":
            size, mb = 0, 8
        else:
            size = min(lib_sizes[fam], key=lambda z: abs(math.log(mesh_tris(fam, z)) - math.log(tris)))
            mb = 16 if fam == "glass" else 32
        res = int(round(2.0 ** rng.uniform(*res_log2)))
        n = int(2.0 ** rng.uniform(*budget_log2))
        out.append(Job(t, fam, size, res, n, mb, seed_base))
        seed_base += n
    return out


def job_scene(lib, fam, size):
    if fam == "glass":
        return scenes.make_glass(lib, freq=size)
    if fam == "fog_strands":
        return scenes.make_fog_strands(lib, n_strands=size)
    return scenes.make_cornell(lib)


def fifo_latencies(arrival_s, service_s):
    """Job latencies of a server that runs one job at a time in arrival order: job i starts
    at max(its arrival, the previous job's finish) and takes service_s[i]."""
    lat = np.empty(len(arrival_s))
    free = 0.0
    for i, (a, d) in enumerate(zip(arrival_s, service_s)):
        start = max(a, free)
        free = start + d
        lat[i] = free - a
    return lat
