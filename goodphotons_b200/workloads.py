"""Seeded job lists of the batched and served workloads (no dataset behind them).

Batched animation: 64 frames of the dispersive-glass scene.  Per frame the glass mesh takes
a rigid rotation about a random axis (0-360 deg) and a translation of +-0.2 m from its
rest position; one BLAS is shared by all frames and each frame's top level is a refit
clone.  Frame resolutions are drawn uniformly from {256, 512, 768, 1024}^2 and photon
budgets log-uniformly from 2^22-2^27.

Served stream: jobs arrive as a Poisson process.  Each picks a scene family (Cornell,
glass, fog + strands) with a mesh size of 1k-2M triangles (log-uniform; glass meshes are
icospheres, so the size snaps to a subdivision level and scenes are shared), a resolution
of 128^2-1024^2 and a photon budget of 2^20-2^28 (both log-uniform).
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
GLASS_LEVELS = {3: 1280, 4: 5120, 5: 20480, 6: 81920, 7: 327680, 8: 1310720}


@dataclass
class Job:
    arrival_s: float
    family: str        # "cornell" | "glass" | "fog_strands"
    size: int          # glass: icosphere level; fog_strands: strand count; cornell: 0
    res: int
    photons: int
    max_bounce: int
    seed_base: int


def _snap_level(tris):
    return min(GLASS_LEVELS, key=lambda lv: abs(math.log(GLASS_LEVELS[lv]) - math.log(tris)))


def served_jobs(n_jobs, rate_hz, seed=0, tris_range=(1e3, 2e6), res_log2=(7.0, 10.0),
                budget_log2=(20.0, 28.0)):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    seed_base = 0
    for _ in range(n_jobs):
        t += rng.exponential(1.0 / rate_hz)
        fam = ("cornell", "glass", "fog_strands")[int(rng.integers(0, 3))]
        tris = math.exp(rng.uniform(math.log(tris_range[0]), math.log(tris_range[1])))
        if fam == "glass":
            size, mb = _snap_level(tris), 16
        elif fam == "fog_strands":
            # curve segments stand for the mesh size: 4 per strand, snapped to powers of 4
            strands = max(250, int(tris / 4))
            size, mb = int(4 ** round(math.log(strands, 4))), 32
        else:
            size, mb = 0, 8
        res = int(round(2.0 ** rng.uniform(*res_log2)))
        n = int(2.0 ** rng.uniform(*budget_log2))
        out.append(Job(t, fam, size, res, n, mb, seed_base))
        seed_base += n
    return out


def job_scene(lib, fam, size):
    if fam == "glass":
        return scenes.make_glass(lib, level=size)
    if fam == "fog_strands":
        return scenes.make_fog_strands(lib, n_strands=size)
    return scenes.make_cornell(lib)
