"""Scene descriptions for the forward light tracer.

`SceneBuilder` assembles the POD arrays of `ftb_scene_desc` (include/ftb200.h) the way the
reference's loaders fill `Scene` after FTSL load: a `quad` is two triangles
(o, o+u, o+u+v) and (o, o+u+v, o+v); an area light is an emitter plus two emissive
triangles with a black diffuse material (ftsl.h:6195-6222).

The synthetic workloads below are seeded stand-ins for the benchmark scenes (there is no
dataset behind them): a Cornell box, a dispersive noisy icosphere in the same box, and a
fog-filled box holding a ball of hair strands.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi

LAMBDA_MIN, LAMBDA_MAX = 360.0, 830.0


def _as_ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None and a.size else None


class SceneDesc:
    """Owns the numpy arrays behind an `ftb_scene_desc` and the struct itself."""

    def __init__(self, tri_v, tri_n, tri_mat, sph, sph_mat, curve, curve_mat, mats,
                 spectra, table_w, table_v, emitters, emitter_cdf, media, meta=None,
                 blas=(), instances=()):
        self.tri_v = np.ascontiguousarray(tri_v, dtype=np.float64).reshape(-1, 9)
        self.tri_n = None if tri_n is None else np.ascontiguousarray(tri_n, np.float64).reshape(-1, 9)
        self.tri_mat = np.ascontiguousarray(tri_mat, dtype=np.int32)
        self.sph = np.ascontiguousarray(sph, dtype=np.float64).reshape(-1, 4)
        self.sph_mat = np.ascontiguousarray(sph_mat, dtype=np.int32)
        self.curve = np.ascontiguousarray(curve, dtype=np.float64).reshape(-1, 10)
        self.curve_mat = np.ascontiguousarray(curve_mat, dtype=np.int32)
        self.mats = (abi.Material * max(1, len(mats)))(*mats)
        self.n_mats = len(mats)
        self.spectra = (abi.Spectrum * max(1, len(spectra)))(*spectra)
        self.n_spectra = len(spectra)
        self.table_w = np.ascontiguousarray(table_w, dtype=np.float64)
        self.table_v = np.ascontiguousarray(table_v, dtype=np.float64)
        self.emitters = (abi.Emitter * max(1, len(emitters)))(*emitters)
        self.n_emitters = len(emitters)
        self.emitter_cdf = np.ascontiguousarray(emitter_cdf, dtype=np.float64)
        self.media = (abi.Medium * max(1, len(media)))(*media)
        self.n_media = len(media)
        self.meta = dict(meta or {})
        # BLAS assets: (tri_v, tri_n or None, tri_mat, handle or None)
        self.blas_arrays = []
        for tv, tn, tm, handle in blas:
            tv = np.ascontiguousarray(tv, dtype=np.float64).reshape(-1, 9)
            tn = None if tn is None else np.ascontiguousarray(tn, np.float64).reshape(-1, 9)
            tm = np.ascontiguousarray(tm, dtype=np.int32)
            self.blas_arrays.append((tv, tn, tm, handle))
        self.blas = (abi.BlasDesc * max(1, len(self.blas_arrays)))()
        for i, (tv, tn, tm, handle) in enumerate(self.blas_arrays):
            b = self.blas[i]
            b.n_tris = len(tv)
            b.tri_v = _as_ptr(tv, C.c_double)
            b.tri_n = _as_ptr(tn, C.c_double) if tn is not None else None
            b.tri_mat = _as_ptr(tm, C.c_int32)
            b.handle = handle.h.value if handle is not None else None
        self.n_blas = len(self.blas_arrays)
        self.instances = (abi.Instance * max(1, len(instances)))(*instances)
        self.n_instances = len(instances)
        d = abi.SceneDesc()
        d.n_tris = len(self.tri_v)
        d.tri_v = _as_ptr(self.tri_v, C.c_double)
        d.tri_n = _as_ptr(self.tri_n, C.c_double) if self.tri_n is not None else None
        d.tri_mat = _as_ptr(self.tri_mat, C.c_int32)
        d.n_spheres = len(self.sph)
        d.sph = _as_ptr(self.sph, C.c_double)
        d.sph_mat = _as_ptr(self.sph_mat, C.c_int32)
        d.n_curves = len(self.curve)
        d.curve = _as_ptr(self.curve, C.c_double)
        d.curve_mat = _as_ptr(self.curve_mat, C.c_int32)
        d.n_mats = self.n_mats
        d.n_spectra = self.n_spectra
        d.mats = C.cast(self.mats, C.POINTER(abi.Material))
        d.spectra = C.cast(self.spectra, C.POINTER(abi.Spectrum))
        d.n_table = len(self.table_w)
        d.table_w = _as_ptr(self.table_w, C.c_double)
        d.table_v = _as_ptr(self.table_v, C.c_double)
        d.n_emitters = self.n_emitters
        d.n_media = self.n_media
        d.emitters = C.cast(self.emitters, C.POINTER(abi.Emitter))
        d.emitter_cdf = _as_ptr(self.emitter_cdf, C.c_double)
        d.media = C.cast(self.media, C.POINTER(abi.Medium))
        d.n_blas = self.n_blas
        d.blas = C.cast(self.blas, C.POINTER(abi.BlasDesc))
        d.n_instances = self.n_instances
        d.instances = C.cast(self.instances, C.POINTER(abi.Instance))
        self.desc = d

    @property
    def n_prims(self):
        return len(self.tri_v) + len(self.sph) + len(self.curve) + self.n_instances

    def ref(self):
        return C.byref(self.desc)

    def total_power(self):
        """Scene::totalPower (scene.h:1509-1511): sum in emitter order."""
        tp = 0.0
        for i in range(self.n_emitters):
            tp += self.emitters[i].power
        return tp


class SceneBuilder:
    def __init__(self):
        self.tri_v, self.tri_n, self.tri_mat = [], [], []
        self.sph, self.sph_mat = [], []
        self.curve, self.curve_mat = [], []
        self.mats, self.spectra = [], []
        self.table_w, self.table_v = [], []
        self.emitter_specs = []   # (Emitter, spd index)
        self.media = []
        self.meta = {}
        self._smooth = False
        self.blas_list = []     # (tri_v, tri_n, tri_mat, handle)
        self.instance_list = []

    # -- spectra ----------------------------------------------------------------------
    def _spec(self, kind, p=(), n=0, offset=0):
        s = abi.Spectrum()
        s.kind, s.n, s.offset = kind, n, offset
        for i, v in enumerate(p):
            s.p[i] = float(v)
        self.spectra.append(s)
        return len(self.spectra) - 1

    def const(self, v):
        return self._spec(abi.SPEC_CONST, (v,))

    def table(self, pairs):
        pairs = sorted((float(w), float(v)) for w, v in pairs)
        ws = [w for w, _ in pairs]
        if len(set(ws)) != len(ws):
            raise ValueError("table spectra need distinct wavelengths")
        off = len(self.table_w)
        self.table_w += ws
        self.table_v += [v for _, v in pairs]
        return self._spec(abi.SPEC_TABLE, (), len(pairs), off)

    def cauchy(self, a, b):
        return self._spec(abi.SPEC_CAUCHY, (a, b))

    def sellmeier(self, b1, b2, b3, c1, c2, c3):
        return self._spec(abi.SPEC_SELLMEIER, (b1, b2, b3, c1, c2, c3))

    def blackbody(self, kelvin, scale=1.0):
        return self._spec(abi.SPEC_BLACKBODY, (kelvin, scale))

    # -- materials ----------------------------------------------------------------------
    def material(self, mtype, reflect=-1, ior=-1, absorb=-1, transmit=-1, roughness=0.0,
                 priority=abi.PRIORITY_UNSET):
        m = abi.Material()
        m.type, m.priority = mtype, priority
        m.reflect, m.ior, m.absorb, m.transmit = reflect, ior, absorb, transmit
        m.roughness = float(roughness)
        self.mats.append(m)
        return len(self.mats) - 1

    def diffuse(self, reflect_spec):
        return self.material(abi.MAT_DIFFUSE, reflect=reflect_spec)

    # -- geometry -----------------------------------------------------------------------
    def tris(self, v, mat, normals=None):
        v = np.asarray(v, dtype=np.float64).reshape(-1, 9)
        self.tri_v.append(v)
        self.tri_mat.append(np.full(len(v), mat, dtype=np.int32))
        if normals is not None:
            self._smooth = True
            self.tri_n.append(np.asarray(normals, np.float64).reshape(-1, 9))
        else:
            self.tri_n.append(np.zeros((len(v), 9)))

    def quad(self, o, u, v, mat):
        o, u, v = (np.asarray(x, dtype=np.float64) for x in (o, u, v))
        a, b, c, d = o, o + u, o + u + v, o + v
        self.tris(np.stack([np.concatenate([a, b, c]), np.concatenate([a, c, d])]), mat)

    def sphere(self, c, r, mat):
        self.sph.append([c[0], c[1], c[2], r])
        self.sph_mat.append(mat)

    def curves(self, segs, mat):
        """segs: (n, 10) p0 p1 r0 r1 u0 u1"""
        segs = np.asarray(segs, dtype=np.float64).reshape(-1, 10)
        self.curve.append(segs)
        self.curve_mat.append(np.full(len(segs), mat, dtype=np.int32))

    def blas(self, v, mat, normals=None, handle=None):
        """A triangle asset in its own local space (Blas, scene.h:996); returns its index.
        `handle` (lib.Blas) shares an already baked device copy of the same triangles."""
        v = np.asarray(v, dtype=np.float64).reshape(-1, 9)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(mat, np.int32), (len(v),)))
        self.blas_list.append((v, normals, m, handle))
        return len(self.blas_list) - 1

    def instance(self, blas, to_world, mat_override=-1):
        """Place BLAS `blas` by the affine `to_world` (12 doubles: 3x3 row-major, then the
        translation; MeshInstance, scene.h:1035); returns the instance index."""
        inst = abi.Instance()
        inst.blas = blas
        inst.mat_override = mat_override
        for i, x in enumerate(np.asarray(to_world, dtype=np.float64).reshape(12)):
            inst.to_world[i] = float(x)
        self.instance_list.append(inst)
        return len(self.instance_list) - 1

    def box(self, center_xz, size, height, angle_deg, mat, y0=0.0):
        """Axis-aligned-in-y box (12 triangles) rotated about +y, outward winding."""
        hx, hz = size[0] / 2.0, size[1] / 2.0
        th = math.radians(angle_deg)
        cs, sn = math.cos(th), math.sin(th)

        def P(x, y, z):
            return np.array([center_xz[0] + cs * x + sn * z, y0 + y,
                             center_xz[1] - sn * x + cs * z])
        c = [P(sx * hx, sy * height, sz * hz) for sy in (0, 1) for sz in (-1, 1) for sx in (-1, 1)]
        # c index: (y, z, x) bits -> 0:(-x,-z,b) 1:(+x,-z,b) 2:(-x,+z,b) 3:(+x,+z,b), +4 top
        faces = [(4, 5, 7, 6), (0, 2, 3, 1), (2, 6, 7, 3), (0, 1, 5, 4), (1, 3, 7, 5), (0, 4, 6, 2)]
        out = []
        for a, b, cc, d in faces:   # reversed order: counter-clockwise seen from outside
            out.append(np.concatenate([c[a], c[cc], c[b]]))
            out.append(np.concatenate([c[a], c[d], c[cc]]))
        self.tris(np.stack(out), mat)

    # -- lights -------------------------------------------------------------------------
    def area_light(self, o, u, v, normal, spd, step=1.0, geometry=True, collimated=False,
                   beam=(1.0, 0.0, 0.0)):
        """`light area { ... }` (ftsl.h:6195-6222)."""
        o, u, v = (np.asarray(x, dtype=np.float64) for x in (o, u, v))
        e = abi.Emitter()
        e.shape = abi.EMIT_QUAD
        e.collimated = 1 if collimated else 0
        e.spd = spd
        e.step = float(step)
        cr = np.cross(u, v)
        e.area = float(math.sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]))
        for i in range(3):
            e.origin[i], e.u[i], e.v[i], e.normal[i], e.beam[i] = o[i], u[i], v[i], normal[i], beam[i]
        if geometry:
            lm = self.material(abi.MAT_DIFFUSE, reflect=self.const(0.0))
            self.quad(o, u, v, lm)
        self.emitter_specs.append(e)
        return len(self.emitter_specs) - 1

    def sphere_light(self, c, r, spd, step=1.0):
        e = abi.Emitter()
        e.shape = abi.EMIT_SPHERE
        e.spd = spd
        e.step = float(step)
        e.radius = float(r)
        e.area = 4.0 * math.pi * r * r
        for i in range(3):
            e.origin[i] = c[i]
        self.emitter_specs.append(e)
        return len(self.emitter_specs) - 1

    def medium(self, sigma_a, sigma_s, g, bmin=None, bmax=None, center=None, radius=None):
        m = abi.Medium()
        m.sigma_a, m.sigma_s, m.g = sigma_a, sigma_s, float(g)
        if bmin is not None:
            m.bound = abi.BOUND_BOX
            for i in range(3):
                m.bmin[i], m.bmax[i] = bmin[i], bmax[i]
        elif center is not None:
            m.bound = abi.BOUND_SPHERE
            for i in range(3):
                m.center[i] = center[i]
            m.radius = float(radius)
        self.media.append(m)
        return len(self.media) - 1

    # -- finish -------------------------------------------------------------------------
    def build(self, lib=None) -> SceneDesc:
        """Bake emitter CDFs and powers through the library (ftb_emission_cdf), which uses
        the reference's EmissionSampler arithmetic, and return the descriptor."""
        from . import lib as _lib
        L = lib or _lib.load()
        tri_v = np.concatenate(self.tri_v) if self.tri_v else np.zeros((0, 9))
        tri_mat = np.concatenate(self.tri_mat) if self.tri_mat else np.zeros(0, np.int32)
        tri_n = (np.concatenate(self.tri_n) if self._smooth else None)
        curve = np.concatenate(self.curve) if self.curve else np.zeros((0, 10))
        curve_mat = np.concatenate(self.curve_mat) if self.curve_mat else np.zeros(0, np.int32)
        sph = np.asarray(self.sph, dtype=np.float64).reshape(-1, 4)
        sph_mat = np.asarray(self.sph_mat, dtype=np.int32)
        # a temporary descriptor that only carries the spectra, for the CDF bake
        tmp = SceneDesc(np.zeros((0, 9)), None, np.zeros(0), np.zeros((0, 4)), np.zeros(0),
                        np.zeros((0, 10)), np.zeros(0), [], self.spectra, self.table_w,
                        self.table_v, [], np.zeros(0), [])
        cdfs, emitters = [], []
        off = 0
        for e in self.emitter_specs:
            cdf, integral = L.emission_cdf(tmp, e.spd, e.step)
            e.cdf_n = len(cdf) - 1
            e.cdf_offset = off
            off += len(cdf)
            e.power = integral * e.area * math.pi   # emitIntegral*area*PI (scene.h:1509)
            cdfs.append(cdf)
            emitters.append(e)
        cdf_all = np.concatenate(cdfs) if cdfs else np.zeros(0)
        return SceneDesc(tri_v, tri_n, tri_mat, sph, sph_mat, curve, curve_mat, self.mats,
                         self.spectra, self.table_w, self.table_v, emitters, cdf_all,
                         self.media, self.meta, blas=self.blas_list, instances=self.instance_list)


def affine(axis=(0.0, 1.0, 0.0), angle_deg=0.0, translate=(0.0, 0.0, 0.0), scale=1.0):
    """12-double to_world map: rotation by angle_deg about `axis` (Rodrigues), a uniform
    scale, then the translation."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    th = math.radians(angle_deg)
    c, s = math.cos(th), math.sin(th)
    x, y, z = a
    R = np.array([[c + x * x * (1 - c), x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                  [y * x * (1 - c) + z * s, c + y * y * (1 - c), y * z * (1 - c) - x * s],
                  [z * x * (1 - c) - y * s, z * y * (1 - c) + x * s, c + z * z * (1 - c)]]) * scale
    return np.concatenate([R.reshape(9), np.asarray(translate, dtype=np.float64)])


# ---------------------------------------------------------------------------------------
# Synthetic workloads
# ---------------------------------------------------------------------------------------
def _step_table(lo, hi, on=0.75, off=0.05, ramp=0.01):
    """Reflectance `on` over [lo, hi] nm and `off` elsewhere, as table breakpoints with a
    `ramp`-nm linear edge."""
    return [(LAMBDA_MIN, off), (lo - ramp, off), (lo, on), (hi, on), (hi + ramp, off),
            (LAMBDA_MAX, off)]


def cornell_box(sb: SceneBuilder, boxes=True, light_kelvin=6500.0, ramp=0.01):
    """2x2x2 m box of 5 quads (open at +z), 0.5x0.5 m blackbody ceiling light."""
    white = sb.diffuse(sb.const(0.75))
    red = sb.diffuse(sb.table(_step_table(600.0, 780.0, ramp=ramp)))
    green = sb.diffuse(sb.table(_step_table(500.0, 570.0, ramp=ramp)))
    sb.quad((0, 0, 0), (0, 0, 2), (2, 0, 0), white)    # floor (+y)
    sb.quad((0, 2, 0), (2, 0, 0), (0, 0, 2), white)    # ceiling (-y)
    sb.quad((0, 0, 0), (2, 0, 0), (0, 2, 0), white)    # back (+z)
    sb.quad((0, 0, 0), (0, 2, 0), (0, 0, 2), red)      # left (+x)
    sb.quad((2, 0, 0), (0, 0, 2), (0, 2, 0), green)    # right (-x)
    if boxes:
        sb.box((1.4, 1.35), (0.6, 0.6), 0.6, 17.0, white)
        sb.box((0.6, 0.6), (0.6, 0.6), 1.2, -17.0, white)
    bb = sb.blackbody(light_kelvin)
    sb.area_light((0.75, 1.998, 0.75), (0.5, 0, 0), (0, 0, 0.5), (0, -1, 0), bb)
    return white


def default_camera(lib, res):
    return lib.look_at((1.0, 1.0, 5.4), (1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 40.0, res, res)


# -- icosphere --------------------------------------------------------------------------
def icosphere(level):
    """Vertices (unit sphere) and faces of an icosahedron subdivided `level` times."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        ue, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[ue[:, 0]] + v[ue[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01 = base + inv[:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:]
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def geodesic_sphere(freq):
    """Vertices (unit sphere) and faces of a class-I geodesic sphere: every face of the
    icosahedron split into freq^2 triangles on a barycentric grid, the grid points pushed
    out to the sphere.  20 freq^2 faces (freq = 2^L gives the face count of icosphere(L)),
    so a mesh of any size in steps of ~2/freq relative is available.  Points shared by two
    faces are merged, so the mesh is watertight; faces are wound outward."""
    v0, f0 = icosphere(0)
    n = int(freq)
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    m = (ii + jj) <= n
    I, J = ii[m], jj[m]
    grid = -np.ones((n + 1, n + 1), dtype=np.int64)
    grid[I, J] = np.arange(len(I))
    ui, uj = np.nonzero((ii + jj) < n)
    up = np.stack([grid[ui, uj], grid[ui + 1, uj], grid[ui, uj + 1]], 1)
    di, dj = np.nonzero((ii + jj) < n - 1)
    down = np.stack([grid[di + 1, dj], grid[di + 1, dj + 1], grid[di, dj + 1]], 1)
    local = np.concatenate([up, down])
    A, B, Cv = v0[f0[:, 0]], v0[f0[:, 1]], v0[f0[:, 2]]
    wa, wb, wc = (n - I - J) / n, I / n, J / n
    P = (A[:, None, :] * wa[None, :, None] + B[:, None, :] * wb[None, :, None] +
         Cv[:, None, :] * wc[None, :, None]).reshape(-1, 3)
    P /= np.linalg.norm(P, axis=1, keepdims=True)
    F = (local[None, :, :] + (np.arange(len(f0)) * len(I))[:, None, None]).reshape(-1, 3)
    keys = np.round(P * 1e9).astype(np.int64)
    _, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    v = P[first]
    f = inv.reshape(-1)[F]
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    inward = np.einsum("ij,ij->i", np.cross(b - a, c - a), a + b + c) < 0.0
    f[inward] = f[inward][:, [0, 2, 1]]
    return v, f


def value_noise3(p, seed, octaves=3, base_freq=4.0):
    """Seeded 3-octave value noise in [0, 1]: a hashed lattice of uniform values,
    trilinearly interpolated with a smoothstep fade, octaves at doubling frequency and
    halving amplitude."""
    rng = np.random.default_rng(seed)
    lattice = rng.random(4096)
    perm = rng.permutation(4096)

    def hash3(ix, iy, iz):
        h = perm[(ix * 73856093 ^ iy * 19349663 ^ iz * 83492791) & 4095]
        return lattice[h]

    total = np.zeros(len(p))
    amp, norm, freq = 1.0, 0.0, base_freq
    for _ in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        fr = q - i0
        w = fr * fr * (3.0 - 2.0 * fr)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    wt = ((w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1]) *
                          (w[:, 2] if dz else 1 - w[:, 2]))
                    acc += wt * hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


GLASS_CENTER = (1.0, 0.55, 1.0)


def blob_tris(level=7, center=(0.0, 0.0, 0.0), radius=0.4, amp=0.05, seed=0, freq=None):
    """Triangles (n x 9) of a subdivided icosphere (or, with `freq`, a geodesic sphere of
    20 freq^2 faces) displaced radially by value noise."""
    v, f = icosphere(level) if freq is None else geodesic_sphere(freq)
    n = value_noise3(v, seed)
    r = radius + amp * (2.0 * n - 1.0)
    pos = np.asarray(center)[None, :] + v * r[:, None]
    return pos[f].reshape(-1, 9)


def glass_material(sb: SceneBuilder):
    return sb.material(abi.MAT_DIELECTRIC, ior=sb.cauchy(1.5, 0.0042), roughness=0.0)


def glass_blob(sb: SceneBuilder, level=7, center=GLASS_CENTER, radius=0.4, amp=0.05,
               seed=0, mat=None, freq=None):
    tv = blob_tris(level, center, radius, amp, seed, freq=freq)
    if mat is None:
        mat = glass_material(sb)
    sb.tris(tv, mat)
    return mat


# -- hair strands -----------------------------------------------------------------------
def strand_ball(sb: SceneBuilder, n_strands, center=(1.0, 1.5, 1.1), ball_r=0.3, seg=4,
                radius=0.0005, length=(0.02, 0.04), jitter_deg=20.0, seed=0, mat=None):
    rng = np.random.default_rng(seed + 1)
    nrm = rng.normal(size=(n_strands, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    root = np.asarray(center)[None, :] + ball_r * nrm

    def jitter(d, max_deg):
        # uniform direction in the cone of half-angle max_deg about d
        a = np.where(np.abs(d[:, 2:3]) < 0.9, np.array([[0.0, 0.0, 1.0]]), np.array([[1.0, 0.0, 0.0]]))
        t = np.cross(d, a)
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        b = np.cross(d, t)
        ct = 1.0 - rng.random(len(d)) * (1.0 - math.cos(math.radians(max_deg)))
        st = np.sqrt(1.0 - ct * ct)
        ph = rng.random(len(d)) * 2.0 * math.pi
        out = t * (st * np.cos(ph))[:, None] + b * (st * np.sin(ph))[:, None] + d * ct[:, None]
        return out / np.linalg.norm(out, axis=1, keepdims=True)

    d = jitter(nrm, jitter_deg)
    L = length[0] + (length[1] - length[0]) * rng.random(n_strands)
    segs = np.zeros((n_strands, seg, 10))
    p = root
    for k in range(seg):
        q = p + d * (L / seg)[:, None]
        segs[:, k, 0:3] = p
        segs[:, k, 3:6] = q
        segs[:, k, 6] = radius
        segs[:, k, 7] = radius
        segs[:, k, 8] = k / seg
        segs[:, k, 9] = (k + 1) / seg
        p = q
        d = jitter(d, 8.0)
    if mat is None:
        mat = sb.diffuse(sb.const(0.4))
    sb.curves(segs.reshape(-1, 10), mat)
    return mat


# -- the benchmark workloads --------------------------------------------------------------
WORKLOADS = {
    # name: (res, photons, max_bounce)
    "cornell": (256, 1 << 24, 8),
    "glass": (1024, 1 << 28, 16),
    "fog_strands": (512, 1 << 26, 32),
}


def make_cornell(lib=None, boxes=True):
    sb = SceneBuilder()
    cornell_box(sb, boxes=boxes)
    sb.meta.update(name="cornell", tris=36 if boxes else 12)
    return sb.build(lib)


def make_glass(lib=None, level=7, seed=0, freq=None):
    """The dispersive-caustics scene: the Cornell room (without the two small boxes, which
    the blob would cut through) holding the noise-displaced glass icosphere of `level`
    subdivisions, or with `freq` a geodesic sphere of 20 freq^2 triangles."""
    sb = SceneBuilder()
    cornell_box(sb, boxes=False)
    glass_blob(sb, level=level, seed=seed, freq=freq)
    sb.meta.update(name="glass", **({"level": level} if freq is None else {"freq": freq}))
    return sb.build(lib)


def make_glass_instanced(lib=None, level=7, seed=0, to_world=None, handle=None):
    """The glass scene with the blob as one instance of a BLAS authored about the origin
    (to_world defaults to a translation to the blob's usual center).  `handle` (lib.Blas
    of blob_tris(level, seed=seed) with material 5) shares a baked copy of the mesh."""
    sb = SceneBuilder()
    cornell_box(sb, boxes=False)
    mat = glass_material(sb)
    tv = None if handle is not None else blob_tris(level, seed=seed)
    b = sb.blas(np.zeros((0, 9)) if tv is None else tv, mat, handle=handle)
    sb.instance(b, affine(translate=GLASS_CENTER) if to_world is None else to_world)
    sb.meta.update(name="glass_instanced", level=level)
    return sb.build(lib)


def make_fog_strands(lib=None, n_strands=250_000, seed=0):
    sb = SceneBuilder()
    cornell_box(sb, boxes=True)
    strand_ball(sb, n_strands, seed=seed)
    sb.medium(sb.const(0.02), sb.const(0.2), 0.6, bmin=(0, 0, 0), bmax=(2, 2, 2))
    sb.meta.update(name="fog_strands", strands=n_strands)
    return sb.build(lib)
