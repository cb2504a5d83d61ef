"""Small seeded scenes shared by the parity tests and the golden-vector script."""
import ctypes as C
import hashlib

import numpy as np

from goodphotons_b200 import abi, scenes


def make_materials(L):
    """Every supported branch: glossy, filter, diffuse-transmit, nested dielectrics with
    priority / interior absorption / frosting, a Sellmeier glass, a diffuse sphere and two
    emitters (power-CDF selection draws)."""
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    glossy = sb.material(abi.MAT_GLOSSY, reflect=sb.const(0.8), roughness=0.3)
    sb.box((1.45, 0.5), (0.5, 0.5), 0.5, 25.0, glossy)
    filt = sb.material(abi.MAT_FILTER, transmit=sb.table([(400, 0.2), (550, 0.9), (700, 0.3)]))
    sb.quad((0.2, 0.1, 1.6), (0.5, 0, 0), (0, 0.8, 0), filt)
    trans = sb.material(abi.MAT_DIFFUSE_TRANSMIT, reflect=sb.const(0.4), transmit=sb.const(0.35))
    sb.quad((1.3, 0.2, 1.7), (0.5, 0, 0.05), (0, 0.7, 0), trans)
    outer = sb.material(abi.MAT_DIELECTRIC, ior=sb.cauchy(1.5, 0.0042), absorb=sb.const(0.3),
                        roughness=0.05, priority=1)
    scenes.glass_blob(sb, level=2, center=(0.7, 0.5, 0.9), radius=0.35, amp=0.04, seed=3, mat=outer)
    inner = sb.material(abi.MAT_DIELECTRIC,
                        ior=sb.sellmeier(1.03961212, 0.231792344, 1.01046945, 0.00600069867,
                                         0.0200179144, 103.560653), priority=2)
    scenes.glass_blob(sb, level=1, center=(0.7, 0.5, 0.9), radius=0.15, amp=0.0, seed=4, mat=inner)
    sb.sphere((1.5, 1.2, 0.6), 0.15, sb.diffuse(sb.const(0.6)))
    sb.sphere_light((0.4, 1.5, 1.4), 0.08, sb.blackbody(3000.0, 0.5))
    return sb.build(L)


def make_instances(L, ramp=0.01, cauchy=True):
    """Instanced meshes (Blas / MeshInstance): a smooth-shaded dielectric blob placed twice
    (a rotation with non-uniform scale, and a scaled copy with a glossy material override)
    and a diffuse box asset rotated about y, beside the world triangles of the box."""
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False, ramp=ramp)
    glass = sb.material(abi.MAT_DIELECTRIC, ior=sb.cauchy(1.5, 0.0042) if cauchy else sb.const(1.5), roughness=0.0)
    v, f = scenes.icosphere(2)
    n = scenes.value_noise3(v, 5)
    r = 0.25 + 0.03 * (2.0 * n - 1.0)
    blob = sb.blas((v * r[:, None])[f].reshape(-1, 9), glass, normals=v[f].reshape(-1, 9))
    box_sb = scenes.SceneBuilder()
    white = sb.diffuse(sb.const(0.7))
    box_sb.box((0.0, 0.0), (0.4, 0.4), 0.6, 0.0, 0, y0=-0.3)
    box = sb.blas(np.concatenate(box_sb.tri_v), white)
    xf = scenes.affine((1.0, 1.0, 0.0), 30.0, (0.6, 0.55, 1.0))
    xf[:9] = (xf[:9].reshape(3, 3) @ np.diag([1.2, 0.8, 1.0])).reshape(9)
    sb.instance(blob, xf)
    glossy = sb.material(abi.MAT_GLOSSY, reflect=sb.const(0.8), roughness=0.25)
    sb.instance(blob, scenes.affine((0.3, -1.0, 0.2), 75.0, (1.45, 0.45, 0.7), scale=0.8), mat_override=glossy)
    sb.instance(box, scenes.affine((0.0, 1.0, 0.0), 20.0, (1.3, 0.31, 1.5)))
    return sb.build(L)


def make_mirrors(L, fog=False):
    """Planar mirrors (the reference's connectSpecularPlane): a Mirror panel in front of the
    back wall, a HalfMirror pane standing in the room and a roughness-0 Glossy tile beside the
    left wall, with the two Cornell boxes; `fog` fills the box with the homogeneous medium, so
    volume vertices connect through the mirrors too."""
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=True)
    mirror = sb.material(abi.MAT_MIRROR, reflect=sb.const(0.9))
    sb.quad((0.3, 0.3, 0.02), (1.4, 0, 0), (0, 1.4, 0), mirror)
    half = sb.material(abi.MAT_HALF_MIRROR, reflect=sb.table([(400, 0.3), (700, 0.7)]))
    sb.quad((1.0, 0.0, 1.2), (0.5, 0, -0.3), (0, 1.0, 0), half)
    tile = sb.material(abi.MAT_GLOSSY, reflect=sb.const(0.8), roughness=0.0)
    sb.quad((0.01, 0.6, 0.6), (0, 0.6, 0), (0, 0, 0.8), tile)
    if fog:
        sb.medium(sb.const(0.02), sb.const(0.2), 0.6, bmin=(0, 0, 0), bmax=(2, 2, 2))
    return sb.build(L)


def make_smooth(L):
    """Smooth shading, modelled on the reference's -checktrinormal (main.cpp:8123): diffuse
    spheres tessellated with exact outward vertex normals (n = p - centre), one wound outward
    and one wound inward without touching its vertex normals, so its geometric normal opposes
    the shading normal everywhere; and a smooth glossy sphere.  Exercises the interpolated
    normal, the oriented geometric normal and the shading-normal adjoint correction."""
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    v, f = scenes.icosphere(2)
    tri = v[f]                              # (n, 3, 3) on the unit sphere, wound outward
    inward = tri[:, [0, 2, 1], :]
    for centre, r, mat, t in (((0.6, 0.4, 1.0), 0.3, sb.diffuse(sb.const(0.7)), tri),
                              ((1.4, 0.35, 0.8), 0.25, sb.diffuse(sb.table([(400, 0.2), (600, 0.8)])), inward),
                              ((1.0, 1.2, 0.6), 0.2, sb.material(abi.MAT_GLOSSY, reflect=sb.const(0.85),
                                                                 roughness=0.15), tri)):
        sb.tris((t * r + np.asarray(centre)).reshape(-1, 9), mat, normals=t.reshape(-1, 9))
    return sb.build(L)


CASES = {
    # name: (builder, res, photons, max_bounce, seed_base, wavelengths per photon)
    "cornell": (lambda L: scenes.make_cornell(L), 32, 8192, 8, 0, 1),
    "cornell_seed": (lambda L: scenes.make_cornell(L), 32, 4096, 8, 123456789, 1),
    "glass": (lambda L: scenes.make_glass(L, level=2), 32, 8192, 16, 0, 1),
    "fog_strands": (lambda L: scenes.make_fog_strands(L, n_strands=500), 32, 8192, 32, 0, 1),
    "materials": (make_materials, 32, 8192, 16, 7, 1),
    "instances": (make_instances, 32, 8192, 16, 11, 1),
    "mirrors": (make_mirrors, 32, 8192, 16, 13, 1),
    "mirrors_fog": (lambda L: make_mirrors(L, fog=True), 32, 8192, 32, 17, 1),
    "mirrors_hero4": (make_mirrors, 32, 8192, 16, 19, 4),
    "smooth": (make_smooth, 32, 8192, 16, 23, 1),
    "smooth_hero4": (make_smooth, 32, 8192, 16, 29, 4),
    # hero-wavelength bundles (Renderer::tracePhotonHero): C wavelengths per photon
    "cornell_hero4": (lambda L: scenes.make_cornell(L), 32, 8192, 8, 3, 4),
    "glass_hero4": (lambda L: scenes.make_glass(L, level=2), 32, 8192, 16, 5, 4),
    "materials_hero3": (make_materials, 32, 8192, 16, 9, 3),
}


# The benchmark configurations at their own size: scene, film, bounce cap.  The photon
# count is the golden vectors' (the per-photon tests trace 2^15).
CONFIG_CASES = {
    # dispersive caustics: level-7 (327,680 triangles) and level-8 (1,310,720) glass, 1024^2
    "cfg_glass_l7": (lambda L: scenes.make_glass(L, level=7), 1024, 2048, 16, 0, 1),
    "cfg_glass_l8": (lambda L: scenes.make_glass(L, level=8), 1024, 2048, 16, 1 << 40, 1),
    # fog + 250k strands (1M round cones), 512^2, 32 bounces
    "cfg_fog_strands": (lambda L: scenes.make_fog_strands(L, n_strands=250_000), 512, 2048, 32, 77, 1),
    # the Cornell box at 256^2, 8 bounces
    "cfg_cornell": (lambda L: scenes.make_cornell(L), 256, 4096, 8, 5, 1),
}


def joint_ties(d, gl, ol, idx):
    """Of the photons `idx` whose logged paths differ between two tracers, those that differ
    only in which of two consecutive segments of one strand was hit at their shared joint
    (the segment of one strand ends where the next begins, so a ray meeting the joint meets
    both round cones at the same point, with distances equal to within ~1e-16 m; a last-bit
    difference in the ray -- CUDA's sin/cos/log against glibc's -- can decide which is
    nearer).  Such photons have the same bounce count, termination and final beta, and the
    same hit sequence up to those swaps.  Only paths of at most 8 hits (all logged) count."""
    base = len(d.tri_v) + len(d.sph)
    curve = d.curve
    nc = len(curve)

    def joint(a, b):
        ia, ib = a - base, b - base
        if not (0 <= ia < nc and 0 <= ib < nc):
            return False
        pa, pb = curve[ia], curve[ib]
        return bool(np.array_equal(pa[3:6], pb[0:3]) or np.array_equal(pb[3:6], pa[0:3]))

    out = []
    for i in idx:
        nh = int(gl["n_hits"][i])
        if nh != int(ol["n_hits"][i]) or gl["fate"][i] != ol["fate"][i] or nh > 8:
            continue
        if not np.isclose(gl["beta"][i], ol["beta"][i], rtol=1e-12, atol=0):
            continue
        ga, oa = gl["prims"][i][:nh], ol["prims"][i][:nh]
        diff = np.nonzero(ga != oa)[0]
        if len(diff) and all(joint(int(ga[k]), int(oa[k])) for k in diff):
            out.append(int(i))
    return out


def camera(L, res):
    return scenes.default_camera(L, res)


def scene_hash(d):
    h = hashlib.sha256()
    for a in (d.tri_v, d.tri_mat, d.sph, d.sph_mat, d.curve, d.curve_mat, d.table_w, d.table_v,
              d.emitter_cdf):
        h.update(np.ascontiguousarray(a).tobytes())
    if d.tri_n is not None:
        h.update(d.tri_n.tobytes())
    for arr, n in ((d.mats, d.n_mats), (d.spectra, d.n_spectra), (d.emitters, d.n_emitters),
                   (d.media, d.n_media)):
        h.update(C.string_at(C.addressof(arr), n * C.sizeof(arr._type_)))
    for tv, tn, tm, _ in d.blas_arrays:
        for a in (tv, tm) + (() if tn is None else (tn,)):
            h.update(np.ascontiguousarray(a).tobytes())
    if d.n_instances:
        h.update(C.string_at(C.addressof(d.instances), d.n_instances * C.sizeof(abi.Instance)))
    return h.hexdigest()
