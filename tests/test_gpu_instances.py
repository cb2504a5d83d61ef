"""Instanced meshes on the GPU beyond the parity case: shared BLAS handles, TLAS refit and
scene clones.  Each must render exactly what a scene created from scratch with the same
transforms renders (the film is fixed point and photons are keyed by index, so equal
paths give equal films bit for bit)."""
import numpy as np
import pytest

from goodphotons_b200 import lib, scenes

pytestmark = pytest.mark.gpu

LEVEL = 3
XF_A = scenes.affine((0.2, 1.0, 0.1), 40.0, (1.05, 0.6, 0.95))
XF_B = scenes.affine((1.0, 0.3, -0.5), 200.0, (0.85, 0.5, 1.15))


def render(sc, res=48, n=200_000, seed=5):
    cam = scenes.default_camera(sc.lib, res)
    film, _, en = sc.render(cam, n, seed_base=seed, max_bounce=16, frac_bits=30)
    return film, list(en.fx)


def test_refit_renders_like_a_fresh_scene(gpu):
    a = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A), 0, gpu)
    b = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_B), 0, gpu)
    fa, ea = render(a)
    a.set_instance_transforms([XF_B])
    fb, eb = render(b)
    fr, er = render(a)
    assert not np.array_equal(fa, fb)
    np.testing.assert_array_equal(fr, fb)
    assert er == eb
    a.set_instance_transforms([XF_A])   # and back
    fa2, ea2 = render(a)
    np.testing.assert_array_equal(fa2, fa)
    assert ea2 == ea
    a.close()
    b.close()


def test_clone_renders_like_a_fresh_scene_and_outlives_its_source(gpu):
    a = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A), 0, gpu)
    b = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_B), 0, gpu)
    fa, _ = render(a)
    c = a.clone_instances([XF_B])
    np.testing.assert_array_equal(render(c)[0], render(b)[0])
    np.testing.assert_array_equal(render(a)[0], fa)   # the source keeps its own transforms
    a.close()
    np.testing.assert_array_equal(render(c)[0], render(b)[0])
    c.close()
    b.close()


def test_shared_blas_handle_equals_baked_arrays(gpu):
    d_arr = scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A)
    mat = int(d_arr.blas_arrays[0][2][0])
    h = lib.Blas(scenes.blob_tris(LEVEL), mat, device=0, lib=gpu)
    d_h = scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A, handle=h)
    s_arr = lib.Scene(d_arr, 0, gpu)
    s_h = lib.Scene(d_h, 0, gpu)
    h.close()   # the scene holds its own reference to the device copy
    fa, ea = render(s_arr)
    fh, eh = render(s_h)
    np.testing.assert_array_equal(fa, fh)
    assert ea == eh
    s_arr.close()
    s_h.close()


def test_batched_frames_equal_solo_renders(gpu):
    """Animation frames: clones of one scene (one shared BLAS, a refit TLAS each) rendered
    together in one ftb_render_batch, frame by frame equal to rendering alone."""
    torch = pytest.importorskip("torch")
    base = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A), 0, gpu)
    rng = np.random.default_rng(3)
    frames, jobs, films = [], [], []
    for k in range(8):
        ax = rng.normal(size=3)
        xf = scenes.affine(ax, rng.uniform(0, 360), np.asarray(scenes.GLASS_CENTER) + rng.uniform(-0.2, 0.2, 3))
        fr = base.clone_instances([xf])
        frames.append(fr)
        res = int(rng.choice([24, 32, 48]))
        cam = scenes.default_camera(gpu, res)
        film = torch.zeros((res, res, 4), dtype=torch.int64, device="cuda:0")
        films.append(film)
        jobs.append(dict(scene=fr, cam=cam, d_film=film.data_ptr(), n=int(rng.integers(20_000, 120_000)),
                         seed_base=1000 * k, max_bounce=16, frac_bits=30))
    stream = torch.cuda.current_stream().cuda_stream
    _, ens = gpu.render_batch(jobs, stream=stream)
    torch.cuda.synchronize()
    for k, (j, film) in enumerate(zip(jobs, films)):
        solo, _, en = j["scene"].render(j["cam"], j["n"], seed_base=j["seed_base"], max_bounce=16, frac_bits=30)
        np.testing.assert_array_equal(film.cpu().numpy(), solo, err_msg=f"frame {k}")
        assert list(ens[k].fx) == list(en.fx)
    for fr in frames:
        fr.close()
    base.close()


def test_bad_instance_arguments_fail_cleanly(gpu):
    sb = scenes.SceneBuilder()
    scenes.cornell_box(sb, boxes=False)
    m = sb.diffuse(sb.const(0.5))
    b = sb.blas(scenes.blob_tris(1), m)
    sb.instance(b + 1, scenes.affine())            # no such BLAS
    with pytest.raises(lib.FtbError):
        lib.Scene(sb.build(gpu), 0, gpu)
    sc = lib.Scene(scenes.make_glass_instanced(gpu, 1), 0, gpu)
    with pytest.raises(lib.FtbError):
        sc.set_instance_transforms(np.zeros((2, 12)))   # only one instance
    bad = scenes.affine()
    bad[3] = np.nan
    with pytest.raises(lib.FtbError):
        sc.set_instance_transforms([bad])
    sc.close()


# ---- anchored to the oracle and the reference ------------------------------------------
# The tests above show that a refit TLAS, a clone and a batched frame render what a fresh
# scene renders.  These show that what they render is the reference's light transport for
# the moved instance: per-photon paths against the oracle built from a descriptor with the
# new transform (MeshInstance::setToWorld, scene.h:1052-1062), films and energy against
# the oracle and against the reference's own tracer, within the parity tolerances of
# test_gpu_parity.py.
def assert_film_close(film, info, xyz_ref, hits_ref):
    xyz, hits = lib.film_to_xyz(film, info)
    np.testing.assert_array_equal(hits, hits_ref)
    tol = hits_ref[..., None] * info.scale + 1e-10 * np.abs(xyz_ref)
    bad = np.abs(xyz - xyz_ref) > tol
    assert not bad.any(), f"{bad.sum()} film values differ"


def check_against_oracle(sc, desc, oracle, reference, res=40, n=1 << 14, seed=9):
    cam = scenes.default_camera(sc.lib, res)
    gl = sc.trace_log(cam, n, seed_base=seed, max_bounce=16)
    ol = oracle.trace(desc, cam, n, seed_base=seed, max_bounce=16, logs=True, threads=4)["logs"]
    same = (gl["n_hits"] == ol["n_hits"]) & (gl["prim_hash"] == ol["prim_hash"]) & (gl["fate"] == ol["fate"])
    assert (~same).sum() <= max(1, int(1e-5 * n)), f"{(~same).sum()} of {n} photon paths differ"
    np.testing.assert_allclose(gl["beta"][same], ol["beta"][same], rtol=1e-12, atol=0)
    film, info, en = sc.render(cam, n, seed_base=seed, max_bounce=16)
    o = oracle.trace(desc, cam, n, seed_base=seed, max_bounce=16, threads=1)
    assert_film_close(film, info, o["xyz"], o["hits"])
    np.testing.assert_allclose(en.as_list(), o["energy"], rtol=1e-9, atol=0)
    r = reference.trace(desc, cam, n, seed_base=seed, max_bounce=16, threads=1)
    assert_film_close(film, info, r["xyz"], r["hits"])
    np.testing.assert_allclose(en.as_list(), r["energy"], rtol=1e-9, atol=0)


def test_refit_and_clone_match_oracle_and_reference(gpu, oracle, reference):
    a = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A), 0, gpu)
    try:
        a.set_instance_transforms([XF_B])                   # refit
        check_against_oracle(a, scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_B), oracle, reference)
        xf_c = scenes.affine((0.7, -0.2, 0.4), 290.0, (1.1, 0.45, 0.9), scale=0.9)
        c = a.clone_instances([xf_c])                       # clone with a third transform
        try:
            check_against_oracle(c, scenes.make_glass_instanced(gpu, LEVEL, to_world=xf_c), oracle, reference)
        finally:
            c.close()
    finally:
        a.close()


def test_batched_frames_match_oracle(gpu, oracle):
    """Four animation frames (clones with seeded rigid transforms, uneven films and
    budgets) in one ftb_render_batch: each frame's film and energy against the oracle's
    render of a descriptor with that frame's transform."""
    torch = pytest.importorskip("torch")
    base = lib.Scene(scenes.make_glass_instanced(gpu, LEVEL, to_world=XF_A), 0, gpu)
    rng = np.random.default_rng(17)
    frames, jobs, films, xfs = [], [], [], []
    try:
        for k in range(4):
            xf = scenes.affine(rng.normal(size=3), rng.uniform(0, 360),
                               np.asarray(scenes.GLASS_CENTER) + rng.uniform(-0.2, 0.2, 3))
            xfs.append(xf)
            fr = base.clone_instances([xf])
            frames.append(fr)
            res = (24, 40, 32, 48)[k]
            film = torch.zeros((res, res, 4), dtype=torch.int64, device="cuda:0")
            films.append(film)
            jobs.append(dict(scene=fr, cam=scenes.default_camera(gpu, res), d_film=film.data_ptr(),
                             n=(9000, 30000, 15000, 22000)[k], seed_base=50_000 * k, max_bounce=16,
                             frac_bits=30))
        infos, ens = gpu.render_batch(jobs, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for k, j in enumerate(jobs):
            desc = scenes.make_glass_instanced(gpu, LEVEL, to_world=xfs[k])
            o = oracle.trace(desc, j["cam"], j["n"], seed_base=j["seed_base"], max_bounce=16, threads=1)
            assert_film_close(films[k].cpu().numpy(), infos[k], o["xyz"], o["hits"])
            np.testing.assert_allclose(ens[k].as_list(), o["energy"], rtol=1e-9, atol=0)
    finally:
        for fr in frames:
            fr.close()
        base.close()
