"""The render server (ftb_server_*): jobs of mixed scenes, sizes and photon budgets,
submitted from several threads while others run, each equal to rendering it alone --
through admission limits, waves shared between jobs and jobs spanning many waves."""
import threading

import numpy as np
import pytest

import cases
from goodphotons_b200 import lib, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident(gpu):
    sc = {
        "cornell": lib.Scene(scenes.make_cornell(gpu), 0, gpu),
        "glass": lib.Scene(scenes.make_glass(gpu, level=3), 0, gpu),
        "materials": lib.Scene(cases.make_materials(gpu), 0, gpu),
        "fog": lib.Scene(scenes.make_fog_strands(gpu, n_strands=300), 0, gpu),
        "instances": lib.Scene(cases.make_instances(gpu), 0, gpu),
        "mirrors": lib.Scene(cases.make_mirrors(gpu), 0, gpu),
    }
    yield sc
    for s in sc.values():
        s.close()


def job_list(gpu, resident):
    rng = np.random.default_rng(9)
    names = sorted(resident)
    out = []
    for k in range(24):
        name = names[k % len(names)]
        res = int(rng.choice([16, 24, 40, 64]))
        n = int(rng.choice([0, 1, 5_000, 60_000, 300_000, 5_000_000 if k == 7 else 200_000]))
        mb = {"cornell": 8, "fog": 32}.get(name, 16)
        out.append((name, res, n, 1000 * k, mb))
    return out


def run_server(gpu, resident, jobs, **cfg):
    srv = lib.Server(device=0, lib=gpu, **cfg)
    films = [np.full((res, res, 4), -1, dtype=np.int64) for _, res, _, _, _ in jobs]
    ids = [None] * len(jobs)

    def submit(idx):
        for i in idx:
            name, res, n, seed, mb = jobs[i]
            ids[i] = srv.submit(resident[name], scenes.default_camera(gpu, res), n, seed_base=seed,
                                max_bounce=mb, host_film=films[i])

    ts = [threading.Thread(target=submit, args=(range(t, len(jobs), 3),)) for t in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    return films, results, st


def check_against_solo(gpu, resident, jobs, films, results):
    for (name, res, n, seed, mb), film, r in zip(jobs, films, results):
        assert r.status == 0, (name, n)
        solo, info, en = resident[name].render(scenes.default_camera(gpu, res), n, seed_base=seed, max_bounce=mb)
        np.testing.assert_array_equal(film, solo, err_msg=f"{name} n={n}")
        assert r.info.frac_bits == info.frac_bits
        assert list(r.energy.fx) == list(en.fx), f"{name} n={n} energy"
        assert r.submit_s <= r.admit_s <= r.finish_s


def test_mixed_jobs_equal_solo_renders(gpu, resident):
    jobs = job_list(gpu, resident)
    films, results, st = run_server(gpu, resident, jobs, wave_slots=1 << 20)
    check_against_solo(gpu, resident, jobs, films, results)
    assert st.completed == len(jobs) and st.failed == 0
    assert st.photons_done == sum(j[2] for j in jobs)


def test_admission_limits_keep_results(gpu, resident):
    """Two jobs admitted at once and a film budget of about three 64^2 films: jobs wait in
    the queue and still come out equal to solo renders."""
    jobs = job_list(gpu, resident)[:12]
    films, results, st = run_server(gpu, resident, jobs, max_active=2, film_budget=3 * 64 * 64 * 32,
                                    wave_slots=1 << 18)
    check_against_solo(gpu, resident, jobs, films, results)
    assert st.completed == len(jobs)


def test_oversized_film_and_timeouts(gpu, resident):
    srv = lib.Server(device=0, lib=gpu, film_budget=32 * 32 * 32)
    with pytest.raises(lib.FtbError, match="TOO_LARGE"):
        srv.submit(resident["cornell"], scenes.default_camera(gpu, 64), 1000)
    jid = srv.submit(resident["glass"], scenes.default_camera(gpu, 32), 20_000_000, max_bounce=16)
    with pytest.raises(lib.FtbError, match="TIMEOUT"):
        srv.wait(jid, timeout=0.0)
    r = srv.wait(jid)
    assert r.status == 0
    with pytest.raises(lib.FtbError):
        srv.wait(jid)   # already collected
    srv.close()


def test_bundles_and_classes_in_the_mix(gpu, resident):
    """Hero bundles (C = 4, 3) among one-wavelength jobs of every kernel class: passes hold
    one class at a time, and each job still equals its solo render."""
    specs = [("glass", 32, 400_000, 4), ("cornell", 24, 300_000, 1), ("fog", 16, 50_000, 1),
             ("cornell", 40, 900_000, 3), ("instances", 24, 200_000, 4), ("materials", 32, 250_000, 1),
             ("mirrors", 32, 300_000, 1), ("mirrors", 24, 300_000, 4)]
    srv = lib.Server(device=0, lib=gpu, wave_slots=1 << 19)
    films, ids = [], []
    for k, (name, res, n, hero) in enumerate(specs):
        films.append(np.full((res, res, 4), -1, dtype=np.int64))
        mb = {"cornell": 8, "fog": 32}.get(name, 16)
        ids.append(srv.submit(resident[name], scenes.default_camera(gpu, res), n, seed_base=777 * k,
                              max_bounce=mb, host_film=films[k], hero_c=hero))
    results = [srv.wait(i) for i in ids]
    srv.close()
    for k, ((name, res, n, hero), film, r) in enumerate(zip(specs, films, results)):
        assert r.status == 0, name
        mb = {"cornell": 8, "fog": 32}.get(name, 16)
        solo, _, en = resident[name].render(scenes.default_camera(gpu, res), n, seed_base=777 * k, max_bounce=mb,
                                            hero_c=hero)
        np.testing.assert_array_equal(film, solo, err_msg=f"{name} hero {hero}")
        assert list(r.energy.fx) == list(en.fx), f"{name} hero {hero} energy"


def test_server_pool_jobs_equal_solo_renders(gpu, resident):
    """multigpu.ServerPool over the devices this box has (one here): jobs routed to a
    device's server render exactly their solo films."""
    from goodphotons_b200 import multigpu
    pool = multigpu.ServerPool([0], lambda key, d: resident[key], lib=gpu, wave_slots=1 << 19)
    specs = [("glass", 24, 200_000), ("mirrors", 32, 150_000), ("fog", 16, 60_000)]
    films, hs = [], []
    for k, (name, res, n) in enumerate(specs):
        films.append(np.full((res, res, 4), -1, dtype=np.int64))
        mb = {"cornell": 8, "fog": 32}.get(name, 16)
        hs.append(pool.submit(name, scenes.default_camera(gpu, res), n, seed_base=31 * k, max_bounce=mb,
                              host_film=films[k]))
    results = [pool.wait(h) for h in hs]
    pool.close()
    for k, ((name, res, n), film, r) in enumerate(zip(specs, films, results)):
        assert r.status == 0, name
        mb = {"cornell": 8, "fog": 32}.get(name, 16)
        solo, _, en = resident[name].render(scenes.default_camera(gpu, res), n, seed_base=31 * k, max_bounce=mb)
        np.testing.assert_array_equal(film, solo, err_msg=name)
        assert list(r.energy.fx) == list(en.fx), name
