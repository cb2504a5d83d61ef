"""Scene residency (ftb_scene_evict / ftb_scene_restore) and the render server's admission by
device-memory footprint: a scene that left the device and came back renders exactly what it
rendered before, and a server whose HBM budget holds only part of its scenes evicts and
restores them between jobs while every job still equals its solo render."""
import numpy as np
import pytest

import cases
from goodphotons_b200 import abi, lib, scenes

from test_gpu_server import check_against_solo, job_list, run_server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def library(gpu):
    sc = {
        "cornell": lib.Scene(scenes.make_cornell(gpu), 0, gpu),
        "glass": lib.Scene(scenes.make_glass(gpu, level=5), 0, gpu),
        "materials": lib.Scene(cases.make_materials(gpu), 0, gpu, build=abi.BUILD_DEVICE),
        "fog": lib.Scene(scenes.make_fog_strands(gpu, n_strands=3000), 0, gpu),
        "instances": lib.Scene(cases.make_instances(gpu), 0, gpu),
    }
    yield sc
    for s in sc.values():
        s.close()


def restore_all(library):
    for s in library.values():
        if not s.resident:
            s.restore()


def test_evicted_scene_renders_the_same_after_restore(gpu, library):
    cam = scenes.default_camera(gpu, 48)
    for name in ("glass", "fog", "materials"):
        sc = library[name]
        before, info, en = sc.render(cam, 100_000, seed_base=7, max_bounce=16)
        sc.evict()
        assert not sc.resident
        with pytest.raises(lib.FtbError) as e:
            sc.render(cam, 10, seed_base=7, max_bounce=16)
        assert e.value.status == abi.ERR_INVALID
        sc.evict()          # evicting twice is a no-op
        sc.restore()
        assert sc.resident
        after, info2, en2 = sc.render(cam, 100_000, seed_base=7, max_bounce=16)
        np.testing.assert_array_equal(after, before, err_msg=name)
        assert list(en2.fx) == list(en.fx)
        sc.evict()          # a second round trip (host copy kept, pooled device memory)
        sc.restore()
        again, _, _ = sc.render(cam, 100_000, seed_base=7, max_bounce=16)
        np.testing.assert_array_equal(again, before, err_msg=name)


def test_scene_with_instances_stays_on_the_device(gpu, library):
    with pytest.raises(lib.FtbError) as e:
        library["instances"].evict()
    assert e.value.status == abi.ERR_UNSUPPORTED
    assert library["instances"].resident


def test_server_admits_by_footprint_and_evicts_idle_scenes(gpu, library):
    restore_all(library)
    probe = lib.Server(device=0, wave_slots=1 << 20, lib=gpu)
    waves = probe.stats().wave_bytes
    probe.close()
    assert waves > 0
    sizes = {k: s.footprint(1, 1).scene_bytes for k, s in library.items()}
    evictable = sorted((k for k in sizes if k != "instances"), key=lambda k: sizes[k])
    films = 4 * 64 * 64 * 32   # four admitted jobs at the largest resolution
    # room for the films, the instanced scene (always resident), the largest other scene and
    # a quarter of the rest: the library does not fit, so the server must evict to run the mix
    rest = sum(sizes[k] for k in evictable[:-1])
    budget = waves + films + sizes["instances"] + sizes[evictable[-1]] + rest // 4
    for k in evictable:   # the library starts in host memory
        library[k].evict()
    jobs = job_list(gpu, library)
    films_out, results, st = run_server(gpu, library, jobs, wave_slots=1 << 20, hbm_budget=budget, max_active=4)
    assert st.completed == len(jobs) and st.failed == 0
    assert st.restores >= len(evictable) and st.evictions > 0, (st.restores, st.evictions)
    assert st.wave_bytes == waves
    restore_all(library)
    check_against_solo(gpu, library, jobs, films_out, results)


def test_server_rejects_a_job_larger_than_its_budget(gpu, library):
    restore_all(library)
    probe = lib.Server(device=0, wave_slots=1 << 20, lib=gpu)
    waves = probe.stats().wave_bytes
    probe.close()
    srv = lib.Server(device=0, wave_slots=1 << 20, hbm_budget=waves + 64 * 64 * 32, lib=gpu)
    try:
        with pytest.raises(lib.FtbError) as e:   # film fits, film + scene does not
            srv.submit(library["glass"], scenes.default_camera(gpu, 64), 1000, max_bounce=16)
        assert e.value.status == abi.ERR_TOO_LARGE
    finally:
        srv.close()
    with pytest.raises(lib.FtbError) as e:      # the wave buffers alone exceed the budget
        lib.Server(device=0, wave_slots=1 << 20, hbm_budget=waves // 2, lib=gpu)
    assert e.value.status == abi.ERR_TOO_LARGE
