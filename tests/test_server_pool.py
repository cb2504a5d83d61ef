"""Serving on several GPUs as replicas (multigpu.ServerPool): each job goes whole to the
device with the least outstanding photons, scenes are asked for once per device, and waits
release the load.  Host logic only, with stand-in servers (no GPU here)."""
import pytest

from goodphotons_b200 import multigpu


class FakeServer:
    def __init__(self, device, **cfg):
        self.device, self.cfg, self.jobs, self.closed = device, cfg, {}, False

    def submit(self, scene, cam, n, **kw):
        assert scene[1] == self.device, "a job must use its own device's copy of the scene"
        jid = len(self.jobs) + 1
        self.jobs[jid] = (scene, cam, n, kw)
        return jid

    def wait(self, jid, timeout=-1.0):
        return ("done", self.device) + self.jobs.pop(jid)[:3]

    def close(self):
        self.closed = True


def test_jobs_go_to_the_least_loaded_device_and_scenes_are_made_once_per_device():
    made = []

    def scene_of(key, device):
        made.append((key, device))
        return (key, device)

    pool = multigpu.ServerPool([0, 1, 2], scene_of, make_server=FakeServer, max_active=8)
    assert all(s.cfg == {"max_active": 8} for s in pool.servers.values())
    hs = [pool.submit("glass", "cam", n, seed_base=k) for k, n in enumerate([100, 10, 10, 50, 5, 5])]
    # 100 -> 0; 10 -> 1; 10 -> 2; 50 -> 1 (load 10 vs 10 vs 100: first of the ties); 5 -> 2; 5 -> 2
    assert [pool.device_of(h) for h in hs] == [0, 1, 2, 1, 2, 2]
    assert pool.load == {0: 100, 1: 60, 2: 20}
    assert sorted(made) == [("glass", 0), ("glass", 1), ("glass", 2)]
    r = pool.wait(hs[0])
    assert r[:2] == ("done", 0) and r[4] == 100 and pool.load[0] == 0
    assert pool.device_of(pool.submit("cornell", "cam", 7)) == 0   # device 0 is idle again
    for h in hs[1:]:
        pool.wait(h)
    assert pool.load == {0: 7, 1: 0, 2: 0}
    servers = list(pool.servers.values())
    pool.close()
    assert all(s.closed for s in servers)


def test_pool_needs_devices():
    with pytest.raises(ValueError):
        multigpu.ServerPool([], lambda k, d: None, make_server=FakeServer)
