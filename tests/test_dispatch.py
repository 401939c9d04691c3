"""The multi-device dispatcher's placement logic on CPU, with fake servers (no GPU): scene affinity,
replication of hot scenes, load accounting, ticket mapping and failures."""
import numpy as np
import pytest

from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200._lib import RtcError
from cortexraytracercuda_b200.dispatch import RenderDispatcher
from cortexraytracercuda_b200.scene import RenderParams


class FakeServer:
    def __init__(self, dev):
        self.dev, self.scenes, self.pending, self.next, self.closed = dev, [], {}, 1, False

    def add_scene(self, scene):
        self.scenes.append(scene)
        return len(self.scenes) - 1

    def submit(self, sid, params, camera=None, out=None):
        out = np.full((params.height, params.width, 4), float(self.dev), np.float32) if out is None else out
        t = self.next
        self.next += 1
        self.pending[t] = (sid, out)
        return t, out

    def poll(self, t):
        return True, {"state": 2, "scene": self.pending.pop(t)[0]}

    def wait(self, t, timeout_ms=-1):
        if timeout_ms == 0:
            raise RtcError(5, "timed out")
        sid, out = self.pending.pop(t)
        return out, {"state": 2, "scene": sid}

    def stats(self):
        return {"scenes": len(self.scenes), "pending": len(self.pending)}

    def close(self):
        self.closed = True


def _d(n=3, **kw):
    return RenderDispatcher(devices=list(range(n)), server_factory=FakeServer, **kw)


P = RenderParams(width=16, height=8, spp=4, max_depth=4)   # 16 x 8 x 4 = 512 paths


def test_affinity_and_first_placement():
    d = _d()
    a, b = d.add_scene(configs.cornell()), d.add_scene(configs.textured())
    ta, _ = d.submit(a, P)
    assert d.homes(a) == [0]                       # least loaded, lowest index
    tb, _ = d.submit(b, P)
    assert d.homes(b) == [1]                       # device 0 now carries work
    ta2, _ = d.submit(a, P)                        # within the replication factor: stays home
    assert d.homes(a) == [0] and d.load == [1024, 512, 0]
    for t in (ta, tb, ta2):
        d.wait(t)
    assert d.load == [0, 0, 0]
    assert [len(s.scenes) for s in d.servers] == [1, 1, 0]


def test_hot_scene_replicates_and_results_come_back():
    d = _d(replicate_at=2.0)
    s = d.add_scene(configs.cornell())
    ts = [d.submit(s, P)[0] for _ in range(6)]
    # the home fills until it carries more than 2x the idle devices' work, then the scene spreads
    assert d.homes(s) == [0, 1, 2] and d.replications == 2
    seen = set()
    for t in ts:
        out, info = d.wait(t)
        assert out.shape == (8, 16, 4) and float(out[0, 0, 0]) == info["device"]
        seen.add(info["device"])
    assert seen == {0, 1, 2} and d.load == [0, 0, 0]
    st = d.stats()
    assert sum(st["routed"]) == 6 and st["homes"][s] == [0, 1, 2]


def test_poll_timeout_and_errors():
    d = _d(n=2)
    s = d.add_scene(configs.cornell())
    t, _ = d.submit(s, P)
    with pytest.raises(RtcError):
        d.wait(t, 0)                               # a timeout keeps the request in flight
    assert d.load[0] == 512
    done, info = d.poll(t)
    assert done and info["device"] == 0 and d.load == [0, 0]
    with pytest.raises(KeyError):
        d.poll(t)                                  # released
    with pytest.raises(KeyError):
        d.submit(7, P)
    with pytest.raises(ValueError):
        RenderDispatcher(devices=[], server_factory=FakeServer)
    d.close()


def test_close_and_factory_failure():
    made = []

    def factory(dev):
        if dev == 2:
            raise RuntimeError("no device 2")
        s = FakeServer(dev)
        made.append(s)
        return s

    with pytest.raises(RuntimeError):
        RenderDispatcher(devices=[0, 1, 2], server_factory=factory)
    assert all(s.closed for s in made)             # servers made before the failure are closed
