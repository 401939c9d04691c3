"""The dispatcher end to end on the GPU: two servers (both on device 0 here, as one GPU is what a test
gets) behind one RenderDispatcher.  Requests spread over the servers by scene affinity and
replication; every image must equal the same request served by a lone server, bit for bit (g++
flavour), whichever server rendered it."""
import numpy as np
import pytest

from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200.dispatch import RenderDispatcher
from cortexraytracercuda_b200.renderer import RenderServer
from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, MODE_COMPAT, RenderParams

pytestmark = pytest.mark.gpu

KW = dict(mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, slots=4096, ring=16, batch=4)
REQ = {"cornell": dict(width=40, height=40, spp=4, max_depth=8),
       "spheres": dict(width=64, height=36, spp=9, max_depth=16),
       "textured": dict(width=40, height=30, spp=4, max_depth=10)}


def _p(name, seed):
    return RenderParams(seed=seed, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, **REQ[name])


def test_dispatcher_results_equal_a_lone_server():
    names = list(REQ)
    work = [(names[k % 3], 2580 + k) for k in range(12)]
    with RenderServer(0, **KW) as lone:
        ids = {n: lone.add_scene(configs.SCENES[n][0]()) for n in names}
        want = [lone.wait(lone.submit(ids[n], _p(n, s))[0], 60000)[0] for n, s in work]
    with RenderDispatcher(devices=[0, 0], replicate_at=1.0, **KW) as d:
        gid = {n: d.add_scene(configs.SCENES[n][0]()) for n in names}
        tickets = [d.submit(gid[n], _p(n, s))[0] for n, s in work]
        got, served = [], set()
        for t in tickets:
            out, info = d.wait(t, 60000)
            got.append(out)
            served.add(info["device"])
        st = d.stats()
    assert served == {0, 1} and st["replications"] >= 1 and sum(st["load_paths"]) == 0
    for (n, s), a, b in zip(work, want, got):
        assert np.array_equal(a, b, equal_nan=True), (n, s)
