"""The render server (rtc_server_*): continuous admission into a running wavefront, results copied to
the caller's buffers, scenes kept resident under an HBM budget with LRU eviction.

The bar: a request's image is the same alone and in the mix (bit for bit), and equal to the plain
single-image render of that scene and camera (bit for bit in the g++ flavour)."""
import threading

import numpy as np
import pytest
import torch

from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200._lib import RtcError
from cortexraytracercuda_b200.renderer import DeviceScene, RenderServer
from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, ENGINE_WAVEFRONT, MODE_COMPAT, Camera, RenderParams

pytestmark = pytest.mark.gpu

NAMES = ["cornell", "spheres", "textured", "icosphere"]
SIZES = {"cornell": (40, 40, 4, 8), "spheres": (64, 36, 9, 16), "textured": (40, 30, 4, 10),
         "icosphere": (48, 32, 16, 12)}


def _params(name, seed=2580):
    w, h, spp, d = SIZES[name]
    return RenderParams(width=w, height=h, spp=spp, max_depth=d, seed=seed, mode=MODE_COMPAT,
                        draw_order=DRAW_ORDER_HOST, engine=ENGINE_WAVEFRONT)


def _orbit(name, angle):
    """A camera orbiting the scene's own look-at point in the horizontal plane."""
    c = configs.SCENES[name][0]().camera
    f, a = np.array(c.look_from, np.float64), np.array(c.look_at, np.float64)
    r = f - a
    ca, sa = np.cos(angle), np.sin(angle)
    rr = np.array([ca * r[0] + sa * r[2], r[1], -sa * r[0] + ca * r[2]])
    return Camera(look_from=tuple(a + rr), look_at=tuple(a), up=c.up, vfov=c.vfov, aspect=c.aspect,
                  aperture=c.aperture, focus=c.focus)


@pytest.fixture(scope="module")
def server():
    s = RenderServer(0, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, slots=4096, ring=16, batch=4)
    ids = {n: s.add_scene(configs.SCENES[n][0]()) for n in NAMES}
    yield s, ids
    s.close()


def _plain(ctx, name, cam):
    sc = configs.SCENES[name][0]()
    if cam is not None:
        sc.camera = cam
    ds = DeviceScene(ctx, sc)
    p = _params(name)
    out = torch.empty((p.height, p.width, 4), dtype=torch.float32, device="cuda")
    ds.render_device(p, out.data_ptr())
    torch.cuda.synchronize()
    ds.close()
    return out.cpu().numpy()


def test_request_alone_in_the_mix_and_vs_plain(ctx, server):
    s, ids = server
    cam = _orbit("icosphere", 1.1)
    t, _ = s.submit(ids["icosphere"], _params("icosphere"), cam)
    alone, info = s.wait(t, 60000)
    assert info["state"] == 3 and info["paths"] == 48 * 32 * 16
    # the same request among many others, submitted while the first ones render
    tickets = []
    for k in range(24):
        n = NAMES[k % 4]
        tickets.append((n, s.submit(ids[n], _params(n), _orbit(n, 0.3 * k))[0]))
        if k == 11:
            tickets.append(("target", s.submit(ids["icosphere"], _params("icosphere"), cam)[0]))
    mixed = None
    for n, t in tickets:
        out, info = s.wait(t, 120000)
        assert info["state"] == 3
        assert info["submit_ms"] <= info["admit_ms"] <= info["done_ms"]
        if n == "target":
            mixed = out
    assert np.array_equal(alone, mixed, equal_nan=True)
    assert np.array_equal(alone, _plain(ctx, "icosphere", cam), equal_nan=True)


def test_scene_camera_and_concurrent_submitters(ctx, server):
    s, ids = server
    results = {}
    errors = []

    def client(k):
        try:
            n = NAMES[k % 4]
            t, _ = s.submit(ids[n], _params(n))
            out, _ = s.wait(t, 120000)
            results[k] = (n, out)
        except Exception as e:   # reported below
            errors.append(e)

    th = [threading.Thread(target=client, args=(k,)) for k in range(8)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert not errors
    want = {n: _plain(ctx, n, None) for n in NAMES}
    for k, (n, out) in results.items():
        assert np.array_equal(out, want[n], equal_nan=True), n


def test_lru_eviction_under_a_small_budget(ctx):
    probe = RenderServer(0, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, slots=2048, ring=8, batch=4)
    base = probe.stats()["resident_bytes"]
    probe.close()
    scenes = [configs.icosphere_scene(level) for level in (3, 4, 5)]   # ~0.2, 0.8, 3 MB on the device
    sizes = [DeviceScene(ctx, sc).info()["device_bytes"] for sc in scenes]
    # room for the slots, the two largest scenes and one output: never all three scenes at once
    out_bytes = 32 * 24 * 16
    assert min(sizes) > out_bytes + 1024, sizes
    budget = base + sorted(sizes)[-1] + sorted(sizes)[-2] + out_bytes + 1024
    with RenderServer(0, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, slots=2048, ring=8, batch=4,
                      hbm_budget_bytes=budget) as s:
        ids = [s.add_scene(sc) for sc in scenes]
        p = RenderParams(width=32, height=24, spp=4, max_depth=8, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST)
        first = {}
        for rnd in range(3):
            for k, sid in enumerate(ids):
                out, info = s.wait(s.submit(sid, p)[0], 60000)
                if rnd == 0:
                    first[k] = out
                else:
                    assert np.array_equal(out, first[k], equal_nan=True)
        st = s.stats()
        assert st["scene_evictions"] > 0 and st["scene_uploads"] > 3
        assert st["peak_resident_bytes"] <= budget
        assert st["completed"] == 9 and st["failed"] == 0


def test_oversize_request_fails_cleanly():
    with RenderServer(0, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST, slots=1024, ring=4,
                      hbm_budget_bytes=64 << 20) as s:
        sid = s.add_scene(configs.cornell())
        big = RenderParams(width=4096, height=4096, spp=1, max_depth=2, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST)
        t, _ = s.submit(sid, big)
        with pytest.raises(RtcError) as e:
            s.wait(t, 30000)
        assert e.value.status == 4
        small = RenderParams(width=16, height=16, spp=1, max_depth=2, mode=MODE_COMPAT, draw_order=DRAW_ORDER_HOST)
        out, info = s.wait(s.submit(sid, small)[0], 30000)
        assert info["state"] == 3
        with pytest.raises(RtcError) as e:
            s.submit(99, small)
        assert e.value.status == 9


@pytest.mark.parametrize("mode", [MODE_COMPAT, 1])
def test_fma_flavours_alone_equals_mix(mode):
    """The server never runs the drain kernel, so in the FMA-contracting flavours too (nvcc flavour,
    clean mode) a request's image is bit-identical alone and in the mix."""
    from cortexraytracercuda_b200.scene import DRAW_ORDER_DEVICE
    with RenderServer(0, mode=mode, draw_order=DRAW_ORDER_DEVICE, slots=3000, ring=8, batch=4) as s:
        ids = {n: s.add_scene(configs.SCENES[n][0]()) for n in NAMES}

        def p(n):
            q = _params(n)
            q.mode, q.draw_order = mode, DRAW_ORDER_DEVICE
            return q

        cam = _orbit("spheres", 2.0)
        alone, _ = s.wait(s.submit(ids["spheres"], p("spheres"), cam)[0], 60000)
        ts = [s.submit(ids[NAMES[k % 4]], p(NAMES[k % 4]))[0] for k in range(10)]
        target = s.submit(ids["spheres"], p("spheres"), cam)[0]
        ts += [s.submit(ids[NAMES[k % 4]], p(NAMES[k % 4]))[0] for k in range(10)]
        mixed, _ = s.wait(target, 60000)
        for t in ts:
            s.wait(t, 60000)
        assert np.array_equal(alone, mixed, equal_nan=True)
