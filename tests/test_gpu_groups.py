"""Sample groups (RTC_FLAG_SAMPLE_GROUPS, clean mode): a pixel's samples split into min(8, spp) groups
that run on separate path slots; each group sums its samples in order and the last group to finish adds
the group sums in group order.

* Every sample is the same computation as without groups (same stream, same kernels), so with the drain
  kernel off the image equals the one-group image up to float re-association of the per-pixel sum.
* The reduction order is fixed, so an image is bit-identical alone and in any mix.
* The allocation-free entry point has no scratch for the partial sums and refuses the flag."""
import ctypes as C

import numpy as np
import pytest
import torch

from cortexraytracercuda_b200 import _lib, configs
from cortexraytracercuda_b200._lib import RtcError
from cortexraytracercuda_b200.renderer import DeviceScene, Job, RenderServer
from cortexraytracercuda_b200.scene import (DRAW_ORDER_DEVICE, ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT,
                                            FLAG_SAMPLE_GROUPS, MODE_CLEAN, RenderParams)

pytestmark = pytest.mark.gpu


def _p(name, flags, **kw):
    p = configs.SCENES[name][1](**kw)
    p.mode, p.draw_order, p.engine, p.flags = MODE_CLEAN, DRAW_ORDER_DEVICE, ENGINE_WAVEFRONT, flags
    return p


def _render(ds, p):
    out = torch.full((p.height, p.width, 4), float("nan"), dtype=torch.float32, device="cuda")
    ds.render_device(p, out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name,kw", [("spheres", dict(width=64, height=36, spp=16, max_depth=16)),
                                     ("cornell", dict(width=40, height=40, spp=12, max_depth=8)),
                                     ("textured", dict(width=40, height=30, spp=5, max_depth=10))])
def test_groups_reassociate_only(ctx, monkeypatch, name, kw):
    monkeypatch.setenv("RTC_WF_DRAIN", "1")   # every bounce in the extend/shade kernels
    ds = DeviceScene(ctx, configs.SCENES[name][0]())
    one = _render(ds, _p(name, 0, **kw))
    grp = _render(ds, _p(name, FLAG_SAMPLE_GROUPS, **kw))
    again = _render(ds, _p(name, FLAG_SAMPLE_GROUPS, **kw))
    ds.close()
    assert np.array_equal(grp, again, equal_nan=True)          # deterministic
    a, b = one[..., :3].astype(np.float64), grp[..., :3].astype(np.float64)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-5 * max(a.mean(), 1e-6)), np.abs(a - b).max()


def test_groups_megakernel_agrees_and_noalloc_refuses(ctx):
    kw = dict(width=48, height=27, spp=16, max_depth=12)
    ds = DeviceScene(ctx, configs.spheres())
    wf = _render(ds, _p("spheres", FLAG_SAMPLE_GROUPS, **kw))
    pm = _p("spheres", FLAG_SAMPLE_GROUPS, **kw)
    pm.engine = ENGINE_MEGAKERNEL
    mk = _render(ds, pm)
    a, b = wf[..., :3].astype(np.float64), mk[..., :3].astype(np.float64)
    assert abs(a.mean() - b.mean()) <= 0.02 * b.mean()
    out = torch.empty((kw["height"], kw["width"], 4), dtype=torch.float32, device="cuda")
    pc = _p("spheres", FLAG_SAMPLE_GROUPS, **kw).to_c()
    lib = _lib.load()
    assert lib.rtc_render_noalloc(ds.handle, C.byref(pc), C.c_void_p(out.data_ptr()), None) == 1
    ds.close()


def test_groups_alone_equals_mix_in_batch_and_server(ctx):
    names = ["cornell", "spheres", "textured"]
    scenes = {n: DeviceScene(ctx, configs.SCENES[n][0]()) for n in names}
    items = [("spheres", dict(width=48, height=27, spp=16, max_depth=12)),
             ("cornell", dict(width=32, height=32, spp=9, max_depth=8)),
             ("textured", dict(width=30, height=20, spp=6, max_depth=10))]

    def batch(sel, **bp):
        jobs, outs = [], []
        for n, kw in sel:
            p = _p(n, FLAG_SAMPLE_GROUPS, **kw)
            o = torch.full((p.height, p.width, 4), float("nan"), dtype=torch.float32, device="cuda")
            outs.append(o)
            jobs.append(Job(scenes[n], p, o.data_ptr()))
        ctx.render_batch(jobs, drain=1, **bp)
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in outs]

    alone = batch(items[:1])[0]
    mixed = batch(items[::-1], slots=900, ring=2)[2]
    assert np.array_equal(alone, mixed, equal_nan=True)
    with RenderServer(0, mode=MODE_CLEAN, draw_order=DRAW_ORDER_DEVICE, slots=3000, ring=8, batch=6,
                      flags=FLAG_SAMPLE_GROUPS) as s:
        ids = {n: s.add_scene(configs.SCENES[n][0]()) for n in names}

        def req(n, kw):
            return RenderParams(mode=MODE_CLEAN, draw_order=DRAW_ORDER_DEVICE, **kw)

        solo, _ = s.wait(s.submit(ids["spheres"], req(*items[0]))[0], 60000)
        ts = [s.submit(ids[n], req(n, kw))[0] for n, kw in items[1:] * 4]
        tgt = s.submit(ids["spheres"], req(*items[0]))[0]
        ts += [s.submit(ids[n], req(n, kw))[0] for n, kw in items[1:] * 4]
        mix, _ = s.wait(tgt, 60000)
        for t in ts:
            s.wait(t, 60000)
        st = s.stats()
    assert np.array_equal(solo, mix, equal_nan=True)
    assert np.array_equal(solo, alone, equal_nan=True)      # same kernels as the batch (no drain in either)
    assert st["failed"] == 0
    for d in scenes.values():
        d.close()
