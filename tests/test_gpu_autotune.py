"""The batch autotuner (cortexraytracercuda_b200/autotune.py): it tries slot counts, poll intervals,
drain thresholds, both BVH node layouts and three block sizes, and keeps the fastest.  Every candidate
must render the same images (g++ flavour: bit for bit), so tuning can only change the speed."""
import numpy as np
import pytest
import torch

from cortexraytracercuda_b200 import autotune, configs
from cortexraytracercuda_b200.renderer import DeviceScene, Job
from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, ENGINE_WAVEFRONT, MODE_COMPAT

pytestmark = pytest.mark.gpu

ITEMS = [("cornell", dict(width=40, height=40, spp=4, max_depth=6)),
         ("spheres", dict(width=48, height=27, spp=4, max_depth=10)),
         ("icosphere", dict(width=36, height=24, spp=9, max_depth=8))]


def test_autotuner_picks_a_candidate_and_every_candidate_renders_the_same(ctx):
    scenes = {n: DeviceScene(ctx, configs.SCENES[n][0]()) for n, _ in ITEMS}
    jobs, outs = [], []
    for n, kw in ITEMS:
        p = configs.SCENES[n][1](**kw)
        p.mode, p.draw_order, p.engine = MODE_COMPAT, DRAW_ORDER_HOST, ENGINE_WAVEFRONT
        o = torch.full((p.height, p.width, 4), float("nan"), dtype=torch.float32, device="cuda")
        outs.append(o)
        jobs.append(Job(scenes[n], p, o.data_ptr()))
    space = {"slots": [1000, 4096], "batch": [6], "drain": [0, 1], "layout": ["binary", "wide"],
             "block": [128, 256, 512]}
    tuned = autotune.autotune_batch(ctx, jobs, space=space, repeats=1, use_cache=False, search="grid")
    assert len(tuned.table) == 24
    assert tuned.slots in space["slots"] and tuned.layout in space["layout"] and tuned.drain in space["drain"]
    assert tuned.block in space["block"]
    assert tuned.ms == min(ms for _, ms in tuned.table)
    want = []
    for (n, kw), j in zip(ITEMS, jobs):
        ref = torch.empty((j.params.height, j.params.width, 4), dtype=torch.float32, device="cuda")
        scenes[n].render_device(j.params, ref.data_ptr())
        torch.cuda.synchronize()
        want.append(ref.cpu().numpy())
    # render once more with every candidate and compare each image with the plain render
    for cfg, _ in tuned.table:
        js = autotune.with_layout(jobs, cfg["layout"])
        ctx.render_batch(js, slots=cfg["slots"], batch=cfg["batch"], drain=cfg["drain"], block=cfg["block"])
        torch.cuda.synchronize()
        for o, w in zip(outs, want):
            assert np.array_equal(o.cpu().numpy(), w, equal_nan=True), cfg
    for s in scenes.values():
        s.close()


def test_autotuner_descent_meets_each_configuration_once(ctx):
    """Coordinate descent times the start point and each knob's values around the best so far; no
    configuration is timed twice, and the result is the fastest one timed."""
    scene = DeviceScene(ctx, configs.cornell())
    p = configs.cornell_params(width=32, height=32, spp=4, max_depth=6)
    o = torch.empty((32, 32, 4), dtype=torch.float32, device="cuda")
    jobs = [Job(scene, p, o.data_ptr())]
    space = {"slots": [512, 1024], "batch": [6, 12], "drain": [0, 1], "layout": ["binary"], "block": [128, 256]}
    tuned = autotune.autotune_batch(ctx, jobs, space=space, repeats=1, use_cache=False,
                                    start={"slots": 1024, "batch": 12, "drain": 0, "layout": "binary", "block": 128})
    keys = [tuple(sorted(c.items())) for c, _ in tuned.table]
    assert len(keys) == len(set(keys)) and 5 <= len(keys) <= 16
    assert tuned.ms == min(ms for _, ms in tuned.table)
    with pytest.raises(ValueError):
        autotune.autotune_batch(ctx, jobs, space=space, use_cache=False, search="random")
    scene.close()
