"""Device BVH builds against the host SAH build: RTC_BVH_DEVICE (Morton sort + PLOC clustering) and
RTC_BVH_DEVICE_LBVH (Morton sort + linear BVH).

Closest hits do not depend on the tree: every primitive test is the same arithmetic whatever the node
it sits under, and the traversal keeps the nearest t.  Only which of several primitives at exactly the
same t is reported can differ (shared mesh edges, coincident surfaces), so:
  * trace_closest: t bit-identical on every ray, the primitive identical wherever t is not a tie;
  * images (g++ flavour, compat, host draw order): a sample that meets a tie can take another path and
    the pixel's stream moves on differently, so >= 99.5% of pixels bit-identical, image mean within 0.5%;
  * the tree is deterministic (stable radix sort, ties broken by position, PLOC nodes numbered by a
    prefix sum): two builds render the same image bit for bit."""
import numpy as np
import pytest
import torch

from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200.renderer import DeviceScene, RenderServer
from cortexraytracercuda_b200.scene import (BVH_DEVICE, BVH_DEVICE_LBVH, BVH_SAH, DRAW_ORDER_DEVICE, DRAW_ORDER_HOST,
                                            FLAG_WIDE_BVH, MODE_COMPAT, ENGINE_WAVEFRONT, RenderParams, Scene)

pytestmark = pytest.mark.gpu

SCENES = ["cornell", "spheres", "icosphere", "textured"]
BUILDERS = [BVH_DEVICE, BVH_DEVICE_LBVH]


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("name", SCENES)
def test_device_bvh_closest_hit_identity(ctx, name, builder):
    from golden.make_golden import golden_rays
    scene = configs.SCENES[name][0]()
    sah = DeviceScene(ctx, scene, BVH_SAH)
    dev = DeviceScene(ctx, scene, builder)
    info = dev.info()
    assert info["bvh_builder"] == builder and sah.info()["bvh_builder"] == BVH_SAH
    # one primitive per leaf, then subtrees of up to 4 merged where the SAH cost favours a leaf
    assert info["num_nodes"] <= info["num_primitives"] - 1 and 1 <= info["max_leaf_size"] <= 4
    rays = golden_rays(name, 50000, seed=19)
    for depth, max_depth in ((1, 1), (0, 8)):
        a, ta = sah.trace_closest(rays, depth, max_depth)
        b, tb = dev.trace_closest(rays, depth, max_depth)
        assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32)), name
        mism = a != b
        print(name, depth, "hits", int((a >= 0).sum()), "tie mismatches", int(mism.sum()))
        assert int(mism.sum()) <= max(3, int(0.001 * len(rays)))
    sah.close()
    dev.close()


@pytest.mark.parametrize("builder", BUILDERS)
def test_device_bvh_large_mesh_identity(ctx, builder):
    """The meshes scene at level 6: four displaced icospheres, 327,680 triangles."""
    scene = configs.meshes(level=6, env_size=(64, 32))
    sah = DeviceScene(ctx, scene, BVH_SAH)
    dev = DeviceScene(ctx, scene, builder)
    i_s, i_d = sah.info(), dev.info()
    print("build ms: SAH", round(i_s["build_ms"], 1), "device", builder, round(i_d["build_ms"], 1),
          "primitives", i_d["num_primitives"])
    assert i_d["bvh_builder"] == builder
    rng = np.random.default_rng(5)
    n = 200000
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform([-6, 0.2, -6], [6, 4, 6], size=(n, 3))
    rays[:, 3] = 1e-4
    rays[:, 4:7] = rng.normal(size=(n, 3))
    rays[:, 7] = 3.402823466e38
    a, ta = sah.trace_closest(rays, 0, 8)
    b, tb = dev.trace_closest(rays, 0, 8)
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert int((a != b).sum()) <= int(0.001 * n)
    sah.close()
    dev.close()


def _img(ds, p):
    out = torch.full((p.height, p.width, 4), float("nan"), dtype=torch.float32, device="cuda")
    ds.render_device(p, out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("name,kw", [("cornell", dict(width=48, height=48, spp=16, max_depth=8)),
                                     ("icosphere", dict(width=60, height=40, spp=9, max_depth=12)),
                                     ("textured", dict(width=64, height=48, spp=9, max_depth=10))])
def test_device_bvh_images(ctx, name, kw, builder):
    scene = configs.SCENES[name][0]()
    p = configs.SCENES[name][1](**kw)
    p.mode, p.draw_order, p.engine = MODE_COMPAT, DRAW_ORDER_HOST, ENGINE_WAVEFRONT
    sah = DeviceScene(ctx, scene, BVH_SAH)
    dev = DeviceScene(ctx, scene, builder)
    dev2 = DeviceScene(ctx, scene, builder)
    a, b, c = _img(sah, p), _img(dev, p), _img(dev2, p)
    assert np.array_equal(b, c, equal_nan=True)                      # deterministic build
    same = np.mean(np.all((a == b) | (np.isnan(a) & np.isnan(b)), axis=-1))
    ma, mb = np.nanmean(a[..., :3].astype(np.float64)), np.nanmean(b[..., :3].astype(np.float64))
    print(name, "identical pixels", same, "means", ma, mb)
    assert same >= 0.995
    assert abs(ma - mb) <= 0.005 * ma
    # no 8-wide copy: the wide flag falls back to the binary nodes and changes nothing
    pw = configs.SCENES[name][1](**kw)
    pw.mode, pw.draw_order, pw.engine, pw.flags = MODE_COMPAT, DRAW_ORDER_HOST, ENGINE_WAVEFRONT, FLAG_WIDE_BVH
    assert np.array_equal(_img(dev, pw), b, equal_nan=True)
    for d in (sah, dev, dev2):
        d.close()


def test_device_bvh_single_primitive_falls_back(ctx):
    s = Scene(name="one sphere")
    s.sphere((0.0, 0.0, -1.0), 0.5, s.lambertian((0.5, 0.5, 0.5)))
    for builder in BUILDERS:
        ds = DeviceScene(ctx, s, builder)
        assert ds.info()["bvh_builder"] == BVH_SAH
        ds.close()


def test_ploc_identical_boxes(ctx):
    """5,000 spheres at one position: every pair is equally close, and the symmetric tie order pairs
    them up so the rounds halve the clusters (depth ~log2 n) instead of merging one pair a round."""
    s = Scene(name="stack")
    mat = s.lambertian((0.5, 0.5, 0.5))
    for _ in range(5000):
        s.sphere((0.0, 0.0, -1.0), 0.5, mat)
    s.sphere((0.0, -100.5, -1.0), 100.0, mat)
    ds = DeviceScene(ctx, s, BVH_DEVICE)
    info = ds.info()
    # PLOC built it (no SAH fallback); the leaf collapse then merges the coincident spheres in fours
    assert info["bvh_builder"] == BVH_DEVICE and info["num_nodes"] <= 5000 and info["max_leaf_size"] <= 4
    rays = np.zeros((64, 8), np.float32)
    rays[:, 2] = 3.0
    rays[:, 3] = 1e-4
    rays[:, 6] = -1.0
    rays[:, 7] = 3.402823466e38
    prim, t = ds.trace_closest(rays, 0, 8)
    assert np.all(prim >= 0) and np.allclose(t, 3.5, rtol=1e-6)
    ds.close()


def test_server_device_builder(ctx):
    """rtc_server_add_scene with the device builder: the request renders like the SAH-built scene."""
    kw = dict(width=48, height=48, spp=9, max_depth=8)
    imgs = []
    for builder in (BVH_SAH, BVH_DEVICE, BVH_DEVICE_LBVH):
        with RenderServer(0, mode=MODE_COMPAT, draw_order=DRAW_ORDER_DEVICE, slots=4096, ring=4,
                          bvh_builder=builder) as s:
            sid = s.add_scene(configs.cornell())
            img, _ = s.wait(s.submit(sid, RenderParams(mode=MODE_COMPAT, draw_order=DRAW_ORDER_DEVICE, **kw))[0],
                            60000)
            imgs.append(np.asarray(img))
    a = imgs[0]
    for b in imgs[1:]:
        same = np.mean(np.all((a == b) | (np.isnan(a) & np.isnan(b)), axis=-1))
        assert same >= 0.99
        assert abs(np.nanmean(a[..., :3]) - np.nanmean(b[..., :3])) <= 0.01 * np.nanmean(a[..., :3])
