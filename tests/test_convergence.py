"""Converged-image checks against the double-precision clean-mode estimator (oracle/fp64_clean.c).

* CPU (pinning the oracle): on the same PCG draws, fp64 and the float C restatement in clean mode
  follow the same paths except where rounding flips a branch, so >= 90% of pixels agree within 1e-3
  relative and the image means within 0.5%.
* GPU (T4): the clean kernels' image at N spp converges to the fp64 estimate: with independent seeds,
  RMSE(kernel, fp64) must not exceed 1.2x the seed-to-seed noise floor RMSE(kernel seed A, kernel seed
  B), and the image means must agree within 4 standard errors (a bias would add to both)."""
import numpy as np
import pytest

import oracles
from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200.scene import ENGINE_WAVEFRONT, MODE_CLEAN, RenderParams, Scene


def _small_spheres():
    return configs.spheres(grid=2)


def _ico_scene():
    return configs.icosphere_scene(level=1)


def _textured():
    # floor off the checker cell boundary: on the boundary the cell parity is rounding noise, whose
    # statistics differ between FMA-contracted float, plain float and double arithmetic
    return configs.textured(floor_y=0.013)


CASES = [
    ("cornell", configs.cornell, 32, 32, 8),
    ("textured", _textured, 32, 24, 10),
    ("spheres", _small_spheres, 40, 24, 16),
    ("icosphere", _ico_scene, 36, 24, 12),
    ("uvmesh", configs.uv_mesh_scene, 36, 24, 10),   # image textures through per-vertex texture coordinates
]


@pytest.fixture(scope="module")
def f64():
    o = oracles.fp64()
    if o is None:
        pytest.skip("oracle/librt_fp64.so not built")
    return o


@pytest.mark.parametrize("name,mk,w,h,depth", CASES)
def test_fp64_oracle_matches_float_restatement(f64, name, mk, w, h, depth):
    port = oracles.port()
    if port is None:
        pytest.skip("oracle/librt_port.so not built")
    sc = mk()
    spp = 16
    a = f64.render(sc, w, h, spp, depth, 2580)
    p = RenderParams(width=w, height=h, spp=spp, max_depth=depth, mode=MODE_CLEAN)
    b, _ = port.scene(sc).render_pixels(p, np.arange(w * h), threads=8, trig=0)
    b = b[:, :3].astype(np.float64)
    close = np.mean(np.all(np.isclose(a, b, rtol=1e-3, atol=1e-6), axis=1))
    print(name, "pixels within 1e-3:", close, "mean", a.mean(), b.mean())
    assert close >= 0.9
    assert abs(a.mean() - b.mean()) <= 0.005 * b.mean()


def _kernel(ctx, sc, w, h, spp, depth, seed, flags=0, engine=ENGINE_WAVEFRONT):
    import torch
    from cortexraytracercuda_b200.renderer import DeviceScene
    ds = DeviceScene(ctx, sc)
    p = RenderParams(width=w, height=h, spp=spp, max_depth=depth, seed=seed, mode=MODE_CLEAN, engine=engine,
                     flags=flags)
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    ds.render_device(p, out.data_ptr())
    torch.cuda.synchronize()
    ds.close()
    return out.cpu().numpy().reshape(-1, 4)[:, :3].astype(np.float64) / spp


@pytest.mark.gpu
@pytest.mark.parametrize("name,mk,w,h,depth", CASES)
def test_clean_kernel_converges_to_fp64(ctx, f64, name, mk, w, h, depth):
    sc = mk()
    spp = 256
    ga = _kernel(ctx, sc, w, h, spp, depth, 1234)
    gb = _kernel(ctx, sc, w, h, spp, depth, 98765)
    ref = f64.render(sc, w, h, spp, depth, 55555) / spp
    noise = np.sqrt(np.mean((ga - gb) ** 2))
    err = np.sqrt(np.mean((ga - ref) ** 2))
    se = np.std(ga - gb) / np.sqrt(ga.size) / np.sqrt(2.0)
    print(name, "RMSE vs fp64", err, "noise floor", noise, "means", ga.mean(), ref.mean(), "stderr", se)
    assert err <= 1.2 * noise
    assert abs(ga.mean() - ref.mean()) <= 4.0 * se * np.sqrt(2.0) + 1e-9


@pytest.mark.parametrize("name,mk", [("spheres", lambda: configs.spheres(grid=6)),
                                     ("icosphere", lambda: configs.icosphere_scene(level=3))])
def test_fp64_tree_finds_the_brute_force_hits(f64, name, mk):
    """The fp64 oracle's bounding-volume tree (scenes of more than 64 primitives) changes how closest
    hits are searched, not which are found: its image equals the brute-force search's except where an
    exact-distance tie resolves to another primitive."""
    scene = mk()
    w, h, spp, depth = 24, 16, 4, 8
    try:
        f64.set_bvh_threshold(1 << 30)
        brute = f64.render(scene, w, h, spp, depth, 5)
        f64.set_bvh_threshold(64)
        tree = f64.render(scene, w, h, spp, depth, 5)
    finally:
        f64.set_bvh_threshold(64)
    same = float(np.mean(np.all(np.nan_to_num(brute, nan=-1.0) == np.nan_to_num(tree, nan=-1.0), axis=1)))
    print(name, "identical pixels", same)
    assert same >= 0.99


def _env_scene():
    """Diffuse and textured objects lit by an environment map with a bright sun lobe and a dim sky, and a
    quad light (so the light/cosine/environment mixture is exercised in full)."""
    from cortexraytracercuda_b200.scene import Camera, Scene
    s = Scene(name="envlit")
    s.dir_light((0.0, 5.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (3.0, 3.0, 3.0), intensity=1.0, invisible=True)
    v, f = configs.displaced_icosphere(2, 0.1)
    s.mesh((v + np.array([-1.2, 1.0, 0.0])).astype(np.float32), f, s.lambertian((0.7, 0.7, 0.7)))
    s.sphere((1.2, 1.0, 0.0), 1.0, s.lambertian(s.checker_colors(0.3, (0.8, 0.2, 0.2), (0.9, 0.9, 0.9))))
    s.quad((-8.0, 0.0, -8.0), (16.0, 0.0, 0.0), (0.0, 0.0, 16.0), s.lambertian((0.5, 0.5, 0.5)))
    s.camera = Camera(look_from=(0.0, 2.5, 6.0), look_at=(0.0, 0.9, 0.0), up=(0, 1, 0), vfov=45.0, aspect=1.5,
                      aperture=0.0, focus=6.0)
    s.set_background_env(configs.sky_sun_envmap(128, 64, sun_sigma=0.08, sun_power=60.0))
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("engine", [ENGINE_WAVEFRONT, 1])
def test_env_sampling_converges_to_fp64_with_less_noise(ctx, f64, engine):
    """RTC_FLAG_ENV_SAMPLING (clean mode): lambertian bounces also sample the environment map by its
    luminance.  The estimate converges to the fp64 oracle's (which samples lights and cosine only: the
    same integral) and, on a scene lit mostly by the map's sun, with less seed-to-seed noise than without."""
    from cortexraytracercuda_b200.scene import FLAG_ENV_SAMPLING
    sc = _env_scene()
    w, h, spp, depth = 36, 24, 256, 8
    ga = _kernel(ctx, sc, w, h, spp, depth, 1234, FLAG_ENV_SAMPLING, engine)
    gb = _kernel(ctx, sc, w, h, spp, depth, 98765, FLAG_ENV_SAMPLING, engine)
    na = _kernel(ctx, sc, w, h, spp, depth, 1234, 0, engine)
    nb = _kernel(ctx, sc, w, h, spp, depth, 98765, 0, engine)
    ref = f64.render(sc, w, h, 4 * spp, depth, 55555) / (4 * spp)
    noise = np.sqrt(np.mean((ga - gb) ** 2))
    noise_plain = np.sqrt(np.mean((na - nb) ** 2))
    err = np.sqrt(np.mean((ga - ref) ** 2))
    se = np.std(ga - gb) / np.sqrt(ga.size) / np.sqrt(2.0)
    print("env sampling: RMSE vs fp64", err, "noise", noise, "noise without", noise_plain, "means", ga.mean(),
          ref.mean())
    assert err <= 1.2 * noise
    assert abs(ga.mean() - ref.mean()) <= 4.0 * se * np.sqrt(2.0) + 1e-9
    assert noise < noise_plain
