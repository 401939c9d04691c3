"""Generates the golden fixtures of tests/golden/ from the reference's own code.

    make -C oracle ref            # builds oracle/_ref/libref_cpu.so from the reference's sources
    python tests/golden/make_golden.py

The reference (flarive/CortexRaytracerCuda) ships no tests, golden images or known-answer vectors, so
its own classes, compiled with g++ (oracle/ref_harness.cpp), produce them here:

* rng_kat.npz    T0: thrust::minstd_rand + uniform_real_distribution<float> draws for seeds
                 1984, 2580, 2580+65535 (10^4 each) and the states whose draw rounds to 1.0f;
                 get_int draws (always `min`); the g++ build's multi-draw helpers
                 (random_in_unit_disk, random_in_unit_sphere, random_cosine_direction,
                 directional_light::random, omni_light::random), 500 calls each.
* scenes.npz     T3: per-pixel FP32 radiance sums (pixel_color before prepare_pixel_color) of the
                 five parity scenes at small sizes, g++ draw order; T2: closest-hit primitive ids
                 and t of 4096 seeded random rays per scene.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from cortexraytracercuda_b200 import configs  # noqa: E402
from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, MODE_COMPAT  # noqa: E402

import oracles  # noqa: E402

# the parity scenes and the sizes the fixtures use
GOLDEN_SCENES = {
    "cornell": dict(width=40, height=40, spp=16, max_depth=8),
    "spheres": dict(width=48, height=27, spp=9, max_depth=16),
    "textured": dict(width=40, height=30, spp=9, max_depth=10),
    "icosphere": dict(width=36, height=24, spp=9, max_depth=12),
    "lights": dict(width=40, height=30, spp=9, max_depth=10),
    "xforms": dict(width=40, height=40, spp=9, max_depth=8),   # boxes and transforms
}
RAYS_PER_SCENE = 4096


def golden_params(name):
    _, mp = configs.SCENES[name]
    p = mp(**GOLDEN_SCENES[name])
    p.mode = MODE_COMPAT
    p.draw_order = DRAW_ORDER_HOST
    return p


def golden_rays(name, n=RAYS_PER_SCENE, seed=11):
    rng = np.random.default_rng(seed)
    lo, hi = {"cornell": ([10, 10, -700], [545, 545, 545]), "spheres": ([-12, 0.05, -12], [12, 4, 12])}.get(
        name, ([-4, 0.0, -4], [4, 4, 6]))
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = o
    rays[:, 3] = 1e-5
    rays[:, 4:7] = d
    rays[:, 7] = 3.402823466e38
    return rays


def main():
    ref = oracles.ref_cpu()
    if ref is None:
        raise SystemExit("oracle/_ref/libref_cpu.so is not built (make -C oracle ref)")
    kat = {}
    for seed in (1984, 2580, 2580 + 65535):
        kat[f"draws_{seed}"] = ref.rng_draws(seed, 10000)
    # states x with float(x - 1) * 2^-31 == 1.0f: a seed s gives x1 = 48271*s mod m; search near the top
    kat["get_int_2580_0_5"] = ref.get_int(2580, 0, 5, 1000)
    for which, nm in enumerate(("disk", "sphere", "cosine", "light", "omni")):
        kat[f"sampler_{nm}"] = ref.sampler_draws(which, 2580, 500)
    np.savez_compressed(HERE / "rng_kat.npz", **kat)

    sc = {}
    for name in GOLDEN_SCENES:
        mk, _ = configs.SCENES[name]
        scene = mk()
        p = golden_params(name)
        rs = ref.scene(scene)
        pix = np.arange(p.width * p.height, dtype=np.int64)
        out, rays = rs.render_pixels(p, pix, 0)
        sc[f"{name}_radiance"] = out
        sc[f"{name}_rays"] = np.array([rays], np.uint64)
        R = golden_rays(name)
        for depth, md in ((1, 1), (0, 8)):
            prim, t = rs.trace_closest(R, depth, md)
            sc[f"{name}_hit_{depth}_{md}_prim"] = prim
            sc[f"{name}_hit_{depth}_{md}_t"] = t
    np.savez_compressed(HERE / "scenes.npz", **sc)
    print("wrote", HERE / "rng_kat.npz", HERE / "scenes.npz")


if __name__ == "__main__":
    main()
