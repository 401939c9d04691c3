"""The drop-in render call, run on the GPU.

* rtc_launchGPU (replacing launchGPU, core/src/gpu.cu:2127) renders the Cornell box at 64x64, 16 spp,
  depth 8 to a PNG.  Its bytes equal the quantised, row-flipped radiance that rtc_render returns for the
  same parameters (compat mode, seed 2580, the nvcc build's draw order), byte for byte.
* The same frame's 8-bit pixels against the reference's own builds: the g++ flavour against the
  reference's g++ build, every pixel; the nvcc flavour's first bounce against the reference's nvcc
  build.  At least 99% of pixels must be byte-equal (the rest differ by last-ulp trig or FMA rounding,
  which a path tracer amplifies).
* The reference's own command-line program reads a `.scene` file and renders it through the library.
  Its main.cpp, scene loading, srenderer and gpu_cuda_renderer are compiled unchanged, with gpu.cu
  replaced by cortexraytracercuda_b200/seam/launchgpu_b200.cpp (oracle/Makefile target `cli`).  Its
  PNG equals, byte for byte, rtc_launchGPU's on the same file read by rtc_scene_file_load in the
  reference's capacity mode.
"""
import ctypes as C
import subprocess

import numpy as np
import pytest

from cortexraytracercuda_b200 import _lib, configs
from cortexraytracercuda_b200.renderer import DeviceScene
from cortexraytracercuda_b200.scene import (DRAW_ORDER_DEVICE, DRAW_ORDER_HOST, MODE_COMPAT,
                                            SCENE_FILE_REFERENCE_CAPACITY, SCENE_FILE_REFERENCE_MESHES, SceneDesc,
                                            SceneFile, decode_png)

import oracles

pytestmark = pytest.mark.gpu

W = H = 64
SPP, DEPTH = 16, 8
CLI = oracles.ORACLE / "_ref" / "cortex_cli_b200"


def quantize(rad, spp):
    """prepare_pixel_color (color.cuh:289-309), int(255.99 * clamp) and the row flip (gpu.cu:2098-2107)."""
    x = rad[..., :3].astype(np.float32).copy()
    x[np.isnan(x)] = 0.0
    x = np.sqrt(x * (np.float32(1.0) / np.float32(spp)))
    x = np.clip(x, np.float32(0.0), np.float32(0.999))
    return (np.float32(255.99) * x).astype(np.int32).astype(np.uint8)[::-1]


def launch(desc_ptr, path, width=W, height=H, spp=SPP, depth=DEPTH):
    lib = _lib.load()
    _lib.check(lib.rtc_launchGPU(desc_ptr, width, height, spp, depth, 16, 16, str(path).encode(), 1))
    return decode_png(path)


def _params(order, spp=SPP, depth=DEPTH):
    p = configs.cornell_params(width=W, height=H, spp=spp, max_depth=depth)
    p.mode, p.draw_order, p.seed = MODE_COMPAT, order, 2580
    return p


def test_launchgpu_png_equals_render(ctx, tmp_path):
    scene = configs.cornell()
    png = launch(SceneDesc(scene).ptr(), tmp_path / "cornell.png")
    assert png.shape == (H, W, 3)
    rad, _ = DeviceScene(ctx, scene).render(_params(DRAW_ORDER_DEVICE))
    assert np.array_equal(png, quantize(rad, SPP))
    assert png.max() > 0


def test_launchgpu_bytes_vs_reference_builds(ctx, refcpu, refgpu, tmp_path):
    scene = configs.cornell()
    ds = DeviceScene(ctx, scene)
    pix = np.arange(W * H, dtype=np.int64)
    # g++ flavour against the reference's g++ build, full depth
    p = _params(DRAW_ORDER_HOST)
    ours = quantize(ds.render(p)[0], SPP)
    ref = quantize(refcpu.scene(scene).render_pixels(p, pix)[0].reshape(H, W, 4), SPP)
    same = float(np.all(ours == ref, axis=-1).mean())
    print("g++ flavour vs reference g++ build: byte-equal pixels", same)
    assert same >= 0.99
    # rtc_launchGPU's own bytes (nvcc flavour), first bounce, against the reference's nvcc build
    png = launch(SceneDesc(scene).ptr(), tmp_path / "first.png", spp=1, depth=2)
    q = _params(DRAW_ORDER_DEVICE, spp=1, depth=2)
    refg = quantize(refgpu.scene(scene).render_pixels(q, pix).reshape(H, W, 4), 1)
    same = float(np.all(png == refg, axis=-1).mean())
    print("launchGPU first bounce vs reference nvcc build: byte-equal pixels", same)
    assert same >= 0.99


ROOM = r'''
image: { width = 64; height = 64; maxDepth = 8; samplesPerPixel = 16;
         background = { color = { r = 0.0; g = 0.0; b = 0.0; }; }; };
camera: { aspectRatio = "1:1"; lookFrom = { x = 278.0; y = 278.0; z = -800.0; };
          lookAt = { x = 278.0; y = 278.0; z = 0.0; }; upAxis = { x = 0.0; y = 1.0; z = 0.0; }; fov = 40.0; };
lights: {
  directionals: ( { name = "QuadLight1"; position = { x = 278.0; y = 554.0; z = 332.0; };
                    u = { x = -130.0; y = 0.0; z = 0.0; }; v = { x = 0.0; y = 0.0; z = -105.0; };
                    intensity = 1.5; color = { r = 15.0; g = 15.0; b = 15.0; }; invisible = true; } );
};
textures: {
  solidColor: ( { name = "white_texture"; color = { r = 0.73; g = 0.73; b = 0.73; }; } );
  checker: ( { name = "floor_checker"; scale = 60.0; oddColor = { r = 0.2; g = 0.3; b = 0.1; };
               evenColor = { r = 0.9; g = 0.9; b = 0.9; }; } );
};
materials: {
  lambertian: ( { name = "green_material"; color = { r = 0.12; g = 0.45; b = 0.15; }; },
                { name = "red_material"; color = { r = 0.65; g = 0.05; b = 0.05; }; },
                { name = "white_material"; texture = "white_texture"; },
                { name = "floor_material"; texture = "floor_checker"; } );
  metal: ( { name = "mirror"; color = { r = 0.8; g = 0.85; b = 0.88; }; fuzziness = 0.05; } );
};
primitives: {
  spheres: ( { name = "Ball1"; position = { x = 190.0; y = 90.0; z = 190.0; }; radius = 90.0; material = "mirror"; },
             { name = "Ball2"; position = { x = 390.0; y = 70.0; z = 330.0; }; radius = 70.0;
               material = "white_material"; } );
  quads: ( { name = "Quad1"; position = { x = 555.0; y = 0.0; z = 0.0; }; u = { x = 0.0; y = 555.0; z = 0.0; };
             v = { x = 0.0; y = 0.0; z = 555.0; }; material = "green_material"; },
           { name = "Quad2"; position = { x = 0.0; y = 0.0; z = 0.0; }; u = { x = 0.0; y = 555.0; z = 0.0; };
             v = { x = 0.0; y = 0.0; z = 555.0; }; material = "red_material"; },
           { name = "Quad3"; position = { x = 0.0; y = 0.0; z = 0.0; }; u = { x = 555.0; y = 0.0; z = 0.0; };
             v = { x = 0.0; y = 0.0; z = 555.0; }; material = "floor_material"; },
           { name = "Quad4"; position = { x = 555.0; y = 555.0; z = 555.0; }; u = { x = -555.0; y = 0.0; z = 0.0; };
             v = { x = 0.0; y = 0.0; z = -555.0; }; material = "white_material"; },
           { name = "Quad5"; position = { x = 0.0; y = 0.0; z = 555.0; }; u = { x = 555.0; y = 0.0; z = 0.0; };
             v = { x = 0.0; y = 555.0; z = 0.0; }; material = "white_material"; } );
};
'''


def test_reference_cli_renders_through_the_library(tmp_path):
    """The reference's own main() -> scene_manager -> srenderer -> gpu_cuda_renderer -> launchGPU, with
    launchGPU served by the library."""
    if not CLI.exists():
        pytest.skip("oracle/_ref/cortex_cli_b200 not built (make -C oracle cli)")
    scene_path = tmp_path / "room.scene"
    scene_path.write_text(ROOM)
    out = tmp_path / "cli.png"
    # the reference's argument parser reads the word after every flag, so -quiet must not come last
    r = subprocess.run([str(CLI), "-quiet", "-scene", str(scene_path), "-height", str(H), "-ratio", "1:1",
                        "-spp", str(SPP), "-maxdepth", str(DEPTH), "-save", str(out)],
                       capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0 and out.exists(), r.stderr
    cli = decode_png(out)
    sf = SceneFile(scene_path, flags=SCENE_FILE_REFERENCE_CAPACITY | SCENE_FILE_REFERENCE_MESHES)
    ours = launch(sf.ptr(), tmp_path / "lib.png")
    sf.close()
    assert cli.shape == (H, W, 3)
    assert np.array_equal(cli, ours)
    assert cli.max() > 0
