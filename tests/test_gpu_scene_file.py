"""A reference `.scene` file, read by rtc_scene_file_load, rendered on the GPU through the C ABI: the
compat kernel against the C restatement (Port, trig=1) on the same description, pixel for pixel, and the
clean mode against the same file's image mean from the Port's clean estimator."""
import numpy as np
import pytest

from cortexraytracercuda_b200.renderer import DeviceScene
from cortexraytracercuda_b200.scene import DRAW_ORDER_HOST, ENGINE_WAVEFRONT, MODE_COMPAT, SceneFile

import oracles

pytestmark = pytest.mark.gpu

ROOM = r'''
image: { width = 48; height = 36; maxDepth = 8; samplesPerPixel = 8;
         background = { color = { r = 0.05; g = 0.06; b = 0.08; }; }; };
camera: { aspectRatio = "4:3"; lookFrom = { x = 0.0; y = 1.5; z = 6.0; }; lookAt = { x = 0.0; y = 0.8; z = 0.0; };
          upAxis = { x = 0; y = 1; z = 0; }; fov = 45.0; aperture = 0.0; focus = 6.0; };
lights: {
  directionals: ( { position = { x = -1.0; y = 3.5; z = -1.0; }; u = { x = 2.0; y = 0.0; z = 0.0; };
                    v = { x = 0.0; y = 0.0; z = 2.0; }; intensity = 3.0; color = { r = 1.0; g = 1.0; b = 1.0; };
                    invisible = false; } );
  omnis: ( { position = { x = 1.5; y = 2.0; z = 1.0; }; radius = 0.2; intensity = 4.0;
             color = { r = 255; g = 200; b = 150; }; } );
  spots: ( { position = { x = -1.5; y = 3.0; z = 1.0; }; direction = { x = 0.3; y = -1.0; z = 0.0; };
             cutoff = 25.0; falloff = 2.0; intensity = 5.0; radius = 0.1; color = { r = 0.9; g = 0.9; b = 1.0; }; } );
};
textures: {
  solidColor: ( { name = "white"; color = { r = 0.73; g = 0.73; b = 0.73; }; },
                { name = "dark"; color = { r = 0.1; g = 0.1; b = 0.12; }; } );
  checker: ( { name = "floor"; scale = 0.4; oddTextureName = "white"; evenTextureName = "dark"; } );
};
materials: {
  lambertian: ( { name = "ground"; texture = "floor"; }, { name = "red"; color = { r = 0.65; g = 0.05; b = 0.05; }; } );
  metal: ( { name = "brushed"; color = { r = 0.8; g = 0.8; b = 0.9; }; fuzziness = 0.15; } );
  glass: ( { name = "clear"; refraction = 1.5; } );
};
primitives: {
  spheres: ( { position = { x = -1.0; y = 0.6; z = 0.0; }; radius = 0.6; material = "red"; },
             { position = { x = 0.4; y = 0.5; z = 0.6; }; radius = 0.5; material = "clear"; },
             { position = { x = 1.3; y = 0.7; z = -0.5; }; radius = 0.7; material = "brushed"; } );
  quads: ( { position = { x = -4.0; y = 0.0; z = -4.0; }; u = { x = 8.0; y = 0.0; z = 0.0; };
             v = { x = 0.0; y = 0.0; z = 8.0; }; material = "ground"; },
           { position = { x = -4.0; y = 0.0; z = -3.0; }; u = { x = 8.0; y = 0.0; z = 0.0; };
             v = { x = 0.0; y = 4.0; z = 0.0; }; material = "red"; } );
};
'''


@pytest.fixture()
def room(tmp_path):
    p = tmp_path / "room.scene"
    p.write_text(ROOM)
    f = SceneFile(p)
    d = f.desc
    assert (d.num_spheres, d.num_quads, d.num_dir_lights, d.num_omni_lights, d.num_spot_lights) == (3, 2, 1, 1, 1)
    return f


def test_scene_file_render_bitexact_vs_port(ctx, room):
    port = oracles.port()
    if port is None:
        pytest.skip("oracle/librt_port.so not built")
    params = room.params()
    params.mode = MODE_COMPAT
    params.draw_order = DRAW_ORDER_HOST
    params.engine = ENGINE_WAVEFRONT
    ours, rgb8 = DeviceScene(ctx, room).render(params, want_rgb8=True)
    assert ours.shape[:2] == (36, 48) and rgb8.shape == (36, 48, 3)
    pix = np.arange(params.width * params.height, dtype=np.int64)
    ref, _ = port.scene(room).render_pixels(params, pix, trig=1)
    st = oracles.parity_stats(ours.reshape(-1, 4), ref)
    print("room.scene", st)
    assert st["frac_exact"] >= 0.999, st
