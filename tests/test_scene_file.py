"""Reading the reference's `.scene` files (rtc_scene_file_load): the libconfig syntax and typing, the
scene_loader's reading of each section, and the conversion shared with the sceneConfig adapter.  CPU only:
the files and OBJ meshes are written here; nothing is rendered.

Where the reference tree is present (or the check program was built from it), the same files are also
read by the reference's own scene_loader + libconfig (oracle/Makefile's `scenefile` target,
oracle/scenefile_check.cpp) and the two descriptions must agree field for field; files the reference
refuses (it throws) must be refused here too."""
import json
import os
import struct
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

import oracles

from cortexraytracercuda_b200._lib import RtcError
from cortexraytracercuda_b200.scene import (DRAW_ORDER_HOST, MAT_DIELECTRIC, MAT_LAMBERTIAN, MAT_METAL, SCENE_FILE_REFERENCE_CAPACITY, SCENE_FILE_REFERENCE_MESHES,
                                            TEX_CHECKER, TEX_IMAGE, TEX_SOLID, SceneFile, decode_png)

SCENE = r'''
# a scene in the reference's format: comments of every kind
image:
{
    width = 320; height = 0x00B4;   // hexadecimal
    maxDepth = 12;
    samplesPerPixel = 16L;          /* 64-bit suffix */
    background = { color = { r = 0.1; g = 0.2; b = 0.3; }; };
};
camera:
{
    aspectRatio = "16:9";
    lookFrom = { x = 0.0; y = 2; z = 9.5; };
    lookAt = { x = 0.0; y = 1.0; z = 0.0; };
    upAxis = { x = 0; y = 1; z = 0; };
    fov = 35.0; aperture = 0.05; focus = 9.0;
};
lights:
{
    directionals: (
        { name = "Quad" "Light"; position = { x = 0.0; y = 5.0; z = 0.0; };
          u = { x = 2.0; y = 0.0; z = 0.0; }; v = { x = 0.0; y = 0.0; z = 2.0; };
          intensity = 2.0; color = { r = 4.0; g = 4.0; b = 4.0; }; invisible = false; },
        { name = "Off"; position = { x = 0.0; y = 9.0; z = 0.0; }; u = { x = 1.0; y = 0.0; z = 0.0; };
          v = { x = 0.0; y = 0.0; z = 1.0; }; intensity = 1.0; color = { r = 1.0; g = 1.0; b = 1.0; }; active = false; }
    );
    omnis: ( { name = "Bulb"; position = { x = 1.0; y = 3.0; z = 1.0; }; radius = 0.25; intensity = 3;
               color = { r = 5.0; g = 4.0; b = 3.0; }; } );
    spots: ( { name = "Spot"; position = { x = 0.0; y = 4.0; z = 2.0; }; direction = { x = 0.0; y = -1.0; z = 0.0; };
               cutoff = 30.0; falloff = 2.0; intensity = 4.0; radius = 0.1; color = { r = 6.0; g = 6.0; b = 6.0; };
               invisible = true; } );
};
textures:
{
    solidColor: ( { name = "white"; color = { r = 0.73; g = 0.73; b = 0.73; }; },
                  { name = "black"; color = { r = 0.05; g = 0.05; b = 0.05; }; } );
    checker: ( { name = "named"; scale = 0.5; oddTextureName = "white"; evenTextureName = "black"; },
               { name = "colors"; scale = 2.0; oddColor = { r = 1.0; g = 0.0; b = 0.0; };
                 evenColor = { r = 0.0; g = 0.0; b = 1.0; }; } );
    image: ( { name = "pic"; filepath = "pic.png"; } );
    noise: ( { name = "perlin"; scale = 1.0; } );
};
materials:
{
    lambertian: ( { name = "matte"; color = { r = 0.5; g = 0.4; b = 0.3; }; },
                  { name = "floor"; texture = "named"; },
                  { name = "painted"; texture = "pic"; } );
    metal: ( { name = "mirror"; color = { r = 0.9; g = 0.9; b = 0.9; }; fuzziness = 2.5; } );
    glass: ( { name = "clear"; refraction = 1.5; } );
    phong: ( { name = "shiny"; } );
};
primitives:
{
    spheres: ( { name = "s1"; position = { x = -1.0; y = 1.0; z = 0.0; }; radius = 1; material = "matte"; },
               { name = "s2"; position = { x = 1.0; y = 1.0; z = 0.0; }; radius = 0.5; material = "clear"; },
               { name = "s3"; position = { x = 3.0; y = 1.0; z = 0.0; }; radius = 0.5; material = "nosuch"; },
               { name = "s4"; position = { x = 5.0; y = 1.0; z = 0.0; }; radius = 0.5; material = "painted"; } );
    quads: ( { name = "ground"; position = { x = -5.0; y = 0.0; z = -5.0; }; u = { x = 10.0; y = 0.0; z = 0.0; };
               v = { x = 0.0; y = 0.0; z = 10.0; }; material = "floor"; } );
    boxes: ( { name = "crate"; position = { x = 0.0; y = 0.5; z = 0.0; }; size = { x = 1.0; y = 1.0; z = 1.0; };
               material = "matte"; } );
};
meshes:
{
    obj: ( { name = "tri"; filepath = "tri.obj"; position = { x = 0.0; y = 2.0; z = 0.0; }; material = "mirror";
             use_smoothing = true; } );
};
'''

OBJ = """v 0 0 0
v 1 0 0
v 0 1 0
vn 0 0 1
f 1//1 2//1 3//1
"""


def _png(path, px):
    """Writes an 8-bit RGB PNG with the Sub filter on every row (exercises the decoder's filters)."""
    h, w, _ = px.shape
    raw = b""
    for y in range(h):
        row = px[y].astype(np.int32).reshape(-1)
        sub = row.copy()
        sub[3:] = (row[3:] - row[:-3]) & 255
        raw += b"\x01" + sub.astype(np.uint8).tobytes()

    def chunk(k, b):
        return struct.pack(">I", len(b)) + k + b + struct.pack(">I", zlib.crc32(k + b) & 0xFFFFFFFF)
    path.write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
                     chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))


@pytest.fixture()
def scene_dir(tmp_path):
    (tmp_path / "demo.scene").write_text(SCENE)
    (tmp_path / "tri.obj").write_text(OBJ)
    px = (np.arange(4 * 3 * 3).reshape(4, 3, 3) * 7 % 256).astype(np.uint8)
    _png(tmp_path / "pic.png", px)
    return tmp_path, px


def _texture(d, i):
    return d.textures[i]


def test_sections_read_like_scene_loader(scene_dir):
    path, px = scene_dir
    f = SceneFile(path / "demo.scene")
    d = f.desc
    assert f.info == {"width": 320, "height": 180, "spp": 16, "max_depth": 12, "num_skipped": len(f.skipped)}
    p = f.params()
    assert (p.width, p.height, p.spp, p.max_depth) == (320, 180, 16, 12)
    # camera: "16:9" -> 16/9; integers read as floats
    assert d.camera.aspect == pytest.approx(16 / 9) and list(d.camera.look_from) == [0.0, 2.0, 9.5]
    assert d.camera.vfov == 35.0 and d.camera.aperture == pytest.approx(0.05) and d.camera.focus == 9.0
    assert list(d.background.color) == pytest.approx([0.1, 0.2, 0.3])
    # lights: the inactive directional light is left out; adjacent string literals join; `intensity = 3`
    # is an integer where scene_loader looks up a float, so the omni light keeps its initial 0
    assert d.num_dir_lights == 1 and d.dir_lights[0].intensity == 2.0 and d.dir_lights[0].invisible == 0
    assert d.num_omni_lights == 1 and d.omni_lights[0].intensity == 0.0 and d.omni_lights[0].invisible == 1
    assert d.num_spot_lights == 1 and d.spot_lights[0].cutoff == 30.0 and d.spot_lights[0].falloff == 2.0
    # spheres: the one with an unknown material is skipped (gpu.cu:531); `radius = 1` reads as 0 (typing)
    assert d.num_spheres == 3 and [d.spheres[i].radius for i in range(3)] == [0.0, 0.5, 0.5]
    mats = [d.materials[d.spheres[i].material] for i in range(3)]
    assert [m.kind for m in mats] == [MAT_LAMBERTIAN, MAT_DIELECTRIC, MAT_LAMBERTIAN]
    assert mats[1].ior == 1.5
    pic = _texture(d, mats[2].texture)
    assert pic.kind == TEX_IMAGE and d.num_images == 1
    img = d.images[pic.image]
    assert (img.width, img.height) == (3, 4)
    got = np.ctypeslib.as_array(img.rgb, shape=(4 * 3 * 3,)).reshape(4, 3, 3)
    assert np.array_equal(got, px)
    # the floor's named checker: checker_texture(scale, odd, even) stores odd in m_even
    floor = d.materials[d.quads[0].material]
    chk = _texture(d, floor.texture)
    assert chk.kind == TEX_CHECKER and chk.scale == 0.5
    assert list(_texture(d, chk.even).color) == pytest.approx([0.73] * 3)    # odd texture "white"
    assert list(_texture(d, chk.odd).color) == pytest.approx([0.05] * 3)     # even texture "black"
    # the OBJ mesh: offset by its position, smooth with its normals, metal fuzz clamped to 1
    assert d.num_meshes == 1
    m = d.meshes[0]
    assert (m.num_vertices, m.num_triangles, m.smooth) == (3, 1, 1)
    assert np.ctypeslib.as_array(m.vertices, shape=(9,)).tolist() == [0, 2, 0, 1, 2, 0, 0, 3, 0]
    metal = d.materials[m.material]
    assert metal.kind == MAT_METAL and metal.fuzz == 1.0
    assert d.num_boxes == 1 and list(d.boxes[0].size) == [1.0, 1.0, 1.0] and d.boxes[0].transform == 0
    assert not any("boxes" in s for s in f.skipped) and any("noise" in s for s in f.skipped)
    assert any("phong" in s for s in f.skipped)
    f.close()


def test_reference_glass_quirk_reproduced_on_request(scene_dir):
    path, _ = scene_dir
    f = SceneFile(path / "demo.scene", flags=SCENE_FILE_REFERENCE_CAPACITY)
    d = f.desc
    assert d.num_spheres == 2          # the glass sphere goes with its material, as in the reference
    assert all(d.materials[d.spheres[i].material].kind != MAT_DIELECTRIC for i in range(2))
    assert any("glass" in s for s in f.skipped)


def test_images_skipped_without_decoder(scene_dir):
    path, _ = scene_dir
    f = SceneFile(path / "demo.scene", decode_images=False)
    assert f.desc.num_images == 0 and f.desc.num_spheres == 2
    assert any("image texture without loader" in s for s in f.skipped)


@pytest.mark.parametrize("text,where", [("image: { width = 3 }\ncamera = { fov = ; };", "line 2"),
                                        ("a = \"open", "unterminated"), ("@include \"x.cfg\"", "@include"),
                                        ("lights = ( 1, 2 ", "closing")])
def test_syntax_errors_name_the_line(tmp_path, text, where):
    (tmp_path / "bad.scene").write_text(text)
    with pytest.raises(RtcError) as e:
        SceneFile(tmp_path / "bad.scene")
    assert where in str(e.value) and e.value.status == 2


def test_missing_file(tmp_path):
    with pytest.raises(RtcError) as e:
        SceneFile(tmp_path / "none.scene")
    assert e.value.status == 7


def test_png_decoder_filters(tmp_path):
    px = np.random.default_rng(1).integers(0, 256, size=(5, 7, 3), dtype=np.uint8)
    _png(tmp_path / "x.png", px)
    assert np.array_equal(decode_png(tmp_path / "x.png"), px)
    assert decode_png(tmp_path / "missing.png") is None


# ---- against the reference's own scene_loader ------------------------------------------------------------
ROOT = Path(__file__).resolve().parent.parent
REF_EXE = ROOT / "oracle" / "_ref" / "scenefile_check"


@pytest.fixture(scope="module")
def ref_loader():
    ref = str(oracles.REFERENCE)
    if (Path(ref) / "core" / "src" / "scenes" / "scene_loader.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "scenefile", f"REF={ref}"], check=True,
                       capture_output=True)
    if not REF_EXE.exists():
        pytest.skip("the reference's scene_loader is not available to build the check program")
    return REF_EXE


def _ref_read(exe, path):
    """The reference's description of `path` (read with the scene's directory as working directory, which
    is where scene_loader resolves relative paths), or None when it refuses the file."""
    r = subprocess.run([str(exe), path.name], cwd=path.parent, capture_output=True, text=True, timeout=60)
    if r.returncode != 0:
        return None
    return json.loads(r.stdout.strip().splitlines()[-1])


def _arr(p, n):
    return [float(p[i]) for i in range(n)]


def _refs(p, n):
    return [int(p[i]) for i in range(n)] if p else []


def _desc_json(f):
    """The fields oracle/scenefile_check.cpp prints, from this library's description."""
    d, info = f.desc, f.info
    return {
        "textures": [{"kind": t.kind, "color": _arr(t.color, 3), "scale": t.scale, "even": t.even, "odd": t.odd,
                      "image": t.image} for t in (d.textures[i] for i in range(d.num_textures))],
        "materials": [{"kind": m.kind, "texture": m.texture, "fuzz": m.fuzz, "ior": m.ior}
                      for m in (d.materials[i] for i in range(d.num_materials))],
        "dir_lights": [{"position": _arr(l.position, 3), "u": _arr(l.u, 3), "v": _arr(l.v, 3),
                        "color": _arr(l.color, 3), "intensity": l.intensity, "invisible": l.invisible}
                       for l in (d.dir_lights[i] for i in range(d.num_dir_lights))],
        "omni_lights": [{"position": _arr(l.position, 3), "color": _arr(l.color, 3), "radius": l.radius,
                         "intensity": l.intensity, "invisible": l.invisible}
                        for l in (d.omni_lights[i] for i in range(d.num_omni_lights))],
        "spot_lights": [{"position": _arr(l.position, 3), "direction": _arr(l.direction, 3),
                         "color": _arr(l.color, 3), "cutoff": l.cutoff, "falloff": l.falloff, "radius": l.radius,
                         "intensity": l.intensity, "invisible": l.invisible}
                        for l in (d.spot_lights[i] for i in range(d.num_spot_lights))],
        "spheres": [{"center": _arr(s.center, 3), "radius": s.radius, "material": s.material}
                    for s in (d.spheres[i] for i in range(d.num_spheres))],
        "quads": [{"q": _arr(q.q, 3), "u": _arr(q.u, 3), "v": _arr(q.v, 3), "material": q.material}
                  for q in (d.quads[i] for i in range(d.num_quads))],
        "boxes": [{"center": _arr(b.center, 3), "size": _arr(b.size, 3), "material": b.material,
                   "transform": b.transform} for b in (d.boxes[i] for i in range(d.num_boxes))],
        "transforms": [{"translate": _arr(x.translate, 3), "rotate": _arr(x.rotate, 3), "scale": _arr(x.scale, 3),
                        "flags": x.flags} for x in (d.transforms[i] for i in range(d.num_transforms))],
        "sphere_transforms": _refs(d.sphere_transforms, d.num_spheres),
        "quad_transforms": _refs(d.quad_transforms, d.num_quads),
        "mesh_transforms": _refs(d.mesh_transforms, d.num_meshes),
        "meshes": [{"vertices": _arr(m.vertices, 3 * m.num_vertices), "num_triangles": m.num_triangles,
                    "material": m.material, "smooth": m.smooth} for m in (d.meshes[i] for i in range(d.num_meshes))],
        "camera": {"look_from": _arr(d.camera.look_from, 3), "look_at": _arr(d.camera.look_at, 3),
                   "up": _arr(d.camera.up, 3), "vfov": d.camera.vfov, "aspect": d.camera.aspect,
                   "aperture": d.camera.aperture, "focus": d.camera.focus},
        "background": _arr(d.background.color, 3),
        "image": {k: info[k] for k in ("width", "height", "spp", "max_depth")},
    }


def _same(a, b, where=""):
    """Equal structures; floats compared as float32 (the check program prints 9 significant digits)."""
    if isinstance(a, dict):
        assert a.keys() == b.keys(), where
        for k in a:
            _same(a[k], b[k], f"{where}.{k}")
    elif isinstance(a, list):
        assert len(a) == len(b), where
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{where}[{i}]")
    elif isinstance(a, float) or isinstance(b, float):
        assert np.float32(a) == np.float32(b), (where, a, b)
    else:
        assert a == b, (where, a, b)


TYPING = r'''
image: { width = 64; height = 48L; maxDepth = 010; samplesPerPixel = 0x10;
         background = { color = { r = 255; g = 128; b = 0; }; }; };
camera: { aspectRatio = "4:3"; lookFrom = { x = 1; y = 2.5; z = 3L; }; fov = 40.0; };
lights: {
  omnis: ( { position = { x = 0.0; y = 1.0; z = 0.0; }; radius = 0.5; intensity = 2;
             color = { r = 1; g = 0.5; b = 0.5; }; invisible = 0; },
           { position = { x = 2.0; y = 1.0; z = 0.0; }; radius = 5e-1; intensity = 2.; color = { r = 9; g = 9; b = 9; }; } );
  spots: ( { position = { x = 0; y = 4; z = 0; }; direction = { x = 0; y = -1; z = 0; }; cutoff = 20; falloff = 1.5;
             intensity = 3.0; radius = .25; color = { r = 0.9; g = 0.8; b = 0.7; }; active = true; }, );
};
textures: {
  solidColor: ( { name = "a\x41\q"; color = { r = 10; g = 20; b = 30; }; },
                { name = "neg"; color = { r = -1; g = 20; b = 30; }; }, );
  checker: ( { name = "chk"; scale = 3; oddColor = { r = 1.0; g = 1.0; b = 1.0; }; evenColor = { r = 0; g = 0; b = 0; }; } );
};
materials: {
  lambertian: ( { name = "m1"; texture = "a\x41\q"; }, { name = "m2"; texture = "neg"; }, { name = "m3"; texture = "chk"; } );
  metal: ( { name = "steel"; color = { r = 200; g = 200; b = 200; }; fuzziness = 0.25; } );
};
primitives: {
  spheres: ( { position = { x = 0.0; y = 0.0; z = 0.0; }; radius = 1.0; material = "m1"; },
             { position = { x = 2; y = 0; z = 0; }; radius = 1.0; material = "m2"; active = 0; },
             { position = { x = 4; y = 0; z = 0; }; radius = 1.0; material = "m3"; active = false; },
             { position = { x = 6; y = 0; z = 0; }; radius = 1.0; material = "steel"; } );
  quads: ( { position = { x = -1; y = 0; z = -1; }; u = { x = 2; y = 0; z = 0; }; v = { x = 0; y = 0; z = 2; };
             material = "m3"; } );
};
'''


def test_libconfig_typing(tmp_path):
    (tmp_path / "t.scene").write_text(TYPING)
    f = SceneFile(tmp_path / "t.scene")
    d = f.desc
    assert f.info["width"] == 64 and f.info["height"] == 48 and f.info["max_depth"] == 8 and f.info["spp"] == 16
    assert list(d.background.color) == pytest.approx([1.0, 128 / 255, 0.0])            # three integers: 0-255
    assert d.camera.aspect == pytest.approx(4 / 3) and list(d.camera.look_from) == [1.0, 2.5, 3.0]
    assert d.camera.focus == 100.0 and list(d.camera.look_at) == [0, 0, 0]              # scene_builder defaults
    o = d.omni_lights[0]
    assert o.intensity == 0.0 and list(o.color) == pytest.approx([0.0, 0.5, 0.5]) and o.invisible == 1
    assert d.omni_lights[1].radius == 0.5 and list(d.omni_lights[1].color) == pytest.approx([9 / 255] * 3)
    assert d.spot_lights[0].cutoff == 0.0 and d.spot_lights[0].radius == 0.25
    assert d.num_spheres == 3           # `active = 0` is an integer: the sphere stays active
    m = [d.materials[d.spheres[i].material] for i in range(3)]
    assert list(d.textures[m[0].texture].color) == pytest.approx([10 / 255, 20 / 255, 30 / 255])
    assert list(d.textures[m[1].texture].color) == [0.0, 0.0, 0.0]                    # -1 and two integers
    assert list(d.textures[m[2].texture].color) == pytest.approx([200 / 255] * 3)      # metal albedo
    chk = d.textures[d.materials[d.quads[0].material].texture]
    assert chk.scale == 0.0                                                             # `scale = 3`


def test_defaults_without_image_and_camera(tmp_path):
    (tmp_path / "e.scene").write_text("# nothing but a comment\n")
    f = SceneFile(tmp_path / "e.scene")
    assert f.info == {"width": 400, "height": 225, "spp": 50, "max_depth": 100, "num_skipped": 0}
    c = f.desc.camera
    assert list(c.look_from) == [0, 0, 10] and c.vfov == 70.0 and c.focus == 100.0
    assert c.aspect == pytest.approx(16 / 9)


CAPACITY = """
materials: { dielectric: ( { name = "unused"; } );
             glass: ( { name = "g1"; refraction = 1.5; }, { name = "g2"; refraction = 1.3; } );
             lambertian: ( { name = "grey"; color = { r = 0.5; g = 0.5; b = 0.5; }; } ); };
primitives: { spheres: ( { position = { x = 0.0; y = 0.0; z = 0.0; }; radius = 1.0; material = "g1"; },
                         { position = { x = 3.0; y = 0.0; z = 0.0; }; radius = 1.0; material = "g2"; },
%s ); };
"""


def _capacity_scene(tmp_path, n_extra):
    extra = ",\n".join(f'{{ position = {{ x = {i}.0; y = 5.0; z = 0.0; }}; radius = 0.25; material = "grey"; }}'
                       for i in range(n_extra))
    p = tmp_path / "cap.scene"
    p.write_text(CAPACITY % extra)
    return p


def test_reference_capacity(tmp_path):
    p = _capacity_scene(tmp_path, 256)          # 258 spheres: the reference's uint8_t count holds 2
    every = SceneFile(p)
    assert every.desc.num_spheres == 258
    ref = SceneFile(p, flags=SCENE_FILE_REFERENCE_CAPACITY)
    d = ref.desc
    assert d.num_spheres == 1                   # g1 fits the dielectric table sized by `dielectric`; g2 does not
    assert d.materials[d.spheres[0].material].kind == MAT_DIELECTRIC
    assert any("table capacity: sphere" in s for s in ref.skipped)


def test_missing_obj_ends_meshes(tmp_path):
    (tmp_path / "tri.obj").write_text(OBJ)
    (tmp_path / "m.scene").write_text('''
materials: { lambertian: ( { name = "grey"; color = { r = 0.5; g = 0.5; b = 0.5; }; } ); };
meshes: { obj: ( { filepath = "tri.obj"; material = "grey"; },
                 { filepath = "gone.obj"; material = "grey"; },
                 { filepath = "tri.obj"; material = "grey"; position = { x = 1.0; y = 0.0; z = 0.0; }; } ); };
''')
    f = SceneFile(tmp_path / "m.scene")
    assert f.desc.num_meshes == 1 and f.desc.meshes[0].smooth == 1     # use_smoothing defaults to true
    assert any("obj file not found" in s for s in f.skipped)


QUAD_OBJ = """v 0 0 0
v 2 0 0
v 2 2 0
v 0 2 0
f 1 2 3 4
"""


def test_reference_meshes_flag(tmp_path):
    """RTC_SCENE_FILE_REFERENCE_MESHES: every entry renders meshes[0]'s file (gpu.cu:626-631) with its own
    material, without its position or transform (scene_factory.cuh:373-385)."""
    (tmp_path / "tri.obj").write_text(OBJ)
    (tmp_path / "quad.obj").write_text(QUAD_OBJ)
    (tmp_path / "m.scene").write_text('''
materials: { lambertian: ( { name = "grey"; color = { r = 0.5; g = 0.5; b = 0.5; }; },
                           { name = "red"; color = { r = 0.9; g = 0.1; b = 0.1; }; } ); };
meshes: { obj: ( { filepath = "tri.obj"; material = "grey"; position = { x = 0.0; y = 3.0; z = 0.0; }; },
                 { filepath = "quad.obj"; material = "red"; use_smoothing = false;
                   position = { x = 1.0; y = 0.0; z = 0.0; };
                   transform = { rotate = { x = 0.0; y = 45.0; z = 0.0; }; }; } ); };
''')
    tri = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
    own = SceneFile(tmp_path / "m.scene")
    d = own.desc
    assert d.num_meshes == 2 and d.meshes[1].num_triangles == 2
    assert np.array_equal(_arr(d.meshes[0].vertices, 9), tri + np.tile(np.float32([0, 3, 0]), 3))
    assert d.mesh_transforms[1] != 0
    ref = SceneFile(tmp_path / "m.scene", flags=SCENE_FILE_REFERENCE_MESHES)
    r = ref.desc
    assert r.num_meshes == 2
    for i in range(2):
        assert r.meshes[i].num_triangles == 1 and r.meshes[i].num_vertices == 3
        assert np.array_equal(_arr(r.meshes[i].vertices, 9), tri)
        assert not r.mesh_transforms or r.mesh_transforms[i] == 0
    assert (r.meshes[0].smooth, r.meshes[1].smooth) == (1, 0)
    assert r.meshes[0].material != r.meshes[1].material
    assert [r.textures[r.materials[r.meshes[i].material].texture].color[0] for i in range(2)] == pytest.approx([0.5, 0.9])


UV_OBJ = """v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0.0 0.0
vt 0.25 0.0
vt 0.25 0.5
vt 0.0 0.5
f 1/1 2/2 3/3 4/4
"""


def test_obj_texture_coordinates(tmp_path):
    """`vt` coordinates reach the mesh (2 per vertex); with RTC_SCENE_FILE_REFERENCE_MESHES they are read as
    mesh_loader reads them, texcoords[3 * i] and [3 * i + 1] from the array of 2 per vertex
    (mesh_loader.cuh:370-371), reads past its end giving 0."""
    (tmp_path / "sq.obj").write_text(UV_OBJ)
    (tmp_path / "m.scene").write_text(
        'materials: { lambertian: ( { name = "grey"; color = { r = 0.5; g = 0.5; b = 0.5; }; } ); };\n'
        'meshes: { obj: ( { filepath = "sq.obj"; material = "grey"; } ); };\n')
    own_file = SceneFile(tmp_path / "m.scene")   # the description lives as long as its file object
    own = own_file.desc
    uv = np.array([0.0, 0.0, 0.25, 0.0, 0.25, 0.5, 0.0, 0.5], np.float32)
    assert own.meshes[0].num_vertices == 4 and np.array_equal(_arr(own.meshes[0].uvs, 8), uv)
    ref_file = SceneFile(tmp_path / "m.scene", flags=SCENE_FILE_REFERENCE_MESHES)
    ref = ref_file.desc
    strided = np.array([uv[0], uv[1], uv[3], uv[4], uv[6], uv[7], 0.0, 0.0], np.float32)
    assert np.array_equal(_arr(ref.meshes[0].uvs, 8), strided)


REFUSED = [
    ("camera: { aperture = 1; };", "aperture"),                   # an integer handed to a float setter
    ("camera: { aspectRatio = 1.5; };", "aspectRatio"),           # not a string
    ("camera: { aspectRatio = \"wide\"; };", "aspectRatio"),      # std::stof refuses it
    ("image: { width = 1.5; };", "width"),
    ("image: { height = 3000000000; };", "out of range"),
    ("camera: { orthographic = 1; };", "orthographic"),
    ("materials: { metal: ( { color = { r = 1.0; g = 1.0; b = 1.0; }; } ); };", "Material name is empty"),
    ("textures: { checker: ( { scale = 1.0; } ); };", "Checker texture name is empty"),
    ("primitives: { spheres: ( { radius = 1.0; active = false; } ); };", "Material name is empty"),
]


@pytest.mark.parametrize("text,what", REFUSED)
def test_refused_like_the_reference(tmp_path, text, what):
    (tmp_path / "bad.scene").write_text(text)
    with pytest.raises(RtcError) as e:
        SceneFile(tmp_path / "bad.scene")
    assert e.value.status == 2 and what in str(e.value)


@pytest.mark.parametrize("text,where", [
    ("a = 1; a = 2;", "duplicate"), ("a = [1, 2.0];", "mismatched"), ("a = [1, (2)];", "scalar"),
    ("a = 09;", "bad value"), ("a = -0x10;", "bad value"), ("a = 1.5e;", "bad value"),
])
def test_grammar_errors(tmp_path, text, where):
    (tmp_path / "g.scene").write_text(text)
    with pytest.raises(RtcError) as e:
        SceneFile(tmp_path / "g.scene")
    assert where in str(e.value)


def test_ratio_edge_cases(tmp_path):
    for text, aspect in [('"16:"', 0.0), ('"2:1:7"', 2.0), ('"-4:3"', 0.0), ('" 3 : 2"', 1.5)]:
        (tmp_path / "r.scene").write_text(f"camera: {{ aspectRatio = {text}; }};")
        assert SceneFile(tmp_path / "r.scene").desc.camera.aspect == pytest.approx(aspect), text


def _write_all(tmp_path):
    """The scene files compared with the reference's loader, with their OBJ and image files."""
    (tmp_path / "tri.obj").write_text(OBJ)
    _png(tmp_path / "pic.png", (np.arange(4 * 3 * 3).reshape(4, 3, 3) * 7 % 256).astype(np.uint8))
    files = {"demo": SCENE, "typing": TYPING, "empty": "# empty\n",
             "meshes": '''materials: { lambertian: ( { name = "grey"; color = { r = 0.5; g = 0.5; b = 0.5; }; } ); };
meshes: { obj: ( { filepath = "tri.obj"; material = "grey"; use_smoothing = false; },
                 { filepath = "gone.obj"; material = "grey"; },
                 { filepath = "tri.obj"; material = "grey"; } ); };''',
             "images": '''textures: { image: ( { name = "p"; filepath = "pic.png"; }, { name = "q"; filepath = "none.png"; },
                            { name = "r"; filepath = "pic.png"; } ); };
materials: { lambertian: ( { name = "pm"; texture = "p"; }, { name = "rm"; texture = "r"; } ); };
primitives: { spheres: ( { position = { x = 0.0; y = 0.0; z = 0.0; }; radius = 1.0; material = "pm"; },
                         { position = { x = 2.0; y = 0.0; z = 0.0; }; radius = 1.0; material = "rm"; } ); };'''}
    paths = {}
    for k, v in files.items():
        paths[k] = tmp_path / f"{k}.scene"
        paths[k].write_text(v)
    paths["capacity"] = _capacity_scene(tmp_path, 256)
    return paths


def test_matches_reference_loader(tmp_path, ref_loader):
    for name, path in _write_all(tmp_path).items():
        ref = _ref_read(ref_loader, path)
        assert ref is not None, name
        mine = SceneFile(path, flags=SCENE_FILE_REFERENCE_CAPACITY, decode_images=False)
        _same(ref, _desc_json(mine), name)


def test_reference_refuses_the_same_files(tmp_path, ref_loader):
    for i, (text, _) in enumerate(REFUSED):
        p = tmp_path / f"bad{i}.scene"
        p.write_text(text)
        assert _ref_read(ref_loader, p) is None, text


def test_scene_file_renders_like_the_reference_cpu(tmp_path, refcpu):
    """The description read from a `.scene` file, rendered by the C restatement (Port, glibc float
    trig) and by the reference's own classes built with g++ (RefCpu): identical pixels."""
    import oracles
    from test_gpu_scene_file import ROOM
    port = oracles.port()
    if port is None:
        pytest.skip("oracle/librt_port.so not built")
    (tmp_path / "room.scene").write_text(ROOM)
    f = SceneFile(tmp_path / "room.scene")
    p = f.params(spp=4, draw_order=DRAW_ORDER_HOST)   # the g++ build's argument evaluation order
    pix = np.arange(0, p.width * p.height, 3, dtype=np.int64)
    ours, _ = port.scene(f).render_pixels(p, pix, threads=4, trig=0)
    ref, _ = refcpu.scene(f).render_pixels(p, pix)
    st = oracles.parity_stats(ours, ref)
    assert st["frac_exact"] >= 0.999, st


def test_reference_scene_files(ref_loader):
    """Every `.scene` file the reference ships (data/scenes), read by both readers from the reference's
    root directory: identical descriptions (its OBJ and image paths, written relative to a build
    directory, are missing on both sides from there)."""
    ref = oracles.REFERENCE
    files = sorted((ref / "data" / "scenes").glob("*.scene"))
    if not files:
        pytest.skip("the reference's scene files are not available")
    cwd = os.getcwd()
    try:
        os.chdir(ref)
        for path in files:
            rel = path.relative_to(ref)
            r = subprocess.run([str(ref_loader), str(rel)], cwd=ref, capture_output=True, text=True, timeout=120)
            assert r.returncode == 0, path.name
            mine = SceneFile(rel, flags=SCENE_FILE_REFERENCE_CAPACITY, decode_images=False)
            _same(json.loads(r.stdout.strip().splitlines()[-1]), _desc_json(mine), path.name)
    finally:
        os.chdir(cwd)
