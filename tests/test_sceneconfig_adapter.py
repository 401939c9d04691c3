"""The C++ sceneConfig adapter (include/rtc_sceneconfig.hpp) compiled against the reference's own
scene_config.h (core/src/scenes/scene_config.h) by oracle/Makefile's `adapter` target.  The check
program builds one sceneConfig and prints the rtc_scene_desc the adapter makes from it; the resolution
rules are those of the reference's load_scene (core/src/gpu.cu:481-751)."""
import json
import os
import subprocess
from pathlib import Path

import pytest

import oracles

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "oracle" / "_ref" / "sceneconfig_check"


@pytest.fixture(scope="module")
def desc():
    ref = str(oracles.REFERENCE)
    if not (Path(ref) / "core" / "src" / "scenes" / "scene_config.h").exists() and not EXE.exists():
        pytest.skip("reference tree not available to compile the adapter check")
    if Path(ref).exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "adapter", f"REF={ref}"], check=True,
                       capture_output=True)
    out = subprocess.run([str(EXE)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def _tex(d, i):
    return d["textures"][i]


def test_objects_in_load_scene_order_and_unresolved_skipped(desc):
    d = desc
    assert len(d["dir_lights"]) == 1
    assert len(d["spheres"]) == 3          # the sphere with a missing material is skipped (gpu.cu:531)
    assert len(d["quads"]) == 5            # so is the quad with an unknown material
    assert [s["radius"] for s in d["spheres"]] == [90.0, 80.0, 60.0]
    assert any("missing" in s for s in d["skipped"]) and any("nosuchmaterial" in s for s in d["skipped"])
    assert "boxes" not in d["skipped"]


def test_boxes_and_transforms(desc):
    """boxPrimitives become rtc_box (after the quads); each rt::transform becomes a 1-based reference
    with the parts it has (scene_factory::applyTransform)."""
    b, = desc["boxes"]
    assert b["center"] == [212.5, 82.5, 147.5] and b["size"] == [165.0, 165.0, 165.0]
    xs = desc["transforms"]
    assert desc["sphere_transforms"] == [1, 0, 0] and b["transform"] == 2
    assert xs[0]["flags"] == 4 and xs[0]["scale"] == [2.0, 1.0, 1.0]
    assert xs[1]["flags"] == 3 and xs[1]["translate"] == [10.0, 0.0, -5.0] and xs[1]["rotate"] == [0.0, 18.0, 0.0]


def test_omni_and_spot_lights(desc):
    o, = desc["omni_lights"]
    assert o["position"] == [100.0, 500.0, 200.0] and o["radius"] == 20.0 and o["intensity"] == 2.0
    assert o["color"] == [4.0, 3.0, 2.0] and o["invisible"] == 0
    s, = desc["spot_lights"]
    assert s["position"] == [400.0, 500.0, 300.0] and s["direction"] == pytest.approx([0.0, -1.0, 0.2], abs=1e-7)
    assert s["cutoff"] == 30.0 and s["falloff"] == 3.0 and s["radius"] == 10.0 and s["intensity"] == 5.0
    assert s["color"] == [6.0, 6.0, 5.0] and s["invisible"] == 1
    assert not any("light" in k for k in desc["skipped"])


def test_directional_light_and_camera(desc):
    L = desc["dir_lights"][0]
    assert L["position"] == [278.0, 554.0, 332.0] and L["u"] == [-130.0, 0.0, 0.0] and L["v"] == [0.0, 0.0, -105.0]
    assert L["color"] == [15.0, 15.0, 15.0] and L["intensity"] == 1.5 and L["invisible"] == 1
    c = desc["camera"]
    assert c["look_from"] == [278.0, 278.0, -800.0] and c["look_at"] == [278.0, 278.0, 0.0]
    assert c["up"] == [0.0, 1.0, 0.0] and c["vfov"] == 40.0 and c["aspect"] == 1.0 and c["focus"] == 10.0
    assert desc["background"]["kind"] == 0
    assert desc["background"]["color"] == pytest.approx([0.1, 0.2, 0.3], abs=1e-7)


def test_materials_resolved_like_fetchMaterial(desc):
    d = desc
    mats = [d["materials"][s["material"]] for s in d["spheres"]]
    glass, mirror, ball = mats
    assert glass["kind"] == 2 and glass["ior"] == 1.5 and glass["texture"] == -1
    assert mirror["kind"] == 1 and mirror["fuzz"] == 1.0          # metal fuzz clamped to 1 (metal.cuh:52)
    assert _tex(d, mirror["texture"])["color"] == pytest.approx([0.8, 0.85, 0.9], abs=1e-7)
    # checker from named textures: checker_texture(scale, odd, even) stores odd in m_even
    chk = _tex(d, ball["texture"])
    assert ball["kind"] == 0 and chk["kind"] == 1 and chk["scale"] == 2.0
    assert _tex(d, chk["even"])["color"] == pytest.approx([0.9, 0.9, 0.9], abs=1e-7)   # "tex_white" (odd name)
    assert _tex(d, chk["odd"])["color"] == pytest.approx([0.1, 0.2, 0.8], abs=1e-7)    # "tex_blue" (even name)


def test_quads_and_checker_from_colours(desc):
    d = desc
    q = d["quads"]
    assert q[0]["q"] == [555.0, 0.0, 0.0] and q[0]["u"] == [0.0, 555.0, 0.0] and q[0]["v"] == [0.0, 0.0, 555.0]
    cols = [_tex(d, d["materials"][x["material"]]["texture"]) for x in q]
    assert cols[0]["color"] == pytest.approx([0.12, 0.45, 0.15], abs=1e-7)   # green
    assert cols[1]["color"] == pytest.approx([0.65, 0.05, 0.05], abs=1e-7)   # red
    floor = cols[2]
    assert floor["kind"] == 1 and floor["scale"] == 0.5
    # colours: odd colour -> m_even, even colour -> m_odd (scene_factory.cuh:619-629)
    assert _tex(d, floor["even"])["color"] == [1.0, 0.0, 0.0]
    assert _tex(d, floor["odd"])["color"] == [0.0, 1.0, 0.0]


def test_obj_meshes_through_the_loader(desc):
    d = desc
    assert len(d["meshes"]) == 1                        # the unreadable file is reported, not added
    m = d["meshes"][0]
    assert m["num_vertices"] == 4 and m["num_triangles"] == 4 and m["smooth"] == 1 and m["has_normals"] == 1
    assert m["v0"] == [10.0, 20.0, 30.0] and m["v3"] == [10.0, 20.0, 31.0]   # offset by the mesh position
    assert m["i1"] == 2
    assert d["materials"][m["material"]]["kind"] == 1   # "mirror" is a metal
    assert any("missing.obj" in s for s in d["skipped"])
