"""Host-side scene generation: the synthetic workloads have the sizes they are measured at."""
import numpy as np

from cortexraytracercuda_b200 import configs
from cortexraytracercuda_b200.scene import MODE_CLEAN, MODE_COMPAT, RenderParams, SceneDesc


def test_cornell_counts():
    s = configs.cornell()
    assert len(s.quads) == 5 and len(s.dir_lights) == 1 and s.num_triangles == 24
    assert s.num_primitives == 30
    p = configs.cornell_params()
    assert (p.width, p.height, p.spp, p.max_depth) == (256, 256, 16, 8)


def test_spheres_counts_and_distribution():
    s = configs.spheres()
    assert len(s.spheres) == 488          # ground + 3 feature + 22x22 grid
    small = [sp for sp in s.spheres if sp[1] == 0.2]
    assert len(small) == 484
    kinds = np.array([s.materials[sp[2]][0] for sp in small])
    frac_lam = (kinds == 0).mean()
    assert 0.7 < frac_lam < 0.9
    p = configs.spheres_params()
    assert (p.width, p.height, p.spp, p.max_depth) == (1280, 720, 64, 50)


def test_icosphere_subdivision_sizes():
    v, f = configs.icosphere(3)
    assert f.shape == (1280, 3) and v.shape == (642, 3)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    # every edge is shared by exactly two faces (closed, manifold)
    e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert np.all(cnt == 2)


def test_displacement_amplitude():
    v, _ = configs.displaced_icosphere(3, 0.15)
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 0.85 - 1e-9 and r.max() <= 1.15 + 1e-9 and r.std() > 0.01


def test_traced_spp_compat_vs_clean():
    assert RenderParams(8, 8, 128, 4, mode=MODE_COMPAT).traced_spp == 121   # gpu.cu:1989
    assert RenderParams(8, 8, 128, 4, mode=MODE_CLEAN).traced_spp == 128


def test_checker_colors_swap():
    s = configs.Scene()
    t = s.checker_colors(10.0, (1, 0, 0), (0, 1, 0))
    kind, scale, even, odd = s.textures[t]
    assert s.textures[even][1] == (1.0, 0.0, 0.0)   # the "odd" colour lands in m_even
    assert s.textures[odd][1] == (0.0, 1.0, 0.0)


def test_desc_roundtrip_counts():
    s = configs.textured()
    d = SceneDesc(s).desc
    assert d.num_spheres == 3 and d.num_quads == 2 and d.num_images == 1 and d.num_dir_lights == 1
    assert d.images[0].width == 64 and d.images[0].height == 48


def test_desc_packed_arrays_match_elementwise_construction():
    """SceneDesc builds its sphere, material and texture arrays from numpy rows; each element's bytes
    equal the ctypes structure built field by field."""
    import ctypes as C

    from cortexraytracercuda_b200.scene import (TEX_CHECKER, TEX_IMAGE, TEX_SOLID, rtc_material, rtc_sphere,
                                                rtc_texture, F3)
    for make in (configs.spheres, configs.cornell, configs.textured, configs.lights_scene):
        s = make()
        d = SceneDesc(s).desc
        for k, (c, r, m) in enumerate(s.spheres):
            assert bytes(d.spheres[k]) == bytes(rtc_sphere(F3(*map(float, c)), r, m))
        for k, m in enumerate(s.materials):
            assert bytes(d.materials[k]) == bytes(rtc_material(*m))
        for k, t in enumerate(s.textures):
            if t[0] == "solid":
                ref = rtc_texture(TEX_SOLID, F3(*map(float, t[1])), 0.0, -1, -1, -1)
            elif t[0] == "checker":
                ref = rtc_texture(TEX_CHECKER, F3(0.0, 0.0, 0.0), t[1], t[2], t[3], -1)
            else:
                ref = rtc_texture(TEX_IMAGE, F3(0.0, 0.0, 0.0), 0.0, -1, -1, t[1])
            assert bytes(d.textures[k]) == bytes(ref)
        assert d.num_spheres == len(s.spheres) and d.num_materials == len(s.materials)
        assert d.num_textures == len(s.textures)
        assert C.sizeof(rtc_sphere) == 20
