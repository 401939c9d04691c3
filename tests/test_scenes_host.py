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
