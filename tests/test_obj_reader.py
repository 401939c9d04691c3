"""The OBJ reader behind rtc_load_obj (CPU only: no device is touched)."""
import numpy as np
import pytest

from cortexraytracercuda_b200 import _lib, configs
from cortexraytracercuda_b200._lib import RtcError
from cortexraytracercuda_b200.scene import load_obj

CUBE = """# unit cube, quads, two objects, relative and absolute indices
mtllib none.mtl
o first
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0 0 1
v 1 0 1
v 1 1 1
v 0 1 1
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 -1
vn 0 0 1
g front
usemtl red
f 1/1/1 4/4/1 3/3/1 2/2/1
f -4/1/2 -3/2/2 -2/3/2 -1/4/2
o second
s 1
f 1//1 2//1 6//1
f 1 6 5
"""


def test_corner_forms_negative_indices_and_fans(tmp_path):
    p = tmp_path / "cube.obj"
    p.write_text(CUBE)
    v, f, n, t = load_obj(p)
    assert f.shape == (6, 3)                           # 2 quads -> 4 triangles, + 2 triangles
    assert n is not None and t is not None
    tri0 = v[f[0]]
    np.testing.assert_array_equal(tri0, [[0, 0, 0], [0, 1, 0], [1, 1, 0]])   # fan (0, 1, 2) of the first quad
    # the relative quad is the z = 1 face
    assert np.all(v[f[2]][:, 2] == 1.0) and np.all(v[f[3]][:, 2] == 1.0)
    np.testing.assert_array_equal(n[f[2][0]], [0, 0, 1])
    # corners with the same (v, vt, vn) are shared; different vt/vn make new vertices
    assert len(v) == 8 + 3 + 3                         # 8 textured corners, 3 with v//vn, 3 bare
    # the bare-index triangle has zero normals and uvs (absent in the file)
    assert np.all(n[f[5][2]] == 0) and np.all(t[f[5][2]] == 0)


def test_round_trip_of_a_generated_mesh(tmp_path):
    v0, f0 = configs.icosphere(2)
    p = tmp_path / "ico.obj"
    with open(p, "w") as fh:
        for x in v0:
            fh.write(f"v {x[0]:.9g} {x[1]:.9g} {x[2]:.9g}\n")
        for a, b, c in f0:
            fh.write(f"f {a + 1} {b + 1} {c + 1}\n")
    v, f, n, t = load_obj(p)
    assert n is None and t is None
    np.testing.assert_allclose(v[f], v0.astype(np.float32)[f0], rtol=0, atol=1e-7)


@pytest.mark.parametrize("text,status", [("v 0 0 0\nf 1 2 3\n", 2), ("v 0 0\n", 2), ("v 0 0 0\nf 1/5 1 1\n", 2),
                                         ("# nothing\n", 2)])
def test_errors(tmp_path, text, status):
    p = tmp_path / "bad.obj"
    p.write_text(text)
    with pytest.raises(RtcError) as e:
        load_obj(p)
    assert e.value.status == status


def test_missing_file():
    with pytest.raises(RtcError) as e:
        load_obj("/nonexistent/mesh.obj")
    assert e.value.status == 7
