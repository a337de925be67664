"""OBJ ingest (ObjMesh::LoadFromObj, EDXUtil/Graphics/ObjMesh.cpp:39-345) on CPU."""
import numpy as np

from tensorray_b200 import scenes

OBJ = """# a unit quad and a triangle
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0 0 1
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
s 1
f 1/1/1 2/2/1 3/3/1 4/4/1
f -5//1 -4//1 -1//1
usemtl red
f 2 3 5
"""


def test_obj_quads_split_and_indices(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text(OBJ)
    m = scenes.load_obj(str(p))
    assert m.positions.shape == (5, 3)
    np.testing.assert_array_equal(m.faces, [[0, 1, 2], [3, 0, 2], [0, 1, 4], [1, 2, 4]])
    # texture v flipped, quad texture corners follow the position corners
    np.testing.assert_allclose(m.uvs[2], [1.0, 0.0])
    np.testing.assert_array_equal(m.uv_faces[:2], [[0, 1, 2], [3, 0, 2]])


def test_obj_spec_builds_scene_arrays(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text(OBJ)
    spec = scenes.SceneSpec()
    spec.bsdfs = [scenes.BsdfSpec()]
    spec.meshes = [scenes.load_obj(str(p))]
    a = spec.arrays()
    assert a["positions"].shape[0] == 5 and a["indices"].size == 12
