"""Shape parameters and accessors on the host, on the CPU: the axis-angle
matrix of CalcRotateAxisAngle (Renderer/Utils.cpp:200-232), the pose and the
differentiable rotation of Primitive::Configure (Primitive.cpp:158-189) as
api.posed_positions applies them, the chain rule of api.pose_grads against
torch autograd of the same composition, and the face, edge and mesh-export
accessors of Primitive (Primitive.cpp:400-469)."""
from types import SimpleNamespace

import numpy as np
import pytest
import torch
from scipy.spatial.transform import Rotation

from tensorray_b200 import api


def _reference_columns(angle, axis):
    """The three columns CalcRotateAxisAngle writes (Utils.cpp:210-229)."""
    x, y, z = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    s, c = np.sin(angle), np.cos(angle)
    c0 = [x * x + (1 - x * x) * c, x * y * (1 - c) + z * s, x * z * (1 - c) - y * s]
    c1 = [x * y * (1 - c) - z * s, y * y + (1 - y * y) * c, y * z * (1 - c) + x * s]
    c2 = [x * z * (1 - c) + y * s, y * z * (1 - c) - x * s, z * z + (1 - z * z) * c]
    return np.stack([c0, c1, c2], 1)


@pytest.mark.parametrize("angle, axis", [(0.3, (0, 1, 0)), (-1.2, (1, 2, 3)), (2.9, (0.5, -0.2, 0.1))])
def test_axis_angle_matrix(angle, axis):
    R = api.rotation_axis_angle(angle, axis).double().numpy()
    np.testing.assert_allclose(R, _reference_columns(angle, axis), atol=1e-6)   # float32 evaluation
    rv = np.asarray(axis, np.float64) / np.linalg.norm(axis) * angle
    np.testing.assert_allclose(R, Rotation.from_rotvec(rv).as_matrix(), atol=1e-6)
    h = 1e-3
    fd = (_reference_columns(angle + h, axis) - _reference_columns(angle - h, axis)) / (2 * h)
    np.testing.assert_allclose(api.rotation_axis_angle(angle, axis, derivative=True).double().numpy(), fd,
                               atol=1e-5)


def _scene_with(raw, sizes):
    sc = SimpleNamespace(_dirty=False, _raw_positions=raw, device=raw.device)
    shapes, v = [], 0
    for i, n in enumerate(sizes):
        shapes.append(api.Shape(sc, i, v, n, 0))
        v += n
    sc.shapes = shapes
    return sc, shapes


def test_unrotated_shapes_upload_their_raw_positions():
    raw = torch.randn(10, 3)
    _, shapes = _scene_with(raw, [4, 6])
    assert api.posed_positions(raw, shapes) is None
    g = torch.randn(10, 3)
    gp, da, dv = api.pose_grads(raw, g, shapes)
    assert torch.equal(gp, g) and torch.equal(da, torch.zeros(2)) and torch.equal(dv, torch.zeros(2, 3))


def test_pose_and_rotation_and_their_chain_rule():
    torch.manual_seed(0)
    raw = torch.randn(30, 3, dtype=torch.float32)
    sc, shapes = _scene_with(raw, [10, 12, 8])
    M = torch.as_tensor(Rotation.from_rotvec([0.2, -0.7, 0.4]).as_matrix(), dtype=torch.float32)
    shapes[0].rotate_matrix = M
    shapes[0].obj_center = shapes[0].get_obj_center()
    assert sc._dirty
    shapes[1].diff_rotation((1.0, 0.5, -0.25))
    shapes[1].rotate_angle = 0.4
    shapes[2].rotate_matrix = np.eye(4)                   # 4x4 input, identity pose
    shapes[2].diff_rotation(torch.tensor([0.0, 0.0, 2.0]))
    posed = api.posed_positions(raw, shapes)

    # the same composition, written out and differentiated by autograd
    p = raw.clone().requires_grad_(True)
    th = torch.tensor([0.0, 0.4, 0.0], requires_grad=True)
    c0 = 0.5 * (raw[:10].min(0).values + raw[:10].max(0).values)
    parts = [(p[:10] - c0) @ M.T + c0]
    for sl, i, axis in ((slice(10, 22), 1, (1.0, 0.5, -0.25)), (slice(22, 30), 2, (0.0, 0.0, 1.0))):
        k = torch.tensor(axis) / torch.linalg.vector_norm(torch.tensor(axis))
        K = torch.zeros(3, 3)
        K[0, 1], K[0, 2], K[1, 0], K[1, 2], K[2, 0], K[2, 1] = -k[2], k[1], k[2], -k[0], -k[1], k[0]
        R = torch.cos(th[i]) * torch.eye(3) + torch.sin(th[i]) * K + (1 - torch.cos(th[i])) * torch.outer(k, k)
        parts.append(p[sl] @ R.T)
    world = torch.cat(parts)
    torch.testing.assert_close(posed, world.detach(), rtol=1e-6, atol=1e-6)

    w = torch.randn(30, 3)
    (world * w).sum().backward()
    gp, da, _ = api.pose_grads(raw, w, shapes)
    torch.testing.assert_close(gp, p.grad, rtol=1e-5, atol=1e-5)
    torch.testing.assert_close(da[1:], th.grad[1:], rtol=1e-5, atol=1e-5)
    assert da[0] == 0.0


def test_moved_vertex_and_its_gradient():
    """vertex_id / vertex_translation (Primitive.cpp:194-199): one vertex moved
    in world space after the rotations; its gradient is that vertex's."""
    torch.manual_seed(1)
    raw = torch.randn(12, 3)
    sc, shapes = _scene_with(raw, [5, 7])
    shapes[1].diff_rotation((0.0, 0.0, 1.0))
    shapes[1].rotate_angle = 0.3
    shapes[1].vertex_id = 4
    t = torch.tensor([0.1, -0.2, 0.05])
    shapes[1].vertex_translation = t
    posed = api.posed_positions(raw, shapes)
    R = api.rotation_axis_angle(0.3, (0.0, 0.0, 1.0))
    expected = raw.clone()
    expected[5:] = raw[5:] @ R.T
    expected[5 + 4] += t
    torch.testing.assert_close(posed, expected)
    g = torch.randn(12, 3)
    gp, da, dv = api.pose_grads(raw, g, shapes)
    torch.testing.assert_close(dv[1], g[9])
    assert torch.equal(dv[0], torch.zeros(3))
    torch.testing.assert_close(gp[5:], g[5:] @ R)      # the moved vertex's raw gradient still goes through R
    with pytest.raises(RuntimeError, match="out of range"):
        shapes[0].vertex_id = 5


def test_rotate_matrix_checks_its_shape():
    raw = torch.zeros(3, 3)
    _, shapes = _scene_with(raw, [3])
    with pytest.raises(RuntimeError, match="3x3 or 4x4"):
        shapes[0].rotate_matrix = np.eye(2)


def _mesh_scene(tmp_path):
    """A fake scene holding two meshes (a quad and a tetrahedron)."""
    from tensorray_b200 import scenes
    quad = scenes.MeshSpec(np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32),
                           np.array([[0, 1, 2], [0, 2, 3]], np.int32))
    tet = scenes.MeshSpec(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.5]], np.float32),
                          np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32))
    raw = torch.as_tensor(np.concatenate([quad.positions, tet.positions]))
    sc = SimpleNamespace(_dirty=False, _raw_positions=raw, device=raw.device,
                         spec=SimpleNamespace(meshes=[quad, tet]))
    shapes = [api.Shape(sc, 0, 0, 4, 2), api.Shape(sc, 1, 4, 4, 4)]
    return sc, shapes


def test_face_and_edge_accessors(tmp_path):
    _, (quad, tet) = _mesh_scene(tmp_path)
    assert tet.get_face_indices().tolist() == [0, 2, 1, 0, 1, 3, 0, 3, 2, 1, 2, 3]
    out = torch.zeros(6, dtype=torch.int32)
    quad.get_face_indices(out)
    assert out.tolist() == [0, 1, 2, 0, 2, 3]
    with pytest.raises(RuntimeError, match="needed"):
        quad.get_face_indices(np.zeros(5, np.int32))
    # a quad has 5 edges, a closed tetrahedron 6; first vertices, then second
    assert quad.get_edge_count() == 5 and tet.get_edge_count() == 6
    ed = np.zeros(12, np.int32)
    tet.get_edge_data(ed)
    assert sorted(zip(ed[:6].tolist(), ed[6:].tolist())) == [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def test_export_mesh_writes_what_load_obj_reads(tmp_path):
    from tensorray_b200 import scenes
    _, (quad, tet) = _mesh_scene(tmp_path)
    path = str(tmp_path / "tet.obj")
    tet.export_mesh(path)
    text = open(path).read().splitlines()
    assert text[3] == "v 0 0 1.5" and text[4] == "f 1 3 2"
    m = scenes.load_obj(path)
    np.testing.assert_array_equal(m.positions, tet._scene.spec.meshes[1].positions)
    np.testing.assert_array_equal(m.faces, tet._scene.spec.meshes[1].faces)


class _FakeLib:
    """Stands in for the library's scene calls: records the positions that
    configure() uploads and hands get_grads() a fixed position gradient."""

    def __init__(self, nv, grad):
        self.nv, self.grad, self.uploaded = nv, grad, None

    def trn_scene_get_grads(self, h, gt, gp, gx, clear, st):
        import ctypes
        ctypes.memmove(gp.value, self.grad.data_ptr(), self.grad.numel() * 4)
        return 0

    def trn_scene_set_translation(self, h, t, st):
        return 0

    def trn_scene_set_positions(self, h, p, st):
        import ctypes
        buf = (ctypes.c_float * (3 * self.nv)).from_address(p.value)
        self.uploaded = torch.tensor(np.frombuffer(buf, np.float32).copy()).reshape(-1, 3)
        return 0

    def trn_scene_configure(self, h, st):
        return 0


def test_scene_uploads_posed_positions_and_chains_its_gradients(monkeypatch):
    """Scene.configure uploads the posed positions and Scene.get_grads chains
    the library's position gradient through the poses, with the angle and
    moved-vertex gradients only when a shape asks for them."""
    import ctypes
    nv = 12
    torch.manual_seed(2)
    raw, g = torch.randn(nv, 3), torch.randn(nv, 3)
    sc = api.Scene.__new__(api.Scene)
    sc.device, sc._h, sc._dirty = torch.device("cpu"), ctypes.c_void_p(1), True
    sc.num_meshes, sc.num_vertices, sc.num_texels = 2, nv, 0
    sc._raw_positions, sc._translation = raw.clone(), torch.zeros(2, 3)
    sc._lib = _FakeLib(nv, g)
    monkeypatch.setattr(api, "_stream", lambda: 0)

    sc.shapes = [api.Shape(sc, 0, 0, 5, 0), api.Shape(sc, 1, 5, 7, 0)]
    sc.configure()
    assert torch.equal(sc._lib.uploaded, raw)
    assert sorted(sc.get_grads()) == ["positions", "texels", "translation"]

    sc.shapes[1].diff_rotation((0, 1, 0))
    sc.shapes[1].rotate_angle = 0.2
    sc.shapes[0].vertex_id = 2
    sc.shapes[0].vertex_translation = (0.5, 0.0, 0.0)
    sc.configure()
    assert torch.equal(sc._lib.uploaded, api.posed_positions(raw, sc.shapes))
    out = sc.get_grads()
    gp, da, dv = api.pose_grads(raw, g, sc.shapes)
    assert torch.equal(out["positions"], gp) and torch.equal(out["rotation_angle"], da)
    assert torch.equal(out["vertex_translation"], dv)


def test_scene_accessors_of_the_binding():
    """get_width(i) / get_height(i) per sensor (Scene.h:127-128), num_bsdf and
    emitters (TensorRay.cpp:153-163), on a scene object built without a GPU."""
    sc = api.Scene.__new__(api.Scene)
    sc.cameras = [SimpleNamespace(width=64, height=32), SimpleNamespace(width=128, height=96)]
    sc.bsdfs = [object(), object(), object()]
    sc.spec = SimpleNamespace(meshes=[SimpleNamespace(light=-1), SimpleNamespace(light=0), SimpleNamespace(light=-1)])
    sc.shapes = ["sphere", "lamp", "ground"]
    assert (sc.get_width(), sc.get_height(), sc.get_width(1), sc.get_height(1)) == (64, 32, 128, 96)
    assert sc.num_bsdf == 3 and sc.emitters == ["lamp"]
