"""Shape rotations through the renderer: a shape posed by rotate_matrix about
obj_center (the multi-pose optimisation of pyTensorRay/renderer_multi_pose.py:
53-98) renders as the same shape given its posed positions, and its vertex
gradient is that scene's chained through the pose; the angle gradient of
diff_rotation (Primitive.cpp:379-383) at angle 0 is the vertex gradient
contracted with k x p."""
import pytest
import torch
from scipy.spatial.transform import Rotation

from tensorray_b200 import api, scenes
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

OPTS = api.RenderOptions(3, 3, 8, 8, 8, 0, 0)
TERMS = (api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator)


def _grads(scene, w):
    scene.clear_grads()
    for cls in TERMS:
        cls().renderD(scene, OPTS, w)
    return scene.get_grads()


def test_pose_renders_as_its_posed_positions_and_chains_the_gradient(built_lib):
    spec = scenes.config1_scene(64, 64)
    posed_scene, plain = api.Scene(spec), api.Scene(spec)
    shape = posed_scene.shapes[0]
    M = torch.as_tensor(Rotation.from_rotvec([0.1, 0.3, -0.2]).as_matrix(), dtype=torch.float32)
    shape.rotate_matrix = M
    shape.obj_center = shape.get_obj_center() + torch.tensor([0.05, 0.0, 0.0])
    posed_scene.configure()
    plain.set_vertex_positions(api.posed_positions(posed_scene._raw_positions, posed_scene.shapes))
    plain.configure()
    img = api.PathTracer().renderC(posed_scene, OPTS)
    torch.testing.assert_close(img, api.PathTracer().renderC(plain, OPTS), rtol=1e-5, atol=1e-6)

    w = torch.rand(img.shape, generator=torch.Generator().manual_seed(1)).to(img.device)
    g_posed = _grads(posed_scene, w)["positions"]
    g_plain = _grads(plain, w)["positions"]
    expected = g_plain.clone()
    sl = shape.vertex_slice()
    expected[sl] = g_plain[sl] @ M.to(g_plain.device)
    assert float(g_plain[sl].abs().sum()) > 0
    assert rel_l2(g_posed, expected) <= 1e-4


def test_rotation_angle_gradient_at_zero(built_lib):
    spec = scenes.config1_scene(64, 64)
    rotating, plain = api.Scene(spec), api.Scene(spec)
    axis = torch.tensor([0.2, 1.0, -0.3])
    rotating.shapes[0].diff_rotation(axis)
    rotating.configure()
    plain.configure()
    w = torch.rand(64 * 64, 3, generator=torch.Generator().manual_seed(2)).to(plain.device).reshape(64, 64, 3)
    g = _grads(rotating, w)
    assert "rotation_angle" in g and g["rotation_angle"].shape == (len(spec.meshes),)
    gv = _grads(plain, w)["positions"]
    sl = plain.shapes[0].vertex_slice()
    k = (axis / torch.linalg.vector_norm(axis)).to(gv.device)
    terms = (gv[sl] * torch.cross(k.expand_as(plain._raw_positions[sl]), plain._raw_positions[sl], dim=1)).sum(1)
    assert abs(float(g["rotation_angle"][0]) - float(terms.sum())) <= 1e-4 * float(terms.abs().sum())
    assert float(g["rotation_angle"][1:].abs().sum()) == 0.0
