"""Multi-view inverse rendering (refit + batched views + Adam on the device):
recover an icosphere that was scaled by 10 % from four target views."""
import pytest
import torch

from tensorray_b200 import api, inverse, scenes

pytestmark = pytest.mark.gpu

RES = 48


def test_inverse_rendering_reduces_loss(built_lib):
    spec = scenes.config1_scene(RES, RES)
    scene = api.Scene(spec)
    scene.configure()
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(4, 4.0, [RES], seed=1)]
    spps = [4] * len(cams)
    # targets from the true shape at high spp
    target = inverse.render_targets(scene, cams, [64] * len(cams), api.RenderOptions(99, 3, 64, 0, 0, 0, 0))
    # start from the sphere scaled by 1.1 (the sphere is mesh 0, the first vertices)
    raw0 = torch.as_tensor(spec.arrays()["positions"]).clone()
    nv_sphere = len(spec.meshes[0].positions)
    start = raw0.clone()
    start[:nv_sphere] *= 1.1
    scene.set_vertex_positions(start)
    scene.configure()

    def eval_loss():
        vs = api.ViewSet(scene, cams, [64] * len(cams))
        img = vs.render(api.TRN_PATH_TRACER, api.RenderOptions(123, 3, 64, 0, 0, 0, 0))
        return float(vs.loss(img, target).sum())

    before = eval_loss()
    opts = api.RenderOptions(0, 3, 4, 4, 4, 0, 0)
    inv = inverse.InverseRenderer(scene, cams, spps, target, opts, lr=4e-3)
    losses = [float(inv.step().sum()) for _ in range(30)]
    scene.set_vertex_positions(inv.x.detach())
    scene.configure()
    after = eval_loss()
    assert all(torch.isfinite(torch.tensor(losses)))
    assert after < 0.7 * before, f"loss {before:.4g} -> {after:.4g} (trajectory {losses[0]:.4g} .. {losses[-1]:.4g})"
    # the recovered sphere radius moves back towards 1
    r = inv.x.detach()[:nv_sphere].norm(dim=1).mean().item()
    assert r < 1.08, f"mean radius {r:.4f}"
