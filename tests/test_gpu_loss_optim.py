"""The optimiser side on the GPU: image losses against the reference's own
loss module's golden vectors (tests/golden), LargeSteps on the device against
the same step on the CPU, and a multi-view inverse-rendering run with the
pyramid L2 loss and LargeSteps that lowers its loss."""
import os

import pytest
import torch

from tensorray_b200 import api, inverse, loss as trl, optim, scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "loss_pyramid.pt")
RES = 48


@pytest.mark.parametrize("kind", ["l1", "l2", "pyramid_l1", "pyramid_l2"])
def test_device_losses_match_reference_goldens(kind):
    for case in torch.load(GOLDEN):
        img, tgt = case["img"].cuda(), case["target"].cuda()
        target = trl.build_pyramid(tgt) if kind.startswith("pyramid") else tgt
        loss, grad = trl.loss_and_grad(kind, img, target, case["weight"])
        ref_loss, ref_grad = case[kind]
        assert abs(float(loss) - ref_loss) <= 1e-5 * abs(ref_loss)
        torch.testing.assert_close(grad.cpu(), ref_grad, rtol=1e-5, atol=1e-6)


def test_largesteps_on_device_matches_cpu():
    P, F = scenes.icosphere(3, 1.0)
    V = torch.as_tensor(P, dtype=torch.float32)
    F = torch.as_tensor(F, dtype=torch.int64)
    g = torch.Generator().manual_seed(4)
    grads = [torch.randn(V.shape, generator=g) for _ in range(4)]
    out = []
    for dev in ("cpu", "cuda"):
        x = V.clone().to(dev).requires_grad_(True)
        opt = optim.LargeSteps(x, F.to(dev), lr=0.05, lmbda=3.0, tol=1e-8)
        for gr in grads:
            x.grad = gr.to(dev)
            opt.step()
        out.append(x.detach().cpu())
    torch.testing.assert_close(out[1], out[0], rtol=1e-4, atol=1e-5)


def test_inverse_rendering_with_pyramid_loss_and_largesteps(built_lib):
    spec = scenes.config1_scene(RES, RES)
    scene = api.Scene(spec)
    scene.configure()
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(4, 4.0, [RES], seed=1)]
    target = inverse.render_targets(scene, cams, [64] * len(cams), api.RenderOptions(99, 3, 64, 0, 0, 0, 0))
    raw0 = torch.as_tensor(spec.arrays()["positions"]).clone()
    nv = len(spec.meshes[0].positions)
    start = raw0.clone()
    start[:nv] *= 1.1
    scene.set_vertex_positions(start)
    scene.configure()
    inv = inverse.InverseRenderer(scene, cams, [4] * len(cams), target, api.RenderOptions(0, 3, 4, 4, 4, 0, 0),
                                  lr=5e-2, loss="pyramid_l2", optimizer="largesteps", lmbda=2.0, shapes=(0,))
    losses = [float(inv.step().sum()) for _ in range(30)]
    assert all(torch.isfinite(torch.tensor(losses)))
    r = inv.x.detach()[:nv].norm(dim=1).mean().item()
    assert r < 1.07, f"mean radius {r:.4f}, losses {losses[0]:.4g} .. {losses[-1]:.4g}"
    assert sum(losses[-5:]) < sum(losses[:5])
    # only the sphere's vertices are optimised
    torch.testing.assert_close(inv.x.detach()[nv:].cpu(), start[nv:])
