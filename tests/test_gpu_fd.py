"""Finite-difference validation of the full gradient (interior + boundary
terms), the recipe of the reference's validate_gpu.py (forward/central
differences at high spp, example/validation/validate_gpu.py:103-132), and
the autograd.Function bridge."""
import numpy as np
import pytest
import torch

from tensorray_b200 import api, scenes
from tensorray_b200 import autograd as tra

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_translation_gradient_matches_central_fd(built_lib, axis):
    """d/dt_axis of L = sum(w * I) for a fixed random weight image w: the sum
    of all five integrators' gradients against central differences of the
    forward render with the same seeds, averaged over independent seeds."""
    W = H = 64
    D = 3
    spec = scenes.config1_scene(W, H)
    scene = api.Scene(spec)
    scene.configure()
    g = torch.Generator().manual_seed(0)
    w = (torch.rand(H, W, 3, generator=g) - 0.5).cuda()
    spp, eps = 1024, 1e-2
    ads, fds = [], []
    for seed in range(4):
        opts = api.RenderOptions(seed, D, spp, spp, spp, spp, spp)
        scene.clear_grads()
        for it in (api.PathTracer(), api.PrimaryEdgeIntegrator(), api.DirectEdgeIntegrator(),
                   api.IndirectEdgeIntegrator(), api.PixelBoundaryIntegrator()):
            it.renderD(scene, opts, w)
        ads.append(float(scene.get_grads()["translation"][0, axis]))
        vals = []
        for sgn in (1, -1):
            t = torch.zeros(3)
            t[axis] = sgn * eps
            scene.shapes[0].translation = t
            scene.configure()
            img = api.PathTracer().renderC(scene, api.RenderOptions(seed, D, spp, 0, 0, 0, 0))
            vals.append(float((img * w).double().sum()))
        scene.shapes[0].translation = torch.zeros(3)
        scene.configure()
        fds.append((vals[0] - vals[1]) / (2 * eps))
    ad, fd = np.mean(ads), np.mean(fds)
    se = np.sqrt(np.var(ads) / len(ads) + np.var(fds) / len(fds))
    assert abs(ad - fd) <= max(0.1 * abs(fd), 3.0 * se) + 1e-3, (ads, fds)


def test_autograd_function_matches_scene_grads(built_lib):
    W = H = 32
    spec = scenes.config2_scene(W, H, tris=5000, tex_size=64)
    scene = api.Scene(spec)
    scene.configure()
    opts = api.RenderOptions(5, 3, 4, 4, 4, 4, 4)
    ctx = tra.RenderContext(scene, opts)
    V = scene._raw_positions.clone().requires_grad_(True)
    T = torch.as_tensor(np.ascontiguousarray(spec.textures[0]), device=scene.device).reshape(-1, 3).clone()
    T.requires_grad_(True)
    target = torch.zeros(H, W, 3, device=scene.device)
    img = tra.render(V, T, ctx)
    loss = 0.5 * ((img - target) ** 2).sum()
    loss.backward()
    # same thing through the scene API
    scene.set_vertex_positions(V.detach())
    scene.configure()
    img2 = api.PathTracer().renderC(scene, opts)
    torch.testing.assert_close(img, img2, rtol=1e-5, atol=1e-6)
    scene.clear_grads()
    for it in ctx.edge_integrators + [api.PathTracer()]:
        it.renderD(scene, opts, img2 - target)
    g = scene.get_grads()
    torch.testing.assert_close(V.grad, g["positions"], rtol=1e-3, atol=1e-4)
    torch.testing.assert_close(T.grad, g["texels"], rtol=1e-3, atol=1e-4)
    assert float(T.grad.abs().sum()) > 0 and float(V.grad.abs().sum()) > 0
