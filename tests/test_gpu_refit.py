"""LBVH refit (Scene::Update / UpdateAccelerationStructure, Scene.cpp:368-469,
535-546) against a full rebuild after the vertices move: ray queries are
bit-exact (closest hit = smallest (t, triangle id), which no BVH topology can
change); images and gradients are sums of float atomics per pixel / per
vertex, so they agree up to summation order."""
import pytest
import torch

from tensorray_b200 import api, scenes
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

W = H = 32
D = 3


def _perturbed(spec, seed):
    g = torch.Generator().manual_seed(seed)
    raw = torch.as_tensor(spec.arrays()["positions"]).clone()
    return raw + 0.03 * torch.randn(raw.shape, generator=g)


def test_refit_matches_rebuild(built_lib):
    spec = scenes.config1_scene(W, H)
    a, b = api.Scene(spec), api.Scene(spec)
    a.configure()
    b.configure()
    for step in range(3):  # several refits in a row on the same topology
        raw = _perturbed(spec, step)
        a.set_vertex_positions(raw)
        b.set_vertex_positions(raw)
        a.configure(refit=True)
        b.configure()
        ga, gb = a.geometry(), b.geometry()
        assert torch.equal(ga["positions"], gb["positions"])
        assert torch.equal(ga["vertex_normals"], gb["vertex_normals"])
        g = torch.Generator().manual_seed(100 + step)
        n = 8192
        org = (torch.rand(n, 3, generator=g) * 4 - 2).cuda()
        dirs = torch.nn.functional.normalize(torch.randn(n, 3, generator=g), dim=1).cuda()
        tmin, tmax = torch.full((n,), 1e-2, device="cuda"), torch.full((n,), 1e32, device="cuda")
        ra, rb = a.intersect(org, dirs, tmin, tmax), b.intersect(org, dirs, tmin, tmax)
        for x, y in zip(ra, rb):
            assert torch.equal(x, y)
        assert torch.equal(a.occluded(org, dirs, tmin, tmax), b.occluded(org, dirs, tmin, tmax))
        opts = api.RenderOptions(step, D, 4, 4, 4, 4, 4)
        ia = api.PathTracer().renderC(a, opts)
        ib = api.PathTracer().renderC(b, opts)
        torch.testing.assert_close(ia, ib, rtol=1e-5, atol=1e-6)
        dLdI = torch.rand(H, W, 3, generator=g).cuda() - 0.3
        for cls in (api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator):
            a.clear_grads()
            b.clear_grads()
            cls().renderD(a, opts, dLdI)
            cls().renderD(b, opts, dLdI)
            pa, pb = a.get_grads()["positions"].cpu(), b.get_grads()["positions"].cpu()
            assert rel_l2(pa, pb) < 1e-5, f"{cls.__name__} grads rel L2 {rel_l2(pa, pb):.2e}"
