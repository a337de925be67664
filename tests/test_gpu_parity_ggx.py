"""GPU parity against the oracle on the textured GGX-microfacet scene of the
single-view benchmark, at a size the oracle finishes in seconds: the BSDF
eval/sample/pdf of Microfacet.cpp:37-165 and BSDF.cpp:232-302, the
nearest-texel lookup of BSDF.cpp:72-98, smooth shading, and the
hand-written reverse mode of the factors, with vertex and texel gradients of
all five integrators."""
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes
from tests.helpers import oracle_camera_from, rel_l2, sample_table

pytestmark = pytest.mark.gpu

W = H = 24
D = 3


@pytest.fixture(scope="module")
def cfg2(built_lib):
    spec = scenes.config2_scene(W, H, tris=2000, tex_size=16)
    scene = api.Scene(spec)
    scene.configure()
    osc = O.OracleScene(spec, requires_grad=("positions", "texels"))
    cam = oracle_camera_from(scene.cameras[0])
    return spec, scene, osc, cam


def test_ggx_forward_parity(cfg2):
    spec, scene, osc, cam = cfg2
    spp = 4
    smp = sample_table(0, W, H, spp, D, 3)
    img_g = api.PathTracer().renderC(scene, api.RenderOptions(0, D, spp, 0, 0, 0, 0), samples=smp.to(scene.device))
    with torch.no_grad():
        osc.configure()
        img_o = O.path_tracer(osc, cam, spp, D, smp)
    a = img_g.reshape(-1, 3).cpu().double()
    b = img_o.double()
    assert float(b.sum()) > 0
    err = (a - b).abs()
    tol = 1e-4 * torch.maximum(a.abs(), b.abs()) + 1e-6
    bad = (err > tol).any(-1).float().mean()
    assert bad <= 0.02, f"{float(bad):.4f} of pixels differ"
    assert abs(float(a.sum() - b.sum())) <= 2e-3 * float(b.sum())


@pytest.mark.parametrize("integrator", [0, 1, 2, 3, 4])
def test_ggx_grad_parity(cfg2, integrator):
    spec, scene, osc, cam = cfg2
    spp = 4
    smp = sample_table(integrator, W, H, spp, D, 4)
    g = torch.Generator().manual_seed(17)
    dLdI = torch.rand(W * H, 3, generator=g) - 0.3
    cls = [api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
           api.PixelBoundaryIntegrator][integrator]
    opts = api.RenderOptions(0, D, spp, spp, spp, spp, spp)
    scene.clear_grads()
    cls().renderD(scene, opts, dLdI.reshape(H, W, 3).to(scene.device), samples=smp.to(scene.device))
    gg = scene.get_grads()
    go, _ = O.grads(osc, cam, integrator, spp, D, smp, dLdI)
    p_g, p_o = gg["positions"].cpu(), go["positions"].detach()
    assert float(p_o.abs().sum()) > 0
    assert rel_l2(p_g, p_o) < 2e-3, f"vertex grads rel L2 {rel_l2(p_g, p_o):.2e}"
    if integrator == 0:  # only the interior term differentiates the texture
        t_g, t_o = gg["texels"].cpu(), go["texels"].detach()
        assert float(t_o.abs().sum()) > 0
        assert rel_l2(t_g, t_o) < 2e-3, f"texel grads rel L2 {rel_l2(t_g, t_o):.2e}"
