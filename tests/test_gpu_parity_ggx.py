"""GPU parity against the oracle on the textured GGX-microfacet scene of the
single-view benchmark, at a size the oracle finishes in seconds: the BSDF
eval/sample/pdf of Microfacet.cpp:37-165 and BSDF.cpp:232-302, the
nearest-texel lookup of BSDF.cpp:72-98, smooth shading, and the
hand-written reverse mode of the factors, with vertex and texel gradients of
all five integrators. Tolerance: 1e-4 relative per pixel and on the
gradients (relative L2 and largest element)."""
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes
from tests.helpers import assert_grad_parity, assert_image_parity, oracle_camera_from, sample_table

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


@pytest.mark.parametrize("depth", [3, 5])
def test_ggx_forward_parity(cfg2, depth):
    spec, scene, osc, cam = cfg2
    spp = 4
    smp = sample_table(0, W, H, spp, depth, 3)
    img_g = api.PathTracer().renderC(scene, api.RenderOptions(0, depth, spp, 0, 0, 0, 0),
                                     samples=smp.to(scene.device))
    with torch.no_grad():
        osc.configure()
        img_o = O.path_tracer(osc, cam, spp, depth, smp)
    assert_image_parity(img_g, img_o, f"ggx 2K tris {W}x{H} D{depth} forward")


@pytest.mark.parametrize("depth", [3, 5])
@pytest.mark.parametrize("integrator", [0, 1, 2, 3, 4])
def test_ggx_grad_parity(cfg2, integrator, depth):
    spec, scene, osc, cam = cfg2
    spp = 4
    smp = sample_table(integrator, W, H, spp, depth, 4)
    g = torch.Generator().manual_seed(17)
    dLdI = torch.rand(W * H, 3, generator=g) - 0.3
    cls = [api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
           api.PixelBoundaryIntegrator][integrator]
    opts = api.RenderOptions(0, depth, spp, spp, spp, spp, spp)
    scene.clear_grads()
    cls().renderD(scene, opts, dLdI.reshape(H, W, 3).to(scene.device), samples=smp.to(scene.device))
    gg = scene.get_grads()
    go, _ = O.grads(osc, cam, integrator, spp, depth, smp, dLdI)
    label = f"ggx 2K tris {W}x{H} D{depth} term {integrator}"
    assert_grad_parity(gg["positions"], go["positions"], label + " vertices")
    if integrator == 0:  # only the interior term differentiates the texture
        assert_grad_parity(gg["texels"], go["texels"], label + " texels")
