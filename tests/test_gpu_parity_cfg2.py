"""GPU parity against the oracle at the single-view benchmark's scene size:
the 100K-triangle displaced sphere with GGX (roughness 0.3) and its 512x512
albedo texture, depth 5 (the benchmark's depth), all five integrators, with
vertex and texel gradients. The camera renders the scene at 20x20 pixels and
2 spp so that the oracle's brute-force ray queries over 100K triangles
finish in seconds. Tolerance: 1e-4 relative per pixel and on the gradients."""
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes
from tests.helpers import assert_grad_parity, assert_image_parity, oracle_camera_from, sample_table

pytestmark = pytest.mark.gpu

W = H = 20
D = 5
SPP = 2


@pytest.fixture(scope="module")
def cfg2_full(built_lib):
    spec = scenes.config2_scene(W, H, tris=100_000)
    assert spec.num_triangles > 99_000 and spec.textures[0].shape[:2] == (512, 512)
    scene = api.Scene(spec)
    scene.configure()
    osc = O.OracleScene(spec, requires_grad=("positions", "texels"))
    cam = oracle_camera_from(scene.cameras[0])
    return spec, scene, osc, cam


def test_cfg2_forward_parity(cfg2_full):
    spec, scene, osc, cam = cfg2_full
    smp = sample_table(0, W, H, SPP, D, 5)
    img_g = api.PathTracer().renderC(scene, api.RenderOptions(0, D, SPP, 0, 0, 0, 0), samples=smp.to(scene.device))
    with torch.no_grad():
        osc.configure()
        img_o = O.path_tracer(osc, cam, SPP, D, smp)
    assert_image_parity(img_g, img_o, f"cfg2 100K tris {W}x{H} D{D} forward")


@pytest.mark.parametrize("integrator", [0, 1, 2, 3, 4])
def test_cfg2_grad_parity(cfg2_full, integrator):
    spec, scene, osc, cam = cfg2_full
    smp = sample_table(integrator, W, H, SPP, D, 6)
    g = torch.Generator().manual_seed(19)
    dLdI = torch.rand(W * H, 3, generator=g) - 0.3
    cls = [api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
           api.PixelBoundaryIntegrator][integrator]
    opts = api.RenderOptions(0, D, SPP, SPP, SPP, SPP, SPP)
    scene.clear_grads()
    cls().renderD(scene, opts, dLdI.reshape(H, W, 3).to(scene.device), samples=smp.to(scene.device))
    gg = scene.get_grads()
    go, _ = O.grads(osc, cam, integrator, SPP, D, smp, dLdI)
    label = f"cfg2 100K tris {W}x{H} D{D} term {integrator}"
    assert_grad_parity(gg["positions"], go["positions"], label + " vertices")
    if integrator == 0:
        assert_grad_parity(gg["texels"], go["texels"], label + " texels")
