"""GPU parity of the trn CUDA path against the CPU oracle (same inputs, same
uniform sample tables), called through the C-ABI via the Python mirror.

Tolerance: every pixel within 1e-4 relative, gradients within 1e-4 relative
L2 and 1e-4 of the largest element (the float atomics of the scatter add in
another order than the oracle's index_add). Paths agree exactly: the
sampling arithmetic is evaluated with the same IEEE operations on both
sides (no multiply-add contraction, deterministic sin/cos/acos)."""
import numpy as np
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes
from tests.helpers import assert_grad_parity, assert_image_parity, oracle_camera_from, sample_table

pytestmark = pytest.mark.gpu

W = H = 32
D = 3
DEPTHS = [3, 5]  # 5 is the depth of the single-view benchmark


@pytest.fixture(scope="module")
def cfg1(built_lib):
    spec = scenes.config1_scene(W, H)
    scene = api.Scene(spec)
    scene.configure()
    osc = O.OracleScene(spec, requires_grad=("translation", "positions"))
    cam = oracle_camera_from(scene.cameras[0])
    return spec, scene, osc, cam


def test_camera_matches_oracle_restatement(cfg1):
    spec, scene, osc, cam = cfg1
    c = spec.cameras[0]
    ref = O.camera_matrices(c.pos, c.target, c.up, c.width, c.height, c.fov)
    for k in ("raster_to_camera", "view_inv", "world_to_sample", "sample_to_camera", "raster_to_world"):
        np.testing.assert_allclose(cam[k], ref[k], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(cam["inv_area"], ref["inv_area"], rtol=1e-5)


def test_geometry_chain(cfg1):
    spec, scene, osc, cam = cfg1
    g = scene.geometry()
    osc.configure()
    np.testing.assert_array_equal(g["positions"].cpu().numpy(), osc.pos.detach().numpy())
    np.testing.assert_allclose(g["face_normals"].cpu().numpy(), osc.fn.detach().numpy(), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(g["areas"].cpu().numpy(), osc.area.detach().numpy(), rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(g["vertex_normals"].cpu().numpy(), osc.vn.detach().numpy(), rtol=1e-5, atol=1e-6)


def _rays(osc, cam, n, seed):
    g = torch.Generator().manual_seed(seed)
    # camera rays with random sub-pixel offsets
    pix = torch.randint(0, W * H, (n,), generator=g)
    d1 = O.camera_ray_dir(cam, pix % W, pix // W, torch.rand(n, generator=g), torch.rand(n, generator=g))
    o1 = torch.from_numpy(cam["pos"]).expand(n, 3).contiguous()
    # random rays from surface points in random directions
    tri = torch.randint(0, osc.idx.shape[0], (n,), generator=g)
    u, v = torch.rand(n, generator=g), torch.rand(n, generator=g)
    flip = u + v > 1
    u, v = torch.where(flip, 1 - u, u), torch.where(flip, 1 - v, v)
    o2 = osc.post_intersect(tri, u, v)["p"].detach()
    d2 = O.normalize(torch.randn(n, 3, generator=g))
    return torch.cat([o1, o2]), torch.cat([d1, d2])


def test_intersect_bit_exact(cfg1):
    spec, scene, osc, cam = cfg1
    osc.configure()
    org, dirs = _rays(osc, cam, 2048, 3)
    n = org.shape[0]
    tmin = torch.full((n,), O.SHADOW_EPS)
    tmax = torch.full((n,), O.RAY_MAX)
    tri_o, u_o, v_o, t_o = osc.intersect(org, dirs, tmin, tmax)
    dev = scene.device
    tri_g, u_g, v_g, t_g = scene.intersect(org.to(dev), dirs.to(dev), tmin.to(dev), tmax.to(dev))
    assert (tri_o >= 0).sum() > n // 4
    np.testing.assert_array_equal(tri_g.cpu().numpy(), tri_o.numpy().astype(np.int32))
    hit = tri_o >= 0
    np.testing.assert_array_equal(u_g.cpu()[hit].numpy(), u_o[hit].numpy())
    np.testing.assert_array_equal(v_g.cpu()[hit].numpy(), v_o[hit].numpy())
    np.testing.assert_array_equal(t_g.cpu()[hit].numpy(), t_o[hit].numpy())
    # occlusion agrees with the closest-hit query inside a finite interval
    tmax2 = torch.where(hit, t_o * 0.999, torch.full_like(t_o, 3.0))
    vis = scene.occluded(org.to(dev), dirs.to(dev), tmin.to(dev), tmax2.to(dev)).cpu()
    tri2, _, _, _ = osc.intersect(org, dirs, tmin, tmax2)
    np.testing.assert_array_equal(vis.numpy(), (tri2 < 0).numpy().astype(np.int32))


def test_hash_sampler_matches_numpy(cfg1):
    spec, scene, osc, cam = cfg1
    opts = api.RenderOptions(7, D, 2, 0, 0, 0, 0)
    pt = api.PathTracer()
    img_hash = pt.renderC(scene, opts)
    table = O.hash_table(7, 0, api.sample_dims(0, D), W * H * 2).to(scene.device)
    img_tab = pt.renderC(scene, opts, samples=table)
    torch.testing.assert_close(img_hash, img_tab, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("depth", DEPTHS)
def test_path_forward_parity(cfg1, depth):
    spec, scene, osc, cam = cfg1
    spp = 4
    smp = sample_table(0, W, H, spp, depth, 1)
    img_g = api.PathTracer().renderC(scene, api.RenderOptions(0, depth, spp, 0, 0, 0, 0),
                                     samples=smp.to(scene.device))
    with torch.no_grad():
        osc.configure()
        img_o = O.path_tracer(osc, cam, spp, depth, smp)
    assert_image_parity(img_g, img_o, f"cfg1 {W}x{H} D{depth} forward")


@pytest.mark.parametrize("depth", DEPTHS)
@pytest.mark.parametrize("integrator", [0, 1, 2, 3, 4])
def test_grad_parity(cfg1, integrator, depth):
    spec, scene, osc, cam = cfg1
    spp = 4
    smp = sample_table(integrator, W, H, spp, depth, 2)
    g = torch.Generator().manual_seed(11)
    dLdI = torch.rand(W * H, 3, generator=g) - 0.3
    cls = [api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
           api.PixelBoundaryIntegrator][integrator]
    opts = api.RenderOptions(0, depth, spp, spp, spp, spp, spp)
    scene.clear_grads()
    cls().renderD(scene, opts, dLdI.reshape(H, W, 3).to(scene.device), samples=smp.to(scene.device))
    gg = scene.get_grads()
    go, _ = O.grads(osc, cam, integrator, spp, depth, smp, dLdI)
    label = f"cfg1 {W}x{H} D{depth} term {integrator}"
    assert_grad_parity(gg["positions"], go["positions"], label + " vertices")
    assert_grad_parity(gg["translation"], go["translation"], label + " translation")


@pytest.mark.parametrize("eps,depth,max_size,thold", [(0.01, 0, 0, 0.0), (0.5, 0, 0, 0.0),
                                                      (0.01, 2, 3000, 1e-4), (0.5, 1, 2100, 1e-5)])
def test_guided_direct_grad_parity(cfg1, eps, depth, max_size, thold):
    """AQ-guided direct boundary term (AdaptiveQuadratureDistribution,
    AQ_distrb.h:83-195): same tree, same leaf weights, same guided samples,
    same grads. depth > 0 refines the tree (36 evaluations per leaf and pass,
    splits appended in leaf order); the last case fills the leaf limit."""
    spec, scene, osc, cam = cfg1
    spp, gspp = 4, 4
    dims = api.sample_dims(api.TRN_DIRECT_EDGE, D, guided=True)
    smp = O.uniform_table(77, dims, api.sample_slots(api.TRN_DIRECT_EDGE, W, H, spp))
    g = torch.Generator().manual_seed(13)
    dLdI = torch.rand(W * H, 3, generator=g) - 0.3
    opts = api.RenderOptions(5, D, spp, spp, spp, spp, spp)
    opts.g_direct, opts.g_direct_spp, opts.g_eps = True, gspp, eps
    opts.g_direct_depth, opts.g_direct_max_size, opts.g_direct_thold = depth, max_size, thold
    scene.clear_grads()
    api.DirectEdgeIntegrator().renderD(scene, opts, dLdI.reshape(H, W, 3).to(scene.device),
                                       samples=smp.to(scene.device))
    gg = scene.get_grads()
    go, _ = O.grads(osc, cam, api.TRN_DIRECT_EDGE, spp, D, smp, dLdI,
                    guiding=(5, gspp, eps, depth, max_size, thold))
    label = f"cfg1 {W}x{H} D{D} guided direct eps {eps} depth {depth}"
    assert_grad_parity(gg["positions"], go["positions"], label + " vertices")
    assert_grad_parity(gg["translation"], go["translation"], label + " translation")
