"""Path cache: a forward render of the interior term keeps its path records and
the gradient call of the same paths runs only the reverse sweep. The reference
re-traces the paths in RenderD (Integrator.h:106-121); the gradients must be
those of the replaying form, and records must never be reused once anything
the paths depend on has changed. Gradients are sums of float atomics, so the
two forms agree up to summation order."""
import pytest
import torch

from tensorray_b200 import api, scenes
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

W = H = 32
D = 3


def _grads(scene):
    g = scene.get_grads()
    return g["positions"].cpu(), g["texels"].cpu()


def _close(a, b, tol=1e-5):
    for x, y in zip(a, b):
        if float(y.abs().sum()) == 0:
            assert float(x.abs().sum()) == 0
        else:
            assert rel_l2(x, y) < tol, f"rel L2 {rel_l2(x, y):.2e}"


def _replayed(spec, opts, dLdI, raw=None):
    """renderD of a scene whose path cache is off (the replaying form)."""
    ref = api.Scene(spec)
    ref.set_path_cache(0)
    if raw is not None:
        ref.set_vertex_positions(raw)
    ref.configure()
    img = api.PathTracer().renderC(ref, opts)
    ref.clear_grads()
    api.PathTracer().renderD(ref, opts, dLdI)
    return img, _grads(ref)


def test_cached_gradient_equals_replay(built_lib):
    spec = scenes.config1_scene(W, H)
    sc = api.Scene(spec)
    sc.configure()
    opts = api.RenderOptions(3, D, 4, 4, 4, 4, 4)
    g = torch.Generator().manual_seed(5)
    dLdI = (torch.rand(H, W, 3, generator=g) - 0.3).cuda()
    img = api.PathTracer().renderC(sc, opts)
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts, dLdI)
    got = _grads(sc)
    ref_img, ref = _replayed(spec, opts, dLdI)
    torch.testing.assert_close(img, ref_img, rtol=1e-5, atol=1e-6)
    _close(got, ref)
    # a second gradient call with other dL/dI reuses the same records
    dLdI2 = (torch.rand(H, W, 3, generator=g) - 0.5).cuda()
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts, dLdI2)
    ref_sc = api.Scene(spec)
    ref_sc.set_path_cache(0)
    ref_sc.configure()
    ref_sc.clear_grads()
    api.PathTracer().renderD(ref_sc, opts, dLdI2)
    _close(_grads(sc), _grads(ref_sc))


def test_records_not_reused_after_changes(built_lib):
    spec = scenes.config1_scene(W, H)
    sc = api.Scene(spec)
    sc.configure()
    g = torch.Generator().manual_seed(6)
    dLdI = (torch.rand(H, W, 3, generator=g) - 0.3).cuda()
    opts = api.RenderOptions(1, D, 4, 4, 4, 4, 4)
    # other seed in the gradient call
    api.PathTracer().renderC(sc, opts)
    opts2 = api.RenderOptions(2, D, 4, 4, 4, 4, 4)
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts2, dLdI)
    _close(_grads(sc), _replayed(spec, opts2, dLdI)[1])
    # other depth
    api.PathTracer().renderC(sc, opts)
    opts3 = api.RenderOptions(1, D - 1, 4, 4, 4, 4, 4)
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts3, dLdI)
    _close(_grads(sc), _replayed(spec, opts3, dLdI)[1])
    # other camera
    api.PathTracer().renderC(sc, opts)
    cam = api.Camera((0.3, 0.2, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), W, H, 45.0)
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts, dLdI, camera=cam)
    ref = api.Scene(spec)
    ref.set_path_cache(0)
    ref.configure()
    ref.clear_grads()
    api.PathTracer().renderD(ref, opts, dLdI, camera=cam)
    _close(_grads(sc), _grads(ref))
    # moved vertices (new scene version)
    api.PathTracer().renderC(sc, opts)
    raw = torch.as_tensor(spec.arrays()["positions"]).clone()
    raw = raw + 0.02 * torch.randn(raw.shape, generator=g)
    sc.set_vertex_positions(raw)
    sc.configure()
    sc.clear_grads()
    api.PathTracer().renderD(sc, opts, dLdI)
    _close(_grads(sc), _replayed(spec, opts, dLdI, raw)[1])


def test_view_set_path_cache(built_lib):
    spec = scenes.config1_scene(W, H)
    sc = api.Scene(spec)
    sc.configure()
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(3, 4.0, [16, 24, 32], seed=4)]
    spps = [2, 4, 3]
    opts = api.RenderOptions(7, D, 0, 0, 0, 0, 0)
    plain = api.ViewSet(sc, cams, spps)
    cached = api.ViewSet(sc, cams, spps)
    cached.set_path_cache(1 << 30)
    g = torch.Generator().manual_seed(8)
    dLdI = (torch.rand(plain.npix, 3, generator=g) - 0.3).cuda()
    ia = plain.render(api.TRN_PATH_TRACER, opts)
    ib = cached.render(api.TRN_PATH_TRACER, opts)
    torch.testing.assert_close(ib, ia, rtol=1e-5, atol=1e-6)
    sc.clear_grads()
    plain.render_grad(api.TRN_PATH_TRACER, opts, dLdI)
    ref = _grads(sc)
    sc.clear_grads()
    cached.render_grad(api.TRN_PATH_TRACER, opts, dLdI)
    _close(_grads(sc), ref)
    # a limit below the records' size renders without them
    cached.set_path_cache(1024)
    cached.render(api.TRN_PATH_TRACER, opts)
    sc.clear_grads()
    cached.render_grad(api.TRN_PATH_TRACER, opts, dLdI)
    _close(_grads(sc), ref)
