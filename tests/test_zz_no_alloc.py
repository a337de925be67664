"""trn_render_grad_noalloc, the gradient entry point for callers that may not
allocate device memory while rendering (hosts whose own allocator owns all
of it, loops that cannot take cudaFree's synchronisation), against
trn_render_grad through the C-ABI on the same scene, camera, options and
dL/dI. Gradients are sums of float atomics whose order differs between
launches, so the comparison is a relative L2 tolerance of 1e-4, on two calls
in a row (the second call finds the scratch the first one left behind).
The file name puts it last in collection order; it also passes alone."""
import ctypes as C

import pytest
import torch

from tensorray_b200 import api, scenes
from tensorray_b200._abi import TrnSamples, check
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

W, H, D, SPP = 48, 32, 3, 4
TOL = 1e-4


@pytest.fixture(scope="module")
def setup(built_lib):
    spec = scenes.config1_scene(W, H)
    scene = api.Scene(spec)
    scene.configure()
    g = torch.Generator().manual_seed(5)
    dLdI = (torch.rand(H * W * 3, generator=g) - 0.3).to(scene.device)
    return scene, dLdI


def _grads(scene, fn, integrator, dLdI, guided=False):
    lib = scene._lib
    cam = scene.cameras[0]
    o = api.RenderOptions(3, D, SPP, SPP, SPP, SPP, SPP)
    o.g_direct = guided
    opts = o._c()
    smp = TrnSamples(None, 0)  # counter-hash sampler
    scene.clear_grads()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(getattr(lib, fn)(scene.handle, C.byref(cam.c), C.byref(opts), integrator, C.byref(smp),
                           C.c_void_p(dLdI.data_ptr()), stream), fn)
    torch.cuda.synchronize()
    g = scene.get_grads()
    return g["positions"].detach().cpu().clone(), g["translation"].detach().cpu().clone()


@pytest.mark.parametrize("integrator,guided", [(api.TRN_PRIMARY_EDGE, False), (api.TRN_PATH_TRACER, False),
                                               (api.TRN_DIRECT_EDGE, False), (api.TRN_DIRECT_EDGE, True),
                                               (api.TRN_INDIRECT_EDGE, False), (api.TRN_PIXEL_EDGE, False)])
def test_noalloc_grad_matches_allocating_entry_point(setup, integrator, guided):
    scene, dLdI = setup
    ref_p, ref_t = _grads(scene, "trn_render_grad", integrator, dLdI, guided)
    assert float(ref_p.abs().sum()) > 0
    for _ in range(2):
        p, t = _grads(scene, "trn_render_grad_noalloc", integrator, dLdI, guided)
        assert rel_l2(p, ref_p) < TOL, f"vertex grads rel L2 {rel_l2(p, ref_p):.2e}"
        assert rel_l2(t, ref_t) < TOL, f"translation grads {t.tolist()} vs {ref_t.tolist()}"


def _call_noalloc(scene, integrator, dLdI):
    lib = scene._lib
    o = api.RenderOptions(3, D, SPP, SPP, SPP, SPP, SPP)
    opts = o._c()
    smp = TrnSamples(None, 0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.trn_render_grad_noalloc(scene.handle, C.byref(scene.cameras[0].c), C.byref(opts), integrator,
                                      C.byref(smp), C.c_void_p(dLdI.data_ptr()), stream), "noalloc")


def test_noalloc_allocates_nothing(setup):
    """Free device memory stays the same across calls, including the first
    calls on a scene that never rendered through trn_render_grad (so no
    per-scene buffer is created lazily either). One earlier call per term on
    another scene has looked up the scratch address and let the driver size
    its local memory for the fused kernels."""
    scene, dLdI = setup
    for integ in range(5):
        _call_noalloc(scene, integ, dLdI)
    torch.cuda.synchronize()
    fresh = api.Scene(scenes.config1_scene(W, H))
    fresh.configure()
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for integ in range(5):
            _call_noalloc(fresh, integ, dLdI)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == before, "trn_render_grad_noalloc allocated device memory"


def test_noalloc_rejects_bad_arguments(setup):
    scene, dLdI = setup
    lib = scene._lib
    cam = scene.cameras[0]
    opts = api.RenderOptions(3, D, SPP, SPP, SPP, SPP, SPP)._c()
    smp = TrnSamples(None, 0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.trn_render_grad_noalloc(scene.handle, C.byref(cam.c), C.byref(opts), 9, C.byref(smp),
                                       C.c_void_p(dLdI.data_ptr()), stream) != 0
    assert lib.trn_render_grad_noalloc(scene.handle, C.byref(cam.c), C.byref(opts), api.TRN_PATH_TRACER,
                                       C.byref(smp), None, stream) != 0
