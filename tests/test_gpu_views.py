"""Batched multi-view launches equal the per-view calls they replace
(pyTensorRay/renderer_multi_view.py:53-61 loops over views one at a time)."""
import pytest
import torch

from oracle import tr_oracle as O
from tensorray_b200 import api, scenes
from tensorray_b200._abi import TrnView
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

D = 3


@pytest.fixture(scope="module")
def setup(built_lib):
    spec = scenes.config1_scene(32, 32)
    scene = api.Scene(spec)
    scene.configure()
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(5, 4.0, [16, 24, 32], seed=3)]
    spps = [2, 4, 2, 4, 2]
    return scene, cams, spps


def _tables(integ, cams, spps, seed):
    per = [O.uniform_table(seed + 17 * i, api.sample_dims(integ, D), api.sample_slots(integ, c.width, c.height, s))
           for i, (c, s) in enumerate(zip(cams, spps))]
    return per, torch.cat(per, 1).contiguous()


def test_updates_every_call_run_ahead_of_the_device(setup):
    """A set whose views change on every call, as in the serving loop, stages
    each table upload in its own pinned slot. Renders and losses issued back
    to back with no synchronisation between them, more of them than there are
    slots and with one growth of the set in between, give the images and
    losses of fresh sets of the same views."""
    scene, cams, spps = setup
    opts = api.RenderOptions(5, D, 0, 0, 0, 0, 0)
    plan = [[0], [1, 2], [3, 4, 0], [2], [4, 1], [0, 3], [1], [2, 3, 4], [0, 1, 2, 3, 4], [3], [4, 2], [1]]

    def pick(idx):
        arr = (TrnView * len(idx))()
        for j, v in enumerate(idx):
            arr[j] = TrnView(cams[v].c, spps[v], 100 + v, -1, 0, 0.0, 0, None, None, None, None, None)
        return [cams[v] for v in idx], [spps[v] for v in idx], arr

    vs = api.ViewSet(scene, *pick(plan[2])[:2], seeds=[100 + v for v in plan[2]])
    out = []
    for idx in plan:
        c, s, arr = pick(idx)
        vs.update(c, s, arr)
        img = vs.render(0, opts)
        loss = vs.loss(img, torch.zeros_like(img))
        out.append((idx, img, loss, [vs.view_image(img, j) for j in range(len(idx))]))
    torch.cuda.synchronize()
    for idx, img, loss, views in out:
        c, s, _ = pick(idx)
        fresh = api.ViewSet(scene, c, s, seeds=[100 + v for v in idx])
        ref = fresh.render(0, opts)
        torch.testing.assert_close(img, ref, rtol=1e-5, atol=1e-6)
        torch.testing.assert_close(loss, fresh.loss(ref, torch.zeros_like(ref)), rtol=1e-5, atol=1e-6)
        for j in range(len(idx)):
            torch.testing.assert_close(views[j], fresh.view_image(ref, j), rtol=1e-5, atol=1e-6)


def test_batched_forward_equals_per_view(setup):
    scene, cams, spps = setup
    vs = api.ViewSet(scene, cams, spps)
    per, cat = _tables(0, cams, spps, 1)
    opts = api.RenderOptions(0, D, 0, 0, 0, 0, 0)
    img = vs.render(0, opts, samples=cat.cuda())
    for v, (c, s) in enumerate(zip(cams, spps)):
        o = api.RenderOptions(0, D, s, 0, 0, 0, 0)
        ref = api.PathTracer().renderC(scene, o, samples=per[v].cuda(), camera=c)
        torch.testing.assert_close(vs.view_image(img, v), ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("integ", [0, 1, 2, 3, 4])
def test_batched_grads_equal_sum_of_per_view(setup, integ):
    scene, cams, spps = setup
    vs = api.ViewSet(scene, cams, spps)
    per, cat = _tables(integ, cams, spps, 5)
    g = torch.Generator().manual_seed(1)
    dLdI = (torch.rand(vs.npix, 3, generator=g) - 0.3).cuda()
    opts = api.RenderOptions(0, D, 0, 0, 0, 0, 0)
    scene.clear_grads()
    vs.render_grad(integ, opts, dLdI, samples=cat.cuda())
    gb = scene.get_grads()["positions"].clone()
    scene.clear_grads()
    cls = [api.PathTracer, api.PrimaryEdgeIntegrator, api.DirectEdgeIntegrator, api.IndirectEdgeIntegrator,
           api.PixelBoundaryIntegrator][integ]
    for v, (c, s) in enumerate(zip(cams, spps)):
        o = api.RenderOptions(0, D, s, s, s, s, s)
        cls().renderD(scene, o, vs.view_image(dLdI, v), samples=per[v].cuda(), camera=c)
    gs = scene.get_grads()["positions"]
    assert float(gs.abs().sum()) > 0
    assert rel_l2(gb.cpu(), gs.cpu()) < 1e-5


def test_view_loss_matches_torch(setup):
    scene, cams, spps = setup
    vs = api.ViewSet(scene, cams, spps)
    img = torch.rand(vs.npix, 3, device="cuda")
    tgt = torch.rand(vs.npix, 3, device="cuda")
    d = torch.empty_like(img)
    loss = vs.loss(img, tgt, d)
    torch.testing.assert_close(d, img - tgt)
    for v in range(len(cams)):
        ref = 0.5 * ((vs.view_image(img, v) - vs.view_image(tgt, v)) ** 2).sum()
        torch.testing.assert_close(loss[v], ref, rtol=1e-4, atol=1e-4)


def test_launch_configs_give_same_image(setup):
    scene, cams, spps = setup
    vs = api.ViewSet(scene, cams, spps)
    opts = api.RenderOptions(4, D, 0, 0, 0, 0, 0)
    ref = vs.render(0, opts)
    for blk, per_sm, chunk in [(64, 8, 1), (256, 4, 4), (128, 16, 2)]:
        img = vs.render(0, opts, launch=api.launch_config(blk, per_sm, chunk))
        torch.testing.assert_close(img, ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("integ", [0, 1, 2, 3, 4])
def test_round_size_does_not_change_gradients(setup, integ):
    """Split kernels in rounds of 2^16 slots (paths) give the gradients of the
    default rounds: a slot's samples do not depend on its round."""
    scene = setup[0]
    cams = [api.Camera(c.pos, c.target, c.up, c.width, c.height, c.fov)
            for c in scenes.fibonacci_cameras(2, 4.0, [256], seed=4)]
    vs = api.ViewSet(scene, cams, [4, 4])
    g = torch.Generator().manual_seed(5)
    dLdI = (torch.rand(vs.npix, 3, generator=g) - 0.3).to(scene.device)
    opts = api.RenderOptions(2, D, 0, 0, 0, 0, 0)
    out = []
    for ln in (None, api.launch_config(0, 0, 0, 16)):
        scene.clear_grads()
        vs.render_grad(integ, opts, dLdI, launch=ln)
        out.append(scene.get_grads()["positions"].clone())
    assert vs.slots(integ) > (1 << 16)
    assert float(out[0].abs().sum()) > 0
    assert rel_l2(out[1].cpu(), out[0].cpu()) < 1e-5


@pytest.mark.parametrize("integ", [0, 1, 2, 3, 4])
def test_per_view_gradient_buffers(setup, integ):
    """Views with their own gradient buffers in one launch: each buffer holds
    exactly its view's gradient (the warp-aggregated scatter must not merge
    lanes that target different views' buffers at the same vertex)."""
    scene, cams, spps = setup
    dev = scene.device
    nv = scene.num_vertices
    bufs = [(torch.zeros(nv, 3, device=dev), torch.zeros(nv, 3, device=dev)) for _ in cams]
    arr = (api.TrnView * len(cams))()
    for i, (c, s) in enumerate(zip(cams, spps)):
        arr[i] = api.TrnView(c.c, s, 40 + i, -1, 0, 0.0, D, bufs[i][0].data_ptr(), bufs[i][1].data_ptr(), None,
                             None, None)
    vs = api.ViewSet(scene, cams, spps, views=arr)
    g = torch.Generator().manual_seed(2)
    dLdI = (torch.rand(vs.npix, 3, generator=g) - 0.3).to(dev)
    opts = api.RenderOptions(0, D, 0, 0, 0, 0, 0)
    scene.clear_grads()
    vs.render_grad(integ, opts, dLdI)
    for i, (c, s) in enumerate(zip(cams, spps)):
        scene.finalize_grads(bufs[i][0], bufs[i][1])
        one = (api.TrnView * 1)(api.TrnView(c.c, s, 40 + i, -1, 0, 0.0, D, None, None, None, None, None))
        vs1 = api.ViewSet(scene, [c], [s], views=one)
        scene.clear_grads()
        vs1.render_grad(integ, opts, vs.view_image(dLdI, i).reshape(-1, 3).contiguous())
        ref = scene.get_grads()["positions"]
        if float(ref.abs().sum()) == 0:
            continue
        assert rel_l2(bufs[i][0].cpu(), ref.cpu()) < 1e-4, f"view {i}: rel L2 {rel_l2(bufs[i][0].cpu(), ref.cpu()):.2e}"


def test_reserved_set_allocates_nothing_later(setup):
    """After ViewSet.reserve, gradient calls of every term allocate no device
    memory and give the gradients of a set that allocates on first use."""
    scene, cams, spps = setup
    dev = scene.device
    opts = api.RenderOptions(5, D, 0, 0, 0, 0, 0)
    g = torch.Generator().manual_seed(4)
    plain = api.ViewSet(scene, cams, spps)
    dLdI = (torch.rand(plain.npix, 3, generator=g) - 0.3).to(dev)
    ref = []
    for integ in range(5):
        scene.clear_grads()
        plain.render_grad(integ, opts, dLdI)
        ref.append(scene.get_grads()["positions"].clone())
    vs = api.ViewSet(scene, cams, spps)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    vs.reserve(D)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert 0 < free0 - free1 < 6e9, f"reserved {free0 - free1} bytes"
    for integ in range(5):
        scene.clear_grads()
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        vs.render_grad(integ, opts, dLdI)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == before, f"term {integ} allocated"
        got = scene.get_grads()["positions"]
        if float(ref[integ].abs().sum()) > 0:
            assert rel_l2(got.cpu(), ref[integ].cpu()) < 1e-4
    with pytest.raises(RuntimeError):
        vs.reserve(17)
