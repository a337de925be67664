"""The continuous-batching server: a request's result is the same alone and
in a mix of other requests, it equals the direct batched-API computation, and
admission respects the HBM budget."""
import pytest
import torch

from tensorray_b200 import api, scenes, serve
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(built_lib):
    s1 = api.Scene(scenes.config1_scene(32, 32))
    s2 = api.Scene(scenes.config2_scene(32, 32, tris=3000, tex_size=16))
    s1.configure()
    s2.configure()
    return {"ico": s1, "disp": s2}


def _req(world, scene, pos, res, spp, depth, seed):
    cam = api.Camera(pos, (0, 0, 0), (0, 1, 0), res, res, 45.0)
    tgt = torch.full((res * res, 3), 0.05, device="cuda")
    return serve.RenderRequest(scene, cam, spp, depth, tgt, seed=seed)


def _probe(world, terms=None):
    r = _req(world, "ico", (0.3, 0.5, 4.0), 32, 12, 3, seed=7)
    if terms is not None:
        r.terms = tuple(terms)
    return r


TERM_SETS = [None, serve.ALL_TERMS]


@pytest.mark.parametrize("terms", TERM_SETS, ids=["three_terms", "all_terms"])
def test_alone_equals_in_the_mix(world, terms):
    alone = serve.Server(world, chunk_spp=4)
    r0 = alone.submit(_probe(world, terms))
    while not alone.idle():
        alone.step()
    mix = serve.Server(world, chunk_spp=4)
    others = [_req(world, "ico", (4.0 * (i % 3 - 1), 1.0, 3.0), 24 + 8 * (i % 2), 4 * (1 + i % 3), 2 + i % 3, 100 + i)
              for i in range(4)]
    others += [_req(world, "disp", (0.0, 1.0, 4.0), 16, 8, 3, 200 + i) for i in range(2)]
    for o in others[:3]:
        mix.submit(o)
    mix.step()  # the probe arrives while others are already on the GPU
    r1 = mix.submit(_probe(world, terms))
    for o in others[3:]:
        mix.submit(o)
    while not mix.idle():
        mix.step()
    torch.cuda.synchronize()
    assert r0.phase == serve.PHASE_DONE and r1.phase == serve.PHASE_DONE
    assert float(r0.image.abs().sum()) > 0
    assert rel_l2(r1.image.cpu(), r0.image.cpu()) < 1e-5
    assert rel_l2(r1.grad_positions.cpu(), r0.grad_positions.cpu()) < 1e-4
    assert abs(float(r1.loss) - float(r0.loss)) <= 1e-5 * abs(float(r0.loss)) + 1e-7


@pytest.mark.parametrize("terms", TERM_SETS, ids=["three_terms", "all_terms"])
def test_server_equals_direct_views(world, terms):
    srv = serve.Server(world, chunk_spp=64)   # one chunk per phase
    r = srv.submit(_probe(world, terms))
    while not srv.idle():
        srv.step()
    sc = world["ico"]
    V = api.TrnView(r.camera.c, r.spp, r.seed, -1, 0, 0.0, r.depth, None, None, None, None, None)
    arr = (api.TrnView * 1)(V)
    vs = api.ViewSet(sc, [r.camera], [r.spp], views=arr)
    opts = api.RenderOptions(0, r.depth, 0, 0, 0, 0, 0)
    img = vs.render(api.TRN_PATH_TRACER, opts)
    torch.testing.assert_close(img, r.image, rtol=1e-5, atol=1e-6)
    sc.clear_grads()
    for t in r.terms:
        vs.render_grad(t, opts, img - r.target)
    g = sc.get_grads()["positions"]
    assert rel_l2(r.grad_positions.cpu(), g.cpu()) < 1e-4


def test_admission_respects_budget(world):
    probe = _probe(world)
    srv = serve.Server(world, chunk_spp=4)
    one = srv.request_bytes(probe)
    srv.budget = int(1.5 * one)            # room for one request at a time
    reqs = [srv.submit(_req(world, "ico", (0.0, 0.5 * i, 4.0), 32, 8, 3, seed=i)) for i in range(3)]
    while not srv.idle():
        assert len(srv.active) <= 1
        srv.step()
    assert srv.stats.peak_bytes <= srv.budget
    assert all(r.phase == serve.PHASE_DONE for r in reqs)
    with pytest.raises(RuntimeError):
        srv.submit(_req(world, "ico", (0, 0, 4), 512, 8, 3, seed=0))
