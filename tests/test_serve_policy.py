"""Scheduling policy of the continuous-batching server on CPU: the
iteration's sample budget is filled shortest-remaining-work first."""
from types import SimpleNamespace

from tensorray_b200 import serve


def _server(budget):
    srv = serve.Server.__new__(serve.Server)  # no CUDA streams needed for the policy
    srv.chunk_spp = 8
    srv.iter_samples = budget
    srv.active = []
    return srv


def _req(rid, res, spp, phase=serve.PHASE_FWD, chunk=0, arrival=0.0, terms=(0, 1, 2)):
    return serve.RenderRequest(scene="s", camera=SimpleNamespace(width=res, height=res), spp=spp, depth=3,
                               target=None, rid=rid, arrival=arrival, phase=phase, chunk=chunk, terms=terms)


def test_srpt_fills_budget_smallest_first():
    srv = _server(budget=3 * 64 * 64 * 8)
    big, small, mid = _req(0, 512, 64), _req(1, 64, 8), _req(2, 64, 32, arrival=1.0)
    srv.active = [big, small, mid]
    chosen = srv._select()
    assert [r.rid for r in chosen] == [1, 2]        # big does not fit beside them
    assert srv._remaining(small) == 64 * 64 * 8 * (1 + 3)


def test_at_least_one_request_advances():
    srv = _server(budget=1)
    srv.active = [_req(0, 512, 64), _req(1, 256, 64, phase=serve.PHASE_GRAD)]
    chosen = srv._select()
    assert len(chosen) == 1 and chosen[0].rid == 1  # the gradient phase has less work left
    srv.active.append(_req(2, 64, 8, phase=serve.PHASE_FINISH))
    assert all(r.phase != serve.PHASE_FINISH for r in srv._select())
