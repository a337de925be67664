"""Multi-rank host logic on CPU with gloo (world size 2): disjoint seeds per
rank, cost-balanced view sharding, and the gradient sum all-reduce."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tensorray_b200 import dist as trd


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = {"positions": torch.full((5, 3), float(rank + 1)), "texels": torch.arange(4.0).reshape(2, 2) * (rank + 1),
         "translation": None}
    r = trd.allreduce_grads(g)
    out[rank] = (r["positions"].clone(), r["texels"].clone())
    dist.barrier()
    dist.destroy_process_group()


def test_allreduce_sums_gradients_over_ranks():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    for rank in range(world):
        pos, tex = out[rank]
        assert torch.equal(pos, torch.full((5, 3), 3.0))
        assert torch.equal(tex, torch.arange(4.0).reshape(2, 2) * 3)


def test_rank_seeds_are_disjoint_and_views_balance():
    seeds = {trd.rank_seed(s, r) for s in range(5) for r in range(8)}
    assert len(seeds) == 40
    costs = [512 * 512 * 64, 128 * 128 * 8, 256 * 256 * 16, 384 * 384 * 32, 128 * 128 * 64, 512 * 512 * 8]
    shards = trd.shard_views(costs, 2)
    assert sorted(sum(shards, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shards]
    # greedy longest-processing-time bound
    assert max(loads) <= sum(costs) / 2 + max(costs) / 2


def test_single_process_allreduce_is_identity():
    g = {"positions": torch.ones(3, 3)}
    assert trd.allreduce_grads(g) is g


# ---- view-sharded inverse-rendering step, render stubbed on the CPU ----------
class _FakeCamera:
    def __init__(self, w, h):
        self.width, self.height = w, h


class _FakeScene:
    """Stands in for api.Scene: raw positions, a gradient buffer that the
    fake view sets accumulate into, and a log of every rendered view."""

    def __init__(self, nv):
        self.device = torch.device("cpu")
        self._raw_positions = torch.linspace(-1.0, 1.0, nv * 3).reshape(nv, 3)
        self.grad = torch.zeros(nv, 3)
        self.rendered = []

    def set_vertex_positions(self, x):
        self._raw_positions = x.detach().clone()

    def configure(self, refit=False):
        pass

    def clear_grads(self):
        self.grad.zero_()

    def get_grads(self):
        return {"positions": self.grad.clone()}


class _FakeViewSet:
    """Stands in for api.ViewSet: view i of the set is global view seeds[i];
    its image, loss and gradient depend only on that index and the positions."""

    def __init__(self, scene, cameras, spps, seeds=None):
        self.scene, self.cameras, self.spps = scene, list(cameras), list(spps)
        self.seeds = list(seeds if seeds is not None else range(len(cameras)))
        self.npix = sum(c.width * c.height for c in cameras)
        self.offsets = [sum(c.width * c.height for c in cameras[:i]) for i in range(len(cameras))]

    def _slices(self):
        off = 0
        for c in self.cameras:
            n = c.width * c.height
            yield slice(off, off + n)
            off += n

    def render(self, integrator, options, launch=None, out=None):
        for v, sl in zip(self.seeds, self._slices()):
            out[sl] = float(v + 1) * self.scene._raw_positions.sum() / 10.0
            self.scene.rendered.append(("fwd", v))
        return out

    def loss(self, image, targets, dLdI):
        dLdI.copy_(image - targets)
        return torch.stack([0.5 * (dLdI[sl] ** 2).sum() for sl in self._slices()])

    def render_grad(self, integrator, options, dLdI, launch=None):
        nv = self.scene.grad.shape[0]
        for v, sl in zip(self.seeds, self._slices()):
            self.scene.grad[v % nv] += dLdI[sl].sum(0) * (integrator + 1)
            self.scene.rendered.append(("grad", integrator, v))


def _views_setup():
    cams = [_FakeCamera(w, w) for w in (4, 2, 3, 5, 1, 2, 4)]
    spps = [8, 64, 16, 4, 32, 8, 16]
    npix = sum(c.width * c.height for c in cams)
    targets = torch.arange(npix * 3, dtype=torch.float32).reshape(npix, 3) / npix
    return cams, spps, targets


def _run_inverse(steps):
    from tensorray_b200 import api, inverse
    cams, spps, targets = _views_setup()
    scene = _FakeScene(5)
    real = api.ViewSet
    api.ViewSet = _FakeViewSet
    try:
        inv = inverse.InverseRenderer(scene, cams, spps, targets, api.RenderOptions(0, 3, 0, 0, 0, 0, 0), lr=1e-2)
        losses = [inv.step().clone() for _ in range(steps)]
    finally:
        api.ViewSet = real
    return inv, scene, losses


def _sharded_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    inv, scene, losses = _run_inverse(3)
    out[rank] = (list(inv.shard.local), scene.rendered, [l.tolist() for l in losses], inv.x.detach().clone(),
                 inv.x.grad.clone())
    dist.barrier()
    dist.destroy_process_group()


def test_view_sharded_inverse_step_matches_one_rank():
    """Two gloo ranks split the views by cost; every view is rendered exactly
    once per step, the summed gradient, the per-view losses and the Adam
    update equal those of a single process rendering every view."""
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_sharded_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    inv1, scene1, losses1 = _run_inverse(3)
    nviews = len(_views_setup()[0])
    locals_ = [out[r][0] for r in range(world)]
    assert sorted(sum(locals_, [])) == list(range(nviews)) and all(locals_)
    # three steps: every view's forward once per step, and its gradient once
    # per step and integrator, on one rank or the other
    fwd = sorted(e[1] for r in range(world) for e in out[r][1] if e[0] == "fwd")
    assert fwd == sorted(list(range(nviews)) * 3)
    grads = sorted((e[1], e[2]) for r in range(world) for e in out[r][1] if e[0] == "grad")
    assert grads == sorted([(i, v) for i in (0, 1, 2) for v in range(nviews)] * 3)
    for r in range(world):
        assert out[r][2] == [l.tolist() for l in losses1]
        torch.testing.assert_close(out[r][3], inv1.x.detach(), rtol=1e-6, atol=1e-7)
        torch.testing.assert_close(out[r][4], inv1.x.grad, rtol=1e-6, atol=1e-6)


class _FakeSpec:
    def __init__(self, faces):
        self.faces = faces

    def arrays(self):
        return {"indices": self.faces}


def test_inverse_step_pyramid_loss_and_largesteps_plumbing():
    """One process, render stubbed: the pyramid loss's dL/dI per view is the
    reverse mode of pyTensorRay/loss.py's pyramid L1 of that view, and the
    LargeSteps option updates the positions as optim.LargeSteps does."""
    from tensorray_b200 import api, inverse, loss as trl, optim
    cams, spps, targets = _views_setup()
    scene = _FakeScene(5)
    faces = torch.tensor([[0, 1, 2], [0, 2, 3], [0, 3, 4], [0, 4, 1]], dtype=torch.int32)
    scene.spec = _FakeSpec(faces.numpy())
    real = api.ViewSet
    api.ViewSet = _FakeViewSet
    try:
        inv = inverse.InverseRenderer(scene, cams, spps, targets, api.RenderOptions(0, 3, 0, 0, 0, 0, 0), lr=1e-2,
                                      loss="pyramid_l1", optimizer="largesteps", lmbda=0.5)
        x0 = inv.x.detach().clone()
        losses = inv.step()
    finally:
        api.ViewSet = real
    assert losses.shape == (len(cams),)
    for i, c in enumerate(cams):
        sl = slice(inv.views.offsets[i], inv.views.offsets[i] + c.width * c.height)
        img = inv.image[sl].view(c.height, c.width, 3)
        tgt = targets[sl].view(c.height, c.width, 3)
        ref_loss, ref_g = trl.loss_and_grad("pyramid_l1", img, trl.build_pyramid(tgt))
        torch.testing.assert_close(inv.dLdI[sl].view(c.height, c.width, 3), ref_g)
        assert abs(float(losses[i]) - float(ref_loss)) <= 1e-6 * abs(float(ref_loss)) + 1e-7
    ref = x0.clone().requires_grad_(True)
    opt = optim.LargeSteps(ref, torch.as_tensor(faces), lr=1e-2, lmbda=0.5)
    ref.grad = inv.x.grad.clone()
    opt.step()
    torch.testing.assert_close(inv.x.detach(), ref.detach())


def _one_view_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from tensorray_b200 import api, inverse
    cams = [_FakeCamera(3, 3)]
    targets = torch.zeros(9, 3)
    scene = _FakeScene(5)
    real = api.ViewSet
    api.ViewSet = _FakeViewSet
    try:
        inv = inverse.InverseRenderer(scene, cams, [4], targets, api.RenderOptions(0, 3, 0, 0, 0, 0, 0), lr=1e-2)
        losses = [inv.step().clone() for _ in range(2)]
    finally:
        api.ViewSet = real
    out[rank] = (list(inv.shard.local), inv.views is None, inv.samples_per_step(), [l.tolist() for l in losses],
                 inv.x.detach().clone())
    dist.barrier()
    dist.destroy_process_group()


def test_rank_without_views_still_joins_the_exchange():
    """More ranks than views: the rank that holds no view renders nothing,
    reports no samples, and still takes part in the gradient and loss
    all-reduces, so every rank ends with the same losses and positions."""
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_one_view_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    holders = [r for r in range(world) if out[r][0]]
    assert len(holders) == 1
    empty = 1 - holders[0]
    assert out[empty][1] and out[empty][2] == 0
    assert out[0][3] == out[1][3]
    torch.testing.assert_close(out[0][4], out[1][4])
