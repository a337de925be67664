"""Multi-GPU plumbing: one process per GPU, sample sharding by seed or by
view, and the single gradient exchange of the path (a sum all-reduce).

The path has no data exchange: ranks render disjoint sample streams of the
same views (or disjoint views) and only the gradient buffers -- a sum over
samples in the reference (IndexedWriteKernel scatter-add,
TensorKernels.cuh:177-209) -- are combined once per optimisation step.
"""
from __future__ import annotations

import os

import torch
import torch.distributed as dist


def rank_info() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(base_seed: int, rank: int) -> int:
    """Disjoint sample streams per rank (the hash sampler is keyed by seed)."""
    return base_seed * 1009 + 7919 * rank + 1


def shard_views(costs: list, world: int) -> list:
    """Assign views to ranks greedily by estimated cost (W*H*spp*depth),
    heaviest first; returns the view indices of every rank."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: load[k])
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def allreduce_grads(grads: dict, group=None) -> dict:
    """Sum every gradient tensor over ranks with one flattened all-reduce."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return grads
    keys = [k for k in sorted(grads) if grads[k] is not None and grads[k].numel()]
    flat = torch.cat([grads[k].reshape(-1) for k in keys])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out = dict(grads)
    off = 0
    for k in keys:
        n = grads[k].numel()
        out[k] = flat[off:off + n].view_as(grads[k])
        off += n
    return out


class ViewShard:
    """The views one rank renders when a multi-view set is split over ranks
    (the reference renders them one after another on one device,
    pyTensorRay/renderer_multi_view.py:53-61). Views go to ranks by estimated
    cost, W*H*spp*depth, heaviest first; every view lands on exactly one rank
    and keeps its global index, which is also its sample seed, so a sharded
    run draws the same samples as the unsharded one. Every rank holds a full
    scene replica; the only exchange is the gradient sum (allreduce_grads)
    and the per-view loss vector (gather_view_values)."""

    def __init__(self, costs: list, world: int, rank: int):
        if not 0 <= rank < world:
            raise ValueError("rank out of range")
        self.nviews, self.world, self.rank = len(costs), int(world), int(rank)
        self.assignment = shard_views(list(costs), self.world)
        self.local = self.assignment[self.rank]

    @staticmethod
    def of(cameras: list, spps: list, depth: int, group=None) -> "ViewShard":
        """The shard of this process in the initialised process group (a
        single shard holding every view when there is none)."""
        costs = [c.width * c.height * int(s) * max(1, int(depth)) for c, s in zip(cameras, spps)]
        if dist.is_available() and dist.is_initialized():
            return ViewShard(costs, dist.get_world_size(group), dist.get_rank(group))
        return ViewShard(costs, 1, 0)

    def pick(self, items: list) -> list:
        """This rank's entries of a per-view list."""
        return [items[i] for i in self.local]


def gather_view_values(shard: ViewShard, local_values: torch.Tensor, group=None) -> torch.Tensor:
    """Per-view values of every view (e.g. losses), from each rank's values of
    its own views: one sum all-reduce of a vector that is zero outside them."""
    full = torch.zeros(shard.nviews, dtype=local_values.dtype, device=local_values.device)
    if shard.local:
        full[torch.as_tensor(shard.local, device=local_values.device)] = local_values.reshape(-1)
    if shard.world > 1:
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full
