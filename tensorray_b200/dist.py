"""Multi-GPU plumbing: one process per GPU, sample sharding by seed, and the
single gradient exchange of the path (a sum all-reduce).

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
