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
