"""Multi-rank host logic on CPU (gloo, world size 2): the batch sharding
used by the multi-GPU benchmark (every rank computes the same partition,
the shards cover every volume once, longest-processing-time balance) and
the max-over-ranks timing reduction."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nitorch_b200.batch import plan_shards


def _costs():
    g = torch.Generator().manual_seed(31)
    sizes = torch.randint(96, 257, (64, 3), generator=g)
    chans = torch.randint(1, 5, (64,), generator=g)
    return [int(s.prod()) * int(c) for s, c in zip(sizes, chans)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = _costs()
        shards, loads = plan_shards(costs, world)
        mine = torch.tensor(shards[rank] + [-1] * (len(costs) - len(shards[rank])))
        gathered = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(gathered, mine)
        # a per-rank "step time" proportional to the rank's load
        t = torch.tensor([loads[rank] / 1e6], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put(([g[g >= 0].tolist() for g in gathered], loads, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_lpt_partition_single_process():
    costs = _costs()
    shards, loads = plan_shards(costs, 4)
    assert sorted(i for s in shards for i in s) == list(range(len(costs)))
    assert max(loads) <= min(loads) + max(costs)
    assert [sum(costs[i] for i in s) for s in shards] == loads


@pytest.mark.timeout(180)
def test_sharding_and_max_timing_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    shards, loads, tmax = q.get(timeout=150)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(shards[0] + shards[1]) == list(range(64))
    assert not set(shards[0]) & set(shards[1])
    assert abs(tmax - max(loads) / 1e6) < 1e-9
    ref, _ = plan_shards(_costs(), 2)
    assert shards == ref
