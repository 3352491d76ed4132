"""Splitting independent problems over ranks (configuration 5 on several GPUs): every problem
goes to exactly one rank, the estimated work is balanced, and two gloo ranks on the CPU agree on
the split and on the aggregated totals the benchmark reports (no GPU)."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from pdekit_b200 import workloads
from pdekit_b200.batch import problem_work, shard_problems


def _problems():
    probs, _, _, _ = workloads.config5(nprob=24, seed=9, min_cells=50, max_cells=3000)
    return probs


def test_shards_partition_and_balance():
    probs = _problems()
    work = [problem_work(p) for p in probs]
    for n in (1, 2, 3, 8):
        shards = shard_problems(probs, n)
        assert len(shards) == n
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(probs)))
        loads = [sum(work[i] for i in sh) for sh in shards]
        # greedy largest-first: no rank exceeds the mean by more than the largest problem
        assert max(loads) <= sum(work) / n + max(work) + 1e-9


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    probs = _problems()
    mine = shard_problems(probs, world)[rank]
    lists = [None] * world
    dist.all_gather_object(lists, mine)
    cells = torch.tensor([float(sum(probs[i].ncells for i in mine))], dtype=torch.float64)
    dist.all_reduce(cells, op=dist.ReduceOp.SUM)
    if rank == 0:
        out.put((lists, float(cells.item()), sum(p.ncells for p in probs)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    lists, cells, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(lists[0] + lists[1]) == list(range(24)) and not set(lists[0]) & set(lists[1])
    assert lists == shard_problems(_problems(), 2)
    assert np.isclose(cells, total)
