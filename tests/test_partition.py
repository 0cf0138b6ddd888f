"""Whole-system partition of a batch across GPUs (rainmd_b200/partition.py): every system on
exactly one rank, the longest-processing-time balance bound, and the same partition computed
independently on each of two gloo ranks."""
import math
import os

import pytest

from rainmd_b200.partition import partition_systems, system_cost


def test_every_system_on_exactly_one_rank_and_balanced():
    costs = [float((7 * k) % 13 + 1) for k in range(41)]
    for ranks in (1, 2, 3, 8, 50):
        parts = partition_systems(costs, ranks)
        assert len(parts) == ranks
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        assert all(p == sorted(p) for p in parts)
        loads = [sum(costs[k] for k in p) for p in parts]
        bound = max(sum(costs) / ranks, max(costs))
        assert max(loads) <= 4.0 / 3.0 * bound + 1e-9
    assert partition_systems(costs, 4) == partition_systems(list(costs), 4)


def test_refusals():
    with pytest.raises(ValueError):
        partition_systems([1.0], 0)
    with pytest.raises(ValueError):
        partition_systems([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        partition_systems([math.inf], 2)


def test_cost_grows_with_atoms_and_grid():
    base = system_cost(3000, 30.0, 0.9, (32, 32, 32))
    assert system_cost(6000, 60.0, 0.9, (32, 32, 32)) > base
    assert system_cost(3000, 30.0, 0.9, (48, 48, 48)) > base
    assert system_cost(0, 30.0, 0.9, (32, 32, 32)) == 0.0


def test_benchmark_batch_splits_evenly():
    """The 64 uneven systems of the batched benchmark over 2, 4 and 8 GPUs: the slowest rank's
    estimated cost within 5% of the mean."""
    import numpy as np

    from rainmd_b200 import synthetic
    from rainmd_b200.topology import build_system
    import bench

    costs = []
    for topo, _ in synthetic.batch(64, seed=0):
        system = build_system(topo, cutoff=0.9)
        box = np.asarray(system["boxVectors"], dtype=np.float64)
        grid = [bench.smooth_at_least(math.ceil(box[4 * d] / 0.1)) for d in range(3)]
        costs.append(system_cost(topo["atomCount"], float(box[0] * box[4] * box[8]), 0.9, grid))
    for ranks in (2, 4, 8):
        loads = [sum(costs[k] for k in p) for p in partition_systems(costs, ranks)]
        assert max(loads) <= 1.05 * sum(loads) / ranks


def _partition_rank(rank, world, port, costs, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition_systems(costs, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = torch.tensor([float(sum(costs[k] for k in mine))], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out.put((rank, gathered, float(t.item())))
    dist.destroy_process_group()


def test_ranks_agree_on_the_partition_over_two_gloo_ranks():
    import multiprocessing as mp
    import random

    costs = [float(k % 5 + 1) * 10.0 for k in range(17)]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_partition_rank, args=(r, 2, port, costs, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    expect = partition_systems(costs, 2)
    slowest = max(sum(costs[k] for k in p) for p in expect)
    for _, gathered, worst in results:
        assert gathered == expect
        assert worst == slowest
    assert sorted(k for p in expect for k in p) == list(range(len(costs)))
