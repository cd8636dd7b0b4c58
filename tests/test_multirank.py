"""Host logic of multi-GPU runs on CPU ranks (gloo, world size 2): the batched
population is partitioned by cost (N^2 x steps) across the ranks, each
instance on exactly one rank, with no data exchange; the timing is the max
over ranks (the only collective)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from higflow_b200 import workloads
    draws = workloads.batched_giesekus()
    mine = bench.shard(draws, rank, world)
    t = bench._max_over_ranks(0.5 + rank, world, 0)
    out[rank] = ([(d.n, d.De, d.alpha) for d in mine], t)
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_partition_one_population_and_share_the_max_time():
    from higflow_b200 import workloads
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][1] == out[1][1] == 1.5            # max over ranks
    draws = workloads.batched_giesekus()
    every = sorted(out[0][0] + out[1][0])
    assert every == sorted((d.n, d.De, d.alpha) for d in draws)   # each instance exactly once
    cost = [sum(n * n for n, _, _ in out[r][0]) for r in range(world)]
    total = sum(d.cells * d.steps for d in draws) / draws[0].steps
    assert max(cost) <= total / world * 1.02        # balanced within 2 %


@pytest.mark.parametrize("parts", [1, 2, 3, 4, 8])
def test_partition_covers_and_balances(parts):
    import numpy as np
    from higflow_b200 import workloads
    rng = np.random.default_rng(5)
    costs = [float(x) for x in rng.integers(1, 1000, size=97)]
    groups = workloads.partition(costs, parts)
    flat = sorted(i for g in groups for i in g)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in g) for g in groups]
    # greedy longest-first: the largest load is at most the mean plus the
    # largest single cost, and within Graham's 4/3 of the optimum's lower bound
    assert max(loads) <= sum(costs) / parts + max(costs)
    assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / parts, max(costs)) + 1e-9
