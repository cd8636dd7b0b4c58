"""Host logic of multi-GPU runs on CPU ranks (gloo, world size 2): every rank
draws its own batch (independent instances, no data exchange) and the timing is
the max over ranks (the only collective)."""
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
    draws = workloads.batched_giesekus(count=8, seed=bench.rank_seed(rank))
    t = bench._max_over_ranks(0.5 + rank, world, 0)
    out[rank] = (tuple(d.n for d in draws), t)
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_shard_their_batches_and_share_the_max_time():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][1] == out[1][1] == 1.5            # max over ranks
    assert out[0][0] != out[1][0]                   # different instance populations
