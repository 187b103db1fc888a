"""The replica path of bench.py --gpus N: the whole-job time is the max over ranks
(CPU, world_size 2 over gloo)."""

from __future__ import annotations

import os

import pytest
import torch.multiprocessing as mp


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    assert bench.dist_env() == (rank, world, rank)
    got = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
    out.put((rank, got))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == [2.0, 10.0]


def test_single_process_is_a_no_op():
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
