"""The multi-GPU plumbing of bench.py on CPU: world size 2 over gloo.

bench.py runs one independent build per rank (replicas of the workload with
different seeds: weak scaling, no collective on the data path) and reports
per-step times as the maximum over ranks.  These checks run the same helpers
with two gloo ranks.
"""

import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        mx = bench.max_over_ranks(torch, float(10 + rank), torch.device("cpu"), world)

        class A:
            n, d, comps = 2000, 50, 5

        x = bench.workload(A, rank)
        out[rank] = (mx, float(x[:10].sum()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_replica_workloads():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0  # every rank reports the slowest
    assert res[0][1] != res[1][1]          # each rank builds its own replica


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(torch, 3.5, torch.device("cpu"), 1) == 3.5
