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


# ── the batched doublet-scoring search split by sample over ranks ────────────

def test_shard_samples_balances_whole_samples():
    import polariseq_b200 as pq

    sizes = [9000, 100, 5000, 5000, 300, 8000, 700]
    parts = pq.shard_samples(sizes, 3)
    assert sorted(s for p in parts for s in p) == list(range(len(sizes)))
    loads = [sum(sizes[s] ** 2 for s in p) for p in parts]
    # largest-first greedy: no rank above the best split by more than the
    # largest sample
    assert max(loads) - min(loads) <= max(sizes) ** 2
    assert pq.shard_samples(sizes, 3) == parts  # deterministic
    assert pq.shard_samples(sizes, 1) == [list(range(len(sizes)))]


def _fake_knn(xs, ks):
    """A stand-in for the device search (no GPU here): each sample's k
    smallest squared-distance indices by brute force in NumPy."""
    out = []
    for x, k in zip(xs, ks):
        d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
        np.fill_diagonal(d2, np.inf)
        idx = np.argsort(d2, axis=1, kind="stable")[:, :k]
        out.append((idx.astype(np.uint32), np.sqrt(np.take_along_axis(d2, idx, 1))))
    return out


def _sharded_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import polariseq_b200 as pq

        rng = np.random.default_rng(3)
        samples = [rng.normal(size=(n, 4)).astype(np.float32) for n in (40, 12, 33, 25, 8)]
        ks = [3, 2, 5, 4, 1]
        res = pq.knn_batched_sharded(samples, ks, rank=rank, world=world, _compute=_fake_knn)
        own = pq.knn_batched_sharded(samples, ks, rank=rank, world=world, gather=False,
                                     _compute=_fake_knn)
        out[rank] = ([r[0].tolist() for r in res], sorted(own))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_batched_search_by_sample():
    """Each rank searches only its share; after the one exchange at the end
    every rank holds every sample's result, equal to a single-rank search."""
    import polariseq_b200 as pq

    world = 2
    port = 29600 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_sharded_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    rng = np.random.default_rng(3)
    samples = [rng.normal(size=(n, 4)).astype(np.float32) for n in (40, 12, 33, 25, 8)]
    want = [r[0].tolist() for r in _fake_knn(samples, [3, 2, 5, 4, 1])]
    assert res[0][0] == res[1][0] == want
    parts = pq.shard_samples([len(s) for s in samples], world)
    assert res[0][1] == parts[0] and res[1][1] == parts[1]
