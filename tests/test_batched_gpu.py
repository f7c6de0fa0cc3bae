"""The batched exact kNN (one persistent launch over many samples) on the GPU.

Each sample's graph is compared with an FP64 brute force (oracle/) as exact
(distance, index) neighbour sets: the search is exact in FP32, so it may
differ from the FP64 order only where two distances agree to FP32 rounding;
distances must match the FP64 ones to FP32 accuracy.  The reference's own
search (doublets.rs:544-650) is pinned the same way, by exact-set tests
(doublets.rs:1666-1710).
"""

import numpy as np
import pytest

import oracle
import polariseq_b200 as pq
from polariseq_b200 import synth

pytestmark = pytest.mark.gpu


def make_samples(seed, count, lo, hi, d=30):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    return [synth.mixture_dirichlet(int(s), d, 10, seed=seed * 100 + i) for i, s in enumerate(sizes)]


def check_sample(x, idx, dist, k):
    n = x.shape[0]
    ref_i, ref_d = oracle.exact_knn_f64(x, np.arange(n, dtype=np.uint32), k)
    same = np.mean([len(set(idx[r]) & set(ref_i[r])) / k for r in range(n)])
    assert same >= 0.999, same
    # every returned distance is within FP32 accuracy of the FP64 distance of
    # its own pair, and the k-th distance matches the FP64 k-th
    true = np.sqrt(((x[:, None, :].astype(np.float64) - x[idx].astype(np.float64)) ** 2).sum(-1))
    assert np.max(np.abs(dist - true) / np.maximum(true, 1e-30)) < 1e-5
    assert np.max(np.abs(dist[:, -1] - np.sqrt(ref_d[:, -1])) / np.sqrt(ref_d[:, -1])) < 1e-5
    assert np.all(np.diff(dist, axis=1) >= 0)
    assert np.all(idx != np.arange(n)[:, None])


@pytest.mark.parametrize("mult", [1, 3])
def test_batched_exact_sets(mult):
    samples = make_samples(1, 10, 200, 3000)
    ks = [mult * max(1, round(0.5 * np.sqrt(len(s)))) for s in samples]
    out = pq.knn_batched(samples, ks, autotune=True)
    for x, k, (idx, dist) in zip(samples, ks, out):
        check_sample(x, idx, dist, k)


def test_graph_and_plain_launch_agree_and_repeat():
    samples = make_samples(2, 6, 100, 2000, d=50)
    ks = [7, 15, 3, 31, 64, 5]
    a = pq.knn_batched(samples, ks, graph=True)
    b = pq.knn_batched(samples, ks, graph=False)
    c = pq.knn_batched(samples, ks, graph=True)
    for (ia, da), (ib, db), (ic, dc) in zip(a, b, c):
        np.testing.assert_array_equal(ia, ib)
        np.testing.assert_array_equal(ia, ic)
        assert da.tobytes() == db.tobytes() == dc.tobytes()


def test_ties_and_tiny_samples():
    rng = np.random.default_rng(3)
    base = rng.normal(size=(40, 8)).astype(np.float32)
    dup = np.concatenate([base, base[:20]])          # exact duplicates: ties at 0
    tiny = rng.normal(size=(2, 8)).astype(np.float32)  # k = 1 of 2 points
    out = pq.knn_batched([dup, tiny], [5, 1])
    idx, dist = out[0]
    ref_i, ref_d = oracle.exact_knn_f64(dup, np.arange(len(dup), dtype=np.uint32), 5)
    np.testing.assert_array_equal(idx, ref_i)  # (distance, index) order, exact here
    assert list(out[1][0][:, 0]) == [1, 0]


def test_rejects_bad_k():
    x = np.zeros((5, 4), np.float32)
    with pytest.raises(ValueError):
        pq.knn_batched([x], [5])
    with pytest.raises(ValueError):
        pq.knn_batched([x], [0])
