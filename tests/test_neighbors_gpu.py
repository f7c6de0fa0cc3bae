"""Bit-exact parity of the CUDA exact kNN (neighbors_dense) with the oracle.

The oracle restates neighbors::neighbors (crates/polariseq-core/src/
neighbors.rs:101-241) with the reference's FP32 summation order, bounded heap
and stable sort; the CUDA path must match it byte for byte (indices, indptr,
distance bits), including ties (duplicate rows), k >= n, ragged tile edges and
both metrics.  The reference's own unit tests (neighbors.rs:243-333) are
restated on the GPU path.
"""

import numpy as np
import pytest

import oracle
import polariseq_b200 as pq
from polariseq_b200 import synth

pytestmark = pytest.mark.gpu


def assert_graph_equal(g, h, what=""):
    np.testing.assert_array_equal(g["indptr"], h["indptr"], err_msg=f"{what} indptr")
    np.testing.assert_array_equal(g["indices"], h["indices"], err_msg=f"{what} indices")
    assert g["data"].tobytes() == h["data"].tobytes(), f"{what}: distance bits differ"
    assert g["n_obs"] == h["n_obs"]


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
@pytest.mark.parametrize("n,d,k", [(3000, 50, 15), (2501, 30, 16), (777, 13, 31), (300, 50, 64)])
def test_matches_oracle(metric, n, d, k):
    emb = synth.mixture_dirichlet(n, d, 12, seed=n + d)
    g = pq.neighbors_dense(emb, k, metric)
    ref = oracle.neighbors_exact(emb, k, metric)
    assert_graph_equal(g, ref, f"{metric} n={n} d={d} k={k}")


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_duplicate_rows_tie_order(metric):
    """Duplicates tie at distance 0 with self: the heap's array order decides
    which one the reference drops, and the GPU heap must agree."""
    rng = np.random.default_rng(5)
    base = rng.normal(size=(60, 8)).astype(np.float32)
    emb = np.concatenate([base, base[:25], base[10:40], base[:5]])
    emb = emb[rng.permutation(len(emb))]
    for k in (2, 5, 17):
        assert_graph_equal(pq.neighbors_dense(emb, k, metric),
                           oracle.neighbors_exact(emb, k, metric), f"{metric} k={k}")


def test_k_at_least_n_and_k_one():
    emb = synth.mixture_dirichlet(40, 5, 3, seed=1)
    assert_graph_equal(pq.neighbors_dense(emb, 100, "euclidean"),
                       oracle.neighbors_exact(emb, 100, "euclidean"), "k > n")
    g = pq.neighbors_dense(emb, 1, "euclidean")  # only self searched: no edges
    assert g["indices"].size == 0 and np.all(g["indptr"] == 0)
    one = pq.neighbors_dense(emb[:1], 15, "euclidean")
    assert one["indices"].size == 0 and list(one["indptr"]) == [0, 0]


def test_reference_finds_nearest_in_simple_embedding():  # neighbors.rs:247-263
    emb = np.array([[0, 0], [1, 0], [10, 10], [0, 1]], np.float32)
    g = pq.neighbors_dense(emb, 3, "euclidean")
    assert g["n_obs"] == 4
    s, e = g["indptr"][0], g["indptr"][1]
    assert set(g["indices"][s:e]) == {1, 3}
    assert np.all(np.abs(g["data"][s:e] - 1.0) < 1e-5)


def test_reference_neighbors_count():  # neighbors.rs:286-300
    emb = (np.arange(30, dtype=np.float32) * 0.1).reshape(10, 3)
    g = pq.neighbors_dense(emb, 5, "euclidean")
    assert np.all(np.diff(g["indptr"]) == 4)


def test_reference_self_excluded():  # neighbors.rs:302-315
    emb = np.array([[0, 0], [1, 0], [2, 0]], np.float32)
    g = pq.neighbors_dense(emb, 2, "euclidean")
    for i in range(3):
        assert i not in g["indices"][g["indptr"][i]:g["indptr"][i + 1]]


def test_reference_cosine_metric():  # neighbors.rs:317-333
    emb = np.array([[1, 0], [2, 0], [-1, 0]], np.float32)
    g = pq.neighbors_dense(emb, 2, "Cosine")
    s = g["indptr"][0]
    assert g["indices"][s] == 1 and abs(g["data"][s]) < 1e-5


def test_reference_errors():  # neighbors.rs:265-284, lib.rs:488-495
    with pytest.raises(RuntimeError, match="n_neighbors must be"):
        pq.neighbors_dense(np.zeros((2, 2), np.float32), 0, "euclidean")
    with pytest.raises(RuntimeError, match="zero rows"):
        pq.neighbors_dense(np.zeros((0, 5), np.float32), 15, "euclidean")
    with pytest.raises(RuntimeError, match="unknown metric"):
        pq.neighbors_dense(np.zeros((2, 2), np.float32), 1, "manhattan")


def test_device_entry_point_matches_host():
    import torch

    emb = synth.mixture_dirichlet(1500, 50, 8, seed=9)
    ctx = pq.default_context(0)
    xd = torch.from_numpy(emb).cuda()
    k = 15
    ip = torch.zeros(1501, dtype=torch.int32, device="cuda")
    ix = torch.zeros(1500 * (k - 1), dtype=torch.int32, device="cuda")
    dx = torch.zeros(1500 * (k - 1), dtype=torch.float32, device="cuda")
    nnz = ctx.neighbors_device(xd, k, pq.METRICS["cosine"], ip, ix, dx)
    torch.cuda.synchronize()
    ref = oracle.neighbors_exact(emb, k, "cosine")
    assert nnz == ref["indices"].size
    assert_graph_equal({"indptr": ip.cpu().numpy().view(np.uint32),
                        "indices": ix.cpu().numpy().view(np.uint32),
                        "data": dx.cpu().numpy(), "n_obs": 1500}, ref, "device")
