"""The tensor-core shortlist form (mode='bf16') on the GPU: graph structure,
determinism and recall@k against the FP64 exact oracle.

Its graph is not the reference's (a different search), so it is checked by
recall@k >= 0.99 against FP64 brute force with (distance, index) order and by
its distances: every returned distance is the exact FP32 distance of its pair
in the reference's summation order."""

import numpy as np
import pytest

import oracle
import polariseq_b200 as pq
from polariseq_b200 import synth

pytestmark = pytest.mark.gpu


def recall(g, data, k, queries):
    ex, _ = oracle.exact_knn_f64(data, queries, k)
    a = g["indices"].reshape(-1, k)[queries]
    return np.mean([len(set(a[i]) & set(ex[i])) / k for i in range(len(queries))])


def check_structure(g, n, k):
    ip, ix, dx = g["indptr"], g["indices"], g["data"]
    assert np.all(np.diff(ip) == k)
    rows = ix.reshape(n, k)
    assert not (rows == np.arange(n)[:, None]).any(), "self-loop"
    assert all(len(set(r)) == k for r in rows[:: max(1, n // 2000)]), "duplicate neighbour"
    assert (np.diff(dx.reshape(n, k), axis=1) >= 0).all(), "not sorted"


@pytest.mark.parametrize("wide", ["1", "0"])
@pytest.mark.parametrize("n,comps", [(20_000, 20), (120_000, 40)])
def test_bf16_form_recall_and_structure(n, comps, wide, monkeypatch):
    """Both tile kernels of the 16-entry shortlists: the wide one (jobs of 256
    query entries, 128-candidate tiles, 16 epilogue warps; the default) and
    the standard one (128 entries, 256-candidate tiles)."""
    monkeypatch.setenv("POLARISEQ_TILES_WIDE", wide)
    x = synth.mixture_lognormal(n, 50, comps, seed=5)
    g = pq.nndescent_dense(x, 15, mode="bf16")
    check_structure(g, n, 15)
    q = np.random.default_rng(1).choice(n, 2000, replace=False).astype(np.uint32)
    assert recall(g, x, 15, q) >= 0.99


def test_bf16_form_distances_are_exact_fp32():
    x = synth.mixture_dirichlet(20_000, 50, 20, 0)
    g = pq.nndescent_dense(x, 15, mode="bf16")
    ix = g["indices"].reshape(-1, 15)
    dx = g["data"].reshape(-1, 15)
    for i in range(0, 20_000, 997):
        for t in range(15):
            want = np.sqrt(oracle.sq_dist(x[i], x[ix[i, t]]))
            assert dx[i, t] == np.float32(want)


def test_bf16_form_is_deterministic():
    x = synth.mixture_lognormal(50_000, 50, 30, seed=2)
    a = pq.nndescent_dense(x, 15, mode="bf16")
    b = pq.nndescent_dense(x, 15, mode="bf16")
    np.testing.assert_array_equal(a["indices"], b["indices"])
    assert a["data"].tobytes() == b["data"].tobytes()


def test_bf16_form_host_chunks_above_2_20_cells():
    """Above 2^20 cells the host-buffer entry point re-ranks in cell-index
    chunks and copies each chunk to the host while the next is re-ranked:
    every chunk's rows must hold their own cell's neighbours (sorted, no self,
    each distance the exact FP32 distance of its pair), at full recall."""
    n = (1 << 20) + 4321
    x = synth.mixture_lognormal(n, 50, 30, seed=9)
    g = pq.nndescent_dense(x, 15, mode="bf16")
    check_structure(g, n, 15)
    ix = g["indices"].reshape(-1, 15)
    dx = g["data"].reshape(-1, 15)
    for i in np.linspace(0, n - 1, 64).astype(np.int64):  # rows of every chunk
        for t in range(15):
            want = np.sqrt(oracle.sq_dist(x[i], x[ix[i, t]]))
            assert dx[i, t] == np.float32(want)
    q = np.random.default_rng(3).choice(n, 300, replace=False).astype(np.uint32)
    assert recall(g, x, 15, q) >= 0.99


def test_bf16_form_host_and_device_entry_points_agree():
    """The build is deterministic (fixed-order reductions throughout): the
    host-buffer entry point, chunked above 2^20 cells, and the device entry
    point give the same graph byte for byte."""
    import torch

    n = (1 << 20) + 4321
    x = synth.mixture_lognormal(n, 50, 30, seed=9)
    h = pq.nndescent_dense(x, 15, mode="bf16")
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    ip = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ix = torch.empty(n * 15, dtype=torch.int32, device=dev)
    dx = torch.empty(n * 15, dtype=torch.float32, device=dev)
    opts = pq._opts(15, 0, 0, 0, 0, 0.001, mode=pq.MODES["bf16"])
    nnz = pq.default_context(0).nndescent_device(xd, opts, ip, ix, dx)
    torch.cuda.synchronize(dev)
    assert nnz == len(h["indices"]) == n * 15
    np.testing.assert_array_equal(ip.cpu().numpy().view(np.uint32), h["indptr"])
    np.testing.assert_array_equal(ix.cpu().numpy().view(np.uint32), h["indices"])
    assert dx.cpu().numpy().tobytes() == h["data"].tobytes()


def test_bf16_form_k30_and_30_pcs():
    x = synth.mixture_lognormal(40_000, 30, 10, seed=3)
    g = pq.nndescent_dense(x, 30, mode="bf16")
    check_structure(g, 40_000, 30)
    q = np.random.default_rng(2).choice(40_000, 1000, replace=False).astype(np.uint32)
    assert recall(g, x, 30, q) >= 0.99


def test_bf16_form_small_inputs_are_exact():
    # one bucket: the shortlist covers every cell, so the graph is the exact kNN
    x = synth.blobs_rust_tests(3000, 8, 4, 1)
    g = pq.nndescent_dense(x, 10, mode="bf16")
    q = np.arange(0, 3000, 7, dtype=np.uint32)
    assert recall(g, x, 10, q) >= 0.999


def test_fp8_form_recall_and_exact_distances():
    """E4M3 tiles (every query and candidate row with its own scale) with the
    exact FP32 re-rank and its default polish round (below 2^20 cells): recall against FP64 and
    exact returned distances."""
    n, k = 120_000, 15
    x = synth.mixture_lognormal(n, 50, 30, seed=11)
    g = pq.nndescent_dense(x, k, mode="fp8")
    check_structure(g, n, k)
    q = np.random.default_rng(3).choice(n, 2000, replace=False)
    assert recall(g, x, k, q) >= 0.99
    # returned distances are the exact FP32 distances of their pairs
    ip, ix = g["indptr"], g["indices"]
    for i in q[:200]:
        js = ix[ip[i]:ip[i + 1]]
        want = np.sqrt([oracle.sq_dist(x[i], x[j]) for j in js]).astype(np.float32)
        np.testing.assert_array_equal(g["data"][ip[i]:ip[i + 1]], want)


def test_fp8_form_k30_recall_and_structure():
    """E4M3 tiles at k = 30 (32-entry shortlists per column half)."""
    n, k = 60_000, 30
    x = synth.mixture_lognormal(n, 50, 20, seed=13)
    g = pq.nndescent_dense(x, k, mode="fp8")
    check_structure(g, n, k)
    q = np.random.default_rng(4).choice(n, 1000, replace=False).astype(np.uint32)
    assert recall(g, x, k, q) >= 0.99


def test_bf16_form_every_row_ascending_at_4m():
    """At 4M cells thousands of cells go through the FP64 boundary step (the
    k-th and (k+1)-th FP32 distances within the FP32 error bound).  FP64 only
    chooses which entries are kept: every row of the whole graph is still
    ascending, without self-loops or repeated neighbours."""
    import torch

    n, k = 4_000_000, 15
    x = synth.mixture_lognormal(n, 50, 60, seed=1000)
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    ip = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ix = torch.empty(n * k, dtype=torch.int32, device=dev)
    dx = torch.empty(n * k, dtype=torch.float32, device=dev)
    ctx = pq.default_context(0)
    opts = pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES["bf16"])
    nnz = ctx.nndescent_device(xd, opts, ip, ix, dx)
    torch.cuda.synchronize(dev)
    assert nnz == n * k
    assert ctx.stats()["shortlist"][6] > 0, "no cell went through the FP64 boundary step"
    rows = ix.view(n, k).long()
    d = dx.view(n, k)
    assert bool((d[:, 1:] >= d[:, :-1]).all()), "a row is not ascending"
    assert not bool((rows == torch.arange(n, device=dev)[:, None]).any()), "self-loop"
    srt = rows.sort(dim=1).values
    assert bool((srt[:, 1:] != srt[:, :-1]).all()), "repeated neighbour"


def test_a_bounded_wait_that_gives_up_returns_timeout_and_the_context_recovers():
    """The tile kernel's bounded waits: the test hook makes every CTA wait on
    an mbarrier that nothing arrives at, with a short poll limit, before it
    issues any copy or MMA.  The wait runs out, the kernel exits with nothing
    in flight, the build returns PQ_ETIMEOUT (DeviceTimeout), and the next
    build on the same context gives the normal graph."""
    import ctypes as C

    from polariseq_b200 import _lib

    n, k = 100_000, 15
    x = synth.mixture_lognormal(n, 50, 20, seed=4)
    ctx = pq.Context(0)
    opts = pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES["bf16"])

    def build():
        ip = np.zeros(n + 1, np.uint32)
        ix = np.zeros(n * k, np.uint32)
        dx = np.zeros(n * k, np.float32)
        nnz = ctx.nndescent_into(x, opts, ip, ix, dx)
        return nnz, ip, ix, dx

    want = build()
    assert _lib.load().pq_ctx_set_test_wait(ctx._h, C.c_uint32(1000)) == _lib.PQ_OK
    with pytest.raises(pq.DeviceTimeout):
        build()
    got = build()
    assert got[0] == want[0]
    for a, b in zip(got[1:], want[1:]):
        assert a.tobytes() == b.tobytes()
    ctx.close()


def test_host_entry_point_with_short_rows_above_2_20_cells():
    """Above 2^20 cells the host-buffer entry point copies rows to the host
    while it re-ranks, only when no row can be short.  Forcing short rows (one
    probe into 40,000 small buckets: some cells see fewer than k others), the
    pre-check sends the build down the count-and-scan path: the result equals
    the device entry point's, and the host arrays past nnz stay untouched."""
    import torch

    n, k = (1 << 20) + 1000, 15
    x = synth.mixture_lognormal(n, 50, 30, seed=17)
    opts = pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES["bf16"], probes=1, buckets=40_000)
    ctx = pq.default_context(0)
    ip = np.zeros(n + 1, np.uint32)
    ix = np.full(n * k, 0xDEADBEEF, np.uint32)
    dx = np.full(n * k, -7.0, np.float32)
    nnz = ctx.nndescent_into(x, opts, ip, ix, dx)
    assert nnz < n * k, "expected some short rows"
    assert (ix[nnz:] == 0xDEADBEEF).all() and (dx[nnz:] == -7.0).all()
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    dip = torch.empty(n + 1, dtype=torch.int32, device=dev)
    dix = torch.empty(n * k, dtype=torch.int32, device=dev)
    ddx = torch.empty(n * k, dtype=torch.float32, device=dev)
    nnz2 = ctx.nndescent_device(xd, opts, dip, dix, ddx)
    torch.cuda.synchronize(dev)
    assert nnz2 == nnz
    np.testing.assert_array_equal(dip.cpu().numpy().view(np.uint32), ip)
    np.testing.assert_array_equal(dix[:nnz].cpu().numpy().view(np.uint32), ix[:nnz])
    assert ddx[:nnz].cpu().numpy().tobytes() == dx[:nnz].tobytes()
