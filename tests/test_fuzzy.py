"""Fuzzy connectivities (umap.rs:283-620): the CPU oracle against the
reference's own tests (umap.rs:1937-2001, 2260-2290), and the CUDA path
against the oracle on the GPU.

Weights are floating point: the structure (indptr, indices) must be identical
and the weights equal to within 1e-6 relative (CUDA's and the host library's
f64 exp may differ in the last bit, the only source of difference).
"""

import numpy as np
import pytest

import oracle
from polariseq_b200 import synth


def knn_graph(n, k, seed):
    x = synth.mixture_dirichlet(n, 8, 4, seed=seed)
    return oracle.nndescent(x, k, seed=seed), x


def hashmap_fuzzy(g, n):
    """umap.rs:1891-1921 restated: fold each edge into its unordered pair in
    edge order, in f32."""
    ip, ix, dx = g["indptr"], g["indices"], g["data"]
    w = [oracle.smooth_knn_dist(dx[ip[i]:ip[i + 1]]) for i in range(n)]
    m = {}
    for i in range(n):
        for t, j in enumerate(ix[ip[i]:ip[i + 1]]):
            key = (min(i, int(j)), max(i, int(j)))
            old = m.get(key, np.float32(0))
            wij = w[i][t]
            m[key] = np.float32(np.float32(old + wij) - np.float32(old * wij))
    return sorted((a, b, v) for (a, b), v in m.items() if v > np.float32(1e-5))


def test_smooth_knn_dist_matches_umap_learn():  # umap.rs:2260-2276
    w = oracle.smooth_knn_dist([0.5, 1.0, 2.0, 4.0])
    want = [1.0, 0.754181, 0.42896995, 0.13878077]
    assert np.all(np.abs(w - want) < 1e-5)
    assert abs(w.sum() - np.log2(5)) < 1e-4
    assert np.all((w >= 0) & (w <= 1)) and w[0] >= w[1] >= w[2]


def test_oracle_matches_hashmap_fold():  # umap.rs:1937-1951
    g, _ = knn_graph(80, 5, 7)
    f = oracle.fuzzy_connectivities(g["indptr"], g["indices"], g["data"], 80)
    got = [(i, int(j), v) for i in range(80)
           for j, v in zip(f["indices"][f["indptr"][i]:f["indptr"][i + 1]],
                           f["data"][f["indptr"][i]:f["indptr"][i + 1]]) if j > i]
    want = hashmap_fuzzy(g, 80)
    assert len(got) == len(want)
    for (a, b, v), (c, d, u) in zip(got, want):
        assert (a, b) == (c, d) and np.float32(v).tobytes() == np.float32(u).tobytes()


def test_oracle_symmetric_sorted_canonical():  # umap.rs:1953-2001
    g, _ = knn_graph(120, 8, 3)
    f = oracle.fuzzy_connectivities(g["indptr"], g["indices"], g["data"], 120)
    ip, ix, w = f["indptr"], f["indices"], f["data"]
    pos = {}
    for i in range(120):
        row = ix[ip[i]:ip[i + 1]]
        assert np.all(row != i) and np.all(np.diff(row.astype(np.int64)) > 0)
        for j, v in zip(row, w[ip[i]:ip[i + 1]]):
            pos[(i, int(j))] = v
    for (i, j), v in pos.items():
        assert pos[(j, i)].tobytes() == v.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("n,k", [(20_000, 15), (3000, 30)])
def test_cuda_matches_oracle(n, k):
    import polariseq_b200 as pq

    x = synth.mixture_dirichlet(n, 50, 12, seed=n + k)
    g = pq.nndescent_dense(x, k)
    ref = oracle.fuzzy_connectivities(g["indptr"], g["indices"], g["data"], n)
    got = pq.fuzzy_connectivities(g["indptr"], g["indices"], g["data"], n)
    np.testing.assert_array_equal(got["indptr"], ref["indptr"])
    np.testing.assert_array_equal(got["indices"], ref["indices"])
    np.testing.assert_allclose(got["data"], ref["data"], rtol=1e-6, atol=0)
    assert np.mean(got["data"] == ref["data"]) > 0.999  # last-bit differences only


@pytest.mark.gpu
def test_device_graph_feeds_connectivities():
    """The graph of the device build goes to the connectivities on the device."""
    import ctypes as C

    import torch

    import polariseq_b200 as pq
    from polariseq_b200 import _lib

    n, k = 30_000, 15
    x = synth.mixture_lognormal(n, 50, 10, seed=5)
    ctx = pq.default_context(0)
    xd = torch.from_numpy(x).cuda()
    ip = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    ix = torch.zeros(n * k, dtype=torch.int32, device="cuda")
    dx = torch.zeros(n * k, dtype=torch.float32, device="cuda")
    nnz = ctx.nndescent_device(xd, pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES["bf16"]),
                               ip, ix, dx)
    cap = 2 * nnz
    oip = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    oix = torch.zeros(cap, dtype=torch.int32, device="cuda")
    ow = torch.zeros(cap, dtype=torch.float32, device="cuda")
    m = C.c_uint64(0)
    rc = _lib.load().pq_fuzzy_connectivities_device(
        ctx._h, n, ip.data_ptr(), ix.data_ptr(), dx.data_ptr(), nnz, oip.data_ptr(),
        oix.data_ptr(), ow.data_ptr(), cap, C.byref(m), None)
    assert rc == 0
    torch.cuda.synchronize()
    h = {k_: v.cpu().numpy() for k_, v in (("ip", ip), ("ix", ix), ("dx", dx))}
    ref = oracle.fuzzy_connectivities(h["ip"].view(np.uint32), h["ix"].view(np.uint32)[:nnz],
                                      h["dx"][:nnz], n)
    mm = int(m.value)
    np.testing.assert_array_equal(oip.cpu().numpy().view(np.uint32), ref["indptr"])
    np.testing.assert_array_equal(oix.cpu().numpy().view(np.uint32)[:mm], ref["indices"])
    np.testing.assert_allclose(ow.cpu().numpy()[:mm], ref["data"], rtol=1e-6, atol=0)
