"""The CPU oracle held to the reference's own tests (CPU only).

Restates crates/polariseq-core/src/nndescent.rs:1005-1200, simd.rs:83-137,
neighbors.rs:243-333 and python/polariseq/tests/test_neighbors.py:32-66
against the C++ restatement in oracle/, and checks it against the committed
golden fixtures in tests/golden/.
"""

import os

import numpy as np
import pytest

import oracle
from polariseq_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def recall_vs(graph, data, k, queries):
    """recall (nndescent.rs:1038-1056): exact by f32 sq_dist, sort by distance."""
    hits = 0
    for i in range(queries):
        d2 = np.array([oracle.sq_dist(data[i], data[j]) for j in range(len(data))], np.float32)
        d2[i] = np.inf
        exact = set(np.argsort(d2, kind="stable")[:k].tolist())
        s, e = graph["indptr"][i], graph["indptr"][i + 1]
        hits += len(exact & set(graph["indices"][s:e].tolist()))
    return hits / (queries * k)


# ── simd.rs:83-137 ──────────────────────────────────────────────────────────
def _vecs(n):
    a = np.array([((i * 7) % 13) * 0.25 - 1.0 for i in range(n)], np.float32)
    b = np.array([((i * 5) % 11) * 0.5 - 2.0 for i in range(n)], np.float32)
    return a, b


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 15, 16, 17, 50, 64, 101])
def test_dot_and_sq_dist_match_naive_for_all_tail_lengths(n):
    a, b = _vecs(n)
    d = float(np.dot(a.astype(np.float64), b.astype(np.float64)))
    assert abs(float(oracle.dot(a, b)) - d) < 1e-3 * max(abs(d), 1.0)
    sq = float(((a.astype(np.float64) - b.astype(np.float64)) ** 2).sum())
    assert abs(float(oracle.sq_dist(a, b)) - sq) < 1e-3 * max(sq, 1.0)


def test_results_are_bit_identical_across_calls():
    a, b = _vecs(1000)
    assert oracle.dot(a, b).tobytes() == oracle.dot(a, b).tobytes()
    assert oracle.sq_dist(a, b).tobytes() == oracle.sq_dist(a, b).tobytes()


def test_sq_dist_lane_order_known_answer():
    """The 8-lane order is observable: it differs from a sequential f32 sum."""
    rng = np.random.default_rng(0)
    found = False
    for _ in range(200):
        a = rng.normal(size=50).astype(np.float32) * 100
        b = rng.normal(size=50).astype(np.float32)
        t = (a - b).astype(np.float32)
        sq = (t * t).astype(np.float32)
        acc = np.zeros(8, np.float32)
        for c in range(6):
            acc = (acc + sq[8 * c:8 * c + 8]).astype(np.float32)
        red = np.float32(np.float32(np.float32(acc[0] + acc[4]) + np.float32(acc[1] + acc[5]))
                         + np.float32(np.float32(acc[2] + acc[6]) + np.float32(acc[3] + acc[7])))
        tail = np.float32(np.float32(0) + sq[48])
        tail = np.float32(tail + sq[49])
        want = np.float32(red + tail)
        assert oracle.sq_dist(a, b) == want
        seq = np.float32(0)
        for v in sq:
            seq = np.float32(seq + v)
        found |= seq != want
    assert found


# ── the RNG (nndescent.rs:80-112) ───────────────────────────────────────────
def test_splitmix_known_values():
    # splitmix64 finaliser of x + golden gamma; the first outputs of the
    # seed-0 SplitMix64 stream are published test vectors of the generator.
    assert oracle.splitmix(0) == 0xE220A8397B1DCDAF
    assert oracle.splitmix(0x9E3779B97F4A7C15) == 0x6E789E6AA1B965F4
    u = oracle.hash_unit(7, 3, 11)
    assert 0.0 <= u < 1.0
    assert oracle.hash_index(1, 2, 3, 10) < 10


# ── the two-pointer partition and its closed form used on the GPU ──────────
def closed_form_partition(a, side):
    """Parallel restatement of partition_in_place (nndescent.rs:389-405), the
    formula the CUDA forest uses (polariseq_b200/csrc/forest.cu)."""
    n = len(a)
    L = side.astype(bool)
    Lpre = np.concatenate([[0], np.cumsum(L)])
    nL = int(Lpre[n])
    A, B = {}, {}
    for p in range(n):
        if p < nL and not L[p]:
            A[p - Lpre[p] + 1] = p
        if p >= nL and L[p]:
            B[nL - Lpre[p]] = p
    c = nL - int(Lpre[nL])
    out = np.empty_like(a)
    for p in range(n):
        if L[p]:
            dst = p if p < nL else A[nL - Lpre[p]]
        elif p < nL:
            j = p - Lpre[p] + 1
            dst = (n if j == 1 else B[j - 1]) - 1
        elif p > nL:
            dst = p - 1
        else:
            dst = (n if c == 0 else B[c]) - 1
        out[dst] = a[p]
    return out, nL


def test_partition_closed_form_matches_two_pointer():
    rng = np.random.default_rng(1)
    for _ in range(3000):
        n = int(rng.integers(1, 48))
        a = rng.permutation(1000)[:n].astype(np.uint32)
        s = (rng.random(n) < rng.random()).astype(np.uint8)
        r1, s1 = oracle.partition(a, s)
        r2, s2 = closed_form_partition(a, s)
        assert s1 == s2
        np.testing.assert_array_equal(r1, r2)


# ── nndescent.rs tests ──────────────────────────────────────────────────────
def test_writing_into_caller_arrays_gives_the_same_graph():
    n, d, k = 1500, 6, 9
    data = synth.blobs_rust_tests(n, d, 4, 3)
    g = oracle.nndescent(data, k, seed=5)
    g2 = oracle.nndescent(data, k, seed=5)
    np.testing.assert_array_equal(g["indptr"], g2["indptr"])
    np.testing.assert_array_equal(g["indices"], g2["indices"])
    assert g["data"].tobytes() == g2["data"].tobytes()


def test_graph_structure_is_valid():
    n, d, k = 2000, 8, 10
    data = synth.blobs_rust_tests(n, d, 5, 1)
    g = oracle.nndescent(data, k, seed=1)
    ip, ix, dx = g["indptr"], g["indices"], g["data"]
    for i in range(n):
        s, e = ip[i], ip[i + 1]
        assert e - s == k
        row = ix[s:e]
        assert i not in row
        assert len(set(row.tolist())) == k
        assert np.all(np.diff(dx[s:e]) >= 0)


def test_recall_is_high_on_structured_data():
    n, d, k = 6000, 20, 15
    rng = np.random.default_rng(9)
    c = (np.arange(n) % 12).astype(np.float32)[:, None]
    j3 = (np.arange(d) % 3).astype(np.float32)[None, :]
    data = (c * 3.0 * j3 + rng.random((n, d), dtype=np.float32) * 4.0).astype(np.float32)
    g = oracle.nndescent(data, k, seed=4)
    assert recall_vs(g, data, k, 300) >= 0.95


def test_the_gather_bound_does_not_change_the_graph():
    n, d, k = 20_000, 12, 10
    data = synth.blobs_rust_tests(n, d, 15, 11)
    copied = oracle.nndescent(data, k, seed=9, gather_max=2**62)
    for gm in [1, 64, 1000]:
        g = oracle.nndescent(data, k, seed=9, gather_max=gm)
        np.testing.assert_array_equal(g["indptr"], copied["indptr"])
        np.testing.assert_array_equal(g["indices"], copied["indices"])
        assert g["data"].tobytes() == copied["data"].tobytes()


def test_is_deterministic_across_thread_counts():
    n, d, k = 3000, 10, 12
    data = synth.blobs_rust_tests(n, d, 7, 5)
    t0 = oracle.max_threads()
    try:
        oracle.set_threads(1)
        g1 = oracle.nndescent(data, k, seed=42)
        oracle.set_threads(max(2, t0))
        g2 = oracle.nndescent(data, k, seed=42)
    finally:
        oracle.set_threads(t0)
    np.testing.assert_array_equal(g1["indices"], g2["indices"])
    assert g1["data"].tobytes() == g2["data"].tobytes()


def test_tiny_inputs_work():
    data = synth.blobs_rust_tests(5, 3, 2, 0)
    g = oracle.nndescent(data, 10)
    assert np.all(np.diff(g["indptr"]) == 4)


def test_single_point_keeps_itself():
    """n = 1: k resolves to 1 and the random fill can only draw the point itself."""
    g = oracle.nndescent(np.ones((1, 4), np.float32), 5)
    assert g["indptr"].tolist() == [0, 1]
    assert g["indices"].tolist() == [0] and g["data"].tolist() == [0.0]


def test_panics_become_errors():
    with pytest.raises(ValueError):
        oracle.nndescent(np.zeros((0, 3), np.float32), 5)
    with pytest.raises(ValueError):
        oracle.nndescent(np.zeros((10, 3), np.float32), 0)


def test_recall_vs_exact_python_mixture():
    """test_neighbors.py:32-39 at reduced size (the oracle is the slow path)."""
    emb = synth.mixture25(5000)
    ex = oracle.neighbors_exact(emb, 16, "euclidean")
    ap = oracle.nndescent(emb, 15, seed=42)
    a = ap["indices"].reshape(-1, 15)
    e = ex["indices"].reshape(-1, 15)
    r = np.array([len(set(a[i]) & set(e[i])) for i in range(len(a))]) / 15
    assert r.mean() >= 0.97 and np.percentile(r, 5) >= 0.85


def test_resolved_defaults_match_the_reference_formulas():
    p = oracle.nndescent_probe(synth.mixture_dirichlet(20_000), 15, stop_after=-1)
    k, m, iters, trees, leaf, stop = p["resolved"]
    assert (k, m, iters, trees, leaf, stop) == (15, 30, 14, 22, 15, 300)


# ── neighbors.rs tests (exact path restatement) ────────────────────────────
def test_exact_finds_nearest_in_simple_embedding():
    emb = np.array([[0, 0], [1, 0], [10, 10], [0, 1]], np.float32)
    g = oracle.neighbors_exact(emb, 3)
    s, e = g["indptr"][0], g["indptr"][1]
    assert set(g["indices"][s:e].tolist()) == {1, 3}
    assert np.allclose(g["data"][s:e], 1.0, atol=1e-5)


def test_exact_counts_and_self_exclusion():
    emb = (np.arange(30, dtype=np.float32) * 0.1).reshape(10, 3)
    g = oracle.neighbors_exact(emb, 5)
    assert np.all(np.diff(g["indptr"]) == 4)
    emb = np.array([[0, 0], [1, 0], [2, 0]], np.float32)
    g = oracle.neighbors_exact(emb, 2)
    for i in range(3):
        assert i not in g["indices"][g["indptr"][i]:g["indptr"][i + 1]]


def test_exact_cosine_metric_works():
    emb = np.array([[1, 0], [2, 0], [-1, 0]], np.float32)
    g = oracle.neighbors_exact(emb, 2, "cosine")
    assert g["indices"][g["indptr"][0]] == 1 and abs(g["data"][g["indptr"][0]]) < 1e-5


def test_fp64_oracle_tie_break_is_distance_then_index():
    """doublets.rs:1702-1710: equal distances resolve by the smaller index."""
    pts = np.array([[0.0], [1.0], [2.0], [3.0], [10.0]], np.float32)
    idx, dist = oracle.exact_knn_f64(pts, np.array([1], np.uint32), 3)
    assert idx[0].tolist() == [0, 2, 3]
    idx, dist = oracle.exact_knn_f64(pts, np.array([2], np.uint32), 2)
    assert idx[0].tolist() == [1, 3]


# ── golden fixtures (tests/golden/make_golden.py) ──────────────────────────
def test_oracle_matches_committed_golden_graphs():
    path = os.path.join(GOLDEN, "nndescent_golden.npz")
    z = np.load(path)
    for name in sorted({k.split("__")[0] for k in z.files}):
        cfg = z[name + "__cfg"]
        n, d, k, seed, gen_seed, ncl = (int(v) for v in cfg)
        data = synth.blobs_rust_tests(n, d, ncl, gen_seed)
        np.testing.assert_array_equal(data, z[name + "__data"])
        g = oracle.nndescent(data, k, seed=seed)
        np.testing.assert_array_equal(g["indptr"], z[name + "__indptr"])
        np.testing.assert_array_equal(g["indices"], z[name + "__indices"])
        assert g["data"].tobytes() == z[name + "__dists"].tobytes()
