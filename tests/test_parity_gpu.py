"""Bit-exact parity of the CUDA plain form with the oracle (GPU).

Every graph is compared byte for byte (indices, indptr and f32 distance bits)
with the C++ restatement of the reference (oracle/), on the same seeded
inputs; intermediate states (forest trees, heaps after the initialisation and
after each round, candidate lists) are compared too, so a mismatch names the
phase.  The reference's own tests (nndescent.rs:1059-1199,
test_neighbors.py:32-66) are restated on the GPU path.
"""

import os

import numpy as np
import pytest

import oracle
import polariseq_b200 as pq
from polariseq_b200 import _lib, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _opts(k=15, seed=0, **kw):
    return pq._opts(k, kw.get("max_iterations", 0), seed, kw.get("max_candidates", 0),
                    kw.get("n_trees", 0), kw.get("delta", 0.001), kw.get("leaf_size", 0))


def assert_graph_equal(g, h, what=""):
    np.testing.assert_array_equal(g["indptr"], h["indptr"], err_msg=f"{what} indptr")
    np.testing.assert_array_equal(g["indices"], h["indices"], err_msg=f"{what} indices")
    assert g["data"].tobytes() == h["data"].tobytes(), f"{what}: distance bits differ"


def assert_heaps_equal(gpu, ref, what):
    for key in ("heap_idx", "heap_dist", "heap_flag"):
        a, b = gpu[key], ref[key]
        if a.tobytes() != b.tobytes():
            bad = np.where((a.view(np.uint8).reshape(len(a), -1)
                            != b.view(np.uint8).reshape(len(b), -1)).any(1))[0]
            r = bad[0]
            raise AssertionError(f"{what}: {key} differs in {len(bad)} rows; first row {r}: "
                                 f"gpu {a[r].tolist()} oracle {b[r].tolist()}")


@pytest.fixture(scope="module")
def c1():
    return synth.mixture_dirichlet(20_000, 50, 20, 0)


@pytest.fixture(scope="module")
def ctx():
    return pq.default_context(0)


# ── forest ──────────────────────────────────────────────────────────────────
@pytest.mark.parametrize("tree", [0, 7, 21])
def test_forest_tree_matches_oracle(ctx, c1, tree):
    ids, leaves = ctx.debug_tree(c1, _opts(15, seed=0), tree)
    rids, rleaves = oracle.build_tree(c1, 15, oracle.splitmix(0 ^ (tree + 1)))
    np.testing.assert_array_equal(ids, rids)
    np.testing.assert_array_equal(leaves, rleaves)


def test_forest_with_six_parallel_levels_matches_oracle(ctx):
    x = synth.mixture_lognormal(600_000, 16, 30, seed=3)
    for tree in (0, 5):
        ids, leaves = ctx.debug_tree(x, _opts(15, seed=11), tree)
        rids, rleaves = oracle.build_tree(x, 15, oracle.splitmix(11 ^ (tree + 1)))
        np.testing.assert_array_equal(ids, rids)
        np.testing.assert_array_equal(leaves, rleaves)


def test_forest_with_ties_and_degenerate_splits(ctx):
    """Duplicated points: margins of exactly zero draw tie bits (parallel levels
    by splitmix(seed ^ id), sequential levels from the Rng) and hyperplanes
    that separate nothing fall back to random_split."""
    rng = np.random.default_rng(5)
    base = rng.normal(size=(40, 6)).astype(np.float32)
    x = base[rng.integers(0, 40, size=30_000)]
    for tree in (0, 3):
        ids, leaves = ctx.debug_tree(x, _opts(10, seed=2), tree)
        rids, rleaves = oracle.build_tree(x, 10, oracle.splitmix(2 ^ (tree + 1)))
        np.testing.assert_array_equal(ids, rids)
        np.testing.assert_array_equal(leaves, rleaves)


# ── heaps after each phase ─────────────────────────────────────────────────
@pytest.mark.parametrize("stop", [-1, 0, 1])
def test_heaps_match_after_phase(ctx, c1, stop):
    g = ctx.probe(c1, _opts(15, seed=0), stop)
    r = oracle.nndescent_probe(c1, 15, stop_after=stop, seed=0)
    assert_heaps_equal(g, r, f"after {'init' if stop < 0 else f'round {stop}'}")
    if stop >= 0:
        np.testing.assert_array_equal(g["cand_new"], r["cand_new"], err_msg="new candidates")
        np.testing.assert_array_equal(g["cand_old"], r["cand_old"], err_msg="old candidates")


# ── whole graphs ───────────────────────────────────────────────────────────
def test_c1_graph_is_bit_exact(c1):
    g = pq.nndescent_dense(c1, 15, 0, 0)
    r = oracle.nndescent(c1, 15, seed=0)
    assert_graph_equal(g, r, "20k x 50 k=15")
    st = pq.default_context(0).stats()
    rp = oracle.nndescent_probe(c1, 15, seed=0)
    assert st["rounds_run"] == rp["rounds_run"]
    assert st["changed"] == rp["round_changed"].tolist()


def test_join_in_small_source_row_chunks_is_bit_exact(c1, monkeypatch):
    """A round whose join records exceed the chunk cap is replayed in
    source-row chunks (index ranges, one after another).  Forcing a cap of
    200,000 records splits every round at 20k x 50 into tens of chunks; the
    graph and the per-round change counts stay those of the oracle."""
    monkeypatch.setenv("POLARISEQ_JOIN_CHUNK", "200000")
    g = pq.nndescent_dense(c1, 15, 0, 0)
    st = pq.default_context(0).stats()
    monkeypatch.delenv("POLARISEQ_JOIN_CHUNK")
    r = oracle.nndescent(c1, 15, seed=0)
    assert_graph_equal(g, r, "20k x 50 k=15, chunked join")
    assert max(st["emitted"]) > 2 * 200_000, "the cap did not force several chunks"
    rp = oracle.nndescent_probe(c1, 15, seed=0)
    assert st["changed"] == rp["round_changed"].tolist()


@pytest.mark.parametrize("n,d,k,seed,ncl", [
    (3000, 10, 12, 42, 7), (2000, 8, 10, 1, 5), (1500, 6, 9, 5, 4), (4000, 13, 30, 3, 6),
    (900, 50, 15, 9, 3), (64, 4, 15, 1, 2),
])
def test_graph_is_bit_exact_on_reference_test_inputs(n, d, k, seed, ncl):
    x = synth.blobs_rust_tests(n, d, ncl, seed)
    assert_graph_equal(pq.nndescent(x, k, seed=seed), oracle.nndescent(x, k, seed=seed),
                       f"{n}x{d} k={k}")


def test_graph_matches_committed_golden_fixtures():
    z = np.load(os.path.join(GOLDEN, "nndescent_golden.npz"))
    for name in sorted({k.split("__")[0] for k in z.files}):
        n, d, k, seed, _, _ = (int(v) for v in z[name + "__cfg"])
        g = pq.nndescent(z[name + "__data"], k, seed=seed)
        h = {"indptr": z[name + "__indptr"], "indices": z[name + "__indices"],
             "data": z[name + "__dists"]}
        assert_graph_equal(g, h, name)


def test_graph_matches_the_literal_restatement_on_reference_test_inputs():
    """The goldens written by the second, independent restatement
    (oracle/nndescent_literal.py) on the reference unit tests' own inputs
    (ChaCha8 make_clustered_data, nndescent.rs:1012-1022): the CUDA graph and
    its per-round change counts are the same, byte for byte."""
    z = np.load(os.path.join(GOLDEN, "reference_inputs_golden.npz"))
    ctx = pq.default_context(0)
    for name in sorted({f.split("__")[0] for f in z.files}):
        n, d, ncl, ds, k, seed = (int(v) for v in z[name + "__cfg"])
        g = pq.nndescent(z[name + "__data"], k, seed=seed)
        h = {"indptr": z[name + "__indptr"], "indices": z[name + "__indices"],
             "data": z[name + "__dists"]}
        assert_graph_equal(g, h, name)
        assert ctx.stats()["changed"] == z[name + "__changed"].tolist(), name


def test_graph_is_bit_exact_at_262k_cells():
    """A whole graph above the sizes of the reference's tests: 262,144 cells x
    50 PCs of the benchmark's generator (the forest's parallel levels, every
    round), byte for byte against the oracle."""
    x = synth.mixture_lognormal(262_144, 50, 40, seed=31)
    g = pq.nndescent_dense(x, 15, 0, 0)
    r = oracle.nndescent(x, 15, seed=0)
    assert_graph_equal(g, r, "262144 x 50 k=15")


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17])
def test_tiny_inputs_match(n):
    x = synth.blobs_rust_tests(n, 3, 2, 0)
    assert_graph_equal(pq.nndescent(x, 10), oracle.nndescent(x, 10), f"n={n}")


def test_options_are_honoured_bit_exactly(c1):
    x = c1[:8000]
    for kw in [dict(max_iterations=2), dict(max_candidates=7), dict(n_trees=3),
               dict(leaf_size=40), dict(delta=0.0)]:
        g = pq.nndescent(x, 15, seed=3, **kw)
        r = oracle.nndescent(x, 15, seed=3, **kw)
        assert_graph_equal(g, r, str(kw))


def test_duplicates_graph_matches():
    rng = np.random.default_rng(5)
    base = rng.normal(size=(300, 6)).astype(np.float32)
    x = base[rng.integers(0, 300, size=12_000)]
    assert_graph_equal(pq.nndescent(x, 10, seed=4), oracle.nndescent(x, 10, seed=4), "dups")


# ── the reference's tests on the GPU path ──────────────────────────────────
def test_writing_into_caller_arrays_gives_the_same_graph():
    n, d, k = 1500, 6, 9
    x = synth.blobs_rust_tests(n, d, 4, 3)
    g = pq.nndescent_dense(x, k, 0, 5)
    cap = n * pq.effective_k(n, k)
    ip = np.full(n + 1, 7, np.uint32)
    ix = np.full(cap + 5, 9, np.uint32)
    dx = np.full(cap + 5, 1.0, np.float32)
    r = pq.nndescent_dense(x, k, 0, 5, out=(ip, ix, dx))
    nnz = r["nnz"]
    assert nnz == len(g["indices"]) and r["n_obs"] == n
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix[:nnz], g["indices"])
    assert dx[:nnz].tobytes() == g["data"].tobytes()
    assert (ix[nnz:] == 9).all() and (dx[nnz:] == 1.0).all()  # untouched past nnz


def test_graph_structure_and_determinism_python_mixture():
    emb = synth.mixture25(5000, seed=3)
    a = pq.nndescent_dense(emb, 15, 0, 7)
    b = pq.nndescent_dense(emb, 15, 0, 7)
    np.testing.assert_array_equal(a["indices"], b["indices"])
    idx = a["indices"].reshape(-1, 15)
    assert not (idx == np.arange(5000)[:, None]).any()
    assert all(len(set(row)) == 15 for row in idx)
    assert (np.diff(a["data"].reshape(-1, 15), axis=1) >= 0).all()


def test_recall_vs_exact_on_25_gaussian_mixture():
    """test_neighbors.py:32-39: 20k x 30, k=15, seed 42."""
    emb = synth.mixture25(20_000)
    approx = pq.nndescent_dense(emb, 15, 0, 42)
    q = np.arange(0, 20_000, 7, dtype=np.uint32)
    ex, _ = oracle.exact_knn_f64(emb, q, 15)
    a = approx["indices"].reshape(-1, 15)[q]
    r = np.array([len(set(a[i]) & set(ex[i])) for i in range(len(q))]) / 15
    assert r.mean() >= 0.97 and np.percentile(r, 5) >= 0.85


def test_noncontiguous_input_is_copied():
    x = synth.blobs_rust_tests(1200, 16, 4, 1)
    g = pq.nndescent_dense(x[:, ::2], 8, 0, 1)
    r = oracle.nndescent(np.ascontiguousarray(x[:, ::2]), 8, seed=1)
    assert_graph_equal(g, r, "strided")


def test_device_entry_point_matches_host_entry_point(c1):
    torch = pytest.importorskip("torch")
    x = torch.from_numpy(c1).cuda()
    n = c1.shape[0]
    ip = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    ix = torch.empty(n * 15, dtype=torch.int32, device="cuda")
    dx = torch.empty(n * 15, dtype=torch.float32, device="cuda")
    ctx = pq.default_context(0)
    nnz = ctx.nndescent_device(x, _opts(15, seed=0), ip, ix, dx,
                               stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    r = oracle.nndescent(c1, 15, seed=0)
    assert nnz == len(r["indices"])
    np.testing.assert_array_equal(ip.cpu().numpy().view(np.uint32), r["indptr"])
    np.testing.assert_array_equal(ix[:nnz].cpu().numpy().view(np.uint32), r["indices"])
    assert dx[:nnz].cpu().numpy().tobytes() == r["data"].tobytes()
