"""A second, independent restatement of the reference NN-Descent
(oracle/nndescent_literal.py: literal, sequential, pure Python) against the
C++ restatement (oracle/nndescent_ref.cpp), byte for byte (CPU only).

The two share no code: agreement on graphs, per-round change counts and
trees (including the forest's parallel levels and the tie draws of duplicated
points) pins each against a misreading in the other.  The reference tests'
own inputs (make_clustered_data on ChaCha8Rng, nndescent.rs:1012-1022) are
restated from the published rand / rand_chacha algorithms; the ChaCha block
function is checked against a library ChaCha20 (the same function with 20
rounds).
"""

import os

import numpy as np
import pytest

import oracle
from oracle import nndescent_literal as lit
from polariseq_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def same_graph(a, b):
    return (np.array_equal(a["indptr"], b["indptr"]) and np.array_equal(a["indices"], b["indices"])
            and a["data"].tobytes() == b["data"].tobytes())


@pytest.mark.parametrize("case", [
    ("clustered 300x6 k=9", lambda: lit.make_clustered_data(300, 6, 4, 5), 9, dict(seed=5)),
    ("mixture 500x8 k=10", lambda: synth.mixture_dirichlet(500, 8, 5, 1), 10, dict(seed=3)),
    ("options 1200x13 k=7", lambda: synth.mixture_dirichlet(1200, 13, 5, 1), 7,
     dict(seed=3, max_candidates=5, n_trees=3, leaf_size=25)),
    ("tiny 5x3 k=10", lambda: lit.make_clustered_data(5, 3, 2, 1), 10, {}),
])
def test_literal_restatement_matches_the_cpp_oracle(case):
    name, make, k, kw = case
    x = make()
    a = lit.nndescent(x, k, **kw)
    b = oracle.nndescent(x, k, **kw)
    assert same_graph(a, b), name
    p = oracle.nndescent_probe(x, k, **kw)
    assert a["round_changed"] == p["round_changed"].tolist(), name


def test_literal_restatement_matches_with_duplicated_points():
    """Duplicated points: zero normals draw tie bits and hyperplanes that
    separate nothing fall back to random splits."""
    rng = np.random.default_rng(5)
    base = rng.normal(size=(20, 6)).astype(np.float32)
    x = base[rng.integers(0, 20, size=400)]
    assert same_graph(lit.nndescent(x, 8, seed=2), oracle.nndescent(x, 8, seed=2))


@pytest.mark.parametrize("n,d,dup", [(20_000, 12, False), (9_000, 5, False), (12_000, 4, True)])
def test_literal_trees_match_including_parallel_levels(n, d, dup):
    """Trees of at least 8,192 cells run the parallel top levels (child seeds
    splitmix(seed ^ 1/2), tie bits splitmix(seed ^ id)) before the sequential
    subtrees."""
    if dup:
        rng = np.random.default_rng(7)
        base = rng.normal(size=(300, d)).astype(np.float32)
        x = base[rng.integers(0, 300, size=n)]
    else:
        x = synth.mixture_lognormal(n, d, 10, seed=n)
    for t in (0, 3):
        s = lit.splitmix(17 ^ (t + 1))
        ids, leaves = lit.build_tree(x, 15, s)
        rids, rleaves = oracle.build_tree(x, 15, s)
        np.testing.assert_array_equal(ids, rids)
        np.testing.assert_array_equal(leaves.ravel(), np.asarray(rleaves).ravel())


def test_chacha_block_function_matches_a_library_chacha20():
    """ChaCha8Rng is ChaCha with 8 rounds; the block function here, run with
    20 rounds, must give the keystream of an independent ChaCha20 (the
    cryptography package: 32-bit counter in the nonce's first 4 bytes, zero
    nonce, which equals the 64-bit counter / 64-bit stream layout below
    2^32 blocks)."""
    cg = pytest.importorskip("cryptography.hazmat.primitives.ciphers")
    key = bytes((7 * i + 3) & 0xFF for i in range(32))
    kw = [int.from_bytes(key[4 * i:4 * i + 4], "little") for i in range(8)]
    for ctr in (0, 1, 2, 1000):
        nonce = ctr.to_bytes(4, "little") + bytes(12)
        ks = cg.Cipher(cg.algorithms.ChaCha20(key, nonce), mode=None).encryptor().update(bytes(64))
        want = [int.from_bytes(ks[4 * i:4 * i + 4], "little") for i in range(16)]
        assert lit.chacha_block(kw, ctr, 0, 20) == want


def test_clustered_data_generator_shape_and_range():
    x = lit.make_clustered_data(40, 7, 4, 3)
    assert x.dtype == np.float32 and x.shape == (40, 7)
    c = (np.arange(40) % 4).astype(np.float32)[:, None] * 10
    assert ((x - c) >= 0).all() and ((x - c) < 1).all()
    np.testing.assert_array_equal(x, lit.make_clustered_data(40, 7, 4, 3))


# ── the reference's unit tests (nndescent.rs:1059-1199) on their own inputs,
#    through the C++ oracle ──────────────────────────────────────────────────

def test_reference_caller_arrays_case_on_its_own_input():
    import ctypes as C

    x = lit.make_clustered_data(1500, 6, 4, 3)
    g = oracle.nndescent(x, 9, seed=5)
    cap = 1500 * 9
    ip = np.full(1501, 7, np.uint32)
    ix = np.full(cap, 9, np.uint32)
    dx = np.full(cap, 1.0, np.float32)
    o = oracle.make_opts(9, 0, 0, 0.001, 0, 0, 0, 5)
    nn = C.c_uint64(0)
    rc = oracle.lib().oracle_nndescent_into(x.ctypes.data, 1500, 6, C.byref(o), ip.ctypes.data,
                                            1501, ix.ctypes.data, cap, dx.ctypes.data, cap,
                                            C.byref(nn), None)
    assert rc == 0
    nnz = nn.value
    assert nnz == len(g["indices"])
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix[:nnz], g["indices"])
    assert dx[:nnz].tobytes() == g["data"].tobytes()


def test_reference_structure_case_on_its_own_input():
    n, k = 2000, 10
    g = oracle.nndescent(lit.make_clustered_data(n, 8, 5, 1), k, seed=1)
    for i in range(n):
        s, e = g["indptr"][i], g["indptr"][i + 1]
        row = g["indices"][s:e]
        assert e - s == k and i not in row and len(set(row.tolist())) == k
        assert (np.diff(g["data"][s:e]) >= 0).all()


def test_reference_recall_case_on_its_own_input():
    x = lit.make_blob_data(6000, 20, 9)
    g = oracle.nndescent(x, 15, seed=4)
    hits = 0
    for i in range(300):
        d2 = ((x.astype(np.float64) - x[i].astype(np.float64)) ** 2).sum(1)
        d2[i] = np.inf
        exact = set(np.argsort(d2, kind="stable")[:15].tolist())
        hits += len(exact & set(g["indices"][g["indptr"][i]:g["indptr"][i + 1]].tolist()))
    assert hits / (300 * 15) >= 0.95


def test_reference_gather_bound_case_on_its_own_input():
    x = lit.make_clustered_data(20_000, 12, 15, 11)
    copied = oracle.nndescent(x, 10, seed=9, gather_max=2 ** 62)
    for gm in (1, 64, 1000):
        assert same_graph(oracle.nndescent(x, 10, seed=9, gather_max=gm), copied), gm


def test_reference_tiny_case_on_its_own_input():
    g = oracle.nndescent(lit.make_clustered_data(5, 3, 2, 0), 10)
    assert (np.diff(g["indptr"]) == 4).all()


def test_committed_reference_input_goldens_match_the_cpp_oracle():
    """The goldens (written by the literal restatement on the reference tests'
    inputs) equal the C++ oracle's graphs and change counts."""
    z = np.load(os.path.join(GOLDEN, "reference_inputs_golden.npz"))
    for name in sorted({f.split("__")[0] for f in z.files}):
        n, d, ncl, ds, k, seed = (int(v) for v in z[name + "__cfg"])
        x = z[name + "__data"]
        np.testing.assert_array_equal(x, lit.make_clustered_data(n, d, ncl, ds))
        g = oracle.nndescent(x, k, seed=seed)
        h = {"indptr": z[name + "__indptr"], "indices": z[name + "__indices"],
             "data": z[name + "__dists"]}
        assert same_graph(g, h), name
        p = oracle.nndescent_probe(x, k, seed=seed)
        assert p["round_changed"].tolist() == z[name + "__changed"].tolist(), name
