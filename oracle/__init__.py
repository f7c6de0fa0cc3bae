"""ORACLE — test infrastructure only.

ctypes bindings to the C++ restatement of the reference's CPU NN-Descent
(``nndescent_ref.cpp``, restating crates/polariseq-core/src/nndescent.rs:78-1003
and simd.rs:14-81), to the FP64 exact kNN / exact f32 search restatement
(``exact_ref.cpp``, neighbors.rs:101-241) and to the fuzzy simplicial set
restatement (``fuzzy_ref.cpp``, umap.rs:283-620); ``mlp_ref.py`` restates the
learned router's gradients in float64 NumPy.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; the product package never does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class OracleOpts(C.Structure):
    """Mirrors NndescentOptions (nndescent.rs:42-76)."""

    _fields_ = [
        ("k", C.c_uint64),
        ("max_candidates", C.c_uint64),
        ("max_iterations", C.c_uint64),
        ("delta", C.c_double),
        ("n_trees", C.c_uint64),
        ("leaf_size", C.c_uint64),
        ("gather_max", C.c_uint64),
        ("seed", C.c_uint64),
    ]


class OracleProbe(C.Structure):
    _fields_ = [
        ("stop_after", C.c_int32),
        ("rounds_run", C.c_int32),
        ("heap_idx", C.c_void_p),
        ("heap_dist", C.c_void_p),
        ("heap_flag", C.c_void_p),
        ("cand_new", C.c_void_p),
        ("cand_old", C.c_void_p),
        ("round_changed", C.c_void_p),
        ("round_emitted", C.c_void_p),
        ("round_pairs", C.c_void_p),
        ("resolved", C.c_uint64 * 6),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        P = C.c_void_p
        L.oracle_nndescent_into.argtypes = [P, C.c_uint64, C.c_uint64, C.POINTER(OracleOpts),
                                            P, C.c_uint64, P, C.c_uint64, P, C.c_uint64,
                                            C.POINTER(C.c_uint64), C.POINTER(OracleProbe)]
        L.oracle_nndescent_into.restype = C.c_int
        L.oracle_build_tree.argtypes = [P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                        C.c_uint64, P, P, C.c_uint64]
        L.oracle_build_tree.restype = C.c_uint64
        L.oracle_effective_k.argtypes = [C.c_uint64, C.c_uint64]
        L.oracle_effective_k.restype = C.c_uint64
        L.oracle_splitmix.argtypes = [C.c_uint64]
        L.oracle_splitmix.restype = C.c_uint64
        L.oracle_hash_unit.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.oracle_hash_unit.restype = C.c_float
        L.oracle_hash_index.argtypes = [C.c_uint64] * 4
        L.oracle_hash_index.restype = C.c_uint64
        L.oracle_sq_dist.argtypes = [P, P, C.c_uint64]
        L.oracle_sq_dist.restype = C.c_float
        L.oracle_dot.argtypes = [P, P, C.c_uint64]
        L.oracle_dot.restype = C.c_float
        L.oracle_partition.argtypes = [P, C.c_uint64, P]
        L.oracle_partition.restype = C.c_uint64
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_max_threads.restype = C.c_int
        L.oracle_exact_knn_f64.argtypes = [P, C.c_uint64, C.c_uint64, P, C.c_uint64, C.c_uint64,
                                           P, P]
        L.oracle_neighbors_exact.argtypes = [P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                             P, P, P]
        L.oracle_neighbors_exact.restype = C.c_int
        L.oracle_smooth_knn_dist.argtypes = [P, C.c_uint64, P]
        L.oracle_smooth_knn_dist.restype = None
        L.oracle_fuzzy.argtypes = [C.c_uint64, P, P, P, P, P, P, C.c_uint64]
        L.oracle_fuzzy.restype = C.c_uint64
        L.oracle_knn_exact_batched.argtypes = [P, C.c_int, C.c_uint32, P, P, P]
        L.oracle_knn_exact_batched.restype = None
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def effective_k(n_obs: int, k: int) -> int:
    return int(lib().oracle_effective_k(n_obs, k))


def set_threads(t: int) -> None:
    lib().oracle_set_threads(int(t))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def make_opts(k=15, max_candidates=0, max_iterations=0, delta=0.001, n_trees=0, leaf_size=0,
              gather_max=0, seed=0) -> OracleOpts:
    return OracleOpts(k, max_candidates, max_iterations, delta, n_trees, leaf_size, gather_max,
                      seed)


def nndescent(data: np.ndarray, k: int = 15, *, max_iterations=0, seed=0, max_candidates=0,
              n_trees=0, delta=0.001, leaf_size=0, gather_max=0) -> dict:
    """The reference's `nndescent` (nndescent.rs:657-686): CSR with nnz entries."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, d = data.shape
    cap = n * effective_k(n, k) if n > 0 else 0
    ip = np.zeros(n + 1, np.uint32)
    ix = np.zeros(max(cap, 1), np.uint32)
    dx = np.zeros(max(cap, 1), np.float32)
    nnz = C.c_uint64(0)
    o = make_opts(k, max_candidates, max_iterations, delta, n_trees, leaf_size, gather_max, seed)
    rc = lib().oracle_nndescent_into(_ptr(data), n, d, C.byref(o), _ptr(ip), n + 1, _ptr(ix),
                                     cap, _ptr(dx), cap, C.byref(nnz), None)
    if rc != 0:
        raise ValueError(f"oracle nndescent rejected the input (code {rc})")
    m = nnz.value
    return {"indptr": ip, "indices": ix[:m].copy(), "data": dx[:m].copy(), "n_obs": n}


def nndescent_probe(data: np.ndarray, k: int = 15, *, stop_after: int = -2, seed=0,
                    max_iterations=0, max_candidates=0, n_trees=0, delta=0.001, leaf_size=0,
                    gather_max=0) -> dict:
    """Run the oracle and return its internal state at `stop_after`
    (-1: after forest + random fill; r: after round r's apply; -2: end)."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, d = data.shape
    ek = effective_k(n, k)
    o = make_opts(k, max_candidates, max_iterations, delta, n_trees, leaf_size, gather_max, seed)
    # resolve first with a stop-at-init probe to learn m and the round count
    pr = OracleProbe()
    pr.stop_after = -1
    ip = np.zeros(n + 1, np.uint32)
    ix = np.zeros(n * ek, np.uint32)
    dx = np.zeros(n * ek, np.float32)
    nnz = C.c_uint64(0)
    res = OracleProbe()
    res.stop_after = -1
    # cheap: the resolve happens before the forest, but the probe returns after init.
    hidx = np.zeros(n * ek, np.uint32)
    hdist = np.zeros(n * ek, np.float32)
    hflag = np.zeros(n * ek, np.uint8)
    rounds_cap = 64
    chg = np.zeros(rounds_cap, np.uint64)
    emi = np.zeros(rounds_cap, np.uint64)
    prs = np.zeros(rounds_cap, np.uint64)
    m_guess = max(1, max_candidates if max_candidates > 0 else min(2 * ek, 60))
    cnew = np.zeros(n * m_guess, np.uint32)
    cold = np.zeros(n * m_guess, np.uint32)
    pr = OracleProbe(stop_after, 0, _ptr(hidx), _ptr(hdist), _ptr(hflag), _ptr(cnew), _ptr(cold),
                     _ptr(chg), _ptr(emi), _ptr(prs))
    rc = lib().oracle_nndescent_into(_ptr(data), n, d, C.byref(o), _ptr(ip), n + 1, _ptr(ix),
                                     n * ek, _ptr(dx), n * ek, C.byref(nnz), C.byref(pr))
    if rc != 0:
        raise ValueError(f"oracle nndescent rejected the input (code {rc})")
    r = pr.rounds_run
    return {
        "heap_idx": hidx.reshape(n, ek), "heap_dist": hdist.reshape(n, ek),
        "heap_flag": hflag.reshape(n, ek), "cand_new": cnew.reshape(n, m_guess),
        "cand_old": cold.reshape(n, m_guess), "rounds_run": r,
        "round_changed": chg[:r].copy(), "round_emitted": emi[:r].copy(),
        "round_pairs": prs[:r].copy(), "resolved": list(pr.resolved),
        "indptr": ip, "indices": ix[:nnz.value].copy(), "data": dx[:nnz.value].copy(),
    }


def build_tree(data: np.ndarray, leaf_size: int, seed: int, gather_max: int = 0):
    """One RP tree (nndescent.rs:643-646): (ids permutation, leaves [L,2])."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, d = data.shape
    ids = np.zeros(n, np.uint32)
    cap = n + 1
    leaves = np.zeros(2 * cap, np.uint32)
    nl = lib().oracle_build_tree(_ptr(data), n, d, leaf_size, seed, gather_max, _ptr(ids),
                                 _ptr(leaves), cap)
    return ids, leaves[: 2 * nl].reshape(nl, 2).copy()


def splitmix(x: int) -> int:
    return int(lib().oracle_splitmix(x & 0xFFFFFFFFFFFFFFFF))


def hash_unit(seed: int, a: int, b: int) -> float:
    return float(lib().oracle_hash_unit(seed, a, b))


def hash_index(seed: int, a: int, b: int, n: int) -> int:
    return int(lib().oracle_hash_index(seed, a, b, n))


def sq_dist(a: np.ndarray, b: np.ndarray) -> np.float32:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return np.float32(lib().oracle_sq_dist(_ptr(a), _ptr(b), a.size))


def dot(a: np.ndarray, b: np.ndarray) -> np.float32:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return np.float32(lib().oracle_dot(_ptr(a), _ptr(b), a.size))


def partition(ids: np.ndarray, sides: np.ndarray) -> tuple[np.ndarray, int]:
    """The reference's two-pointer partition (nndescent.rs:389-405)."""
    ids = np.ascontiguousarray(ids, np.uint32).copy()
    sides = np.ascontiguousarray(sides, np.uint8)
    s = lib().oracle_partition(_ptr(ids), ids.size, _ptr(sides))
    return ids, int(s)


def exact_knn_f64(data: np.ndarray, queries: np.ndarray, k: int):
    """FP64 exact kNN (self excluded, (distance, index) order)."""
    data = np.ascontiguousarray(data, np.float32)
    q = np.ascontiguousarray(queries, np.uint32)
    n, d = data.shape
    oi = np.zeros((q.size, k), np.uint32)
    od = np.zeros((q.size, k), np.float64)
    lib().oracle_exact_knn_f64(_ptr(data), n, d, _ptr(q), q.size, k, _ptr(oi), _ptr(od))
    return oi, od


def neighbors_exact(emb: np.ndarray, n_neighbors: int, metric: str = "euclidean") -> dict:
    """The reference's exact search (neighbors.rs:101-147)."""
    emb = np.ascontiguousarray(emb, np.float32)
    n, d = emb.shape
    kws = min(n_neighbors, n)
    ip = np.zeros(n + 1, np.uint32)
    ix = np.zeros(max(1, n * max(kws - 1, 0)), np.uint32)
    dx = np.zeros(max(1, n * max(kws - 1, 0)), np.float32)
    rc = lib().oracle_neighbors_exact(_ptr(emb), n, d, n_neighbors, int(metric == "cosine"),
                                      _ptr(ip), _ptr(ix), _ptr(dx))
    if rc != 0:
        raise ValueError(f"oracle neighbors rejected the input (code {rc})")
    m = int(ip[-1])
    return {"indptr": ip, "indices": ix[:m].copy(), "data": dx[:m].copy(), "n_obs": n}


def smooth_knn_dist(dists) -> np.ndarray:
    """umap.rs:551-620: membership strengths of one row of ascending distances."""
    d = np.ascontiguousarray(dists, np.float32)
    out = np.zeros(d.size, np.float32)
    lib().oracle_smooth_knn_dist(_ptr(d), d.size, _ptr(out))
    return out


def fuzzy_connectivities(indptr, indices, data, n_obs: int) -> dict:
    """umap.rs:122-138 fuzzy_connectivities_from: the symmetric CSR."""
    ip = np.ascontiguousarray(indptr, np.uint32)
    ix = np.ascontiguousarray(indices, np.uint32)
    dx = np.ascontiguousarray(data, np.float32)
    cap = max(2 * int(ip[-1]), 1)
    oip = np.zeros(n_obs + 1, np.uint32)
    oix = np.zeros(cap, np.uint32)
    ow = np.zeros(cap, np.float32)
    nnz = lib().oracle_fuzzy(n_obs, _ptr(ip), _ptr(ix), _ptr(dx), _ptr(oip), _ptr(oix), _ptr(ow), cap)
    return {"indptr": oip, "indices": oix[:nnz].copy(), "data": ow[:nnz].copy()}


def knn_exact_batched(samples, ks) -> list:
    """The reference's tiled exact per-sample kNN (doublets.rs:544-650,
    restated in knn_exact_ref.cpp) over every sample, all threads: a list of
    (n_s, k_s) u32 index arrays, itself excluded, (distance, index) order."""
    L = lib()
    d = samples[0].shape[1]
    data = np.ascontiguousarray(np.concatenate(samples).astype(np.float32, copy=False))
    offs = np.zeros(len(samples) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in samples])
    kk = np.asarray(ks, np.uint32)
    out = np.zeros(int(sum(len(s) * int(k) for s, k in zip(samples, ks))), np.uint32)
    L.oracle_knn_exact_batched(_ptr(data), int(d), len(samples), _ptr(offs), _ptr(kk), _ptr(out))
    res, o = [], 0
    for s, k in zip(samples, ks):
        m = len(s) * int(k)
        res.append(out[o:o + m].reshape(len(s), int(k)))
        o += m
    return res
