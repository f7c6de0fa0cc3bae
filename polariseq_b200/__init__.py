"""polariseq_b200 — a B200 (sm_100a) drop-in for Polariseq's NN-Descent kNN-graph builder.

Python surface of the reference's PyO3 binding
(crates/polariseq-python/src/lib.rs:503-566)::

    nndescent_dense(embedding, k, max_iterations=0, seed=0, max_candidates=0,
                    n_trees=0, delta=0.001, out=None) -> dict

Without ``out``: ``{"indptr": u32[n+1], "indices": u32[nnz], "data": f32[nnz],
"n_obs": n}`` — the CSR distance graph, Euclidean distances ascending per row.
With ``out=(indptr, indices, data)`` the graph is written in place and
``{"nnz", "n_obs"}`` is returned; entries past nnz are left untouched.  A bad
``out`` raises ``ValueError`` with the reference's message; inputs on which the
reference core panics (empty data, ``k == 0``) raise :class:`PanicException`,
as PyO3 turns the core's panic into ``pyo3_runtime.PanicException``.

Every call runs on the GPU through the C ABI (include/polariseq_knn.h); the
GIL is released for the whole build (ctypes drops it around foreign calls).
"""

from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib

__all__ = [
    "PanicException", "DeviceError", "DeviceTimeout", "Context", "nndescent_dense", "nndescent",
    "effective_k", "default_context", "neighbors_dense", "knn_batched", "knn_batched_sharded",
    "shard_samples", "fuzzy_connectivities", "scrublet_scores",
]


class PanicException(BaseException):
    """Raised where the reference core panics (pyo3_runtime.PanicException
    also derives from BaseException)."""


class DeviceError(RuntimeError):
    pass


class DeviceTimeout(DeviceError):
    """A bounded device-side wait gave up (PQ_ETIMEOUT); the context stays
    usable."""


def effective_k(n_obs: int, k: int) -> int:
    """Neighbours per row the graph can hold (nndescent.rs:648-650)."""
    return int(_lib.load().pq_effective_k(int(n_obs), int(k)))


def _opts(k, max_iterations, seed, max_candidates, n_trees, delta, leaf_size=0, gather_max=0,
          mode=_lib.PQ_MODE_PLAIN, init=_lib.PQ_INIT_RP, probes=0,
          refine_rounds=-1, buckets=0) -> _lib.NndOpts:
    o = _lib.NndOpts()
    _lib.load().pq_nnd_opts_default(C.byref(o))
    o.k = int(k)
    o.max_iterations = int(max_iterations)
    o.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    o.max_candidates = int(max_candidates)
    o.n_trees = int(n_trees)
    o.delta = float(delta)
    o.leaf_size = int(leaf_size)
    o.gather_max = int(gather_max)
    o.mode = int(mode)
    o.init = int(init)
    o.probes = int(probes)
    o.refine_rounds = int(refine_rounds)
    o.buckets = int(buckets)
    return o


class Context:
    """One device context: a CUDA stream plus a device workspace reused
    across calls.  Calls on one context are serialised."""

    def __init__(self, device: int = 0):
        L = _lib.load()
        h = C.c_void_p()
        rc = L.pq_ctx_create(int(device), C.byref(h))
        if rc != _lib.PQ_OK:
            raise DeviceError(f"pq_ctx_create(device={device}) failed with status {rc}; "
                              "a CUDA device is required (there is no CPU fallback)")
        self._h = h
        self.device = device
        self._lock = threading.Lock()

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().pq_ctx_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc == _lib.PQ_OK:
            return
        msg = _lib.load().pq_ctx_last_error(self._h).decode(errors="replace")
        if rc == _lib.PQ_EINVAL:
            raise PanicException(f"{what}: {msg}")
        if rc == _lib.PQ_ENOTSUP:
            raise NotImplementedError(f"{what}: {msg}")
        if rc == _lib.PQ_ENOMEM:
            raise MemoryError(f"{what}: {msg}")
        if rc == _lib.PQ_ETIMEOUT:
            raise DeviceTimeout(f"{what}: {msg}")
        raise DeviceError(f"{what} failed (status {rc}): {msg}")

    def stats(self) -> dict:
        s = _lib.NndStats()
        self._check(_lib.load().pq_ctx_stats(self._h, C.byref(s)), "stats")
        r = s.rounds_run
        return {
            "rounds_run": r, "n_trees": s.n_trees, "k": s.k, "max_candidates": s.max_candidates,
            "n_iters": s.n_iters, "leaf_size": s.leaf_size, "stop_at": s.stop_at,
            "changed": list(s.changed[:r]), "emitted": list(s.emitted[:r]),
            "pairs": list(s.pairs[:r]), "ms_forest": s.ms_forest, "ms_leaves": s.ms_leaves,
            "ms_rounds": s.ms_rounds, "ms_extract": s.ms_extract, "ms_total": s.ms_total,
            "shortlist": list(s.shortlist), "learn_loss_first": s.learn_loss_first,
            "learn_loss_last": s.learn_loss_last, "ms_learn_train": s.ms_learn_train,
            "ms_learn_route": s.ms_learn_route, "est_recall": s.est_recall,
            "est_recall_learned": s.est_recall_learned, "est_recall_rp": s.est_recall_rp,
            "fell_back": s.fell_back, "learned_rounds": s.learned_rounds,
        }

    # -- host-buffer build (the drop-in) ------------------------------------
    def nndescent_into(self, data: np.ndarray, opts: _lib.NndOpts, indptr: np.ndarray,
                       indices: np.ndarray, dists: np.ndarray) -> int:
        n, d = data.shape
        nnz = C.c_uint64(0)
        with self._lock:
            rc = _lib.load().pq_nndescent_into(
                self._h, data.ctypes.data, n, d, C.byref(opts), indptr.ctypes.data, indptr.size,
                indices.ctypes.data, indices.size, dists.ctypes.data, dists.size, C.byref(nnz))
            self._check(rc, "nndescent")
        return int(nnz.value)

    # -- device-buffer build (torch CUDA tensors) ---------------------------
    def nndescent_device(self, data, opts: _lib.NndOpts, indptr, indices, dists,
                         stream=None) -> int:
        """`data`, `indptr`, `indices`, `dists`: contiguous CUDA tensors
        (float32 [n,d], int32/uint32 [n+1], [>= n*k], float32 [>= n*k])."""
        n, d = int(data.shape[0]), int(data.shape[1])
        nnz = C.c_uint64(0)
        sp = None if stream is None else C.c_void_p(int(stream))
        with self._lock:
            rc = _lib.load().pq_nndescent_into_device(
                self._h, data.data_ptr(), n, d, C.byref(opts), indptr.data_ptr(),
                indices.data_ptr(), dists.data_ptr(), C.byref(nnz), sp)
            self._check(rc, "nndescent_device")
        return int(nnz.value)

    # -- exact kNN (neighbors::neighbors) -----------------------------------
    def _check_neighbors(self, rc: int) -> None:
        if rc == _lib.PQ_EINVAL:  # NeighborsError -> RuntimeError (lib.rs:493-495)
            msg = _lib.load().pq_ctx_last_error(self._h).decode(errors="replace")
            raise RuntimeError(f"neighbors failed: {msg}")
        self._check(rc, "neighbors")

    def neighbors_into(self, data: np.ndarray, n_neighbors: int, metric: int,
                       indptr: np.ndarray, indices: np.ndarray, dists: np.ndarray) -> int:
        n, d = data.shape
        nnz = C.c_uint64(0)
        with self._lock:
            rc = _lib.load().pq_neighbors_into(
                self._h, data.ctypes.data, n, d, int(n_neighbors), int(metric),
                indptr.ctypes.data, indptr.size, indices.ctypes.data, indices.size,
                dists.ctypes.data, dists.size, C.byref(nnz))
            self._check_neighbors(rc)
        return int(nnz.value)

    def neighbors_device(self, data, n_neighbors: int, metric: int, indptr, indices, dists,
                         stream=None) -> int:
        """`data` float32 [n, d], `indptr` [n+1], `indices`/`dists` [>= n*(k-1)]:
        contiguous CUDA tensors."""
        n, d = int(data.shape[0]), int(data.shape[1])
        nnz = C.c_uint64(0)
        sp = None if stream is None else C.c_void_p(int(stream))
        with self._lock:
            rc = _lib.load().pq_neighbors_into_device(
                self._h, data.data_ptr(), n, d, int(n_neighbors), int(metric),
                indptr.data_ptr(), indices.data_ptr(), dists.data_ptr(), C.byref(nnz), sp)
            self._check_neighbors(rc)
        return int(nnz.value)

    # -- batched exact kNN over many samples -------------------------------
    def knn_batched_device(self, data, offsets: np.ndarray, ks: np.ndarray, indices, dists,
                           autotune: bool = False, graph: bool = True, stream=None) -> int:
        """All samples' rows back to back in `data` (float32 [N, d] CUDA
        tensor); `offsets` (uint64 [S+1]) and `ks` (uint32 [S]) on the host;
        `indices`/`dists` CUDA tensors of sum(n_s * k_s).  Returns the tile
        shape used."""
        offsets = np.ascontiguousarray(offsets, np.uint64)
        ks = np.ascontiguousarray(ks, np.uint32)
        flags = (_lib.PQ_BATCH_AUTOTUNE if autotune else 0) | (_lib.PQ_BATCH_GRAPH if graph else 0)
        shape = C.c_int32(-1)
        sp = None if stream is None else C.c_void_p(int(stream))
        with self._lock:
            rc = _lib.load().pq_knn_batched_into_device(
                self._h, data.data_ptr(), int(data.shape[1]), int(ks.size), offsets.ctypes.data,
                ks.ctypes.data, indices.data_ptr(), dists.data_ptr(), flags, C.byref(shape), sp)
            if rc == _lib.PQ_EINVAL:
                msg = _lib.load().pq_ctx_last_error(self._h).decode(errors="replace")
                raise ValueError(f"knn_batched: {msg}")
            self._check(rc, "knn_batched")
        return int(shape.value)

    # -- fuzzy connectivities ------------------------------------------------
    def fuzzy_connectivities(self, indptr, indices, data, n_obs: int) -> dict:
        ip = np.ascontiguousarray(indptr, np.uint32)
        ix = np.ascontiguousarray(indices, np.uint32)
        dx = np.ascontiguousarray(data, np.float32)
        cap = max(2 * int(ip[n_obs]), 1)
        oip = np.zeros(n_obs + 1, np.uint32)
        oix = np.zeros(cap, np.uint32)
        ow = np.zeros(cap, np.float32)
        nnz = C.c_uint64(0)
        with self._lock:
            rc = _lib.load().pq_fuzzy_connectivities(
                self._h, n_obs, ip.ctypes.data, ix.ctypes.data, dx.ctypes.data, oip.ctypes.data,
                oix.ctypes.data, ow.ctypes.data, cap, C.byref(nnz))
            self._check(rc, "fuzzy_connectivities")
        m = int(nnz.value)
        return {"indptr": oip, "indices": oix[:m].copy(), "data": ow[:m].copy()}

    # -- parity probes (test hooks) ----------------------------------------
    def probe(self, data: np.ndarray, opts: _lib.NndOpts, stop_after: int) -> dict:
        data = np.ascontiguousarray(data, np.float32)
        n, d = data.shape
        k = effective_k(n, opts.k)
        m = max(1, opts.max_candidates if opts.max_candidates > 0 else min(2 * k, 60))
        hi = np.zeros((n, k), np.uint32)
        hd = np.zeros((n, k), np.float32)
        hf = np.zeros((n, k), np.uint8)
        cn = np.zeros((n, m), np.uint32)
        co = np.zeros((n, m), np.uint32)
        with self._lock:
            rc = _lib.load().pq_nndescent_probe(
                self._h, data.ctypes.data, n, d, C.byref(opts), int(stop_after), hi.ctypes.data,
                hd.ctypes.data, hf.ctypes.data, cn.ctypes.data, co.ctypes.data)
            self._check(rc, "probe")
        return {"heap_idx": hi, "heap_dist": hd, "heap_flag": hf, "cand_new": cn,
                "cand_old": co}

    def debug_tree(self, data: np.ndarray, opts: _lib.NndOpts, tree: int):
        data = np.ascontiguousarray(data, np.float32)
        n, d = data.shape
        ids = np.zeros(n, np.uint32)
        cap = n + 1
        leaves = np.zeros(2 * cap, np.uint32)
        nl = C.c_uint64(0)
        with self._lock:
            rc = _lib.load().pq_debug_tree(self._h, data.ctypes.data, n, d, C.byref(opts),
                                           int(tree), ids.ctypes.data, leaves.ctypes.data, cap,
                                           C.byref(nl))
            self._check(rc, "debug_tree")
        return ids, leaves[: 2 * nl.value].reshape(-1, 2).copy()


_default: dict[int, Context] = {}
_default_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _default_lock:
        ctx = _default.get(device)
        if ctx is None:
            ctx = Context(device)
            _default[device] = ctx
        return ctx


def _as_embedding(embedding) -> np.ndarray:
    a = embedding
    if not isinstance(a, np.ndarray):
        raise TypeError("argument 'embedding': expected a numpy.ndarray of float32")
    if a.ndim != 2:
        raise TypeError(f"argument 'embedding': expected a 2-D array, got {a.ndim}-D")
    if a.dtype != np.float32:
        raise TypeError(f"argument 'embedding': expected float32, got {a.dtype}")
    # read in place when contiguous, else copy (lib.rs:526-533)
    return a if a.flags["C_CONTIGUOUS"] else np.ascontiguousarray(a)


def _as_out(arr, dtype, name):
    if not isinstance(arr, np.ndarray) or arr.ndim != 1 or arr.dtype != dtype:
        raise TypeError(f"out: '{name}' must be a 1-D numpy array of {np.dtype(dtype).name}")
    if not arr.flags["C_CONTIGUOUS"] or not arr.flags["WRITEABLE"]:
        raise TypeError(f"out: '{name}' must be contiguous and writeable")
    return arr


MODES = {"plain": _lib.PQ_MODE_PLAIN, "bf16": _lib.PQ_MODE_BF16, "fp8": _lib.PQ_MODE_FP8}
INITS = {"rp": _lib.PQ_INIT_RP, "learned": _lib.PQ_INIT_LEARNED}


def nndescent_dense(embedding, k, max_iterations=0, seed=0, max_candidates=0, n_trees=0,
                    delta=0.001, out=None, *, device: int = 0, mode: str = "plain",
                    init: str = "rp", probes: int = 0, refine_rounds: int = -1, buckets: int = 0):
    """Approximate kNN graph by NN-Descent, bit-exact with the reference
    (crates/polariseq-python/src/lib.rs:503-566).

    ``mode='plain'`` (default) reproduces the reference graph bit for bit;
    ``mode='bf16'`` is the tensor-core shortlist form (bucketed BF16 distance
    tiles, exact FP32 re-rank, FP64 boundary) with the same output layout."""
    emb = _as_embedding(embedding)
    n_obs, _ = emb.shape
    opts = _opts(k, max_iterations, seed, max_candidates, n_trees, delta, mode=MODES[mode],
                 init=INITS[init], probes=probes, refine_rounds=refine_rounds, buckets=buckets)
    cap = n_obs * effective_k(n_obs, k)
    # the same order as the binding: the out sizes are validated (ValueError)
    # before the core runs and panics on empty data or k == 0
    if out is not None:
        ip, ix, dx = out
        ip = _as_out(ip, np.uint32, "indptr")
        ix = _as_out(ix, np.uint32, "indices")
        dx = _as_out(dx, np.float32, "data")
        if ip.size != n_obs + 1 or ix.size < cap or dx.size < cap:
            raise ValueError(f"outputs must hold {n_obs + 1} row pointers and {cap} neighbours")
    if n_obs == 0 or emb.shape[1] == 0:
        raise PanicException("empty data")
    if int(k) == 0:
        raise PanicException("k must be >= 1")
    ctx = default_context(device)
    if out is not None:
        nnz = ctx.nndescent_into(emb, opts, ip, ix, dx)
        return {"nnz": nnz, "n_obs": n_obs}
    ip = np.zeros(n_obs + 1, np.uint32)
    ix = np.zeros(cap, np.uint32)
    dx = np.zeros(cap, np.float32)
    nnz = ctx.nndescent_into(emb, opts, ip, ix, dx)
    return {"indptr": ip, "indices": ix[:nnz], "data": dx[:nnz], "n_obs": n_obs}


METRICS = {"euclidean": _lib.PQ_METRIC_EUCLIDEAN, "cosine": _lib.PQ_METRIC_COSINE}


def fuzzy_connectivities(indptr, indices, data, n_obs, *, device: int = 0) -> dict:
    """The symmetrised fuzzy connectivities of a kNN distance graph, as the
    reference's ``fuzzy_connectivities`` (crates/polariseq-python/src/
    lib.rs:568-589, umap.rs:122-138): ``{"indptr", "indices", "data"}``, a
    symmetric CSR with both directions stored, rows sorted by column."""
    ip = np.asarray(indptr)
    if ip.size != int(n_obs) + 1:
        raise ValueError("indptr must have n_obs + 1 entries")
    return default_context(device).fuzzy_connectivities(indptr, indices, data, int(n_obs))


def knn_batched(samples, ks, *, device: int = 0, autotune: bool = False, graph: bool = True):
    """Exact kNN within each sample, all samples in one persistent launch
    (the per-sample search of doublet scoring, doublets.rs:544-650).

    ``samples``: list of float32 [n_s, d] arrays (d <= 64); ``ks``: the k of
    each sample (1 <= k < n_s).  Returns a list of ``(indices, distances)``
    pairs, [n_s, k_s] each: local indices of the k nearest other points,
    ascending by (distance, index), Euclidean distances."""
    import torch

    arrs = [np.ascontiguousarray(a, np.float32) for a in samples]
    if not arrs:
        return []
    d = arrs[0].shape[1]
    sizes = np.array([a.shape[0] for a in arrs], np.uint64)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    ks = np.asarray(ks, np.uint32)
    total = int(np.sum(sizes * ks.astype(np.uint64)))
    dev = torch.device("cuda", device)
    x = torch.from_numpy(np.concatenate(arrs, 0)).to(dev)
    oi = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    od = torch.empty(max(total, 1), dtype=torch.float32, device=dev)
    default_context(device).knn_batched_device(x, offsets, ks, oi, od, autotune=autotune,
                                               graph=graph)
    oi = oi.cpu().numpy().view(np.uint32)
    od = od.cpu().numpy()
    out, o = [], 0
    for a, k in zip(arrs, ks):
        m = a.shape[0] * int(k)
        out.append((oi[o:o + m].reshape(a.shape[0], int(k)), od[o:o + m].reshape(a.shape[0], int(k))))
        o += m
    return out


def scrublet_scores(u, w, totals, mv, pairs, ks, rho: float = 0.1, *, device: int = 0,
                    debug: bool = False):
    """Doublet scores of many samples after their PCA, on the GPU (the steps
    of Scrublet's score_batch, crates/polariseq-core/src/doublets.rs:
    1040-1127): each sample's cells and simulated doublets as points, their
    exact kNN within the sample (k_adj = round_half_even(k (1 + n_sim / n))),
    and the Bayesian score from the simulated neighbours.

    Per sample s: ``u[s]`` f64 [n, p] (projected scaled counts), ``w[s]`` and
    ``totals[s]`` f64 [n], ``mv[s]`` f64 [p], ``pairs[s]`` int [n_sim, 2]
    (parents of each simulated doublet), ``ks[s]`` the neighbour count.
    Returns a list of dicts {"obs": f64 [n], "sim": f64 [n_sim], "k_adj"}
    (with ``debug``, also the f32 points and the neighbour indices)."""
    import torch

    S = len(u)
    p = int(np.asarray(u[0]).shape[1])
    dev = torch.device("cuda", device)
    nc = np.array([len(a) for a in u], np.uint64)
    ns = np.array([len(a) for a in pairs], np.uint64)
    kk = np.ascontiguousarray(ks, np.uint32)

    def cat(xs, dt):
        return torch.from_numpy(np.ascontiguousarray(np.concatenate(
            [np.asarray(a, dt).reshape(len(a), -1) if np.asarray(a).ndim > 1
             else np.asarray(a, dt) for a in xs]))).to(dev)

    du, dw, dt_ = cat(u, np.float64), cat(w, np.float64), cat(totals, np.float64)
    dmv = torch.from_numpy(np.ascontiguousarray(np.stack(mv).astype(np.float64))).to(dev)
    dpr = cat(pairs, np.uint32) if int(ns.sum()) else None
    so = torch.empty(int(nc.sum()), dtype=torch.float64, device=dev)
    ss = torch.empty(int(ns.sum()), dtype=torch.float64, device=dev)
    kadj = np.zeros(S, np.uint32)
    npt = int(nc.sum() + ns.sum())
    pts = torch.empty((npt, p), dtype=torch.float32, device=dev) if debug else None
    # every sample's k_adj is at most 512 and below its point count
    nk = int(sum((int(a) + int(b)) * min(512, int(a) + int(b) - 1) for a, b in zip(nc, ns)))
    knn = torch.empty(max(nk, 1), dtype=torch.int32, device=dev) if debug else None
    ctx = default_context(device)
    with ctx._lock:
        rc = _lib.load().pq_scrublet_scores_device(
            ctx._h, S, p, nc.ctypes.data, ns.ctypes.data, kk.ctypes.data, du.data_ptr(),
            dw.data_ptr(), dt_.data_ptr(), dmv.data_ptr(),
            None if dpr is None else dpr.data_ptr(), float(rho), so.data_ptr(), ss.data_ptr(),
            kadj.ctypes.data, None if pts is None else pts.data_ptr(),
            None if knn is None else knn.data_ptr(), None)
        if rc == _lib.PQ_EINVAL:
            msg = _lib.load().pq_ctx_last_error(ctx._h).decode(errors="replace")
            raise ValueError(f"scrublet_scores: {msg}")
        ctx._check(rc, "scrublet_scores")
    torch.cuda.synchronize(dev)
    so, ss = so.cpu().numpy(), ss.cpu().numpy()
    out, a, b, pa, ka = [], 0, 0, 0, 0
    knn_h = knn.cpu().numpy().view(np.uint32) if debug else None
    pts_h = pts.cpu().numpy() if debug else None
    for s in range(S):
        n, m, k = int(nc[s]), int(ns[s]), int(kadj[s])
        r = {"obs": so[a:a + n], "sim": ss[b:b + m], "k_adj": k}
        if debug:
            r["points"] = pts_h[pa:pa + n + m]
            r["knn"] = knn_h[ka:ka + (n + m) * k].reshape(n + m, k)
        out.append(r)
        a, b, pa, ka = a + n, b + m, pa + n + m, ka + (n + m) * k
    return out


def shard_samples(sizes, world: int) -> list:
    """The samples each of `world` ranks takes: every sample whole (its
    search needs all of its points), largest cost (points squared) first, to
    the rank with the least cost so far (ties to the lower rank).  A list of
    ascending sample indices per rank; deterministic, so every rank computes
    the same split without communication."""
    order = sorted(range(len(sizes)), key=lambda s: (-int(sizes[s]) ** 2, s))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(s)
        load[r] += int(sizes[s]) ** 2
    return [sorted(p) for p in parts]


def knn_batched_sharded(samples, ks, *, rank: int, world: int, device: int = 0,
                        gather: bool = True, autotune: bool = False, graph: bool = True,
                        _compute=None):
    """knn_batched over `world` GPUs (one process per GPU, torch.distributed
    initialised): the samples are split whole between the ranks
    (shard_samples) and each rank searches its share in one persistent
    launch; no collective touches the search itself.  With `gather`, the
    results are exchanged once at the end (all_gather_object) and every rank
    returns the full list in sample order; else a dict {sample: (indices,
    distances)} of its own share."""
    parts = shard_samples([len(a) for a in samples], world)
    mine = parts[rank]
    run = _compute if _compute is not None else (
        lambda xs, kk: knn_batched(xs, kk, device=device, autotune=autotune, graph=graph))
    local = dict(zip(mine, run([samples[s] for s in mine], [ks[s] for s in mine]))) if mine else {}
    if not gather or world == 1:
        return local if not gather else [local[s] for s in range(len(samples))]
    import torch.distributed as dist

    allparts = [None] * world
    dist.all_gather_object(allparts, local)
    merged = {}
    for part in allparts:
        merged.update(part)
    return [merged[s] for s in range(len(samples))]


def neighbors_dense(embedding, n_neighbors, metric, *, device: int = 0) -> dict:
    """Exact kNN graph, bit-exact with the reference's ``neighbors_dense``
    (crates/polariseq-python/src/lib.rs:474-501, neighbors.rs:101-241).

    Every cell searches its ``min(n_neighbors, n_obs)`` nearest including
    itself; the closest is dropped, so each row holds ``min(n_neighbors,
    n_obs) - 1`` entries, ascending.  ``metric`` is ``"euclidean"`` (distances
    are sqrt of the squared distance) or ``"cosine"`` (1 - cosine similarity),
    case-insensitive.  Returns ``{"indptr", "indices", "data", "n_obs"}``."""
    if not isinstance(embedding, np.ndarray) or embedding.ndim != 2:
        raise TypeError("argument 'embedding': expected a 2-D numpy.ndarray of float32")
    if embedding.dtype != np.float32:
        raise TypeError(f"argument 'embedding': expected float32, got {embedding.dtype}")
    m = METRICS.get(str(metric).lower())
    if m is None:
        raise RuntimeError(f"unknown metric: {metric}")
    emb = np.ascontiguousarray(embedding)  # the binding copies the array (lib.rs:484)
    n_obs = emb.shape[0]
    kws = min(int(n_neighbors), n_obs)
    nnz_cap = max(n_obs * max(kws - 1, 0), 1)
    ip = np.zeros(n_obs + 1, np.uint32)
    ix = np.zeros(nnz_cap, np.uint32)
    dx = np.zeros(nnz_cap, np.float32)
    nnz = default_context(device).neighbors_into(emb, int(n_neighbors), m, ip, ix, dx)
    return {"indptr": ip, "indices": ix[:nnz], "data": dx[:nnz], "n_obs": n_obs}


def nndescent(data: np.ndarray, k: int = 15, *, max_candidates=0, max_iterations=0, delta=0.001,
              n_trees=0, leaf_size=0, gather_max=0, seed=0, device: int = 0,
              mode: str = "plain", init: str = "rp", probes: int = 0,
              refine_rounds: int = -1) -> dict:
    """The Rust-level ``nndescent(data, n_obs, n_dim, &NndescentOptions)``
    (nndescent.rs:657-686) with every option, returning the NeighborGraph
    fields (indptr, indices, data, n_obs)."""
    emb = _as_embedding(data)
    n_obs = emb.shape[0]
    if n_obs == 0 or emb.shape[1] == 0:
        raise PanicException("empty data")
    if int(k) == 0:
        raise PanicException("k must be >= 1")
    opts = _opts(k, max_iterations, seed, max_candidates, n_trees, delta, leaf_size, gather_max,
                 mode=MODES[mode], init=INITS[init], probes=probes, refine_rounds=refine_rounds)
    cap = n_obs * effective_k(n_obs, k)
    ip = np.zeros(n_obs + 1, np.uint32)
    ix = np.zeros(cap, np.uint32)
    dx = np.zeros(cap, np.float32)
    nnz = default_context(device).nndescent_into(emb, opts, ip, ix, dx)
    return {"indptr": ip, "indices": ix[:nnz], "data": dx[:nnz], "n_obs": n_obs}
