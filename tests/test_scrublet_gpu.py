"""Doublet scoring after PCA on the GPU (Scrublet's score_batch,
crates/polariseq-core/src/doublets.rs:1040-1127) against a NumPy
restatement of the same steps.

The points are f32 from f64 arithmetic in the reference's order, so they are
compared bit for bit; the kNN is exact in FP32 and is compared as exact
(distance, index) sets against an FP64 brute force (as the batched search's
own tests do); the scores are compared bit for bit with the reference's
formula evaluated on the returned neighbours, and their k_adj with
round_half_even(k (1 + n_sim / n)).
"""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def round_half_even(x):
    """doublets.rs:477-485 (numpy's round)."""
    return max(int(np.round(x)), 0)


def make_sample(rng, n, p, ratio):
    u = rng.normal(size=(n, p))
    totals = rng.uniform(800.0, 6000.0, size=n)
    w = 1e6 / totals
    mv = rng.normal(size=p) * 50.0
    m = int(n * ratio)
    pairs = rng.integers(0, n, size=(m, 2)).astype(np.uint32)
    return u, w, totals, mv, pairs


def points_ref(u, w, totals, mv, pairs):
    cells = (w[:, None] * u - mv[None, :]).astype(np.float32)
    x, y = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64)
    s = 1e6 / (totals[x] + totals[y])
    dbl = (s[:, None] * (u[x] + u[y]) - mv[None, :]).astype(np.float32)
    return np.concatenate([cells, dbl])


def score_ref(knn, n, k_adj, ratio, rho):
    nd = (knn >= n).sum(1).astype(np.float64)
    q = (nd + 1.0) / (float(k_adj) + 2.0)
    a = 1.0 - rho
    return q * rho / ratio / (a - q * (a - rho / ratio))


def test_scrublet_scores_match_the_reference_steps():
    import polariseq_b200 as pq

    rng = np.random.default_rng(12)
    # (cells, doublets per cell, k): every sample has p = 30 components
    specs = [(300, 2.0, 8), (1200, 2.0, 17), (75, 1.5, 4), (2000, 2.0, 22)]
    samples = [make_sample(rng, n, 30, r) for n, r, _ in specs]
    ks = [k for *_, k in specs]
    rho = 0.06
    out = pq.scrublet_scores([s[0] for s in samples], [s[1] for s in samples],
                             [s[2] for s in samples], [s[3] for s in samples],
                             [s[4] for s in samples], ks, rho, debug=True)
    for (u, w, t, mv, pairs), k, r in zip(samples, ks, out):
        n, m = len(u), len(pairs)
        ratio = m / n
        k_adj = min(max(round_half_even(k * (1 + ratio)), 1), n + m - 1)
        assert r["k_adj"] == k_adj
        pts = points_ref(u, w, t, mv, pairs)
        assert r["points"].tobytes() == pts.tobytes(), "points differ from the f64 steps"
        ex, _ = oracle.exact_knn_f64(pts, np.arange(n + m, dtype=np.uint32), k_adj)
        same = np.mean([len(set(r["knn"][i]) & set(ex[i])) / k_adj for i in range(n + m)])
        assert same >= 0.999, same
        sc = score_ref(r["knn"], n, k_adj, ratio, rho)
        assert r["obs"].tobytes() == sc[:n].tobytes()
        assert r["sim"].tobytes() == sc[n:].tobytes()


def test_scrublet_scores_reject_bad_inputs():
    import polariseq_b200 as pq

    rng = np.random.default_rng(1)
    u, w, t, mv, pairs = make_sample(rng, 50, 8, 2.0)
    with pytest.raises(ValueError):
        pq.scrublet_scores([u], [w], [t], [mv], [pairs], [5], rho=1.5)
    with pytest.raises(ValueError):
        pq.scrublet_scores([u], [w], [t], [mv], [pairs], [0], rho=0.1)
