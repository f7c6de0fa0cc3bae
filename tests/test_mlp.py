"""Learned routing MLP: the CPU oracle's gradients against finite differences
(CPU), and the hand-written CUDA forward/backward kernels against the oracle
(GPU), then what the trained router gains over nearest-centroid probes (GPU).
"""

import ctypes as C

import numpy as np
import pytest

from oracle import mlp_ref


def small_problem(d=50, rows=64, T=16, seed=0):
    rng = np.random.default_rng(seed)
    n = sum(e - a for a, e in mlp_ref.layout(d))
    params = (rng.normal(size=n) * 0.05).astype(np.float32)
    X = rng.normal(size=(rows, d)).astype(np.float32)
    tb = np.full((rows, T), 0xFFFFFFFF, np.uint32)
    tw = np.zeros((rows, T), np.float32)
    for r in range(rows):
        m = rng.integers(1, T + 1)
        b = rng.choice(mlp_ref.OUT, size=m, replace=False)
        w = rng.random(m)
        tb[r, :m] = b
        tw[r, :m] = w / w.sum()
    return params, X, tb, tw


def test_oracle_gradients_match_finite_differences():
    params, X, tb, tw = small_problem(d=6, rows=5, T=4)
    g, loss, _ = mlp_ref.forward_backward(params, X, tb, tw, round_weights=False)
    p64 = params.astype(np.float64)
    rng = np.random.default_rng(1)
    for i in rng.choice(len(params), 40, replace=False):
        e = 1e-6
        a, b = p64.copy(), p64.copy()
        a[i] += e
        b[i] -= e
        la = mlp_ref.forward_backward(a, X, tb, tw, round_weights=False)[1].mean()
        lb = mlp_ref.forward_backward(b, X, tb, tw, round_weights=False)[1].mean()
        fd = (la - lb) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


@pytest.mark.gpu
def test_cuda_gradients_match_oracle():
    import polariseq_b200 as pq
    from polariseq_b200 import _lib

    d, rows, T = 50, 300, 16
    params, X, tb, tw = small_problem(d=d, rows=rows, T=T, seed=3)
    ref_g, ref_loss, ref_z = mlp_ref.forward_backward(params, X, tb, tw)
    L = _lib.load()
    assert L.pq_mlp_params(d) == params.size
    g = np.zeros(params.size, np.float32)
    loss = np.zeros(rows, np.float32)
    z = np.zeros((rows, mlp_ref.OUT), np.float32)
    ctx = pq.default_context(0)
    rc = L.pq_mlp_grad(ctx._h, d, params.ctypes.data, X.ctypes.data, rows, tb.ctypes.data,
                       tw.ctypes.data, T, g.ctypes.data, loss.ctypes.data, z.ctypes.data)
    assert rc == 0
    # tensor-core products (BF16 operands, FP32 accumulation) against the FP64
    # oracle that rounds the same operands to BF16: what remains is the FP32
    # accumulation and the odd operand that rounds to the other BF16
    # neighbour (its FP32 and FP64 values straddle a rounding boundary).
    # Tolerances: logits 2e-3 (relative and absolute), per-row loss 1e-3, each
    # parameter block's gradient 5e-3 of its largest entry.
    np.testing.assert_allclose(z, ref_z, rtol=2e-3, atol=2e-3)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-3, atol=1e-3)
    for (a, e) in mlp_ref.layout(d):
        err = np.max(np.abs(g[a:e] - ref_g[a:e])) / (np.max(np.abs(ref_g[a:e])) + 1e-30)
        assert err < 5e-3, (a, e, err)


@pytest.mark.gpu
def test_learned_router_training_and_recall():
    """What the trained network gains over the method without it: the router
    starts as the nearest-centroid prior (first-epoch loss) and training lowers
    the cross-entropy to where a cell's neighbours live; with the same 1024
    k-means buckets and probe count, its probes keep the nearest-centroid
    probes' recall (on Gaussian-mixture embeddings, where the centroid ranking
    is already close to the neighbour-bucket ranking, the recall gain is small)."""
    import torch

    import polariseq_b200 as pq
    from bench import recall_fp64
    from polariseq_b200 import synth

    n, k, P = 400_000, 15, 6
    x = synth.mixture_lognormal(n, 50, 40, seed=21)
    xd = torch.from_numpy(x).cuda()
    ctx = pq.default_context(0)

    def run(init):
        g = pq.nndescent_dense(x, k, mode="bf16", init=init, probes=P, refine_rounds=0,
                               buckets=1024)
        return recall_fp64(torch, xd, g["indices"], g["data"], k, 4000)[0], ctx.stats()

    base, _ = run("rp")
    learned, st = run("learned")
    assert st["learn_loss_last"] < st["learn_loss_first"] - 0.01, st
    assert learned > base - 0.01, (learned, base)


@pytest.mark.gpu
def test_learned_init_nndescent_gains_over_rp_init():
    """The learned-init NN-Descent against the method without it, the
    reference's RP-forest initialisation, under the same NN-Descent options:
    the router's top buckets give initial lists (exact within those buckets)
    from which the reference's rounds converge in fewer rounds to a higher
    recall@15 against FP64.  The sampled recall estimate the fallback decides
    on agrees with FP64, and the fallback ran exactly when it fell below
    0.99 (keeping the learned graph, whose estimate is the higher)."""
    import torch

    import polariseq_b200 as pq
    from bench import recall_fp64
    from polariseq_b200 import synth

    n, k = 1_000_000, 15
    x = synth.mixture_lognormal(n, 50, 40, seed=23)
    xd = torch.from_numpy(x).cuda()
    ctx = pq.default_context(0)

    def run(init):
        g = pq.nndescent_dense(x, k, init=init)
        return recall_fp64(torch, xd, g["indices"], g["data"], k, 4000)[0], ctx.stats()

    rec_rp, st_rp = run("rp")
    rec_l, st_l = run("learned")
    assert st_l["learned_rounds"] < st_rp["rounds_run"], (st_l["learned_rounds"],
                                                          st_rp["rounds_run"])
    assert rec_l > rec_rp + 0.02, (rec_l, rec_rp)
    assert abs(st_l["est_recall_learned"] - rec_l) < 0.01, (st_l["est_recall_learned"], rec_l)
    assert (st_l["fell_back"] == 0) == (st_l["est_recall_learned"] >= 0.99), st_l
    assert st_l["fell_back"] in (0, 1), st_l


@pytest.mark.gpu
def test_learned_init_falls_back_to_rp_init(monkeypatch):
    """Below the recall target (forced here above 1) the RP-initialised build
    runs too, and the graph with the higher sampled recall is kept: the
    result is byte for byte one of the two builds, the one its statistics
    name."""
    import polariseq_b200 as pq
    from polariseq_b200 import synth

    n, k = 100_000, 15
    x = synth.mixture_lognormal(n, 50, 20, seed=29)
    ctx = pq.default_context(0)
    rp = pq.nndescent_dense(x, k, max_iterations=2)
    learned = pq.nndescent_dense(x, k, max_iterations=2, init="learned")
    monkeypatch.setenv("POLARISEQ_LEARNED_MIN_RECALL", "2")
    got = pq.nndescent_dense(x, k, max_iterations=2, init="learned")
    st = ctx.stats()
    assert st["fell_back"] in (1, 2)
    assert st["est_recall_rp"] > 0
    want = rp if st["fell_back"] == 2 else learned
    assert st["est_recall"] == max(st["est_recall_rp"], st["est_recall_learned"])
    np.testing.assert_array_equal(got["indptr"], want["indptr"])
    np.testing.assert_array_equal(got["indices"], want["indices"])
    assert got["data"].tobytes() == want["data"].tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("d", [50, 48])
def test_sampled_recall_matches_an_exact_count(d):
    """The sampled recall the fallback decides on (1,024 evenly strided cells
    from a seeded offset, their exact k nearest against all cells) equals the
    count of the graph's hits among the FP64 k nearest of the same cells, up
    to FP32-vs-FP64 order at the boundary.  d = 50 runs the register-row scan,
    d = 48 the shared-memory one."""
    import oracle
    import polariseq_b200 as pq
    from polariseq_b200 import synth

    n, k, seed = 70_000, 15, 7
    x = synth.mixture_lognormal(n, d, 20, seed=31)
    g = pq.nndescent_dense(x, k, init="learned", seed=seed)
    st = pq.default_context(0).stats()
    Q = 1024
    off = oracle.splitmix(seed ^ 0x5A4D504C) % n
    q = np.array([(off + t * n // Q) % n for t in range(Q)], np.uint32)
    want, _ = oracle.exact_knn_f64(x, q, k)
    ip, ix = g["indptr"], g["indices"]
    hits = sum(len(set(ix[ip[i]:ip[i + 1]].tolist()) & set(want[t].tolist()))
               for t, i in enumerate(q.tolist()))
    est = hits / (Q * k)
    # est_recall is the estimate of the graph returned (learned, or the RP
    # build's when the fallback kept that)
    assert abs(st["est_recall"] - est) <= 5e-4, (st["est_recall"], est)
