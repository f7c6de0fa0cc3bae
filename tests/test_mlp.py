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
    # FP32 accumulation against FP64: relative error per parameter block
    np.testing.assert_allclose(z, ref_z, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(loss, ref_loss, rtol=1e-5, atol=1e-5)
    for (a, e) in mlp_ref.layout(d):
        err = np.max(np.abs(g[a:e] - ref_g[a:e])) / (np.max(np.abs(ref_g[a:e])) + 1e-30)
        assert err < 1e-3, (a, e, err)


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
