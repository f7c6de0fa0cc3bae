"""ORACLE — test infrastructure only, never shipped and never on the product path.

A float64 NumPy restatement of the learned-routing MLP's forward and backward
pass (polariseq_b200/csrc/mlp.cu): d -> 256 -> 256 -> 1024 with ReLU, weights
and the products' activation / gradient operands rounded to BF16 (round to
nearest even) and biases kept in FP32 as on the GPU, softmax cross-entropy
against sparse soft targets, gradients of the mean loss with respect to the
FP32 master parameters (the BF16 rounding is passed straight through).  The
MLP has no counterpart in the reference; this is the CPU check of the
hand-written CUDA kernels' gradients.
"""

import numpy as np

H, OUT = 256, 1024


def layout(d):
    sizes = [d * H, H, H * H, H, H * OUT, OUT]
    offs = np.cumsum([0] + sizes)
    return [(int(offs[i]), int(offs[i + 1])) for i in range(6)]


def bf16(a):
    """Round float32 values to BF16 (nearest even), returned as float64."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, d, round_weights=True):
    (a1, e1), (a2, e2), (a3, e3), (a4, e4), (a5, e5), (a6, e6) = layout(d)
    p = np.asarray(params, np.float32)
    w = (lambda x: bf16(x)) if round_weights else (lambda x: x.astype(np.float64))
    return (w(p[a1:e1]).reshape(d, H), p[a2:e2].astype(np.float64),
            w(p[a3:e3]).reshape(H, H), p[a4:e4].astype(np.float64),
            w(p[a5:e5]).reshape(H, OUT), p[a6:e6].astype(np.float64))


def forward_backward(params, X, tb, tw, round_weights=True, round_acts=None):
    """Returns (grad [params], loss per row, logits).

    round_acts (default: as round_weights) rounds every activation and output
    gradient to BF16 where it feeds a product, as the tensor-core kernels do:
    X, H1 and H2 as forward operands, dZ, dH2 and dH1 as backward operands
    (the ReLU masks and the bias gradients use the unrounded values)."""
    if round_acts is None:
        round_acts = round_weights
    rnd = bf16 if round_acts else (lambda a: a)
    X = np.asarray(X, np.float64)
    rows, d = X.shape
    W1, b1, W2, b2, W3, b3 = unpack(params, d, round_weights)
    Xr = rnd(X)
    H1 = np.maximum(Xr @ W1 + b1, 0)
    H1r = rnd(H1)
    H2 = np.maximum(H1r @ W2 + b2, 0)
    H2r = rnd(H2)
    Z = H2r @ W3 + b3
    T = np.zeros_like(Z)
    for r in range(rows):
        for b, w in zip(tb[r], tw[r]):
            if b != 0xFFFFFFFF:
                T[r, b] += w
    m = Z.max(1, keepdims=True)
    lse = m[:, 0] + np.log(np.exp(Z - m).sum(1))
    loss = lse - (T * Z).sum(1)
    dZ = (np.exp(Z - lse[:, None]) - T) / rows
    dZr = rnd(dZ)
    gW3 = H2r.T @ dZr
    gb3 = dZ.sum(0)
    dH2 = (dZr @ W3.T) * (H2 > 0)
    dH2r = rnd(dH2)
    gW2 = H1r.T @ dH2r
    gb2 = dH2.sum(0)
    dH1 = (dH2r @ W2.T) * (H1 > 0)
    gW1 = Xr.T @ rnd(dH1)
    gb1 = dH1.sum(0)
    grad = np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return grad, loss, Z
