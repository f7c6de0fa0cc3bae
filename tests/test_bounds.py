"""The rounding bounds behind the tensor-core form's entry pruning
(polariseq_b200/csrc/chosen.cu, k_prune_keep), checked on the CPU with an
emulation of the tile kernel's arithmetic: rows rounded to BF16 (nearest
even), products accumulated in FP32, the candidate's norm carried as a
BF16 hi + lo pair.

1. Tile distances (rows centred on the probe bucket's centroid):
   d~ >= f(d) with f(t) = t - 2^-6 sqrt(t) a - 2^-15 a^2 - 2^-9 (|q|^2 + |y|^2),
   a = |q| + |y| (q, y the centred rows).
2. Nearest-centroid assignment (rows centred on the global mean, norms u, w):
   |d~ - d| <= 2^-7 sqrt(d) (u + w) + 2^-16 (u + w)^2 + 2^-18 (u^2 + w^2),
   half of the slack the pruning allows.
"""

import numpy as np
import pytest


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def tile_distance(q, y):
    """The tile kernel's squared distance of rows q (query) and y (candidate):
    |q~|^2 - 2 (q~.y~ - (hi + lo) / 2), FP32 accumulation."""
    qb, yb = bf16(q), bf16(y)
    qn = np.float32(np.sum(qb.astype(np.float32) ** 2, dtype=np.float32))
    yn = np.float32(np.sum(yb.astype(np.float32) ** 2, dtype=np.float32))
    hi = bf16(yn)
    lo = bf16(np.float32(yn - hi))
    acc = np.float32(0.0)
    for a, b in zip(qb, yb):
        acc = np.float32(acc + np.float32(a) * np.float32(b))
    acc = np.float32(acc - np.float32(0.5) * hi - np.float32(0.5) * lo)
    return float(np.float32(qn - np.float32(2.0) * acc))


@pytest.mark.parametrize("scale", [0.1, 1.0, 10.0])
def test_tile_distance_lower_bound(scale):
    rng = np.random.default_rng(7)
    worst = np.inf
    for _ in range(400):
        d = 50
        q = (rng.normal(0, scale, d) * rng.uniform(0.2, 3.0)).astype(np.float32)
        y = (q + rng.normal(0, scale * rng.uniform(0.01, 2.0), d)).astype(np.float32)
        exact = float(np.sum((q.astype(np.float64) - y) ** 2))
        qq, yy = float(np.sum(q.astype(np.float64) ** 2)), float(np.sum(y.astype(np.float64) ** 2))
        a = np.sqrt(qq) + np.sqrt(yy)
        f = exact - 2 ** -6 * np.sqrt(exact) * a - 2 ** -15 * a * a - 2 ** -9 * (qq + yy)
        approx = tile_distance(q, y)
        assert approx >= f, (approx, f, exact)
        worst = min(worst, approx - f)
    assert worst >= 0.0


@pytest.mark.parametrize("offset", [0.0, 5.0, 30.0])
def test_assignment_error_bound(offset):
    """Global-mean-centred rows far from the origin (offset) make the rounding
    error large relative to the distance; the bound must still hold."""
    rng = np.random.default_rng(11)
    for _ in range(400):
        d = 50
        centre = rng.normal(0, 1, d) * offset / np.sqrt(d)
        u = (centre + rng.normal(0, 1, d)).astype(np.float32)
        w = (u + rng.normal(0, rng.uniform(0.05, 3.0), d)).astype(np.float32)
        exact = float(np.sum((u.astype(np.float64) - w) ** 2))
        un, wn = float(np.linalg.norm(u.astype(np.float64))), float(np.linalg.norm(w.astype(np.float64)))
        approx = tile_distance(u, w)
        err = 2 ** -7 * np.sqrt(exact) * (un + wn) + 2 ** -16 * (un + wn) ** 2 + 2 ** -18 * (un * un + wn * wn)
        assert abs(approx - exact) <= err, (approx, exact, err)


def test_magic_remainder_of_the_warp_split_draws():
    """The one-warp RP splits (polariseq_b200/csrc/forest.cu, draw_pair_la)
    take x mod n for node sizes n < 2^16 from m = floor((2^32 - 1) / n):
    q = floor(x m / 2^32) is floor(x / n) or one below, so one conditional
    subtraction gives the remainder; a 64-bit draw is reduced as
    ((hi mod n) * (2^32 mod n) + lo mod n) mod n.  Checked here against
    Python's % for every n below 2^16 on edge and random 64-bit draws."""
    rng = np.random.default_rng(7)
    n = np.arange(2, 1 << 16, dtype=np.uint64)[:, None]
    m = np.uint64(0xFFFFFFFF) // n
    x = np.concatenate([
        np.array([0, 1, 0xFFFFFFFF, 0x100000000, 0xFFFFFFFFFFFFFFFF], np.uint64),
        rng.integers(0, 1 << 63, 27, dtype=np.uint64) * np.uint64(2)
        + rng.integers(0, 2, 27, dtype=np.uint64)])[None, :]

    def mod_magic(v):
        r = v - ((v * m) >> np.uint64(32)) * n
        return np.where(r >= n, r - n, r)

    r1 = np.uint64(0xFFFFFFFF) - m * n + np.uint64(1)
    t32 = np.where(r1 == n, np.uint64(0), r1)
    assert np.array_equal(t32, np.uint64(1 << 32) % n)
    lo32 = np.uint64(0xFFFFFFFF)
    hi = mod_magic(x >> np.uint64(32))
    lo = mod_magic(x & lo32)
    got = mod_magic(hi * t32 + lo)
    want = np.array([[int(xv) % int(nv) for xv in x[0]] for nv in n[:, 0]], np.uint64)
    assert np.array_equal(got, want)
