"""Seeded synthetic PCA-like embeddings standing in for the reference's datasets.

No public dataset is needed or available offline; these generators produce the
shapes and value distributions of the workloads the kNN builder is measured on:

* ``mixture_dirichlet`` — n cells x d PCs, a mixture of ``n_comp`` Gaussians with
  Dirichlet(1) weights, means N(0, 4^2) per dimension and per-dimension standard
  deviation j^-0.5 (j = 1..d, a PCA-like spectrum).  20,000 x 50, 20 components,
  seed 0 is the small bit-exactness case.
* ``mixture_lognormal`` — the same spectrum with log-normal(0, 1) cluster sizes
  (normalised) and a fraction of doublet-like cells drawn as midpoints of two
  random cells from different clusters (1.3M x 50 / 40 components, 4M x 50 / 60
  components, 10M x 50 / 100 components).
* ``blobs_rust_tests`` — the clustered inputs of the reference's own unit tests
  (crates/polariseq-core/src/nndescent.rs:1012-1022: cluster*10 + U[0,1)), with a
  numpy PCG64 stream in place of ChaCha8 (the reference's test RNG is a Rust
  crate that is not available here).
* ``mixture25`` — the Python tests' 25-Gaussian mixture
  (python/polariseq/tests/test_neighbors.py:18-23).
"""

from __future__ import annotations

import numpy as np


def _spectrum(d: int) -> np.ndarray:
    return (np.arange(1, d + 1, dtype=np.float64) ** -0.5).astype(np.float32)


def mixture_dirichlet(n: int = 20_000, d: int = 50, n_comp: int = 20, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(n_comp))
    means = rng.normal(0.0, 4.0, size=(n_comp, d)).astype(np.float32)
    lab = rng.choice(n_comp, size=n, p=w)
    x = rng.standard_normal(size=(n, d), dtype=np.float32)
    x *= _spectrum(d)[None, :]
    x += means[lab]
    return np.ascontiguousarray(x, dtype=np.float32)


def mixture_lognormal(n: int, d: int = 50, n_comp: int = 40, seed: int = 0,
                      doublet_frac: float = 0.05, chunk: int = 1 << 20) -> np.ndarray:
    rng = np.random.default_rng(seed)
    sizes = rng.lognormal(0.0, 1.0, size=n_comp)
    w = sizes / sizes.sum()
    means = rng.normal(0.0, 4.0, size=(n_comp, d)).astype(np.float32)
    lab = rng.choice(n_comp, size=n, p=w).astype(np.int32)
    spec = _spectrum(d)
    x = np.empty((n, d), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        blk = rng.standard_normal(size=(e - s, d), dtype=np.float32)
        blk *= spec[None, :]
        blk += means[lab[s:e]]
        x[s:e] = blk
    n_dbl = int(round(doublet_frac * n))
    if n_dbl > 0 and n_comp > 1:
        who = rng.choice(n, size=n_dbl, replace=False)
        a = rng.integers(0, n, size=n_dbl)
        b = rng.integers(0, n, size=n_dbl)
        same = lab[a] == lab[b]
        # redraw b until the two parents come from different clusters
        for _ in range(64):
            if not same.any():
                break
            b[same] = rng.integers(0, n, size=int(same.sum()))
            same = lab[a] == lab[b]
        mid = (x[a].astype(np.float32) + x[b].astype(np.float32)) * np.float32(0.5)
        x[who] = mid
    return x


def blobs_rust_tests(n: int, d: int, n_clusters: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    c = (np.arange(n) % n_clusters).astype(np.float32)[:, None]
    return np.ascontiguousarray(c * 10.0 + rng.random((n, d), dtype=np.float32), np.float32)


def mixture25(n: int, d: int = 30, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centers = rng.normal(size=(25, d)) * 5
    lab = rng.integers(0, 25, size=n)
    return (centers[lab] + rng.normal(size=(n, d))).astype(np.float32)
