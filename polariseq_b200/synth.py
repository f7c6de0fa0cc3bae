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


def doublet_samples(count: int = 64, lo: int = 2000, hi: int = 60000, genes: int = 2000,
                    d: int = 30, comps: int = 10, seed: int = 0, device: str = "cuda"):
    """Per-sample embeddings of the doublet-scoring workload: each sample has
    n_s cells (log-uniform in [lo, hi]) from a `comps`-component mixture of
    negative-binomial counts (r = 2, gene means log-normal) plus 2 n_s
    simulated doublets (sums of two random parent cells' counts), all
    log1p-normalised (counts per 10^4) and projected by one seeded random
    orthonormal genes x d basis.  Generated on the GPU with torch; returns a
    list of float32 numpy arrays of 3 n_s rows."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).round().astype(int)
    basis, _ = torch.linalg.qr(torch.randn(genes, d, generator=g, device=device))
    base = torch.exp(torch.randn(genes, generator=g, device=device)) * 0.5
    out = []
    for n in sizes:
        w = torch.from_numpy(rng.dirichlet(np.ones(comps))).float().to(device)
        mu = base[None, :] * torch.exp(0.5 * torch.randn(comps, genes, generator=g, device=device))
        comp = torch.multinomial(w, int(n), replacement=True, generator=g)
        parts = []
        cells = []
        for c0 in range(0, int(n), 8192):
            m = mu[comp[c0:c0 + 8192]]
            lam = torch._standard_gamma(torch.full_like(m, 2.0), generator=g) * (m / 2.0)
            cells.append(torch.poisson(lam, generator=g))
        cells = torch.cat(cells)
        pa = torch.randint(0, int(n), (2 * int(n),), generator=g, device=device)
        pb = torch.randint(0, int(n), (2 * int(n),), generator=g, device=device)
        for c0 in range(0, 3 * int(n), 8192):
            idx = torch.arange(c0, min(c0 + 8192, 3 * int(n)), device=device)
            cnt = torch.where((idx < n)[:, None], cells[idx.clamp(max=int(n) - 1)],
                              cells[pa[(idx - n).clamp(min=0, max=2 * int(n) - 1)]] +
                              cells[pb[(idx - n).clamp(min=0, max=2 * int(n) - 1)]])
            tot = cnt.sum(1, keepdim=True).clamp(min=1.0)
            parts.append(torch.log1p(cnt / tot * 1e4) @ basis)
        out.append(torch.cat(parts).float().cpu().numpy())
    return out
