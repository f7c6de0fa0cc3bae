"""Generates tests/golden/nndescent_golden.npz from the CPU oracle.

The reference (Rust) cannot be built in this environment and ships no
NN-Descent golden vectors, so these fixtures record the oracle's graphs on
small seeded inputs (the reference unit tests' clustered generator,
nndescent.rs:1012-1022, on numpy's PCG64): they pin the oracle against
regressions and give the GPU tests a fixed expected output.

Run: python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from polariseq_b200 import synth  # noqa: E402

# name: (n, d, k, seed, generator seed, clusters)
CASES = {
    "caller_arrays": (1500, 6, 9, 5, 3, 4),
    "tail13": (700, 13, 7, 1, 2, 3),
    "pcs50": (600, 50, 15, 0, 0, 20),
    "tiny": (5, 3, 10, 0, 0, 2),
}


def main():
    out = {}
    for name, cfg in CASES.items():
        n, d, k, seed, gs, ncl = cfg
        data = synth.blobs_rust_tests(n, d, ncl, gs)
        g = oracle.nndescent(data, k, seed=seed)
        out[name + "__cfg"] = np.array(cfg, np.int64)
        out[name + "__data"] = data
        out[name + "__indptr"] = g["indptr"]
        out[name + "__indices"] = g["indices"]
        out[name + "__dists"] = g["data"]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nndescent_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
