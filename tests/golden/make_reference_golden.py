"""Generates tests/golden/reference_inputs_golden.npz with the literal Python
restatement of the reference (oracle/nndescent_literal.py), which shares no
code with the C++ oracle or the CUDA kernels.

The inputs are the reference unit tests' own (nndescent.rs:1012-1022:
make_clustered_data on ChaCha8Rng::seed_from_u64, restated from the published
rand / rand_chacha algorithms) with the tests' sizes, options and seeds, where
the pure-Python restatement finishes in seconds:

  caller_arrays  writing_into_caller_arrays_gives_the_same_graph (1500 x 6, 4
                 clusters, data seed 3, k = 9, seed 5)
  tiny           tiny_inputs_work (5 x 3, 2 clusters, data seed 0, k = 10)
  structure_1k   the structure test's generator (5 clusters, data seed 1, k =
                 10, seed 1) at 1,000 cells

Run: python tests/golden/make_reference_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import nndescent_literal as lit  # noqa: E402

# name: (n, d, clusters, data seed, k, seed)
CASES = {
    "caller_arrays": (1500, 6, 4, 3, 9, 5),
    "tiny": (5, 3, 2, 0, 10, 0),
    "structure_1k": (1000, 8, 5, 1, 10, 1),
}


def main():
    out = {}
    for name, cfg in CASES.items():
        n, d, ncl, ds, k, seed = cfg
        data = lit.make_clustered_data(n, d, ncl, ds)
        g = lit.nndescent(data, k, seed=seed)
        out[name + "__cfg"] = np.array(cfg, np.int64)
        out[name + "__data"] = data
        out[name + "__indptr"] = g["indptr"]
        out[name + "__indices"] = g["indices"]
        out[name + "__dists"] = g["data"]
        out[name + "__changed"] = np.array(g["round_changed"], np.int64)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "reference_inputs_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
