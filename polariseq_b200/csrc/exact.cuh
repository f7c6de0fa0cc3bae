// Exact brute-force kNN (neighbors::neighbors) launch interface.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pq {

constexpr int EXACT_MAX_DIM = 512;  // n_dim limit of the staged-tile kernel
constexpr int EXACT_MAX_K = 256;    // k_with_self limit (per-warp shared-memory heap)

size_t exact_knn_smem(int d, int kws);
// Loads the kernels and raises their shared-memory limit on the current
// device (once per device, before the first launch).
cudaError_t exact_knn_prepare();
// Enqueues the search on `st`: indptr (n+1), indices / dists (n * (kws-1)).
// `norms` (n floats) is scratch for the cosine metric (unused for Euclidean);
// every element the kernels read is written first in the same launch sequence.
cudaError_t launch_exact_knn(const float* X, uint64_t n, int d, int kws, int cosine,
                             float* norms, uint32_t* indptr, uint32_t* indices, float* dists,
                             cudaStream_t st);

}  // namespace pq
