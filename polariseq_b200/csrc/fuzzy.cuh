// Fuzzy simplicial set of a device kNN distance graph (fuzzy.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pq {

size_t fuzzy_temp_bytes(uint64_t n, uint64_t nnz);
// Writes the symmetric CSR (row pointers n + 1, at most out_cap entries) and
// *h_nnz; synchronises `st` once between the counting and the writing pass.
// cudaErrorNotSupported: a row of the input has more than 256 entries;
// cudaErrorInvalidValue: the result needs more than out_cap entries.
cudaError_t launch_fuzzy(uint64_t n, uint64_t nnz, const uint32_t* indptr, const uint32_t* indices,
                         const float* data, uint8_t* temp, uint32_t* out_indptr,
                         uint32_t* out_indices, float* out_weights, uint64_t out_cap,
                         uint64_t* d_total, int* d_err, uint64_t* h_nnz, cudaStream_t st);

}  // namespace pq
