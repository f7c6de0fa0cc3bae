// Order-preserving device primitives: exclusive scan and a stable LSD radix
// sort of (u32 key, u64 value) pairs.  The stable sort is what lets a whole
// round of updates be generated in parallel and then replayed per destination
// row in the reference's generation order (nndescent.rs:307-324 applies each
// destination's updates chunk by chunk, i.e. in generation order).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pq {

// Bytes of temporary storage scan_exclusive_u32 needs for n elements.
size_t scan_temp_bytes(size_t n);
// out[i] = sum(in[0..i)); *total_dev (may be null) receives the u64 total.
// `in` and `out` may alias.  Returns a cudaError_t.
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, void* temp,
                               uint64_t* total_dev, cudaStream_t st);
// The same over u64 values.
cudaError_t scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, void* temp,
                               uint64_t* total_dev, cudaStream_t st);

// Bytes of temporary storage radix_sort_pairs needs for n pairs.
size_t radix_temp_bytes(size_t n);
// Stable sort of (keys, vals) by the low `key_bits` bits of the keys.  The
// sorted result ends in (keys, vals) (the alternate buffers are scratch of
// the same sizes).
cudaError_t radix_sort_pairs(uint32_t* keys, uint64_t* vals, uint32_t* keys_alt,
                             uint64_t* vals_alt, size_t n, int key_bits, void* temp,
                             cudaStream_t st);

}  // namespace pq
