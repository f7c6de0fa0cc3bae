// Fuzzy simplicial set (scanpy's obsp['connectivities']) of a kNN distance
// graph held on the device: umap.rs:283-620 (fuzzy_connectivities_from).
//
//   1. membership strengths, one thread per row: smooth_knn_dist in f64 (the
//      64-step bisection of sigma, rho = the nearest non-zero distance, floor
//      at 1e-3 x the mean distance including the self distance), weights cast
//      to f32;
//   2. the transpose: a stable radix sort of the edges by target, so that row
//      j of the transpose lists its sources in increasing order, as the
//      reference's counting sort does;
//   3. each symmetric row by merging the row's own entries (sorted by column
//      in registers) with its transposed entries, folding equal columns with
//      the fuzzy union acc + w - acc * w in f32 (own entries first) and
//      pruning at 1e-5; one pass counts the rows, an exclusive scan gives the
//      row pointers, a second pass writes them.
// The f32 arithmetic is separately rounded (no FMA), as in the reference; the
// f64 exp of CUDA and of the host C library may differ in the last bit, so
// weights are compared with a tolerance.
#include <cuda_runtime.h>

#include "common.cuh"
#include "fuzzy.cuh"
#include "primitives.cuh"

namespace pq {
namespace {

constexpr int ROW_MAX = 256;  // own entries per row merged in registers/local memory

__global__ void k_strengths(const uint32_t* __restrict__ indptr, const float* __restrict__ data,
                            uint64_t n, float* __restrict__ w) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = indptr[i], e = indptr[i + 1];
    if (s == e) return;
    const uint32_t len = e - s;
    const double target = log2(double(len + 1));
    double rho = 0.0;
    for (uint32_t t = s; t < e; ++t)
        if (double(data[t]) > 0.0) {
            rho = double(data[t]);
            break;
        }
    double lo = 0.0, hi = __longlong_as_double(0x7ff0000000000000ll), mid = 1.0;
    for (int it = 0; it < 64; ++it) {
        double psum = 0.0;
        for (uint32_t t = s; t < e; ++t) {
            const double x = double(data[t]) - rho;
            psum += x > 0.0 ? exp(-(x / mid)) : 1.0;
        }
        if (fabs(psum - target) < 1e-5) break;
        if (psum > target) {
            hi = mid;
            mid = (lo + hi) / 2.0;
        } else {
            lo = mid;
            mid = isinf(hi) ? mid * 2.0 : (lo + hi) / 2.0;
        }
    }
    double sum = 0.0;
    for (uint32_t t = s; t < e; ++t) sum += double(data[t]);
    const double mean = sum / double(len + 1);
    const double sigma = rho > 0.0 ? fmax(mid, 1e-3 * mean) : mid;
    for (uint32_t t = s; t < e; ++t) {
        const double x = double(data[t]) - rho;
        w[t] = (x <= 0.0 || sigma == 0.0) ? 1.0f : float(exp(-(x / sigma)));
    }
}

__global__ void k_edge_keys(const uint32_t* __restrict__ indices, uint64_t nnz,
                            uint32_t* __restrict__ keys, uint64_t* __restrict__ vals) {
    const uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    keys[e] = indices[e];
    vals[e] = e;
}

__global__ void k_edge_rows(const uint32_t* __restrict__ indptr, uint64_t n,
                            uint32_t* __restrict__ row) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t e = indptr[i]; e < indptr[i + 1]; ++e) row[e] = uint32_t(i);
}

// Row pointers of the transpose from the sorted targets (each entry once).
__global__ void k_bounds(const uint32_t* __restrict__ keys, uint64_t nnz, uint32_t n,
                         uint32_t* __restrict__ off) {
    const uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e > nnz) return;
    const uint32_t lo = e == 0 ? 0u : keys[e - 1] + 1;
    const uint32_t hi = e == nnz ? n : keys[e];
    for (uint32_t v = lo; v <= hi; ++v) off[v] = uint32_t(e);
}

template <bool WRITE>
__global__ void k_merge(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                        const float* __restrict__ w, const uint32_t* __restrict__ t_off,
                        const uint64_t* __restrict__ t_edge, const uint32_t* __restrict__ e_row,
                        uint64_t n, uint32_t* __restrict__ count,
                        const uint32_t* __restrict__ out_off, uint32_t* __restrict__ out_idx,
                        float* __restrict__ out_w, int* __restrict__ err) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = indptr[i], e = indptr[i + 1];
    const uint32_t na = e - s;
    if (na > uint32_t(ROW_MAX)) {
        atomicExch(err, 1);
        return;
    }
    uint32_t oc[ROW_MAX];
    float ow[ROW_MAX];
    // the row's own entries sorted by column (insertion sort; columns are unique)
    for (uint32_t t = 0; t < na; ++t) {
        const uint32_t c = indices[s + t];
        const float v = w[s + t];
        int p = int(t) - 1;
        while (p >= 0 && oc[p] > c) {
            oc[p + 1] = oc[p];
            ow[p + 1] = ow[p];
            --p;
        }
        oc[p + 1] = c;
        ow[p + 1] = v;
    }
    const uint32_t ts = t_off[i], te = t_off[i + 1];
    uint32_t a = 0, b = ts, o = 0;
    const uint32_t base = WRITE ? out_off[i] : 0;
    while (a < na || b < te) {
        const uint32_t tcol = b < te ? e_row[t_edge[b]] : 0xFFFFFFFFu;
        const uint32_t col = (a < na && (b >= te || oc[a] <= tcol)) ? oc[a] : tcol;
        float acc = 0.0f;
        while (a < na && oc[a] == col) {
            acc = __fsub_rn(__fadd_rn(acc, ow[a]), __fmul_rn(acc, ow[a]));
            ++a;
        }
        while (b < te && e_row[t_edge[b]] == col) {
            const float v = w[t_edge[b]];
            acc = __fsub_rn(__fadd_rn(acc, v), __fmul_rn(acc, v));
            ++b;
        }
        if (acc > 1e-5f) {
            if (WRITE) {
                out_idx[base + o] = col;
                out_w[base + o] = acc;
            }
            ++o;
        }
    }
    if (!WRITE) count[i] = o;
}

}  // namespace

size_t fuzzy_temp_bytes(uint64_t n, uint64_t nnz) {
    return nnz * (4 + 8 + 4 + 8 + 4 + 4) + (n + 2) * 4 * 3 + radix_temp_bytes(nnz) +
           scan_temp_bytes(n + 1) + 1024;
}

cudaError_t launch_fuzzy(uint64_t n, uint64_t nnz, const uint32_t* indptr, const uint32_t* indices,
                         const float* data, uint8_t* temp, uint32_t* out_indptr,
                         uint32_t* out_indices, float* out_weights, uint64_t out_cap,
                         uint64_t* d_total, int* d_err, uint64_t* h_nnz, cudaStream_t st) {
    auto carve = [&](size_t bytes) {
        uint8_t* p = temp;
        temp += (bytes + 255) & ~size_t(255);
        return p;
    };
    float* w = reinterpret_cast<float*>(carve(nnz * 4));
    uint32_t* keys = reinterpret_cast<uint32_t*>(carve(nnz * 4));
    uint64_t* vals = reinterpret_cast<uint64_t*>(carve(nnz * 8));
    uint32_t* keys2 = reinterpret_cast<uint32_t*>(carve(nnz * 4));
    uint64_t* vals2 = reinterpret_cast<uint64_t*>(carve(nnz * 8));
    uint32_t* erow = reinterpret_cast<uint32_t*>(carve(nnz * 4));
    uint32_t* t_off = reinterpret_cast<uint32_t*>(carve((n + 1) * 4));
    uint32_t* cnt = reinterpret_cast<uint32_t*>(carve((n + 1) * 4));
    uint8_t* rtemp = carve(radix_temp_bytes(nnz));
    uint8_t* stemp = carve(scan_temp_bytes(n + 1));
    cudaError_t e;
    if ((e = cudaMemsetAsync(d_err, 0, 4, st)) != cudaSuccess) return e;
    const unsigned B = 256;
    k_strengths<<<unsigned((n + B - 1) / B), B, 0, st>>>(indptr, data, n, w); count_launch();
    if (nnz > 0) {
        k_edge_keys<<<unsigned((nnz + B - 1) / B), B, 0, st>>>(indices, nnz, keys, vals);
        count_launch();
        int bits = 0;
        while (bits < 32 && ((n - 1) >> bits) != 0) ++bits;
        if ((e = radix_sort_pairs(keys, vals, keys2, vals2, nnz, bits > 0 ? bits : 1, rtemp, st)) !=
            cudaSuccess)
            return e;
        k_edge_rows<<<unsigned((n + B - 1) / B), B, 0, st>>>(indptr, n, erow); count_launch();
    }
    k_bounds<<<unsigned((nnz + 1 + B - 1) / B), B, 0, st>>>(keys, nnz, uint32_t(n), t_off);
    count_launch();
    k_merge<false><<<unsigned((n + B - 1) / B), B, 0, st>>>(indptr, indices, w, t_off, vals, erow, n,
                                                           cnt, nullptr, nullptr, nullptr, d_err);
    count_launch();
    if ((e = cudaMemsetAsync(cnt + n, 0, 4, st)) != cudaSuccess) return e;
    if ((e = scan_exclusive_u32(cnt, out_indptr, n + 1, stemp, d_total, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h_nnz, d_total, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    int herr = 0;
    if ((e = cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    if (herr) return cudaErrorNotSupported;          // a row with more than ROW_MAX entries
    if (*h_nnz > out_cap) return cudaErrorInvalidValue;
    k_merge<true><<<unsigned((n + B - 1) / B), B, 0, st>>>(indptr, indices, w, t_off, vals, erow, n,
                                                          nullptr, out_indptr, out_indices,
                                                          out_weights, d_err);
    count_launch();
    return cudaGetLastError();
}

}  // namespace pq
