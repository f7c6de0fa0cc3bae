// Exact brute-force kNN: neighbors::neighbors (crates/polariseq-core/src/
// neighbors.rs:101-147) bit for bit.
//
// For every query cell the reference scans all cells j = 0..n-1 in order,
// keeps a bounded max-heap of k_with_self = min(n_neighbors, n) entries
// (push with sift-up while short, else replace the root when d < root and
// sift down; neighbors.rs:160-212), stable-sorts it ascending, takes sqrt for
// Euclidean, and drops the first (closest) entry.  Distances use the
// reference's FP32 summation order (simd.rs): squared Euclidean, or cosine
// 1 - dot / (sqrt(|a|^2) sqrt(|b|^2)) (neighbors.rs:231-241).
//
// One warp per query, eight queries per CTA.  The CTA stages 32 candidate rows
// at a time in shared memory (16-byte padded rows, coalesced loads); lane j
// computes the distance to candidate j0 + j.  The heap update keeps the
// sequential semantics exactly: while the heap is short every candidate is
// pushed in order; after that a ballot finds the first lane (in j order) that
// beats the current root, lane 0 replaces and sifts, and the lanes before it
// are settled (the root only decreases, so a candidate that lost once loses
// again).  Cosine searches read per-row |x|^2 from a scratch array computed
// once (same summation order, so the values equal the reference's per-pair
// dot(b, b)).
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "exact.cuh"
#include "polariseq_knn.h"

namespace pq {
namespace {

constexpr int EW = 8;   // queries (warps) per CTA
constexpr int ET = 32;  // candidates per staged tile
constexpr uint32_t FULL = 0xFFFFFFFFu;

// Stage rows [r0, r0 + cnt) of the row-major n x d matrix into `dst` with
// row stride dp (zero padded).
__device__ __forceinline__ void stage_rows(const float* __restrict__ X, int d, int dp,
                                           uint64_t r0, uint32_t cnt, uint32_t rows,
                                           float* __restrict__ dst) {
    for (int t = threadIdx.x; t < int(rows) * dp; t += blockDim.x) {
        const int r = t / dp, c = t - r * dp;
        dst[t] = (uint32_t(r) < cnt && c < d) ? X[(r0 + r) * uint64_t(d) + c] : 0.0f;
    }
}

// |x|^2 of every row, dot(x, x) in the reference order (simd.rs:20-36:
// eight partial sums, ((a0+a4)+(a1+a5))+((a2+a6)+(a3+a7)), then the tail),
// with scalar loads (rows of the caller's matrix need not be 16-byte aligned).
__global__ void k_row_dots(const float* __restrict__ X, uint64_t n, int d,
                           float* __restrict__ norms) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = X + i * uint64_t(d);
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int full = d >> 3;
    for (int c = 0; c < full; ++c)
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const float v = r[8 * c + l];
            acc[l] = __fadd_rn(acc[l], __fmul_rn(v, v));
        }
    float tail = 0.0f;
    for (int j = full * 8; j < d; ++j) tail = __fadd_rn(tail, __fmul_rn(r[j], r[j]));
    const float s = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                              __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
    norms[i] = __fadd_rn(s, tail);
}

// Heap of one warp in shared memory (lane 0 mutates it), reference rules.
__device__ __forceinline__ void heap_push_up(float* hd, uint32_t* hi, int len, float d,
                                             uint32_t j) {
    int c = len;
    hd[c] = d;
    hi[c] = j;
    while (c > 0) {
        const int p = (c - 1) / 2;
        if (hd[c] > hd[p]) {
            const float tv = hd[c];
            hd[c] = hd[p];
            hd[p] = tv;
            const uint32_t ti = hi[c];
            hi[c] = hi[p];
            hi[p] = ti;
            c = p;
        } else {
            break;
        }
    }
}
__device__ __forceinline__ void heap_replace_down(float* hd, uint32_t* hi, int len, float d,
                                                  uint32_t j) {
    hd[0] = d;
    hi[0] = j;
    int p = 0;
    for (;;) {
        const int l = 2 * p + 1, r = 2 * p + 2;
        int m = p;
        if (l < len && hd[l] > hd[m]) m = l;
        if (r < len && hd[r] > hd[m]) m = r;
        if (m == p) break;
        const float tv = hd[p];
        hd[p] = hd[m];
        hd[m] = tv;
        const uint32_t ti = hi[p];
        hi[p] = hi[m];
        hi[m] = ti;
        p = m;
    }
}

template <int D>
__global__ void __launch_bounds__(EW * 32) k_exact_knn(const float* __restrict__ X, uint32_t n,
                                                       int d, int dp, int kws, int cosine,
                                                       const float* __restrict__ norms,
                                                       uint32_t* __restrict__ out_idx,
                                                       float* __restrict__ out_dist) {
    extern __shared__ __align__(16) float sm[];
    float* sq = sm;                 // EW x dp query rows
    float* st = sq + EW * dp;       // ET x dp candidate rows
    float* hd_all = st + ET * dp;   // EW x kws heap distances
    uint32_t* hi_all = reinterpret_cast<uint32_t*>(hd_all + EW * kws);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t q0 = uint64_t(blockIdx.x) * EW;
    const uint64_t q = q0 + w;
    const bool qv = q < n;
    stage_rows(X, d, dp, q0, uint32_t(n - q0 < EW ? n - q0 : EW), EW, sq);
    float* hd = hd_all + w * kws;
    uint32_t* hi = hi_all + w * kws;
    const float* qr = sq + w * dp;
    const float qn = (cosine && qv) ? norms[q] : 0.0f;
    int hlen = 0;  // warp-uniform
    for (uint64_t j0 = 0; j0 < n; j0 += ET) {
        const uint32_t cnt = uint32_t(n - j0 < ET ? n - j0 : ET);
        __syncthreads();  // the previous tile is consumed
        stage_rows(X, d, dp, j0, cnt, ET, st);
        __syncthreads();
        if (!qv) continue;
        float dd = 0.0f;
        if (uint32_t(lane) < cnt) {
            const float* cr = st + lane * dp;
            if (!cosine) {
                dd = sq_dist_exact_t<D>(qr, cr, d);
            } else {
                const float dt = dot_exact_t<D>(qr, cr, d);
                const float den = __fmul_rn(__fsqrt_rn(qn), __fsqrt_rn(norms[j0 + lane]));
                dd = den > 0.0f ? __fsub_rn(1.0f, __fdiv_rn(dt, den)) : 1.0f;
            }
        }
        uint32_t pending = cnt == 32 ? FULL : ((1u << cnt) - 1u);
        // while the heap is short, every candidate is pushed in order
        while (pending && hlen < kws) {
            const int l = __ffs(pending) - 1;
            pending &= pending - 1;
            const float dl = __shfl_sync(FULL, dd, l);
            if (lane == 0) heap_push_up(hd, hi, hlen, dl, uint32_t(j0 + l));
            ++hlen;
            __syncwarp();
        }
        // then the first remaining lane that beats the current root, in order
        while (pending) {
            const float root = hd[0];
            const uint32_t m = __ballot_sync(FULL, ((pending >> lane) & 1u) && dd < root);
            if (!m) break;
            const int l = __ffs(m) - 1;
            pending &= ~((l == 31) ? FULL : ((2u << l) - 1u));
            const float dl = __shfl_sync(FULL, dd, l);
            if (lane == 0) heap_replace_down(hd, hi, hlen, dl, uint32_t(j0 + l));
            __syncwarp();
        }
    }
    if (!qv) return;
    // stable ascending sort (insertion), sqrt for Euclidean, drop the closest
    if (lane == 0) {
        for (int a = 1; a < hlen; ++a) {
            const float x = hd[a];
            const uint32_t y = hi[a];
            int b = a - 1;
            while (b >= 0 && hd[b] > x) {
                hd[b + 1] = hd[b];
                hi[b + 1] = hi[b];
                --b;
            }
            hd[b + 1] = x;
            hi[b + 1] = y;
        }
    }
    __syncwarp();
    const uint64_t per = uint64_t(kws - 1);
    for (int t = 1 + lane; t < hlen; t += 32) {
        out_idx[q * per + (t - 1)] = hi[t];
        out_dist[q * per + (t - 1)] = cosine ? hd[t] : __fsqrt_rn(hd[t]);
    }
}

__global__ void k_exact_indptr(uint32_t* __restrict__ indptr, uint64_t n, uint32_t per) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i <= n) indptr[i] = uint32_t(i * per);
}

template <int D>
cudaError_t launch_d(const float* X, uint64_t n, int d, int kws, int cosine, float* norms,
                     uint32_t* indptr, uint32_t* indices, float* dists, cudaStream_t st) {
    const int dp = (d + 3) / 4 * 4;
    if (cosine) {
        k_row_dots<<<uint32_t((n + 255) / 256), 256, 0, st>>>(X, n, d, norms);
        count_launch();
    }
    k_exact_knn<D><<<uint32_t((n + EW - 1) / EW), EW * 32, exact_knn_smem(d, kws), st>>>(
        X, uint32_t(n), d, dp, kws, cosine, norms, indices, dists);
    count_launch();
    k_exact_indptr<<<uint32_t((n + 256) / 256), 256, 0, st>>>(indptr, n, uint32_t(kws - 1));
    count_launch();
    return cudaGetLastError();
}

}  // namespace

size_t exact_knn_smem(int d, int kws) {
    const int dp = (d + 3) / 4 * 4;
    return size_t(EW + ET) * dp * 4 + size_t(EW) * kws * 8;
}

cudaError_t exact_knn_prepare() {
    cudaFuncAttributes fa;
    cudaError_t e;
    if ((e = cudaFuncGetAttributes(&fa, k_row_dots)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, k_exact_indptr)) != cudaSuccess) return e;
    const int smax = int(exact_knn_smem(EXACT_MAX_DIM, EXACT_MAX_K));
    if ((e = cudaFuncSetAttribute(k_exact_knn<50>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smax)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_exact_knn<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
}

cudaError_t launch_exact_knn(const float* X, uint64_t n, int d, int kws, int cosine,
                             float* norms, uint32_t* indptr, uint32_t* indices, float* dists,
                             cudaStream_t st) {
    if (n == 0 || n > 0xFFFFFFFEull || d < 1 || d > EXACT_MAX_DIM || kws < 1 ||
        kws > EXACT_MAX_K)
        return cudaErrorInvalidValue;
    if (d == 50) return launch_d<50>(X, n, d, kws, cosine, norms, indptr, indices, dists, st);
    return launch_d<0>(X, n, d, kws, cosine, norms, indptr, indices, dists, st);
}

}  // namespace pq

// ── allocation-free variant ─────────────────────────────────────────────────
// Scratch of pq_neighbors_into_device_noalloc: the cosine metric's per-row
// |x|^2, for at most EXACT_NOALLOC_MAX_ROWS rows (1 MiB).  It lives in every
// device that loads the library, from load until process exit.  In host code
// the name below stands for a host-side shadow, not the device array: the
// device address comes from cudaGetSymbolAddress at set-up.
namespace pq {
namespace {

constexpr uint64_t EXACT_NOALLOC_MAX_ROWS = uint64_t(1) << 18;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) float g_noalloc_norms[EXACT_NOALLOC_MAX_ROWS];

std::mutex g_noalloc_mu;
float* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Once per device, with that device current: the scratch array's device
// address, and the kernels loaded with their shared-memory limit raised.
cudaError_t noalloc_setup(int dev, float** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        float* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_norms);
        if (e != cudaSuccess) return e;
        if ((e = exact_knn_prepare()) != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace pq

extern "C" int pq_neighbors_into_device_noalloc(const float* d_data, uint64_t n_obs,
                                                uint64_t n_dim, uint64_t n_neighbors,
                                                int32_t metric, uint32_t* d_indptr,
                                                uint32_t* d_indices, float* d_dists,
                                                uint64_t* nnz_out, void* stream) {
    using namespace pq;
    if (!d_data || !d_indptr || !d_indices || !d_dists || !nnz_out) return PQ_EINVAL;
    if (n_obs == 0 || n_dim == 0 || n_neighbors == 0) return PQ_EINVAL;
    if (metric != PQ_METRIC_EUCLIDEAN && metric != PQ_METRIC_COSINE) return PQ_EINVAL;
    if (n_obs > EXACT_NOALLOC_MAX_ROWS) return PQ_ETOOBIG;
    const uint64_t kws = n_neighbors < n_obs ? n_neighbors : n_obs;
    if (kws > uint64_t(EXACT_MAX_K) || n_dim > uint64_t(EXACT_MAX_DIM)) return PQ_ENOTSUP;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return PQ_EDEVICE;
    }
    float* norms = nullptr;
    if (noalloc_setup(dev, &norms) != cudaSuccess) {
        cudaGetLastError();
        return PQ_EDEVICE;
    }
    // every norm the search reads is written first, on the same stream
    if (launch_exact_knn(d_data, n_obs, int(n_dim), int(kws), metric == PQ_METRIC_COSINE, norms,
                         d_indptr, d_indices, d_dists,
                         static_cast<cudaStream_t>(stream)) != cudaSuccess) {
        cudaGetLastError();
        return PQ_EDEVICE;
    }
    *nnz_out = n_obs * (kws - 1);
    return PQ_OK;
}
