// Sampled recall of a built graph, on the device: the exact k nearest of Q
// sampled cells (FP32 distances in the reference's summation order,
// simd.rs:43-62; ties by index; the cell itself excluded) against all n
// cells, and the fraction of them the graph's rows hold.  The learned-init
// NN-Descent uses it to decide whether to fall back to the RP-forest
// initialisation.
//
//   k_sample_scan_reg (d = 50): CTA (128 queries, split s of the cells); one
//     thread per query holds the query row in registers and its ascending
//     list of the 32 best (distance bits, index) keys; the split's cells are
//     staged in shared memory 128 rows at a time (contiguous rows, coalesced
//     float4 loads) and every thread reads the same row at the same time (a
//     broadcast); one list per (query, split);
//   k_sample_scan (other d): CTA (query group of 32, split s); 8 threads per
//     query with their own lists, the query rows also in shared memory;
//   k_sample_merge: one CTA per query sorts its S x 8 x 32 keys (bitonic, in
//     shared memory) and counts how many of the k best its graph row holds.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "ctx.cuh"
#include "kernels.cuh"

namespace pq {
namespace {

constexpr int QG = 32;   // queries per scan CTA
constexpr int TPQ = 8;   // threads per query
constexpr int LK = 32;   // keys kept per thread (k <= 32)
constexpr int CH = 128;  // cells staged per chunk
constexpr int SCAN_T = QG * TPQ;
constexpr int QB = 128;  // queries per register-row scan CTA
constexpr int MERGE_T = 512;
constexpr int MERGE_MAX = 4096;  // keys per query in the merge (S <= 16)

template <int D>
__global__ void __launch_bounds__(SCAN_T) k_sample_scan(const float* __restrict__ X, int d, int dp,
                                                        uint32_t n, const uint32_t* __restrict__ q,
                                                        uint32_t Q, uint32_t S,
                                                        uint64_t* __restrict__ out) {
    extern __shared__ __align__(16) float sm[];
    float* qrows = sm;             // QG x dp
    float* crows = sm + QG * dp;   // CH x dp
    const int tid = threadIdx.x, ql = tid / TPQ, j = tid % TPQ;
    const uint32_t qi = blockIdx.x * QG + ql;
    const uint32_t s = blockIdx.y;
    const uint32_t c0 = uint32_t(uint64_t(n) * s / S), c1 = uint32_t(uint64_t(n) * (s + 1) / S);
    const int q4 = dp / 4;
    for (int t = tid; t < QG * q4; t += SCAN_T) {
        const int r = t / q4, c = t - r * q4;
        const uint32_t g = blockIdx.x * QG + r;
        reinterpret_cast<float4*>(qrows)[t] =
            g < Q ? reinterpret_cast<const float4*>(X + size_t(q[g]) * dp)[c]
                  : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const uint32_t self = qi < Q ? q[qi] : 0xFFFFFFFFu;
    uint64_t L[LK];
#pragma unroll
    for (int r = 0; r < LK; ++r) L[r] = ~0ull;
    for (uint32_t b0 = c0; b0 < c1; b0 += CH) {
        const uint32_t len = min(uint32_t(CH), c1 - b0);
        __syncthreads();
        for (int t = tid; t < int(len) * q4; t += SCAN_T) {
            const int r = t / q4, c = t - r * q4;
            reinterpret_cast<float4*>(crows)[t] =
                reinterpret_cast<const float4*>(X + size_t(b0 + r) * dp)[c];
        }
        __syncthreads();
        if (qi < Q) {
            for (uint32_t r = j; r < len; r += TPQ) {
                const uint32_t id = b0 + r;
                if (id == self) continue;
                const float dd = sq_dist_exact_t<D>(qrows + ql * dp, crows + r * dp, d);
                const uint64_t key = (uint64_t(__float_as_uint(dd)) << 32) | id;
                if (key < L[LK - 1]) {
                    // insert: entries after the place move up one, the last drops
#pragma unroll
                    for (int t = LK - 1; t > 0; --t) {
                        const bool up = key < L[t - 1];
                        const bool here = !up && key < L[t];
                        L[t] = up ? L[t - 1] : (here ? key : L[t]);
                    }
                    if (key < L[0]) L[0] = key;
                }
            }
        }
    }
    if (qi < Q) {
        uint64_t* o = out + ((size_t(qi) * S + s) * TPQ + j) * LK;
#pragma unroll
        for (int r = 0; r < LK; ++r) o[r] = L[r];
    }
}

// Squared distance of a register-held query row to a row in shared memory,
// in sq_dist_exact_t's order ((a - b)^2 is symmetric bit for bit).
template <int D>
__device__ __forceinline__ float sq_dist_reg(const float (&q)[D], const float* __restrict__ c) {
    constexpr int FULL = D / 8;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float4* c4 = reinterpret_cast<const float4*>(c);
#pragma unroll
    for (int b = 0; b < FULL; ++b) {
        const float4 y0 = c4[2 * b], y1 = c4[2 * b + 1];
        const float y[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const float t = __fsub_rn(q[8 * b + l], y[l]);
            acc[l] = __fadd_rn(acc[l], __fmul_rn(t, t));
        }
    }
    float tail = 0.0f;
#pragma unroll
    for (int j = FULL * 8; j < D; ++j) {
        const float t = __fsub_rn(q[j], c[j]);
        tail = __fadd_rn(tail, __fmul_rn(t, t));
    }
    const float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                              __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
    return __fadd_rn(r, tail);
}

template <int D>
__global__ void __launch_bounds__(QB) k_sample_scan_reg(const float* __restrict__ X, int dp,
                                                        uint32_t n,
                                                        const uint32_t* __restrict__ q,
                                                        uint32_t Q, uint32_t S,
                                                        uint64_t* __restrict__ out) {
    extern __shared__ __align__(16) float sm[];  // CH x dp
    const int tid = threadIdx.x;
    const uint32_t qi = blockIdx.x * QB + tid;
    const uint32_t s = blockIdx.y;
    const uint32_t c0 = uint32_t(uint64_t(n) * s / S), c1 = uint32_t(uint64_t(n) * (s + 1) / S);
    const uint32_t self = qi < Q ? q[qi] : 0xFFFFFFFFu;
    const float* qrow = X + size_t(qi < Q ? self : 0u) * dp;
    float qr[D];
#pragma unroll
    for (int j = 0; j < D; ++j) qr[j] = qi < Q ? qrow[j] : 0.0f;
    uint64_t L[LK];
#pragma unroll
    for (int r = 0; r < LK; ++r) L[r] = ~0ull;
    const int q4 = dp / 4;
    for (uint32_t b0 = c0; b0 < c1; b0 += CH) {
        const uint32_t len = min(uint32_t(CH), c1 - b0);
        __syncthreads();
        const float4* src = reinterpret_cast<const float4*>(X + size_t(b0) * dp);
        for (int t = tid; t < int(len) * q4; t += QB) reinterpret_cast<float4*>(sm)[t] = src[t];
        __syncthreads();
        if (qi < Q) {
            for (uint32_t r = 0; r < len; ++r) {
                const float dd = sq_dist_reg<D>(qr, sm + r * dp);
                const uint32_t id = b0 + r;
                const uint64_t key = (uint64_t(__float_as_uint(dd)) << 32) | id;
                if (key < L[LK - 1] && id != self) {
#pragma unroll
                    for (int t = LK - 1; t > 0; --t) {
                        const bool up = key < L[t - 1];
                        const bool here = !up && key < L[t];
                        L[t] = up ? L[t - 1] : (here ? key : L[t]);
                    }
                    if (key < L[0]) L[0] = key;
                }
            }
        }
    }
    if (qi < Q) {
        uint64_t* o = out + (size_t(qi) * S + s) * LK;
#pragma unroll
        for (int r = 0; r < LK; ++r) o[r] = L[r];
    }
}

// Query blockIdx.x: sorts its m = S * TPQ * LK keys, takes the k best and
// counts how many of them appear in its graph row (CSR); hits added to *hits.
__global__ void __launch_bounds__(MERGE_T) k_sample_merge(const uint64_t* __restrict__ keys,
                                                          uint32_t m, int k,
                                                          const uint32_t* __restrict__ q,
                                                          const uint32_t* __restrict__ indptr,
                                                          const uint32_t* __restrict__ indices,
                                                          unsigned long long* __restrict__ hits) {
    __shared__ uint64_t v[MERGE_MAX];
    __shared__ unsigned cnt;
    uint32_t m2 = 1;
    while (m2 < m) m2 <<= 1;
    const uint64_t* src = keys + size_t(blockIdx.x) * m;
    for (uint32_t t = threadIdx.x; t < m2; t += MERGE_T) v[t] = t < m ? src[t] : ~0ull;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (uint32_t size = 2; size <= m2; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t t = threadIdx.x; t < m2; t += MERGE_T) {
                const uint32_t p = t ^ stride;
                if (p > t) {
                    const bool up = (t & size) == 0;
                    const uint64_t a = v[t], b = v[p];
                    if ((a > b) == up) {
                        v[t] = b;
                        v[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    const uint32_t i = q[blockIdx.x];
    const uint32_t r0 = indptr[i], r1 = indptr[i + 1];
    for (int t = threadIdx.x; t < k; t += MERGE_T) {
        if (v[t] == ~0ull) continue;
        const uint32_t want = uint32_t(v[t]);
        bool found = false;
        for (uint32_t e = r0; e < r1; ++e) found |= indices[e] == want;
        if (found) atomicAdd(&cnt, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0 && cnt) atomicAdd(hits, (unsigned long long)cnt);
}

}  // namespace

double sampled_recall(pq_ctx* c, const float* X, int d, int dp, uint32_t n, int k,
                      const uint32_t* d_indptr, const uint32_t* d_indices, uint32_t Q,
                      uint64_t seed) {
    using namespace pqh;
    cudaStream_t st = c->stream;
    if (k > LK) throw DeviceError{"sampled recall supports k <= 32"};
    Q = std::min(Q, n);
    if (Q == 0 || n < 2) return 1.0;
    // seeded distinct sample: evenly strided cells with a hashed offset
    std::vector<uint32_t> hq(Q);
    const uint64_t off = splitmix(seed ^ 0x5a4d504cull) % n;
    for (uint32_t t = 0; t < Q; ++t) hq[t] = uint32_t((off + uint64_t(t) * n / Q) % n);
    const bool reg = d == 50;
    const uint32_t groups = (Q + (reg ? QB : QG) - 1) / (reg ? QB : QG);
    // lists per (query, split): 1 (register rows) or TPQ
    const uint32_t per = reg ? 1u : uint32_t(TPQ);
    // about three CTAs per SM (148 SMs)
    uint32_t S = std::max<uint32_t>(1, (reg ? 444u : 296u + groups - 1) / groups);
    S = std::min<uint32_t>(S, MERGE_MAX / (per * LK));
    S = std::min<uint32_t>(S, std::max<uint32_t>(1, n / CH));
    uint32_t* dq = c->get<uint32_t>("sr_q", Q);
    uint64_t* keys = c->get<uint64_t>("sr_keys", size_t(Q) * S * per * LK);
    unsigned long long* hits = c->d_acc + 2;
    ck(cudaMemcpyAsync(dq, hq.data(), size_t(Q) * 4, cudaMemcpyHostToDevice, st), "sample");
    ck(cudaMemsetAsync(hits, 0, 8, st), "hits");
    const size_t smem = size_t(QG + CH) * dp * sizeof(float);
    dim3 grid(groups, S);
    if (reg) {
        const size_t sm2 = size_t(CH) * dp * sizeof(float);
        cudaFuncSetAttribute(k_sample_scan_reg<50>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(sm2));
        k_sample_scan_reg<50><<<grid, QB, sm2, st>>>(X, dp, n, dq, Q, S, keys);
    } else if (d == 50) {
        cudaFuncSetAttribute(k_sample_scan<50>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem));
        k_sample_scan<50><<<grid, SCAN_T, smem, st>>>(X, d, dp, n, dq, Q, S, keys);
    } else {
        cudaFuncSetAttribute(k_sample_scan<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem));
        k_sample_scan<0><<<grid, SCAN_T, smem, st>>>(X, d, dp, n, dq, Q, S, keys);
    }
    count_launch();
    k_sample_merge<<<Q, MERGE_T, 0, st>>>(keys, S * per * LK, k, dq, d_indptr, d_indices, hits);
    count_launch();
    unsigned long long h = 0;
    ck(cudaMemcpyAsync(&h, hits, 8, cudaMemcpyDeviceToHost, st), "hits");
    ck(cudaStreamSynchronize(st), "sampled recall");
    const uint64_t kk = std::min<uint64_t>(uint64_t(k), uint64_t(n) - 1);
    return double(h) / double(uint64_t(Q) * kk);
}

}  // namespace pq
