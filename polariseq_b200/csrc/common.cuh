// Shared device helpers for the sm_100a kNN-graph builder.
//
// Exactness contract: every f32 distance and dot product is computed in the
// reference's order (crates/polariseq-core/src/simd.rs:14-81): eight independent
// lane accumulators over chunks of 8, the fixed reduce
// ((a0+a4)+(a1+a5))+((a2+a6)+(a3+a7)), then a sequentially summed tail; every
// operation rounded separately (no FMA contraction: the Rust reference never
// fuses).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PQ_EMPTY 0xFFFFFFFFu

namespace pq {

// Kernels launched by this library (for the launch-count statistic).
extern unsigned long long g_launches;
inline void count_launch() { ++g_launches; }

// ── deterministic hashing RNG (nndescent.rs:80-112) ───────────────────────
__host__ __device__ __forceinline__ uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// hash_unit (nndescent.rs:89-93): the top 24 bits of the hash over 2^24.
__host__ __device__ __forceinline__ float hash_unit(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t h = splitmix(seed ^ splitmix(a) ^ splitmix(b * 0x9E3779B97F4A7C15ull));
    return float(uint32_t(h >> 40)) * (1.0f / 16777216.0f);
}

// hash_index (nndescent.rs:95-98).
__host__ __device__ __forceinline__ uint64_t hash_index(uint64_t seed, uint64_t a, uint64_t b,
                                                        uint64_t n) {
    return splitmix(seed ^ splitmix(a) ^ splitmix(b + 0x12345678ull)) % n;
}

// x mod n for n < 2^32, exact: one 32-bit remainder, then two 16-bit long
// division steps whose partial dividends (< 2^48) are exact in double; the
// double quotient is corrected to the exact integer quotient.
__device__ __forceinline__ uint32_t mod_u64_u32(uint64_t x, uint32_t n) {
    uint32_t r = uint32_t(x >> 32) % n;
    const double dn = double(n);
#pragma unroll
    for (int step = 1; step >= 0; --step) {
        const uint64_t t = (uint64_t(r) << 16) | ((x >> (16 * step)) & 0xFFFFull);
        uint64_t q = uint64_t(double(t) / dn);
        int64_t rem = int64_t(t) - int64_t(q * n);
        if (rem < 0) rem += n;
        if (rem >= int64_t(n)) rem -= n;
        r = uint32_t(rem);
    }
    return r;
}

// x mod n with a reciprocal rn = RN(1 / n) shared by several draws of one
// n: three steps of 32, 16 and 16 bits, each partial dividend t < 2^48 so
// that trunc(t * rn) is within one of floor(t / n) (relative error below
// 2^-51); one correction either way makes each remainder exact.
__device__ __forceinline__ uint32_t mod_u64_u32_r(uint64_t x, uint32_t n, double rn) {
    uint64_t r = 0;
#pragma unroll
    for (int step = 2; step >= 0; --step) {
        const uint64_t t = step == 2 ? (x >> 32) : ((r << 16) | ((x >> (16 * step)) & 0xFFFFull));
        const int64_t q = int64_t(double(t) * rn);
        int64_t rem = int64_t(t) - q * int64_t(n);
        if (rem < 0) rem += n;
        if (rem >= int64_t(n)) rem -= n;
        r = uint64_t(rem);
    }
    return uint32_t(r);
}

// Rng (nndescent.rs:101-112): the state is replaced by splitmix(state).
struct Rng {
    uint64_t s;
    __host__ __device__ __forceinline__ uint64_t next_u64() {
        s = splitmix(s);
        return s;
    }
    __host__ __device__ __forceinline__ uint64_t below(uint64_t n) {
#ifdef __CUDA_ARCH__
        if (n <= 0xFFFFFFFFull) return mod_u64_u32(next_u64(), uint32_t(n));
#endif
        return next_u64() % n;
    }
};

// ── packed f32x2 arithmetic, round-to-nearest-even per half ───────────────
typedef unsigned long long f2;

__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(f2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// Final reduce of the packed accumulators (a0,a1) (a2,a3) (a4,a5) (a6,a7)
// into ((a0+a4)+(a1+a5))+((a2+a6)+(a3+a7)).
__device__ __forceinline__ float reduce8_packed(f2 a01, f2 a23, f2 a45, f2 a67) {
    float x, y, z, w;
    f2_unpack(f2_add(a01, a45), x, y);  // (a0+a4, a1+a5)
    f2_unpack(f2_add(a23, a67), z, w);  // (a2+a6, a3+a7)
    return __fadd_rn(__fadd_rn(x, y), __fadd_rn(z, w));
}

// Squared Euclidean distance of two padded rows (16-byte aligned), exact
// reference order (simd.rs:43-62).  `d` is the logical dimension.  Every
// operation is a separately rounded scalar intrinsic, which the compiler
// never contracts into an FMA.
__device__ __forceinline__ float sq_dist_exact(const float* __restrict__ a,
                                               const float* __restrict__ b, int d) {
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int full = d >> 3;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
#pragma unroll 4
    for (int c = 0; c < full; ++c) {
        float4 x0 = a4[2 * c], x1 = a4[2 * c + 1];
        float4 y0 = b4[2 * c], y1 = b4[2 * c + 1];
        float t[8] = {__fsub_rn(x0.x, y0.x), __fsub_rn(x0.y, y0.y), __fsub_rn(x0.z, y0.z),
                      __fsub_rn(x0.w, y0.w), __fsub_rn(x1.x, y1.x), __fsub_rn(x1.y, y1.y),
                      __fsub_rn(x1.z, y1.z), __fsub_rn(x1.w, y1.w)};
#pragma unroll
        for (int l = 0; l < 8; ++l) acc[l] = __fadd_rn(acc[l], __fmul_rn(t[l], t[l]));
    }
    float tail = 0.0f;
    for (int j = full << 3; j < d; ++j) {
        float t = __fsub_rn(a[j], b[j]);
        tail = __fadd_rn(tail, __fmul_rn(t, t));
    }
    float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                        __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
    return __fadd_rn(r, tail);
}

// Dot product, exact reference order (simd.rs:20-36).
__device__ __forceinline__ float dot_exact(const float* __restrict__ a,
                                           const float* __restrict__ b, int d) {
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int full = d >> 3;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
#pragma unroll 4
    for (int c = 0; c < full; ++c) {
        float4 x0 = a4[2 * c], x1 = a4[2 * c + 1];
        float4 y0 = b4[2 * c], y1 = b4[2 * c + 1];
        acc[0] = __fadd_rn(acc[0], __fmul_rn(x0.x, y0.x));
        acc[1] = __fadd_rn(acc[1], __fmul_rn(x0.y, y0.y));
        acc[2] = __fadd_rn(acc[2], __fmul_rn(x0.z, y0.z));
        acc[3] = __fadd_rn(acc[3], __fmul_rn(x0.w, y0.w));
        acc[4] = __fadd_rn(acc[4], __fmul_rn(x1.x, y1.x));
        acc[5] = __fadd_rn(acc[5], __fmul_rn(x1.y, y1.y));
        acc[6] = __fadd_rn(acc[6], __fmul_rn(x1.z, y1.z));
        acc[7] = __fadd_rn(acc[7], __fmul_rn(x1.w, y1.w));
    }
    float tail = 0.0f;
    for (int j = full << 3; j < d; ++j) tail = __fadd_rn(tail, __fmul_rn(a[j], b[j]));
    float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                        __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
    return __fadd_rn(r, tail);
}

// dot_exact with a compile-time dimension (fully unrolled); D == 0 falls back
// to the runtime-d version.
template <int D>
__device__ __forceinline__ float dot_exact_t(const float* __restrict__ a,
                                             const float* __restrict__ b, int d) {
    if constexpr (D == 0) {
        return dot_exact(a, b, d);
    } else {
        constexpr int FULL = D / 8;
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const float4* b4 = reinterpret_cast<const float4*>(b);
#pragma unroll
        for (int c = 0; c < FULL; ++c) {
            float4 x0 = a4[2 * c], x1 = a4[2 * c + 1];
            float4 y0 = b4[2 * c], y1 = b4[2 * c + 1];
            acc[0] = __fadd_rn(acc[0], __fmul_rn(x0.x, y0.x));
            acc[1] = __fadd_rn(acc[1], __fmul_rn(x0.y, y0.y));
            acc[2] = __fadd_rn(acc[2], __fmul_rn(x0.z, y0.z));
            acc[3] = __fadd_rn(acc[3], __fmul_rn(x0.w, y0.w));
            acc[4] = __fadd_rn(acc[4], __fmul_rn(x1.x, y1.x));
            acc[5] = __fadd_rn(acc[5], __fmul_rn(x1.y, y1.y));
            acc[6] = __fadd_rn(acc[6], __fmul_rn(x1.z, y1.z));
            acc[7] = __fadd_rn(acc[7], __fmul_rn(x1.w, y1.w));
        }
        float tail = 0.0f;
#pragma unroll
        for (int j = FULL * 8; j < D; ++j) tail = __fadd_rn(tail, __fmul_rn(a[j], b[j]));
        float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                            __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
        return __fadd_rn(r, tail);
    }
}

// sq_dist_exact with a compile-time dimension (fully unrolled); D == 0 falls
// back to the runtime-d version.
template <int D>
__device__ __forceinline__ float sq_dist_exact_t(const float* __restrict__ a,
                                                 const float* __restrict__ b, int d) {
    if constexpr (D == 0) {
        return sq_dist_exact(a, b, d);
    } else {
        constexpr int FULL = D / 8;
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const float4* b4 = reinterpret_cast<const float4*>(b);
#pragma unroll
        for (int c = 0; c < FULL; ++c) {
            float4 x0 = a4[2 * c], x1 = a4[2 * c + 1];
            float4 y0 = b4[2 * c], y1 = b4[2 * c + 1];
            float t[8] = {__fsub_rn(x0.x, y0.x), __fsub_rn(x0.y, y0.y), __fsub_rn(x0.z, y0.z),
                          __fsub_rn(x0.w, y0.w), __fsub_rn(x1.x, y1.x), __fsub_rn(x1.y, y1.y),
                          __fsub_rn(x1.z, y1.z), __fsub_rn(x1.w, y1.w)};
#pragma unroll
            for (int l = 0; l < 8; ++l) acc[l] = __fadd_rn(acc[l], __fmul_rn(t[l], t[l]));
        }
        float tail = 0.0f;
#pragma unroll
        for (int j = FULL * 8; j < D; ++j) {
            float t = __fsub_rn(a[j], b[j]);
            tail = __fadd_rn(tail, __fmul_rn(t, t));
        }
        float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                            __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
        return __fadd_rn(r, tail);
    }
}

// Hyperplane offset -(sum_j (nv_j * 0.5) * (xa_j + xb_j)) with the reference's
// sequential f32 sum (Rust's `sum` folds left from -0.0), nv_j = xa_j - xb_j.
template <int D>
__device__ __forceinline__ float hyper_offset_t(const float* __restrict__ xa,
                                                const float* __restrict__ xb, int d) {
    float s = -0.0f;
    if constexpr (D == 0) {
        for (int j = 0; j < d; ++j) {
            float a = xa[j], b = xb[j];
            s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fsub_rn(a, b), 0.5f), __fadd_rn(a, b)));
        }
    } else {
#pragma unroll 10
        for (int j = 0; j < D; ++j) {
            float a = xa[j], b = xb[j];
            s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fsub_rn(a, b), 0.5f), __fadd_rn(a, b)));
        }
    }
    return -s;
}

// Flagged neighbour-heap push on one row (HeapRowsMut::push, nndescent.rs:168-205):
// reject d >= root or an index already present; else replace the root and
// sift down with strict `>`.
__device__ __forceinline__ bool heap_push(uint32_t* idx, float* dist, uint8_t* flg, int k,
                                          uint32_t j, float d, uint8_t flag) {
    if (d >= dist[0]) return false;
    for (int s = 0; s < k; ++s)
        if (idx[s] == j) return false;
    int p = 0;
    for (;;) {
        int l = 2 * p + 1, r = 2 * p + 2, sw = p;
        float dsw = d;  // the value travelling down from the root
        if (l < k && dist[l] > dsw) { sw = l; dsw = dist[l]; }
        if (r < k && dist[r] > dsw) { sw = r; }
        if (sw == p) break;
        idx[p] = idx[sw];
        dist[p] = dist[sw];
        flg[p] = flg[sw];
        p = sw;
    }
    idx[p] = j;
    dist[p] = d;
    flg[p] = flag;
    return true;
}

// heap_push on a row whose entries sit `stride` elements apart (a column of
// a transposed shared-memory tile).
__device__ __forceinline__ bool heap_push_strided(uint32_t* idx, float* dist, uint8_t* flg, int k,
                                                  int stride, uint32_t j, float d, uint8_t flag) {
    if (d >= dist[0]) return false;
    for (int s = 0; s < k; ++s)
        if (idx[s * stride] == j) return false;
    int p = 0;
    for (;;) {
        int l = 2 * p + 1, r = 2 * p + 2, sw = p;
        float dsw = d;
        if (l < k && dist[l * stride] > dsw) { sw = l; dsw = dist[l * stride]; }
        if (r < k && dist[r * stride] > dsw) { sw = r; }
        if (sw == p) break;
        idx[p * stride] = idx[sw * stride];
        dist[p * stride] = dist[sw * stride];
        flg[p * stride] = flg[sw * stride];
        p = sw;
    }
    idx[p * stride] = j;
    dist[p * stride] = d;
    flg[p * stride] = flag;
    return true;
}

// cand_push on a strided row.
__device__ __forceinline__ void cand_push_strided(uint32_t* idx, float* prio, int m, int stride,
                                                  uint32_t j, float p) {
    if (p >= prio[0]) return;
    for (int s = 0; s < m; ++s)
        if (idx[s * stride] == j) return;
    int q = 0;
    for (;;) {
        int l = 2 * q + 1, r = 2 * q + 2, sw = q;
        float psw = p;
        if (l < m && prio[l * stride] > psw) { sw = l; psw = prio[l * stride]; }
        if (r < m && prio[r * stride] > psw) { sw = r; }
        if (sw == q) break;
        idx[q * stride] = idx[sw * stride];
        prio[q * stride] = prio[sw * stride];
        q = sw;
    }
    idx[q * stride] = j;
    prio[q * stride] = p;
}

// Candidate-heap push (CandidateHeap::push_row, nndescent.rs:244-269).
__device__ __forceinline__ void cand_push(uint32_t* idx, float* prio, int m, uint32_t j,
                                          float p) {
    if (p >= prio[0]) return;
    for (int s = 0; s < m; ++s)
        if (idx[s] == j) return;
    int q = 0;
    for (;;) {
        int l = 2 * q + 1, r = 2 * q + 2, sw = q;
        float psw = p;
        if (l < m && prio[l] > psw) { sw = l; psw = prio[l]; }
        if (r < m && prio[r] > psw) { sw = r; }
        if (sw == q) break;
        idx[q] = idx[sw];
        prio[q] = prio[sw];
        q = sw;
    }
    idx[q] = j;
    prio[q] = p;
}

}  // namespace pq
