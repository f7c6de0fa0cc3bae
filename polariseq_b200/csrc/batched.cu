// Batched exact kNN: many independent samples of uneven size (the per-sample
// neighbour graphs of doublet scoring, doublets.rs:544-650 knn_exact, and of
// per-batch neighbour steps) in ONE persistent, work-queued launch.
//
// Semantics per sample (as knn_exact): every point's k nearest other points
// of the same sample, exact, ties broken by index, ascending; indices are
// local to the sample.  Distances are squared Euclidean sums of (q - x)^2 in
// FP32 (FMA); the graph is checked against an FP64 brute force as exact sets.
//
// Work items are (sample, block of NW*QW queries), ordered largest sample
// first; persistent CTAs take the next item from a device counter.  A CTA
// stages 128 candidate rows at a time in shared memory, dimension-major with a
// padded stride (coalesced reads, conflict-free lane access); each warp
// computes QW queries x 32 candidates per step (lane = candidate, the queries
// broadcast from shared memory as [dim][QW]) and keeps, per query, the kp
// smallest (distance, index) keys: with kp <= 256 (and at most 32 registers
// of keys per lane) in registers, sorted across the warp's lanes — a key
// below the k-th is inserted by one shuffle and KPL compare-and-selects per
// lane, with no shared-memory round trips — otherwise in a bounded max-heap
// in shared memory with the sequential rule (push while short, then replace
// the root when a key is smaller, lanes visited in index order) and sorted
// by a warp bitonic network at the end.  Either way the result is the exact k
// smallest keys.  The tile shape (QW, NW) is chosen by an autotuner that
// times each shape on the largest work items of the call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "batched.cuh"
#include "common.cuh"

namespace pq {
namespace {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr int ET = 128;       // candidate rows staged per step
constexpr int ETP = ET + 1;   // column stride of the transposed tile (no bank conflicts)

struct BatchArgs {
    const float* X;          // all samples' rows, row-major, d floats each
    int d;
    const uint64_t* s_off;   // sample row offsets (n_samples + 1)
    const uint32_t* s_k;     // neighbours per point of each sample
    const uint64_t* s_out;   // output offset of each sample's first row
    const uint32_t* item_s;  // work item: sample
    const uint32_t* item_q;  // work item: first local query
    uint32_t n_items;
    uint32_t* counter;       // next work item (starts at zero)
    int kp;                  // heap capacity per query: power of two >= max k
    uint32_t* out_idx;
    float* out_dist;
};

__device__ __forceinline__ uint64_t dkey(float d, uint32_t j) {
    return (uint64_t(__float_as_uint(d)) << 32) | j;
}

__device__ __forceinline__ void heap_up(uint64_t* h, int c) {
    while (c > 0) {
        const int p = (c - 1) >> 1;
        if (h[c] > h[p]) {
            const uint64_t t = h[c];
            h[c] = h[p];
            h[p] = t;
            c = p;
        } else {
            break;
        }
    }
}
__device__ __forceinline__ void heap_down(uint64_t* h, int len) {
    int p = 0;
    for (;;) {
        const int l = 2 * p + 1, r = l + 1;
        int m = p;
        if (l < len && h[l] > h[m]) m = l;
        if (r < len && h[r] > h[m]) m = r;
        if (m == p) break;
        const uint64_t t = h[p];
        h[p] = h[m];
        h[m] = t;
        p = m;
    }
}

// Ascending warp bitonic sort of len keys padded with the largest key to kp
// (a power of two).
__device__ __forceinline__ void sort_keys(uint64_t* h, int len, int kp, int lane) {
    for (int t = len + lane; t < kp; t += 32) h[t] = ~0ull;
    __syncwarp();
    for (int size = 2; size <= kp; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < kp / 2; t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t x = h[lo], y = h[hi];
                if ((x > y) == up) {
                    h[lo] = y;
                    h[hi] = x;
                }
            }
            __syncwarp();
        }
}

// Register selection (kp <= 32 * KPL): a query's kp best keys sorted
// ascending across the warp, lane l holding places l*KPL .. l*KPL+KPL-1.  A new
// key x (smaller than the k-th) shifts every larger key up one place, the
// last lane's last place passing to the next lane: KPL compare-and-selects
// per lane and one shuffle, no shared memory.
template <int KPL>
__device__ __forceinline__ void sorted_insert(uint64_t (&v)[KPL], uint64_t x, int lane) {
    uint64_t prev = __shfl_up_sync(FULL, v[KPL - 1], 1);
    if (lane == 0) prev = 0;
#pragma unroll
    for (int t = KPL - 1; t >= 0; --t) {
        const uint64_t below = t > 0 ? v[t - 1] : prev;
        v[t] = x < below ? below : (x < v[t] ? x : v[t]);
    }
}
// The key at place k-1 (the k-th smallest), broadcast to the warp.
template <int KPL>
__device__ __forceinline__ uint64_t kth_key(const uint64_t (&v)[KPL], int k) {
    const int p = k - 1, owner = p / KPL, place = p - owner * KPL;
    uint64_t mine = v[0];
#pragma unroll
    for (int t = 1; t < KPL; ++t)
        if (place == t) mine = v[t];
    return __shfl_sync(FULL, mine, owner);
}

template <int DP, int QW, int NW, int KPL>
__global__ void __launch_bounds__(NW * 32) k_batched_knn(BatchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    float* sq = reinterpret_cast<float*>(smem);          // NW x DP x QW (dim-major per warp)
    float* st = sq + NW * DP * QW;                        // DP x ETP: the tile, transposed
    uint64_t* heaps = reinterpret_cast<uint64_t*>(st + ((DP * ETP + 1) & ~1));  // NW x QW x kp
    __shared__ uint32_t s_item;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kp = a.kp;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();
        if (item >= a.n_items) break;
        const uint32_t s = a.item_s[item], q0 = a.item_q[item];
        const uint64_t base = a.s_off[s];
        const uint32_t ns = uint32_t(a.s_off[s + 1] - base);
        const int k = int(a.s_k[s]);
        // queries of this CTA, [warp][dim][QW], zero padded
        for (int t = threadIdx.x; t < NW * QW * DP; t += blockDim.x) {
            const int ww = t / (QW * DP), rem = t - ww * QW * DP;
            const int dim = rem / QW, qi = rem - dim * QW;
            const uint32_t q = q0 + uint32_t(ww * QW + qi);
            sq[t] = (q < ns && dim < a.d) ? a.X[(base + q) * uint64_t(a.d) + dim] : 0.0f;
        }
        int hlen[QW];
        // register selection (KPL > 0): the sorted places and the k-th key
        uint64_t kv[QW][KPL > 0 ? KPL : 1];
        uint64_t thr[QW];
#pragma unroll
        for (int qi = 0; qi < QW; ++qi) {
            hlen[qi] = 0;
            thr[qi] = ~0ull;
#pragma unroll
            for (int t = 0; t < (KPL > 0 ? KPL : 1); ++t) kv[qi][t] = ~0ull;
        }
        const float* qw = sq + w * DP * QW;
        for (uint32_t j0 = 0; j0 < ns; j0 += ET) {
            const uint32_t cnt = ns - j0 < uint32_t(ET) ? ns - j0 : uint32_t(ET);
            __syncthreads();  // the previous tile is consumed
            // rows are read coalesced and stored dimension-major
            for (int t = threadIdx.x; t < ET * DP; t += blockDim.x) {
                const int r = t / DP, dim = t - r * DP;
                st[dim * ETP + r] = (uint32_t(r) < cnt && dim < a.d)
                                        ? a.X[(base + j0 + r) * uint64_t(a.d) + dim]
                                        : 0.0f;
            }
            __syncthreads();
#pragma unroll 1
            for (int sub = 0; sub < ET / 32; ++sub) {
                const uint32_t jl = uint32_t(sub * 32 + lane);
                const uint32_t j = j0 + jl;
                float acc[QW];
#pragma unroll
                for (int qi = 0; qi < QW; ++qi) acc[qi] = 0.0f;
#pragma unroll
                for (int t = 0; t < DP; ++t) {
                    float qv[QW];
                    if constexpr (QW % 4 == 0) {
#pragma unroll
                        for (int u = 0; u < QW; u += 4) {
                            const float4 v = *reinterpret_cast<const float4*>(qw + t * QW + u);
                            qv[u] = v.x;
                            qv[u + 1] = v.y;
                            qv[u + 2] = v.z;
                            qv[u + 3] = v.w;
                        }
                    } else {
#pragma unroll
                        for (int qi = 0; qi < QW; ++qi) qv[qi] = qw[t * QW + qi];
                    }
                    const float cv = st[t * ETP + jl];
#pragma unroll
                    for (int qi = 0; qi < QW; ++qi) {
                        const float df = qv[qi] - cv;
                        acc[qi] = fmaf(df, df, acc[qi]);
                    }
                }
                const uint32_t live = __ballot_sync(FULL, jl < cnt);
#pragma unroll
                for (int qi = 0; qi < QW; ++qi) {
                    const uint32_t q = q0 + uint32_t(w * QW + qi);
                    if (q >= ns) continue;  // warp-uniform
                    const uint64_t key = dkey(acc[qi], j);
                    if constexpr (KPL > 0) {
                        // lanes below the k-th key, in index order, each
                        // re-checked against the k-th after an insertion
                        uint32_t pending = live & ~__ballot_sync(FULL, j == q) &
                                           __ballot_sync(FULL, key < thr[qi]);
                        while (pending) {
                            const int l = __ffs(pending) - 1;
                            const uint64_t x = __shfl_sync(FULL, key, l);
                            sorted_insert<KPL>(kv[qi], x, lane);
                            thr[qi] = kth_key<KPL>(kv[qi], k);
                            pending &= (l == 31) ? 0u : ~((2u << l) - 1u);
                            pending &= __ballot_sync(FULL, key < thr[qi]);
                        }
                        continue;
                    }
                    uint64_t* h = heaps + size_t(w * QW + qi) * kp;
                    uint32_t pending = live & ~__ballot_sync(FULL, j == q);
                    // while short, every candidate is pushed in index order
                    while (pending && hlen[qi] < k) {
                        const int l = __ffs(pending) - 1;
                        pending &= pending - 1;
                        const uint64_t kl = __shfl_sync(FULL, key, l);
                        if (lane == 0) {
                            h[hlen[qi]] = kl;
                            heap_up(h, hlen[qi]);
                        }
                        ++hlen[qi];
                        __syncwarp();
                    }
                    // then the first remaining lane that beats the root, in order
                    while (pending) {
                        const uint64_t root = h[0];
                        const uint32_t m = __ballot_sync(FULL, ((pending >> lane) & 1u) && key < root);
                        if (!m) break;
                        const int l = __ffs(m) - 1;
                        pending &= (l == 31) ? 0u : ~((2u << l) - 1u);
                        const uint64_t kl = __shfl_sync(FULL, key, l);
                        if (lane == 0) {
                            h[0] = kl;
                            heap_down(h, hlen[qi]);
                        }
                        __syncwarp();
                    }
                }
            }
        }
        // write each query's k nearest: the register places as they stand, or
        // the heap sorted (padded to kp)
        if constexpr (KPL > 0) {
#pragma unroll
            for (int qi = 0; qi < QW; ++qi) {
                const uint32_t q = q0 + uint32_t(w * QW + qi);
                if (q >= ns) continue;
                const uint64_t o = a.s_out[s] + uint64_t(q) * uint64_t(k);
#pragma unroll
                for (int t = 0; t < KPL; ++t) {
                    const int p = lane * KPL + t;
                    if (p < k) {
                        const uint64_t v = kv[qi][t];
                        const bool ok = v != ~0ull;
                        a.out_idx[o + p] = ok ? uint32_t(v) : 0xFFFFFFFFu;
                        a.out_dist[o + p] = ok ? __fsqrt_rn(__uint_as_float(uint32_t(v >> 32)))
                                               : __int_as_float(0x7f800000);
                    }
                }
            }
        } else {
#pragma unroll 1
            for (int qi = 0; qi < QW; ++qi) {
                const uint32_t q = q0 + uint32_t(w * QW + qi);
                if (q >= ns) continue;
                uint64_t* h = heaps + size_t(w * QW + qi) * kp;
                sort_keys(h, hlen[qi], kp, lane);
                const uint64_t o = a.s_out[s] + uint64_t(q) * uint64_t(k);
                for (int t = lane; t < k; t += 32) {
                    const uint64_t v = h[t];
                    const bool ok = t < hlen[qi];
                    a.out_idx[o + t] = ok ? uint32_t(v) : 0xFFFFFFFFu;
                    a.out_dist[o + t] = ok ? __fsqrt_rn(__uint_as_float(uint32_t(v >> 32)))
                                           : __int_as_float(0x7f800000);
                }
                __syncwarp();
            }
        }
    }
}

template <int DP, int QW, int NW, int KPL>
size_t smem_bytes(int kp) {
    return size_t(NW) * DP * QW * 4 + size_t((DP * ETP + 1) & ~1) * 4 +
           (KPL > 0 ? 0 : size_t(NW) * QW * kp * 8);
}

struct Shape {
    int qw, nw;
};
constexpr Shape SHAPES[] = {{4, 4}, {8, 4}, {4, 8}, {8, 8}};

template <int DP, int QW, int NW, int KPL>
cudaError_t launch_kpl(const BatchArgs& a, int sms, cudaStream_t st) {
    const size_t sm = smem_bytes<DP, QW, NW, KPL>(a.kp);
    cudaError_t e = cudaFuncSetAttribute(k_batched_knn<DP, QW, NW, KPL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batched_knn<DP, QW, NW, KPL>,
                                                      NW * 32, sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const uint32_t grid =
        uint32_t(std::min<uint64_t>(uint64_t(per_sm) * sms, std::max<uint32_t>(a.n_items, 1)));
    k_batched_knn<DP, QW, NW, KPL><<<grid, NW * 32, sm, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

// Places per lane of the register selection for a heap capacity kp, 0 (the
// shared-memory heap) when the QW queries' places would exceed 32 registers
// of keys per lane.
constexpr int reg_places(int qw, int kp) {
    return kp <= 64 ? 2 : (kp <= 128 ? (qw * 4 <= 32 ? 4 : 0) : (kp <= 256 && qw * 8 <= 32 ? 8 : 0));
}

template <int DP, int QW, int NW>
cudaError_t launch_shape(const BatchArgs& a, int sms, cudaStream_t st) {
    switch (reg_places(QW, a.kp)) {
        case 2: return launch_kpl<DP, QW, NW, 2>(a, sms, st);
        case 4: return launch_kpl<DP, QW, NW, 4>(a, sms, st);
        case 8: return launch_kpl<DP, QW, NW, 8>(a, sms, st);
        default: return launch_kpl<DP, QW, NW, 0>(a, sms, st);
    }
}

template <int DP>
cudaError_t launch_dp(const BatchArgs& a, int shape, int sms, cudaStream_t st) {
    switch (shape) {
        case 0: return launch_shape<DP, 4, 4>(a, sms, st);
        case 1: return launch_shape<DP, 8, 4>(a, sms, st);
        case 2: return launch_shape<DP, 4, 8>(a, sms, st);
        default: return launch_shape<DP, 8, 8>(a, sms, st);
    }
}

}  // namespace

int batched_shapes() { return int(sizeof(SHAPES) / sizeof(SHAPES[0])); }

int batched_queries_per_item(int shape) { return SHAPES[shape].qw * SHAPES[shape].nw; }

bool batched_shape_fits(int shape, int d, int kp) {
    const int DP = d <= 32 ? 32 : 64;
    const Shape sh = SHAPES[shape];
    const size_t heap = reg_places(sh.qw, kp) > 0 ? 0 : size_t(sh.nw) * sh.qw * kp * 8;
    const size_t sm = size_t(sh.nw) * DP * sh.qw * 4 + size_t((DP * ETP + 1) & ~1) * 4 + heap;
    return sm <= 200 * 1024;
}

cudaError_t launch_batched_knn(const BatchLaunch& b, int shape, cudaStream_t st) {
    BatchArgs a{};
    a.X = b.X;
    a.d = b.d;
    a.s_off = b.s_off;
    a.s_k = b.s_k;
    a.s_out = b.s_out;
    a.item_s = b.item_s;
    a.item_q = b.item_q;
    a.n_items = b.n_items;
    a.counter = b.counter;
    a.kp = b.kp;
    a.out_idx = b.out_idx;
    a.out_dist = b.out_dist;
    if (b.d < 1 || b.d > 64 || shape < 0 || shape >= batched_shapes()) return cudaErrorInvalidValue;
    if (b.d <= 32) return launch_dp<32>(a, shape, b.sms, st);
    return launch_dp<64>(a, shape, b.sms, st);
}

}  // namespace pq
