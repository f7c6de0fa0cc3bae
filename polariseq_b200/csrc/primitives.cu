// Exclusive scan and stable LSD radix sort (see primitives.cuh).
#include "primitives.cuh"
#include "common.cuh"

namespace pq {
namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_IPT = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;

// Inclusive block scan of one u64 per thread; returns the exclusive prefix and
// writes the block total to *total.
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t* warp_sums,
                                                    uint64_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        uint64_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;  // inclusive warp totals
    }
    __syncthreads();
    uint64_t wp = w > 0 ? warp_sums[w - 1] : 0;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    return wp + x - v;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_k(const T* in, size_t n,
                                                              uint64_t* sums) {
    __shared__ uint64_t ws[32];
    size_t base = size_t(blockIdx.x) * SCAN_TILE;
    uint64_t s = 0;
    for (int i = threadIdx.x; i < SCAN_TILE; i += SCAN_THREADS) {
        size_t g = base + i;
        if (g < n) s += uint64_t(in[g]);
    }
    uint64_t tot;
    block_excl_scan(s, ws, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_down_k(const T* in, T* out, size_t n,
                                                            const uint64_t* offs,
                                                            uint64_t* total_dev) {
    __shared__ T tile[SCAN_TILE];
    __shared__ uint64_t ws[32];
    size_t base = size_t(blockIdx.x) * SCAN_TILE;
    for (int i = threadIdx.x; i < SCAN_TILE; i += SCAN_THREADS) {
        size_t g = base + i;
        tile[i] = g < n ? in[g] : T(0);
    }
    __syncthreads();
    T v[SCAN_IPT];
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        v[j] = tile[threadIdx.x * SCAN_IPT + j];
        s += uint64_t(v[j]);
    }
    uint64_t tot;
    uint64_t run = block_excl_scan(s, ws, &tot) + (offs ? offs[blockIdx.x] : 0);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SCAN_IPT; ++j) {
        tile[threadIdx.x * SCAN_IPT + j] = T(run);
        run += uint64_t(v[j]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SCAN_TILE; i += SCAN_THREADS) {
        size_t g = base + i;
        if (g < n) out[g] = tile[i];
    }
    if (total_dev && threadIdx.x == 0) *total_dev = tot + (offs ? offs[blockIdx.x] : 0);
}

size_t round32(size_t x) { return (x + 31) / 32 * 32; }

template <typename T>
cudaError_t scan_impl(const T* in, T* out, size_t n, uint64_t* temp, uint64_t* total_dev,
                      cudaStream_t st) {
    if (n == 0) {
        if (total_dev) return cudaMemsetAsync(total_dev, 0, sizeof(uint64_t), st);
        return cudaSuccess;
    }
    size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        scan_down_k<T><<<1, SCAN_THREADS, 0, st>>>(in, out, n, nullptr, total_dev); count_launch();
        return cudaGetLastError();
    }
    uint64_t* sums = temp;
    scan_reduce_k<T><<<unsigned(nb), SCAN_THREADS, 0, st>>>(in, n, sums); count_launch();
    cudaError_t e = scan_impl<uint64_t>(sums, sums, nb, temp + round32(nb), total_dev, st);
    if (e != cudaSuccess) return e;
    scan_down_k<T><<<unsigned(nb), SCAN_THREADS, 0, st>>>(in, out, n, sums, nullptr); count_launch();
    return cudaGetLastError();
}

// ── radix sort ─────────────────────────────────────────────────────────────
constexpr int RS_WARPS = 8;
constexpr int RS_IPT = 16;
constexpr int RS_THREADS = RS_WARPS * 32;
constexpr int RS_TILE = RS_THREADS * RS_IPT;
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;

__global__ void __launch_bounds__(RS_THREADS) rs_upsweep(const uint32_t* keys, size_t n,
                                                         int shift, uint32_t* hist,
                                                         uint32_t ntiles) {
    __shared__ uint32_t h[RS_BINS];
    h[threadIdx.x] = 0;
    __syncthreads();
    size_t base = size_t(blockIdx.x) * RS_TILE;
    for (int i = threadIdx.x; i < RS_TILE; i += RS_THREADS) {
        size_t g = base + i;
        if (g < n) atomicAdd(&h[(keys[g] >> shift) & (RS_BINS - 1)], 1u);
    }
    __syncthreads();
    hist[size_t(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Warp multi-split: items of a tile are ranked in (warp, step, lane) order,
// which is their input order, so equal digits keep their relative order.
__global__ void __launch_bounds__(RS_THREADS) rs_downsweep(
    const uint32_t* __restrict__ kin, const uint64_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint64_t* __restrict__ vout, size_t n, int shift, const uint32_t* __restrict__ offs,
    uint32_t ntiles) {
    __shared__ uint32_t cnt[RS_WARPS][RS_BINS];
    __shared__ uint32_t goff[RS_BINS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&cnt[0][0])[i] = 0;
    goff[threadIdx.x] = offs[size_t(threadIdx.x) * ntiles + blockIdx.x];
    __syncthreads();
    const size_t base = size_t(blockIdx.x) * RS_TILE + size_t(w) * 32 * RS_IPT;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t key[RS_IPT], rnk[RS_IPT];
#pragma unroll
    for (int s = 0; s < RS_IPT; ++s) {
        size_t g = base + size_t(s) * 32 + lane;
        bool valid = g < n;
        uint32_t k = valid ? kin[g] : 0u;
        key[s] = k;
        uint32_t dg = (k >> shift) & (RS_BINS - 1);
        unsigned peers = __match_any_sync(0xFFFFFFFFu, valid ? dg : 0x10000u + lane);
        uint32_t before = valid ? cnt[w][dg] : 0u;
        __syncwarp();
        if (valid && (__ffs(peers) - 1) == lane) cnt[w][dg] = before + __popc(peers);
        __syncwarp();
        rnk[s] = before + __popc(peers & lt);
    }
    __syncthreads();
    {  // per digit: warp counts -> exclusive warp offsets
        uint32_t run = 0;
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            uint32_t c = cnt[ww][threadIdx.x];
            cnt[ww][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < RS_IPT; ++s) {
        size_t g = base + size_t(s) * 32 + lane;
        if (g < n) {
            uint32_t dg = (key[s] >> shift) & (RS_BINS - 1);
            uint32_t dst = goff[dg] + cnt[w][dg] + rnk[s];
            kout[dst] = key[s];
            vout[dst] = vin[g];
        }
    }
}

}  // namespace

size_t scan_temp_bytes(size_t n) {
    size_t total = 0;
    while (n > size_t(SCAN_TILE)) {
        n = (n + SCAN_TILE - 1) / SCAN_TILE;
        total += round32(n);
    }
    return (total + 64) * sizeof(uint64_t);
}

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, void* temp,
                               uint64_t* total_dev, cudaStream_t st) {
    return scan_impl<uint32_t>(in, out, n, static_cast<uint64_t*>(temp), total_dev, st);
}

cudaError_t scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, void* temp,
                               uint64_t* total_dev, cudaStream_t st) {
    return scan_impl<uint64_t>(in, out, n, static_cast<uint64_t*>(temp), total_dev, st);
}

size_t radix_temp_bytes(size_t n) {
    size_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    size_t hist = size_t(RS_BINS) * ntiles;
    return round32(hist) * sizeof(uint32_t) + scan_temp_bytes(hist) + 256;
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint64_t* vals, uint32_t* keys_alt,
                             uint64_t* vals_alt, size_t n, int key_bits, void* temp,
                             cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    size_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    size_t hist_n = size_t(RS_BINS) * ntiles;
    uint32_t* hist = static_cast<uint32_t*>(temp);
    void* stemp = reinterpret_cast<char*>(temp) + round32(hist_n) * sizeof(uint32_t);
    uint32_t *ki = keys, *ko = keys_alt;
    uint64_t *vi = vals, *vo = vals_alt;
    int passes = (key_bits + RS_BITS - 1) / RS_BITS;
    if (passes < 1) passes = 1;
    for (int p = 0; p < passes; ++p) {
        int shift = p * RS_BITS;
        rs_upsweep<<<unsigned(ntiles), RS_THREADS, 0, st>>>(ki, n, shift, hist, uint32_t(ntiles)); count_launch();
        cudaError_t e = scan_exclusive_u32(hist, hist, hist_n, stemp, nullptr, st);
        if (e != cudaSuccess) return e;
        rs_downsweep<<<unsigned(ntiles), RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, shift, hist,
                                                               uint32_t(ntiles)); count_launch();
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    if (ki != keys) {
        cudaMemcpyAsync(keys, ki, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, vi, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
    }
    return cudaGetLastError();
}

}  // namespace pq
