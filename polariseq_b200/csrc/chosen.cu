// Chosen form: a tensor-core shortlist over buckets, exact FP32 re-rank and an
// FP64 boundary step.
//
//   1. buckets: Lloyd k-means on an evenly strided sample of the cells (FP32),
//      then every cell's P nearest centroids by the tensor-core tile kernel
//      (one bucket holding all centroids); the nearest is its primary bucket;
//   2. layout: cells sorted by primary bucket (stable radix sort); each cell's
//      BF16 row centred on its bucket's centroid; query entries (cell, probe)
//      grouped by probe bucket, centred on the probe's centroid;
//   3. the tile kernel (ivf.cu) keeps each entry's S nearest by approximate
//      |q~|^2 + |x~|^2 - 2 q~.x~;
//   4. re-rank: per cell, the R best of its P*S shortlist by approximate
//      distance get their exact FP32 squared distance in the reference's
//      summation order (simd.rs:43-62), sorted by (distance, index); where the
//      k-th and (k+1)-th differ by less than the FP32 error bound, FP64
//      distances choose which of the band's entries are kept, and the kept
//      entries are written in ascending FP32 order;
//   5. optional NN-Descent rounds (the plain form's round kernels) polish the
//      lists; the extract writes the CSR graph.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstdio>
#include <optional>

#include "ctx.cuh"
#include "ivf.cuh"
#include "kernels.cuh"
#include "primitives.cuh"

namespace pq {
namespace {

constexpr float FP32_BOUND = 1e-5f;  // relative band of the FP64 boundary step

// The k-means sample: KB blocks of bl consecutive rows, block b starting at
// row b * s (padded rows).
__global__ void k_block_rows(const float* __restrict__ X, int dp, uint64_t s, uint32_t bl,
                             uint32_t ns, float* __restrict__ out) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(ns) * dp) return;
    const uint32_t j = uint32_t(t / dp), c = uint32_t(t - size_t(j) * dp);
    const uint64_t row = uint64_t(j / bl) * s + (j % bl);
    out[t] = X[row * dp + c];
}

// n rows of d columns -> padded rows of dp (zeros past d).
__global__ void k_pad_cols(const float* __restrict__ src, uint32_t n, int d, int dp,
                           float* __restrict__ dst) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(n) * dp) return;
    const size_t i = t / dp;
    const int j = int(t - i * dp);
    dst[t] = j < d ? src[i * d + j] : 0.0f;
}

// Evenly strided sample of the padded rows.
__global__ void k_sample_rows(const float* __restrict__ X, int dp, uint32_t n, uint32_t ns,
                              float* __restrict__ out) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(ns) * dp) return;
    const uint32_t j = uint32_t(t / dp), c = uint32_t(t - size_t(j) * dp);
    const uint64_t i = uint64_t(j) * n / ns;
    out[t] = X[i * dp + c];
}

// Column sums of padded rows (for the mean used as the centroid search's BF16 centre).
// Column means of n rows: one 256-thread block per column, each thread
// summing a fixed stride of rows, then a fixed tree (deterministic).
__global__ void k_col_mean(const float* __restrict__ X, uint32_t n, int dp, float* mean) {
    __shared__ float part[256];
    const int j = blockIdx.x;
    float s = 0.f;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s += X[size_t(i) * dp + j];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (int(threadIdx.x) < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) mean[j] = part[0] / float(n);
}

// Lloyd update sums from the tensor-core nearest-centroid labels: keys =
// label (C for none), values = sample index, to be sorted stably by label.
__global__ void k_label_pairs(const uint32_t* __restrict__ lab, uint32_t ns, uint32_t C,
                              uint32_t* __restrict__ keys, uint64_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    keys[i] = lab[i] < C ? lab[i] : C;
    vals[i] = i;
}
// Per centroid (one warp): its members' sums in sample order (deterministic)
// and their count; off = the label bounds of the sorted pairs.
__global__ void k_kmeans_sums(const float* __restrict__ xs, int d, int dp,
                              const uint64_t* __restrict__ members,
                              const uint32_t* __restrict__ off, uint32_t C,
                              float* __restrict__ sums, uint32_t* __restrict__ cnt) {
    const uint32_t b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= C) return;
    const uint32_t m0 = off[b], m1 = off[b + 1];
    for (int j = lane; j < d; j += 32) {
        float s = 0.f;
        for (uint32_t m = m0; m < m1; ++m) s += xs[size_t(members[m]) * dp + j];
        sums[size_t(b) * dp + j] = s;
    }
    if (lane == 0) cnt[b] = m1 - m0;
}

// Query-entry keys and values (slot = position * P + rank) from the probes.  Primary
// entries (rank 0) sort first, by (bucket, second-nearest centroid) exactly
// as the candidates do, so that a primary job's own cells form its first
// candidate tile; the others follow by (probe bucket, the cell's primary
// bucket), so that a job's queries come from one neighbouring bucket and meet
// the candidates on that side of the probe bucket first.
// Entry e = (candidate position p, probe rank r), p = e / P, of cell
// perm[p]: key (primary entries) = the cell's candidate key, (others) =
// (C + probe bucket) * C + primary bucket; value = its slot p * P + r (= e).
// Generated in candidate order, so that after the stable sort the entries of
// one (probe, primary) pair follow the primary bucket's candidate order.
__global__ void k_entry_keys(const uint32_t* __restrict__ probes,
                             const uint32_t* __restrict__ perm, size_t ne, int P, uint32_t C,
                             uint32_t* __restrict__ keys, uint64_t* __restrict__ vals) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const size_t p = e / P;
    const uint32_t r = uint32_t(e - p * P);
    const size_t i = perm[p];
    const uint32_t a = probes[i * P];
    if (r == 0)
        keys[e] = a * C + (P > 1 ? probes[i * P + 1] : 0u);
    else
        keys[e] = (C + probes[i * P + r]) * C + a;
    vals[e] = e;
}

// The embedding rows in candidate order (xp[p] = X[perm[p]], dp floats each).
__global__ void k_gather_rows(const float4* __restrict__ X, const uint32_t* __restrict__ perm,
                              uint32_t n, int dq, float4* __restrict__ xp) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(n) * dq) return;
    const size_t p = t / dq;
    xp[t] = X[size_t(perm[p]) * dq + (t - p * dq)];
}

// First candidate tile of each job of the non-primary pass: where the probe
// bucket's candidates whose second-nearest centroid is the job's primary
// bucket begin (candidate key = bucket * C + second-nearest centroid).
__global__ void k_job_tstart(const uint32_t* __restrict__ job_bucket,
                             const uint32_t* __restrict__ job_qstart, uint32_t njobs,
                             const uint32_t* __restrict__ ekeys, uint32_t C,
                             const uint32_t* __restrict__ c_off,
                             const uint32_t* __restrict__ pair_off, uint32_t tile_cols,
                             uint32_t* __restrict__ tstart) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const uint32_t b = job_bucket[j];
    const uint32_t a = ekeys[job_qstart[j]] % C;
    tstart[j] = (pair_off[size_t(b) * C + a] - c_off[b]) / tile_cols;
}

// Seed thresholds of the non-primary entries: the R-th best approximate
// distance of the cell's primary shortlist (a candidate of another bucket can
// only enter the cell's R best if it beats that); +inf when the primary
// shortlist holds fewer than R.  Per candidate position p (the cell perm[p]);
// entry_of and sn are indexed by slot p * P + rank.
__global__ void k_seed_thresholds(const uint32_t* __restrict__ entry_of, uint32_t n, int P,
                                  const float* __restrict__ sd, const uint8_t* __restrict__ sn,
                                  int S, int R, float* __restrict__ cseed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t e0 = entry_of[size_t(i) * P];  // i: the position
    // the R-th smallest of the entry's two ascending runs (live prefixes)
    const float* r0 = sd + size_t(e0) * 2 * S;
    const float* r1 = r0 + S;
    const int n0 = sn[size_t(i) * P * 2], n1 = sn[size_t(i) * P * 2 + 1];
    int x = 0, y = 0;
    float t = __int_as_float(0x7f800000);
    if (n0 + n1 >= R) {
        for (int o = 0; o < R; ++o) {
            const float vx = x < n0 ? r0[x] : __int_as_float(0x7f800000);
            const float vy = y < n1 ? r1[y] : __int_as_float(0x7f800000);
            if (vx <= vy) {
                t = vx;
                ++x;
            } else {
                t = vy;
                ++y;
            }
        }
    }
    cseed[i] = t;
}

// Exact FP32 squared distance of the cell at every candidate position p
// (row xp[p], cell perm[p]) to each of its P probe centroids (d[p * P + r]),
// each bucket's squared radius over its own cells (rad2[b] = max over cells
// whose primary is b) and the largest |y - mean|^2 of its cells (umax2[b],
// from un, per cell); non-negative floats order as their bits.  One warp per
// position: each half-warp takes every other probe, lane h holding
// dimensions 4h..4h+3 (16-byte loads of the row and the centroid), the sum
// reduced over the half-warp.  Needs dp <= 64.
__global__ void k_probe_dist(const float* __restrict__ xp, const uint32_t* __restrict__ perm,
                             int d, int dp, uint32_t n, const uint32_t* __restrict__ probes, int P,
                             const float* __restrict__ cent, const float* __restrict__ un,
                             float* __restrict__ dist, unsigned* __restrict__ rad2,
                             unsigned* __restrict__ umax2) {
    // one warp per candidate position; the block's 8 positions are
    // consecutive, mostly of one bucket, so the bucket maxima are reduced in
    // the block first and each run of equal buckets does one atomic pair
    __shared__ uint32_t sb[8];
    __shared__ unsigned sr[8], su[8];
    const int w = threadIdx.x >> 5;
    const uint32_t p = blockIdx.x * (blockDim.x / 32) + w;
    const bool valid = p < n;
    const int lane = threadIdx.x & 31, h = lane & 15, half = lane >> 4;
    const unsigned hm = 0xFFFFu << (lane & 16);
    if (valid) {
        const uint32_t i = perm[p];
        // every probe id at once (P <= 16), each round takes its two by shuffle
        const uint32_t pr = lane < P ? probes[size_t(i) * P + lane] : 0u;
        float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (4 * h < dp) x4 = reinterpret_cast<const float4*>(xp + size_t(p) * dp)[h];
        const float xs[4] = {x4.x, x4.y, x4.z, x4.w};
        // both halves run the same number of rounds (the shuffles need their lanes)
        for (int r0 = 0; r0 < P; r0 += 2) {
            const int r = r0 + half;
            const bool live = r < P;
            const uint32_t c = __shfl_sync(0xFFFFFFFFu, pr, live ? r : 0);
            float s = 0.f;
            if (live && 4 * h < dp) {
                const float4 c4 = reinterpret_cast<const float4*>(cent + size_t(c) * dp)[h];
                const float cs[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (4 * h + u < d) {
                        const float df = xs[u] - cs[u];
                        s = fmaf(df, df, s);
                    }
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(hm, s, o);
            if (live && h == 0) {
                dist[size_t(p) * P + r] = s;
                if (r == 0 && lane == 0) {
                    sb[w] = c;
                    sr[w] = __float_as_uint(s);
                    su[w] = __float_as_uint(un[i]);
                }
            }
        }
    }
    __syncthreads();
    // one atomic pair per run of equal buckets among the block's positions
    if (threadIdx.x < 8) {
        const int t = threadIdx.x;
        const uint32_t nv = min(8u, n > blockIdx.x * 8u ? n - blockIdx.x * 8u : 0u);
        if (uint32_t(t) < nv && (t == 0 || sb[t] != sb[t - 1])) {
            unsigned mr = sr[t], mu = su[t];
            for (uint32_t q = t + 1; q < nv && sb[q] == sb[t]; ++q) {
                mr = max(mr, sr[q]);
                mu = max(mu, su[q]);
            }
            atomicMax(&rad2[sb[t]], mr);
            atomicMax(&umax2[sb[t]], mu);
        }
    }
}

// Exact distances between centroids: cd[a * C + b] = |c_a - c_b|.
__global__ void k_cent_dist(const float* __restrict__ cent, uint32_t C, int d, int dp,
                            float* __restrict__ cd) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(C) * C) return;
    const size_t a = t / C, b = t - a * C;
    float s = 0.f;
    for (int j = 0; j < d; ++j) {
        const float df = cent[a * dp + j] - cent[b * dp + j];
        s = fmaf(df, df, s);
    }
    cd[t] = sqrtf(s);
}

// The largest of m non-negative floats (one block).
__global__ void k_max_nonneg(const float* __restrict__ v, uint32_t m, unsigned* __restrict__ out) {
    unsigned best = 0;
    for (uint32_t t = threadIdx.x; t < m; t += blockDim.x) best = max(best, __float_as_uint(v[t]));
    atomicMax(out, best);
}

// Which other-probe entries can hold a candidate that the tile pass would
// admit.  Two exact lower bounds on |x - y| for every candidate y of bucket B
// (x's own bucket A):
//  - ball: y lies within B's radius r_B of c_B: |x - y| >= |x - c_B| - r_B;
//  - bisector: y was assigned to B by BF16 distances (rows centred on the
//    global mean, |y - mean| + |c - mean| <= U_B), so |y - c_B|^2 <=
//    |y - c_A|^2 + delta with delta = 2^-6 (2 r_B + L) U_B + 2^-14 U_B^2
//    (twice the rounding bound, using |y - c_A| <= r_B + L, L = |c_A - c_B|),
//    and then |x - y| >= (|x - c_B|^2 - |x - c_A|^2 - delta) / (2 L).
// The pass admits y only if its BF16 distance (rows centred on c_B) is below
// the cell's seed; that distance is at least f(|x - y|^2) with
// f(t) = t - 2^-6 sqrt(t) a - 2^-15 a^2 - 2^-9 (|x - c_B|^2 + r_B^2),
// a = |x - c_B| + r_B (twice the worst case of the rounding of both rows to
// BF16, each coordinate within 2^-8 relative, plus the FP32 accumulation and
// the split norm columns), and f grows with t where it is positive.  So an
// entry with f(lb^2) >= seed (lb the larger bound) admits nothing and is
// dropped: keep[j] = 0.  Entries j are the sorted other-probe entries (key =
// (C + B) * C + A, value = slot p * P + rank); distances are FP32 (their
// rounding is covered by the 2^-20 and 2^-18 terms).
__global__ void k_prune_keep(const uint32_t* __restrict__ keys, const uint64_t* __restrict__ vals,
                             size_t m, int P, uint32_t C, const float* __restrict__ dist,
                             const unsigned* __restrict__ rad2, const unsigned* __restrict__ umax2,
                             const unsigned* __restrict__ wmax2, const float* __restrict__ cd,
                             const float* __restrict__ cseed, uint32_t* __restrict__ keep) {
    const size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const uint64_t v = vals[j];
    const uint64_t i = v / uint64_t(P);
    const uint32_t key = keys[j];
    const uint32_t b = key / C - C, pa = key % C;
    const float dxb = dist[v], dxa = dist[i * P];
    const float r2 = __uint_as_float(rad2[b]);
    const float dx = sqrtf(dxb), rb = sqrtf(r2);
    float lb = dx * (1.0f - 0x1p-20f) - rb * (1.0f + 0x1p-20f);
    const float L = cd[size_t(pa) * C + b];
    if (L > 0.f) {
        const float ub = sqrtf(__uint_as_float(umax2[b])) + sqrtf(__uint_as_float(*wmax2));
        const float delta = 0x1p-6f * (2.0f * rb + L) * ub + 0x1p-14f * ub * ub +
                            0x1p-18f * (dxa + dxb);
        lb = fmaxf(lb, (dxb - dxa - delta) / (2.0f * L * (1.0f + 0x1p-20f)));
    }
    uint32_t k = 1;
    if (lb > 0.f) {
        const float t = lb * lb, a = dx + rb;
        const float f = t - 0x1p-6f * lb * a - 0x1p-15f * a * a - 0x1p-9f * (dxb + r2);
        if (f >= cseed[i]) k = 0;
    }
    keep[j] = k;
}

// Stable compaction of the kept entries: pos = exclusive scan of keep.
__global__ void k_compact_entries(const uint32_t* __restrict__ keys,
                                  const uint64_t* __restrict__ vals, size_t m,
                                  const uint32_t* __restrict__ keep,
                                  const uint32_t* __restrict__ pos, uint32_t* __restrict__ okeys,
                                  uint64_t* __restrict__ ovals) {
    const size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= m || !keep[j]) return;
    okeys[pos[j]] = keys[j];
    ovals[pos[j]] = vals[j];
}

// Admission bound of each laid-out other-probe entry: its cell's seed.
__global__ void k_entry_thr(const uint32_t* __restrict__ slot, size_t m, int P,
                            const float* __restrict__ cseed, float* __restrict__ qthr) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < m) qthr[e] = cseed[slot[e] / uint32_t(P)];
}

__global__ void k_kmeans_update(float* __restrict__ cent, const float* __restrict__ sums,
                                const uint32_t* __restrict__ cnt, uint32_t C, int d, int dp) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(C) * dp) return;
    const uint32_t c = uint32_t(t / dp), j = uint32_t(t - size_t(c) * dp);
    if (j < uint32_t(d) && cnt[c] > 0) cent[t] = sums[t] / float(cnt[c]);
}

// BF16 rows (64 dims, zero padded) of (row(src_i) - center(c_i)), and their
// squared norms computed in FP32 from the rounded values.  Columns d and d+1
// carry the augmentation of the tensor-core tiles: -1/2, -1/2 for a query row
// (aug 1), and hi, lo with hi + lo = the row's norm for a candidate row (aug 2).
// A half-warp per row (lane h: columns 4h..4h+3, one 16-byte load of the row
// and of the centre, one 8-byte store), grid-stride over the rows; needs
// dp <= 64 and d <= 62.
__global__ void k_to_bf16(const float* __restrict__ X, int d, int dp,
                          const uint32_t* __restrict__ src, const uint32_t* __restrict__ cid,
                          const float* __restrict__ cent, size_t rows, int aug,
                          __nv_bfloat16* __restrict__ out, float* __restrict__ norm) {
    const int h = threadIdx.x & 15;
    const unsigned hm = 0xFFFFu << (threadIdx.x & 16);  // this half-warp's lanes
    const size_t nh = (size_t(gridDim.x) * blockDim.x) >> 4;
    for (size_t r = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 4; r < rows; r += nh) {
        const uint32_t i = src ? src[r] : uint32_t(r);
        const uint32_t c = cid ? cid[r] : 0u;
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (4 * h < dp) {
            const float4 x4 = *reinterpret_cast<const float4*>(X + size_t(i) * dp + 4 * h);
            const float4 c4 = *reinterpret_cast<const float4*>(cent + size_t(c) * dp + 4 * h);
            v[0] = x4.x - c4.x;
            v[1] = x4.y - c4.y;
            v[2] = x4.z - c4.z;
            v[3] = x4.w - c4.w;
        }
        __nv_bfloat16 bv[4];
        float s = 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            bv[u] = __float2bfloat16_rn(4 * h + u < d ? v[u] : 0.f);
            const float f = __bfloat162float(bv[u]);
            s = fmaf(f, f, s);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(hm, s, o);
        const __nv_bfloat16 hi = __float2bfloat16_rn(s);
        const __nv_bfloat16 lo = __float2bfloat16_rn(s - __bfloat162float(hi));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = 4 * h + u;
            if (aug == 1 && (j == d || j == d + 1)) bv[u] = __float2bfloat16_rn(-0.5f);
            if (aug == 2 && j == d) bv[u] = hi;
            if (aug == 2 && j == d + 1) bv[u] = lo;
        }
        uint2 w;
        w.x = uint32_t(__bfloat16_as_ushort(bv[0])) | (uint32_t(__bfloat16_as_ushort(bv[1])) << 16);
        w.y = uint32_t(__bfloat16_as_ushort(bv[2])) | (uint32_t(__bfloat16_as_ushort(bv[3])) << 16);
        *reinterpret_cast<uint2*>(out + r * 64 + 4 * h) = w;
        if (h == 0) norm[r] = s;
    }
}

// Grid of the BF16 conversion: 16 rows per 256-thread block, at most 4096 blocks.
inline unsigned cvt_blocks(size_t rows) {
    const size_t b = (rows + 15) / 16;
    return unsigned(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

// The s_out nearest of two ascending runs of S per row (distinct ids).
__global__ void k_merge_runs(const float* __restrict__ rd, const uint32_t* __restrict__ ri,
                             uint32_t rows, int S, int s_out, float* __restrict__ od,
                             uint32_t* __restrict__ oi) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const size_t base = size_t(r) * 2 * S;
    int x = 0, y = 0;
    for (int o = 0; o < s_out; ++o) {
        const float vx = x < S ? rd[base + x] : __int_as_float(0x7f800000);
        const float vy = y < S ? rd[base + S + y] : __int_as_float(0x7f800000);
        const uint32_t ix = x < S ? ri[base + x] : 0xFFFFFFFFu;
        const uint32_t iy = y < S ? ri[base + S + y] : 0xFFFFFFFFu;
        const bool takex = vx < vy || (vx == vy && ix <= iy);
        od[size_t(r) * s_out + o] = takex ? vx : vy;
        oi[size_t(r) * s_out + o] = takex ? ix : iy;
        if (takex) ++x;
        else ++y;
    }
}

// Power-of-two E4M3 scale 2^floor(log2(448 / absmax)) (exact in FP32), 1 for
// an all-zero row.
__device__ __forceinline__ float e4m3_scale(float amax) {
    return amax > 0.f ? exp2f(floorf(log2f(448.0f / amax))) : 1.0f;
}

// E4M3 rows (128 one-byte columns, zero padded) of (row(src_i) - centre(c_i))
// scaled by the row's own power-of-two scale; inv_scale (may be null)
// receives 1/scale, norm the FP32 |dequantised row|^2 times `norm_mult`.  A
// half-warp per row (lane h: columns 4h..4h+3, one 16-byte load of the row
// and of the centre; columns 64..127 are zero), grid-stride over the rows;
// needs dp <= 64.
__global__ void k_to_fp8(const float* __restrict__ X, int d, int dp,
                         const uint32_t* __restrict__ src, const uint32_t* __restrict__ cid,
                         const float* __restrict__ cent, size_t rows,
                         uint32_t* __restrict__ out,
                         float* __restrict__ inv_scale, float* __restrict__ norm,
                         float norm_mult) {
    const int h = threadIdx.x & 15;
    const unsigned hm = 0xFFFFu << (threadIdx.x & 16);  // this half-warp's lanes
    const size_t nh = (size_t(gridDim.x) * blockDim.x) >> 4;
    for (size_t r = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 4; r < rows; r += nh) {
        const uint32_t i = src ? src[r] : uint32_t(r), c = cid[r];
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (4 * h < dp) {
            const float4 x4 = *reinterpret_cast<const float4*>(X + size_t(i) * dp + 4 * h);
            const float4 c4 = *reinterpret_cast<const float4*>(cent + size_t(c) * dp + 4 * h);
            v[0] = x4.x - c4.x;
            v[1] = x4.y - c4.y;
            v[2] = x4.z - c4.z;
            v[3] = x4.w - c4.w;
        }
        float m = 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (4 * h + u >= d) v[u] = 0.f;
            m = fmaxf(m, fabsf(v[u]));
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(hm, m, o));
        const float sc = e4m3_scale(m);
        uint32_t word = 0;
        float s = 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const __nv_fp8_storage_t q =
                __nv_cvt_float_to_fp8(v[u] * sc, __NV_SATFINITE, __NV_E4M3);
            const __half_raw hr = __nv_cvt_fp8_to_halfraw(q, __NV_E4M3);
            const float deq = __half2float(__half(hr)) / sc;
            s = fmaf(deq, deq, s);
            word |= uint32_t(q) << (8 * u);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(hm, s, o);
        out[r * 32 + h] = word;
        out[r * 32 + 16 + h] = 0u;
        if (h == 0) {
            norm[r] = s * norm_mult;
            if (inv_scale) inv_scale[r] = 1.0f / sc;
        }
    }
}

// Candidate keys: (primary bucket, second-nearest centroid), so that cells of
// a bucket lying towards the same neighbour sit together.
__global__ void k_primary_keys(const uint32_t* __restrict__ probes, int P, uint32_t n, uint32_t C,
                               uint32_t* __restrict__ keys, uint64_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = probes[size_t(i) * P] * C + (P > 1 ? probes[size_t(i) * P + 1] : 0u);
    vals[i] = i;
}

// Offsets of every value v = key / div in a sorted key array: off[v] = first
// position with key / div >= v, for v in [0, nv]; each off entry is written
// exactly once (by the position where the value steps past it, or the last).
__global__ void k_key_bounds(const uint32_t* __restrict__ keys, size_t ne, uint32_t div,
                             uint32_t nv, uint32_t* __restrict__ off) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e > ne) return;
    const uint32_t lo = e == 0 ? 0u : keys[e - 1] / div + 1;
    const uint32_t hi = e == ne ? nv : keys[e] / div;
    for (uint32_t v = lo; v <= hi; ++v) off[v] = uint32_t(e);
}

// Candidate position p -> its cell perm[p] (and back: pos_of) and bucket
// cbucket[p].
__global__ void k_cand_layout(const uint64_t* __restrict__ vals, uint32_t n, uint32_t C,
                              const uint32_t* __restrict__ keys, uint32_t* __restrict__ perm,
                              uint32_t* __restrict__ pos_of, uint32_t* __restrict__ cbucket) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t i = uint32_t(vals[p]);
    perm[p] = i;
    pos_of[i] = p;
    cbucket[p] = keys[p] / C;
}

__global__ void k_entry_layout(const uint64_t* __restrict__ vals, const uint32_t* __restrict__ keys,
                               size_t ne, uint32_t e0, int P, uint32_t C,
                               uint32_t* __restrict__ qpos, uint32_t* __restrict__ qbucket,
                               uint32_t* __restrict__ qself, uint32_t* __restrict__ entry_of,
                               uint32_t* __restrict__ slot) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const uint64_t v = vals[e];  // slot: candidate position * P + probe rank
    const uint32_t pos = uint32_t(v / P), r = uint32_t(v % P);
    const uint32_t kb = keys[e] / C;
    qpos[e] = pos;
    qbucket[e] = kb >= C ? kb - C : kb;
    qself[e] = r == 0 ? pos : 0xFFFFFFFFu;  // rank 0 is the primary bucket
    entry_of[v] = e0 + uint32_t(e);
    slot[e] = uint32_t(v);
}

// Bitonic sort (ascending) of 32 keys held one per lane.
__device__ __forceinline__ uint64_t warp_sort32(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const uint64_t o = __shfl_xor_sync(0xFFFFFFFFu, v, stride);
            const bool lower = (lane & stride) == 0;
            const bool up = (lane & size) == 0 || size == 32;
            v = (lower == up) ? (o < v ? o : v) : (o > v ? o : v);
        }
    return v;
}

// Bitonic sort (ascending) of 64 keys held two per lane (element e of lane l
// is index l + 32 e).
__device__ __forceinline__ void warp_sort64(uint64_t (&v)[2]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 64; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int idx = lane + 32 * e;
                const bool up = (idx & size) == 0;
                if (stride >= 32) {
                    if (e == 0) {  // partner is the other element of this lane
                        const bool swap = up ? v[0] > v[1] : v[0] < v[1];
                        if (swap) {
                            const uint64_t t = v[0];
                            v[0] = v[1];
                            v[1] = t;
                        }
                    }
                } else {
                    const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, v[e], stride);
                    const bool lower = (idx & stride) == 0;
                    const uint64_t lo = v[e] < other ? v[e] : other;
                    const uint64_t hi = v[e] < other ? other : v[e];
                    v[e] = (lower == up) ? lo : hi;
                }
            }
        }
    }
}

// Exact FP64 squared distance of two padded rows.
__device__ __forceinline__ double sq_dist_f64(const float* a, const float* b, int d) {
    double s = 0.0;
    for (int j = 0; j < d; ++j) {
        const double t = double(a[j]) - double(b[j]);
        s += t * t;
    }
    return s;
}

// Re-rank, one warp per cell (cells visited in bucket order): merge the
// ascending shortlist runs of the P probes (SO / RS runs of RS per probe) to
// the R best approximate candidates, give
// them exact FP32 squared distances in the reference's summation order, sort
// by (distance, index), and where the k-th and (k+1)-th differ by less than
// the FP32 error bound let FP64 distances choose which of that band's entries
// are kept.  Writes the k nearest per cell, ascending by FP32 distance.
template <int D>
__global__ void __launch_bounds__(128) k_rerank(
    const float* __restrict__ X, const float* __restrict__ xp, int d, int dp, uint32_t n, int k,
    int P, int SO, int RS, int R,
    const uint32_t* __restrict__ entry_of, const float* __restrict__ sd,
    const uint32_t* __restrict__ si, const uint8_t* __restrict__ sn,
    const uint32_t* __restrict__ perm, const uint32_t* __restrict__ pos_of, uint32_t w0,
    uint32_t* __restrict__ out_idx, float* __restrict__ out_dist,
    unsigned long long* boundary_fixes) {
    __shared__ uint32_t band_i[4][64];
    __shared__ double band_d[4][64];
    __shared__ float band_f[4][64];
    __shared__ uint64_t band_key[4][64];
    // item it in [w0, n): a candidate position (pos_of null) or a cell
    const uint32_t it = w0 + blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (it >= n) return;
    const uint32_t wg = pos_of ? pos_of[it] : it;  // the cell's candidate position
    const uint32_t i = pos_of ? it : perm[wg];     // the cell
    // 1. the R best approximate candidates of the shortlist runs (lane L <
    //    P * NR owns run L % NR of probe L / NR; runs are RS long (a multiple
    //    of 4), ascending, an entry's NR runs RS * NR apart, and the first
    //    sn[position * P * NR + L] entries of run L are its finite ones).  The
    //    live prefixes are copied into shared memory (four entries per vector
    //    load, all issued at once) and sorted as (distance bits, position)
    //    keys — 64 at most, else the runs are merged head by head.
    const int NR = SO / RS;
    const bool owner = lane < P * NR;
    size_t base = 0;
    int fin = 0;
    if (owner) {
        base = size_t(entry_of[size_t(wg) * P + lane / NR]) * SO + size_t(lane % NR) * RS;
        fin = sn[size_t(wg) * P * NR + lane];
    }
    uint32_t cand[2] = {0xFFFFFFFFu, 0xFFFFFFFFu};
    int off = fin;  // inclusive prefix sum of the live counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xFFFFFFFFu, off, o);
        if (lane >= o) off += t;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, off, 31);
    off -= fin;
    if (total <= 64) {
        uint64_t* slot = band_key[w];
        slot[lane] = ~0ull;
        slot[lane + 32] = ~0ull;
        __syncwarp();
        // RS / 4 lanes per run (16 bytes each), 128 / RS runs per pass: each
        // load touches a few cache lines rather than one per lane
        const int nruns = P * NR;
        const int lpr = RS / 4, rpp = 32 / lpr;
        for (int r0 = 0; r0 < nruns; r0 += rpp) {
            const int r = r0 + lane / lpr, c = lane % lpr;
            const uint32_t blo = __shfl_sync(0xFFFFFFFFu, uint32_t(base), r & 31);
            const uint32_t bhi = __shfl_sync(0xFFFFFFFFu, uint32_t(base >> 32), r & 31);
            const int fr = __shfl_sync(0xFFFFFFFFu, fin, r & 31);
            const int orr = __shfl_sync(0xFFFFFFFFu, off, r & 31);
            if (r < nruns) {
                const size_t br = (size_t(bhi) << 32) | blo;
                for (int q = c; 4 * q < fr; q += lpr) {
                    const float4 v4 = *reinterpret_cast<const float4*>(sd + br + 4 * q);
                    const uint4 i4 = *reinterpret_cast<const uint4*>(si + br + 4 * q);
                    const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
                    const uint32_t ii[4] = {i4.x, i4.y, i4.z, i4.w};
#pragma unroll
                    for (int t = 0; t < 4; ++t)
                        if (4 * q + t < fr)
                            slot[orr + 4 * q + t] =
                                (uint64_t(__float_as_uint(fmaxf(vv[t], 0.0f))) << 32) | ii[t];
                }
            }
        }
        __syncwarp();
        uint64_t key[2] = {slot[lane], slot[lane + 32]};
        __syncwarp();
        warp_sort64(key);
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (lane + 32 * h < R && key[h] != ~0ull) cand[h] = uint32_t(key[h]);
    } else {
        uint32_t head = 0;
        for (int t = 0; t < R; ++t) {
            float v = __int_as_float(0x7f800000);
            uint32_t id = 0xFFFFFFFFu;
            if (head < uint32_t(fin)) {
                v = sd[base + head];
                id = si[base + head];
            }
            // warp argmin by (value, candidate)
            float bv = v;
            uint32_t bid = id;
            int bl = lane;
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
                const uint32_t oid = __shfl_xor_sync(0xFFFFFFFFu, bid, o);
                const int ol = __shfl_xor_sync(0xFFFFFFFFu, bl, o);
                if (ov < bv || (ov == bv && oid < bid)) {
                    bv = ov;
                    bid = oid;
                    bl = ol;
                }
            }
            if (bid == 0xFFFFFFFFu) break;  // every list exhausted
            if (lane == bl) ++head;
            if ((t & 31) == lane) cand[t >> 5] = bid;
        }
    }
    // 2. exact FP32 distances (reference order) of this lane's candidates
    //    (rows from the candidate-ordered copy: this cell is position wg)
    const float* xi = xp + size_t(wg) * dp;
    uint64_t key[2];
    {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            key[h] = ~0ull;
            if (cand[h] != 0xFFFFFFFFu) {
                const uint32_t j = perm[cand[h]];
                const float dd = sq_dist_exact_t<D>(xi, xp + size_t(cand[h]) * dp, d);
                key[h] = (uint64_t(__float_as_uint(dd)) << 32) | j;
            }
        }
    }
    // 3. sort by (distance, index): non-negative floats order as their bits
    //    (R <= 32: one key per lane, the second places are empty)
    if (R <= 32)
        key[0] = warp_sort32(key[0]);
    else
        warp_sort64(key);
    // 4. FP64 band at the k-th boundary
    const uint64_t kk1 = __shfl_sync(0xFFFFFFFFu, (k - 1) >= 32 ? key[1] : key[0], (k - 1) & 31);
    const uint64_t kk =
        k < 64 ? __shfl_sync(0xFFFFFFFFu, k >= 32 ? key[1] : key[0], k & 31) : ~0ull;
    const float fk1 = __uint_as_float(uint32_t(kk1 >> 32));
    const float fk = __uint_as_float(uint32_t(kk >> 32));
    if (kk != ~0ull && fk - fk1 <= FP32_BOUND * fk) {
        const float lo = fk1 * (1.0f - FP32_BOUND), hi = fk * (1.0f + FP32_BOUND);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            band_i[w][lane + 32 * h] = uint32_t(key[h]);
            band_f[w][lane + 32 * h] = __uint_as_float(uint32_t(key[h] >> 32));
        }
        __syncwarp();
        if (lane == 0) {
            int b0 = k - 1, b1 = k;
            while (b0 > 0 && band_f[w][b0 - 1] >= lo) --b0;
            while (b1 + 1 < 64 && band_i[w][b1 + 1] != 0xFFFFFFFFu && band_f[w][b1 + 1] <= hi) ++b1;
            for (int t = b0; t <= b1; ++t)
                band_d[w][t] = sq_dist_f64(xi, X + size_t(band_i[w][t]) * dp, d);
            for (int a = b0 + 1; a <= b1; ++a) {
                const double x = band_d[w][a];
                const float xf = band_f[w][a];
                const uint32_t y = band_i[w][a];
                int b = a - 1;
                while (b >= b0 && (band_d[w][b] > x || (band_d[w][b] == x && band_i[w][b] > y))) {
                    band_d[w][b + 1] = band_d[w][b];
                    band_f[w][b + 1] = band_f[w][b];
                    band_i[w][b + 1] = band_i[w][b];
                    --b;
                }
                band_d[w][b + 1] = x;
                band_f[w][b + 1] = xf;
                band_i[w][b + 1] = y;
            }
            // FP64 decides which band entries fill places b0..k-1; they are
            // written in ascending FP32 order (FP64, then index, on equal
            // FP32 values), so every row stays ascending (nndescent.rs:989).
            // Entries before b0 lie below the band's FP32 range.
            for (int a = b0 + 1; a < k; ++a) {
                const double x = band_d[w][a];
                const float xf = band_f[w][a];
                const uint32_t y = band_i[w][a];
                int b = a - 1;
                while (b >= b0 &&
                       (band_f[w][b] > xf ||
                        (band_f[w][b] == xf &&
                         (band_d[w][b] > x || (band_d[w][b] == x && band_i[w][b] > y))))) {
                    band_d[w][b + 1] = band_d[w][b];
                    band_f[w][b + 1] = band_f[w][b];
                    band_i[w][b + 1] = band_i[w][b];
                    --b;
                }
                band_d[w][b + 1] = x;
                band_f[w][b + 1] = xf;
                band_i[w][b + 1] = y;
            }
            atomicAdd(boundary_fixes, 1ull);
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h)
            key[h] = (uint64_t(__float_as_uint(band_f[w][lane + 32 * h])) << 32) |
                     band_i[w][lane + 32 * h];
    }
    // 5. the k nearest, ascending
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int t = lane + 32 * h;
        if (t < k) {
            const bool ok = key[h] != ~0ull;
            out_idx[size_t(i) * k + t] = ok ? uint32_t(key[h]) : PQ_EMPTY;
            out_dist[size_t(i) * k + t] =
                ok ? __uint_as_float(uint32_t(key[h] >> 32)) : __int_as_float(0x7f800000);
        }
    }
}

// Entries of each ascending list (the EMPTY slots come last).
__global__ void k_list_count(const uint32_t* __restrict__ li, uint32_t n, int k,
                             uint32_t* __restrict__ cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c = 0;
    for (int s = 0; s < k; ++s) c += li[size_t(i) * k + s] != PQ_EMPTY ? 1u : 0u;
    cnt[i] = c;
}

// CSR rows straight from the ascending lists: Euclidean distances (sqrt).
__global__ void k_list_extract(const uint32_t* __restrict__ li, const float* __restrict__ ld,
                               uint32_t n, int k, const uint32_t* __restrict__ off,
                               const uint32_t* __restrict__ cnt, uint32_t* __restrict__ indptr,
                               uint32_t* __restrict__ indices, float* __restrict__ dists) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= size_t(n) * k) return;
    const size_t i = e / k;
    const uint32_t s = uint32_t(e - i * k);
    if (s < cnt[i]) {
        indices[off[i] + s] = li[e];
        dists[off[i] + s] = __fsqrt_rn(ld[e]);
    }
    if (s == 0) {
        indptr[i + 1] = off[i] + cnt[i];
        if (i == 0) indptr[0] = 0;
    }
}

// CSR rows [a, b) of full lists (k entries each, so row i starts at i * k):
// Euclidean distances (sqrt).  A row with an empty place sets *short_rows
// (the caller then lays the CSR out from the counts instead).
__global__ void k_list_dense(const uint32_t* __restrict__ li, const float* __restrict__ ld,
                             uint32_t a, uint32_t b, int k, uint32_t* __restrict__ indptr,
                             uint32_t* __restrict__ indices, float* __restrict__ dists,
                             unsigned* __restrict__ short_rows) {
    const size_t e = size_t(a) * k + size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= size_t(b) * k) return;
    const size_t i = e / k;
    const uint32_t v = li[e];
    if (v == PQ_EMPTY) atomicOr(short_rows, 1u);
    indices[e] = v;
    dists[e] = __fsqrt_rn(ld[e]);
    if (e - i * k == 0) {
        indptr[i + 1] = uint32_t((i + 1) * k);
        if (i == 0) indptr[0] = 0;
    }
}

// Sets *flag when a cell's shortlist runs hold fewer than k live entries in
// all (the tile kernel never lists a cell itself and a candidate lies in one
// bucket only, so the cell's row will have fewer than k neighbours).
__global__ void k_short_rows(const uint8_t* __restrict__ sn, uint32_t n, int runs, int k,
                             unsigned* __restrict__ flag) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int t = 0;
    for (int l = 0; l < runs; ++l) t += sn[size_t(p) * runs + l];
    if (t < k) atomicOr(flag, 1u);
}

// Events owned by one scope: destroyed on every exit, exceptions included.
struct EventSet {
    std::vector<cudaEvent_t> ev;
    explicit EventSet(int count) : ev(count, nullptr) {
        for (auto& e : ev) pqh::ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
    ~EventSet() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
};

// Sorted (ascending) lists -> neighbour heaps: a descending array is a valid
// max-heap; every entry starts new.
__global__ void k_list_to_heap(const uint32_t* __restrict__ li, const float* __restrict__ ld,
                               uint32_t n, int k, uint32_t* __restrict__ hidx,
                               float* __restrict__ hdist, uint8_t* __restrict__ hflag) {
    const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= size_t(n) * k) return;
    const size_t i = e / k;
    const int s = int(e - i * k);
    const size_t src = i * k + (k - 1 - s);
    hidx[e] = li[src];
    hdist[e] = ld[src];
    hflag[e] = li[src] != PQ_EMPTY ? 1 : 0;
}

}  // namespace
}  // namespace pq

namespace pqh {

using namespace pq;

uint64_t build_chosen(pq_ctx* c, const float* data, bool data_on_host, uint64_t n64, uint64_t d64,
                      const pq_nnd_opts& o, uint32_t* d_indptr, uint32_t* d_indices,
                      float* d_dists, HostGraph* host) {
    cudaStream_t st = c->stream;
    const uint32_t n = uint32_t(n64);
    const int d = int(d64), dp = int((d64 + 3) / 4 * 4);
    const int k = int(effective_k(n64, o.k));
    pq_nnd_stats& S_ = c->stats;
    std::memset(&S_, 0, sizeof(S_));
    S_.k = k;
    Timer tot(st), tm(st);
    tot.start();
    const unsigned long long launches0 = g_launches;

    // host data: the k-means sample (blocks of rows) is copied first; the
    // whole embedding follows on the second stream in XCH row chunks, one
    // event each, while k-means runs, and each chunk's cells are assigned to
    // their centroids as soon as the chunk has landed
    constexpr int XCH = 8;
    EventSet xev(data_on_host ? XCH + 1 : 0);
    auto xrow = [&](int i) { return uint32_t(uint64_t(n) * uint32_t(i) / XCH); };
    float* X = data_on_host ? c->get<float>("X", size_t(n) * dp)
                            : load_embedding(c, data, false, n, d, dp);

    // ── 1. buckets ──
    tm.start();
    std::optional<KGScope> kg_sec;
    kg_sec.emplace(c, PQ_KG_BUCKETS);
    const bool learned = o.init == PQ_INIT_LEARNED;
    // PQ_MODE_PLAIN here is the learned-init NN-Descent: BF16 tiles over the
    // router's top buckets give the initial lists, the rounds run to
    // convergence
    const bool nnd = o.mode == PQ_MODE_PLAIN;
    // learned probes: the MLP's 1024 buckets; else about 4096 cells per bucket
    const uint32_t C = learned ? 1024u
                       : o.buckets > 0 ? std::min<uint32_t>(uint32_t(o.buckets), n)
                                       : std::max<uint32_t>(1, uint32_t(std::llround(double(n) / 4096.0)));
    // probes: 13 (14 for k > 15; 16 from 6M cells, where the buckets are
    // closer together); at 4M x 50 recall@15 is 0.9925 / 0.9944 / 0.9957 with
    // 12 / 13 / 14 probes, recall@30 0.9929 / 0.9945 with 13 / 14
    const uint32_t P_auto =
        nnd ? 12u : learned ? 6u : (n >= 6000000u ? 16u : (k > 15 ? 14u : 13u));
    const int P = int(std::min<uint32_t>(o.probes > 0 ? uint32_t(o.probes) : P_auto, std::min(C, 16u)));
    // the k-means sample: 256 blocks of consecutive rows spread evenly over
    // the embedding (all rows up to twice the target size) — from host data
    // one copy of 256 long runs
    constexpr uint32_t KB = 256;
    const uint32_t ns_target = std::max<uint32_t>(65536, 128 * C);
    const bool all_rows = n <= 2ull * ns_target;
    const uint32_t bl = all_rows ? n : (ns_target + KB - 1) / KB;  // rows per block
    const uint64_t s_stride = all_rows ? 0 : n / KB;                 // block starts
    const uint32_t ns = all_rows ? n : bl * KB;
    if (d > 62) throw DeviceError{"the tensor-core form supports n_dim <= 62"};
    if (uint64_t(C) * C * 2 >= 0xFFFFFFFFull)
        throw DeviceError{"the tensor-core form supports n_obs below 190M"};
    int num_sms = 148;
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, c->device);
    float* xs = c->get<float>("km_sample", size_t(ns) * dp);
    float* cent = c->get<float>("km_cent", size_t(C) * dp);
    float* sums = c->get<float>("km_sums", size_t(C) * dp);
    uint32_t* cnt = c->get<uint32_t>("km_cnt", C);
    uint32_t* zeros = c->get<uint32_t>("zeros", std::max<uint32_t>(C, n));
    ck(cudaMemsetAsync(zeros, 0, size_t(std::max<uint32_t>(C, n)) * 4, st), "zeros");
    uint32_t* noself = c->get<uint32_t>("noself", n);
    ck(cudaMemsetAsync(noself, 0xFF, size_t(n) * 4, st), "noself");
    if (data_on_host) {
        float* xraw = c->get<float>("km_sample_raw", size_t(ns) * d);
        const size_t run = size_t(bl) * d * 4;
        ck(cudaMemcpy2DAsync(xraw, run, data, all_rows ? run : size_t(s_stride) * d * 4, run,
                             all_rows ? 1 : KB, cudaMemcpyHostToDevice, st),
           "copy sample");
        // the embedding's chunks start once the sample is across
        ck(cudaEventRecord(xev.ev[0], st), "event");
        ck(cudaStreamWaitEvent(c->stream2, xev.ev[0], 0), "event");
        for (int i = 0; i < XCH; ++i) {
            load_embedding_rows(c, data, n, d, dp, xrow(i), xrow(i + 1), c->stream2);
            ck(cudaEventRecord(xev.ev[i + 1], c->stream2), "event");
        }
        k_pad_cols<<<blocks(size_t(ns) * dp, 256), 256, 0, st>>>(xraw, ns, d, dp, xs); count_launch();
    } else {
        k_block_rows<<<blocks(size_t(ns) * dp, 256), 256, 0, st>>>(X, dp, s_stride, bl, ns, xs);
        count_launch();
    }
    // the sample's mean: the BF16 centre of the centroid search
    float* mean = c->get<float>("mean", dp);
    k_col_mean<<<dp, 256, 0, st>>>(xs, ns, dp, mean); count_launch();
    k_sample_rows<<<blocks(size_t(C) * dp, 256), 256, 0, st>>>(xs, dp, ns, C, cent); count_launch();
    __nv_bfloat16* xsb = c->get<__nv_bfloat16>("km_sample_bf16", size_t(ns) * 64);
    float* xsn = c->get<float>("km_sample_norm", ns);
    k_to_bf16<<<cvt_blocks(ns), 256, 0, st>>>(xs, d, dp, nullptr, zeros, mean, ns, 1, xsb, xsn); count_launch();
    __nv_bfloat16* cb = c->get<__nv_bfloat16>("cent_bf16", size_t(C) * 64);
    float* cbn = c->get<float>("cent_norm", C);
    float* lab_d = c->get<float>("km_lab_d", ns);
    uint32_t* lab = c->get<uint32_t>("km_lab", ns);
    // one-bucket nearest-centroid search on the tensor cores: queries [0, nq)
    // against all C centroids, S_out nearest per query
    // BF16 tiles with 16-entry shortlists run the wide kernel (jobs of 256
    // query entries, candidate tiles of 128)
    const bool wide_tiles = [] {
        const char* e = std::getenv("POLARISEQ_TILES_WIDE");
        return !(e && e[0] == '0');
    }();
    auto centroid_search = [&](const __nv_bfloat16* qrows, const float* qnorm, uint32_t nq,
                               int s_out, float* od, uint32_t* oi) {
        const int sr = s_out == 1 ? 1 : 16;  // per column half: the nearest, or up to 16
        const int wide = sr == 16 && wide_tiles ? 1 : 0;
        const uint32_t JR = uint32_t(ivf_job_rows(wide)), TC = uint32_t(ivf_tile_cols(wide));
        const uint32_t nj = (nq + JR - 1) / JR;
        std::vector<uint32_t> hb(nj, 0), hq(nj), he(nj);
        for (uint32_t j = 0; j < nj; ++j) {
            hq[j] = j * JR;
            he[j] = std::min(nq, j * JR + JR);
        }
        uint32_t* jb = c->get<uint32_t>("ajob_b", nj);
        uint32_t* jq = c->get<uint32_t>("ajob_q", nj);
        uint32_t* je = c->get<uint32_t>("ajob_e", nj);
        uint32_t* offs = c->get<uint32_t>("aoffs", 4);
        uint32_t ho[4] = {0, C, 0, 0};
        ck(cudaMemcpyAsync(jb, hb.data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
        ck(cudaMemcpyAsync(jq, hq.data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
        ck(cudaMemcpyAsync(je, he.data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
        ck(cudaMemcpyAsync(offs, ho, 16, cudaMemcpyHostToDevice, st), "jobs");
        CUtensorMap tq, tcm;
        if (!make_bf16_map(&tq, qrows, nq, JR) || !make_bf16_map(&tcm, cb, C, TC))
            throw DeviceError{"cuTensorMapEncodeTiled failed"};
        IvfTileArgs a{};
        a.job_bucket = jb;
        a.job_qstart = jq;
        a.job_qend = je;
        a.njobs = nj;
        a.c_off = offs;
        a.qnorm = qnorm;
        a.qself = noself;
        a.S = sr;
        a.wide = wide;
        a.out_d = c->get<float>("arun_d", size_t(nq) * 2 * 16);
        a.out_i = c->get<uint32_t>("arun_i", size_t(nq) * 2 * 16);
        a.err = c->d_err;
        if (std::getenv("POLARISEQ_TRACE")) {
            a.trace = c->get<unsigned long long>("ivf_trace", IVF_TRACE_N);
            ck(cudaMemsetAsync(a.trace, 0, IVF_TRACE_N * 8, st), "trace");
        }
        ck(launch_ivf_tiles(tq, tcm, a, std::min<int>(num_sms, int(nj)), st), "centroid tiles");
        k_merge_runs<<<blocks(nq, 256), 256, 0, st>>>(a.out_d, a.out_i, nq, sr, s_out, od, oi); count_launch();
        ck(cudaStreamSynchronize(st), "centroid tiles");  // the host job arrays are reused
        if (a.trace) {
            unsigned long long h[IVF_TRACE_N];
            ck(cudaMemcpy(h, a.trace, sizeof(h), cudaMemcpyDeviceToHost), "trace");
            std::fprintf(stderr,
                         "[chosen] centroid search (%u queries, S %d) block 0: jobs %llu tiles %llu "
                         "| cycles epi-wait %llu epi-work %llu epi-end %llu flagged-chunk %llu "
                         "total %llu | warp 0: slow chunks %llu admits %llu\n",
                         nq, sr, h[IVF_T_JOBS], h[IVF_T_TILES], h[IVF_T_EPI_WAIT],
                         h[IVF_T_EPI_WORK], h[IVF_T_EPI_END], h[IVF_T_SLOW_CYC], h[IVF_T_TOTAL],
                         h[IVF_T_SLOW], h[IVF_T_ADMITS]);
        }
    };
    ck(cudaMemsetAsync(c->d_err, 0, 4, st), "err");
    // the Lloyd sums in a fixed order: members sorted by label
    uint32_t* lk = c->get<uint32_t>("km_lk", ns);
    uint64_t* lv = c->get<uint64_t>("km_lv", ns);
    uint32_t* lk2 = c->get<uint32_t>("km_lk2", ns);
    uint64_t* lv2 = c->get<uint64_t>("km_lv2", ns);
    uint8_t* ltemp = c->get<uint8_t>("km_ltemp", radix_temp_bytes(ns));
    uint32_t* loff = c->get<uint32_t>("km_loff", size_t(C) + 1);
    const int lloyd = 8;
    for (int it = 0; it < lloyd; ++it) {
        k_to_bf16<<<cvt_blocks(C), 256, 0, st>>>(cent, d, dp, nullptr, zeros, mean, C, 2, cb, cbn); count_launch();
        centroid_search(xsb, xsn, ns, 1, lab_d, lab);
        k_label_pairs<<<blocks(ns, 256), 256, 0, st>>>(lab, ns, C, lk, lv); count_launch();
        ck(radix_sort_pairs(lk, lv, lk2, lv2, ns, key_bits(C), ltemp, st), "sort labels");
        k_key_bounds<<<blocks(size_t(ns) + 1, 256), 256, 0, st>>>(lk, ns, 1, C, loff); count_launch();
        k_kmeans_sums<<<blocks(C, 8), 256, 0, st>>>(xs, d, dp, lv, loff, C, sums, cnt); count_launch();
        k_kmeans_update<<<blocks(size_t(C) * dp, 256), 256, 0, st>>>(cent, sums, cnt, C, d, dp); count_launch();
    }
    k_to_bf16<<<cvt_blocks(C), 256, 0, st>>>(cent, d, dp, nullptr, zeros, mean, C, 2, cb, cbn); count_launch();
    // every cell's P nearest centroids, ascending; the first is its primary bucket
    __nv_bfloat16* qa = c->get<__nv_bfloat16>("assign_q", size_t(n) * 64);
    float* qan = c->get<float>("assign_qn", n);
    uint32_t* probes = c->get<uint32_t>("probes", size_t(n) * P);
    float* probe_d = c->get<float>("probe_d", size_t(n) * P);
    double ms_train = 0.0, ms_route = 0.0;
    if (!learned && data_on_host) {
        // chunk by chunk as the embedding lands
        for (int i = 0; i < XCH; ++i) {
            const uint32_t r0 = xrow(i), r1 = xrow(i + 1);
            ck(cudaStreamWaitEvent(st, xev.ev[i + 1], 0), "event");
            if (r1 <= r0) continue;
            k_to_bf16<<<cvt_blocks(r1 - r0), 256, 0, st>>>(X + size_t(r0) * dp, d, dp, nullptr,
                                                           zeros, mean, r1 - r0, 1,
                                                           qa + size_t(r0) * 64, qan + r0);
            count_launch();
            centroid_search(qa + size_t(r0) * 64, qan + r0, r1 - r0, P,
                            probe_d + size_t(r0) * P, probes + size_t(r0) * P);
        }
    } else {
        if (data_on_host) ck(cudaStreamWaitEvent(st, xev.ev[XCH], 0), "event");
        k_to_bf16<<<cvt_blocks(n), 256, 0, st>>>(X, d, dp, nullptr, zeros, mean, n, 1, qa, qan);
        count_launch();
    }
    if (learned) {  // own bucket by k-means, the other probes from the MLP
        uint32_t* prim = c->get<uint32_t>("primary", n);
        float* prim_d = c->get<float>("primary_d", n);
        centroid_search(qa, qan, n, 1, prim_d, prim);
        ms_route = learned_probes(c, X, d, dp, n, C, prim, prim_d, cent, P, o.seed, probes,
                                  &ms_train, &S_.learn_loss_first, &S_.learn_loss_last);
    } else if (!data_on_host) {
        centroid_search(qa, qan, n, P, probe_d, probes);
    }
    int herr0 = 0;
    ck(cudaMemcpy(&herr0, c->d_err, 4, cudaMemcpyDeviceToHost), "err");
    if (herr0) throw DeviceError{"centroid tiles: a bounded wait gave up", herr0 == 2};
    const size_t ne = size_t(n) * P;
    uint32_t* ekeys = c->get<uint32_t>("ekeys", ne);
    uint64_t* evals = c->get<uint64_t>("evals", ne);
    uint32_t* ekeys2 = c->get<uint32_t>("ekeys2", ne);
    uint64_t* evals2 = c->get<uint64_t>("evals2", ne);
    kg_sec.reset();
    S_.ms_forest = tm.stop();

    // ── 2. layout ──
    tm.start();
    kg_sec.emplace(c, PQ_KG_LAYOUT);
    void* stemp = c->get<uint8_t>("scan_temp_c", scan_temp_bytes(std::max<size_t>(ne, C + 1)));
    uint32_t* ckeys = c->get<uint32_t>("ckeys_c", n);
    uint64_t* cvals = c->get<uint64_t>("cvals_c", n);
    uint32_t* ckeys2 = c->get<uint32_t>("ckeys_c2", n);
    uint64_t* cvals2 = c->get<uint64_t>("cvals_c2", n);
    k_primary_keys<<<blocks(n, 256), 256, 0, st>>>(probes, P, n, C, ckeys, cvals); count_launch();
    ck(radix_sort_pairs(ckeys, cvals, ckeys2, cvals2, n, key_bits(uint64_t(C) * C - 1),
                        c->get<uint8_t>("radix_c", radix_temp_bytes(std::max<size_t>(n, ne))), st),
       "sort cand");
    uint32_t* c_off = c->get<uint32_t>("c_off", C + 1);
    k_key_bounds<<<blocks(size_t(n) + 1, 256), 256, 0, st>>>(ckeys, n, C, C, c_off); count_launch();
    // where each (bucket, second-nearest centroid) group of candidates begins
    uint32_t* pair_off = c->get<uint32_t>("pair_off", size_t(C) * C + 1);
    k_key_bounds<<<blocks(size_t(n) + 1, 256), 256, 0, st>>>(ckeys, n, 1, C * C, pair_off); count_launch();
    uint32_t* perm = c->get<uint32_t>("cperm", n);
    uint32_t* cbucket = c->get<uint32_t>("cbucket", n);
    uint32_t* pos_of = c->get<uint32_t>("pos_of", n);
    k_cand_layout<<<blocks(n, 256), 256, 0, st>>>(cvals, n, C, ckeys, perm, pos_of, cbucket); count_launch();
    // the embedding in candidate order: the conversions below and the re-rank
    // read it in runs instead of gathering rows
    float* xp = c->get<float>("xp_f32", size_t(n) * dp);
    k_gather_rows<<<blocks(size_t(n) * (dp / 4), 256), 256, 0, st>>>(
        reinterpret_cast<const float4*>(X), perm, n, dp / 4, reinterpret_cast<float4*>(xp));
    count_launch();
    k_entry_keys<<<blocks(ne, 256), 256, 0, st>>>(probes, perm, ne, P, C, ekeys, evals); count_launch();
    const bool fp8 = o.mode == PQ_MODE_FP8;
    __nv_bfloat16* xc = nullptr;
    uint32_t* xc8 = nullptr;
    float* xch = nullptr;     // E4M3: |x~|^2 / 2 per candidate
    float* cscale = nullptr;  // E4M3: 1 / the candidate row's own scale
    if (!fp8) {
        xc = c->get<__nv_bfloat16>("xc_bf16", size_t(n) * 64);
        float* xcn = c->get<float>("xc_norm", n);
        k_to_bf16<<<cvt_blocks(n), 256, 0, st>>>(xp, d, dp, nullptr, cbucket, cent, n, 2, xc, xcn); count_launch();
    } else {
        // every candidate row with its own power-of-two scale (its absmax)
        xc8 = c->get<uint32_t>("xc_fp8", size_t(n) * 32);
        xch = c->get<float>("xc_half", n);
        cscale = c->get<float>("xc_scale", n);
        k_to_fp8<<<cvt_blocks(n), 256, 0, st>>>(xp, d, dp, nullptr, cbucket, cent, n, xc8, cscale,
                                                xch, 0.5f); count_launch();
    }
    // query entries grouped by probe bucket (stable: cell order within a bucket);
    // the n primary entries (keys below C * C) come first, in candidate order
    ck(radix_sort_pairs(ekeys, evals, ekeys2, evals2, ne, key_bits(2 * uint64_t(C) * C - 1),
                        c->get<uint8_t>("radix_c", radix_temp_bytes(std::max<size_t>(n, ne))), st),
       "sort entries");
    uint32_t* qpos = c->get<uint32_t>("qpos", ne);  // entry -> its cell's candidate position
    uint32_t* qbucket = c->get<uint32_t>("qbucket", ne);
    uint32_t* qself = c->get<uint32_t>("qself", ne);
    uint32_t* entry_of = c->get<uint32_t>("entry_of", ne);
    uint32_t* eslot = c->get<uint32_t>("entry_slot", ne);  // entry -> position * P + probe rank
    uint32_t* q_off = c->get<uint32_t>("q_off", 2 * C + 1);
    __nv_bfloat16* qb = nullptr;
    uint32_t* qb8 = nullptr;
    float* qscale = nullptr;
    float* qbn = c->get<float>("q_norm", ne);
    if (!fp8) {
        qb = c->get<__nv_bfloat16>("q_bf16", ne * 64);
    } else {
        qb8 = c->get<uint32_t>("q_fp8", ne * 32);
        qscale = c->get<float>("q_scale", ne);
    }
    // the query entries [e0, e0 + m) laid out (from keys/vals) and their rows
    // converted
    auto lay_entries = [&](const uint32_t* keys, const uint64_t* vals, uint32_t e0, size_t m) {
        if (m == 0) return;
        k_entry_layout<<<blocks(m, 256), 256, 0, st>>>(vals, keys, m, e0, P, C, qpos + e0,
                                                       qbucket + e0, qself + e0, entry_of,
                                                       eslot + e0);
        count_launch();
        if (!fp8) {
            k_to_bf16<<<cvt_blocks(m), 256, 0, st>>>(xp, d, dp, qpos + e0, qbucket + e0, cent, m,
                                                      1, qb + size_t(e0) * 64, qbn + e0);
        } else {
            k_to_fp8<<<cvt_blocks(m), 256, 0, st>>>(xp, d, dp, qpos + e0, qbucket + e0, cent, m,
                                                    qb8 + size_t(e0) * 32, qscale + e0,
                                                    qbn + e0, 1.0f);
        }
        count_launch();
    };
    // primary entries now; the other probes after the primary pass, which
    // bounds them
    lay_entries(ekeys, evals, 0, n);
    k_key_bounds<<<blocks(ne + 1, 256), 256, 0, st>>>(ekeys, ne, C, 2 * C, q_off); count_launch();
    // exact distances of every cell to its probe centroids, bucket radii
    float* pdist = c->get<float>("probe_dist", ne);
    unsigned* rad2 = c->get<unsigned>("bucket_rad2", 2 * size_t(C) + 1);
    unsigned* umax2 = rad2 + C;      // per bucket: max |y - mean|^2 of its cells
    unsigned* wmax2 = rad2 + 2 * C;  // max |c - mean|^2 over the centroids
    ck(cudaMemsetAsync(rad2, 0, (2 * size_t(C) + 1) * 4, st), "rad2");
    k_probe_dist<<<blocks(n, 8), 256, 0, st>>>(xp, perm, d, dp, n, probes, P, cent, qan, pdist,
                                                rad2, umax2);
    count_launch();
    k_max_nonneg<<<1, 256, 0, st>>>(cbn, C, wmax2); count_launch();
    float* cdist = c->get<float>("cent_dist", size_t(C) * C);
    k_cent_dist<<<blocks(size_t(C) * C, 256), 256, 0, st>>>(cent, C, d, dp, cdist); count_launch();
    std::vector<uint32_t> hq(2 * C + 1);
    ck(cudaMemcpyAsync(hq.data(), q_off, size_t(2 * C + 1) * 4, cudaMemcpyDeviceToHost, st),
       "q_off");
    ck(cudaStreamSynchronize(st), "layout");
    std::vector<uint32_t> hc(C + 1);
    ck(cudaMemcpy(hc.data(), c_off, size_t(C + 1) * 4, cudaMemcpyDeviceToHost), "c_off");
    // jobs of one pass from its entries' bucket bounds (hq[key] for key in
    // [key0, key0 + C)): JR entries of one probe bucket each, against
    // candidate tiles of TC
    const int wide_pass = (!fp8 && ivf_shortlist(k + 1) == 16 && wide_tiles) ? 1 : 0;
    const uint32_t JR = uint32_t(ivf_job_rows(wide_pass)), TC = uint32_t(ivf_tile_cols(wide_pass));
    std::vector<uint32_t> jb[2], jq[2], je[2], jt0;
    uint64_t tile_pairs = 0, maxb = 0, cells = 0, pass_pairs[2] = {0, 0};
    auto make_jobs = [&](int pass, const std::vector<uint32_t>& bounds, uint32_t key0,
                         uint32_t base) {
        for (uint32_t b = 0; b < C; ++b) {
            const uint32_t key = b + key0;
            const uint64_t nct = (hc[b + 1] - hc[b] + TC - 1) / TC;
            maxb = std::max<uint64_t>(maxb, hc[b + 1] - hc[b]);
            for (uint32_t q0 = base + bounds[key]; q0 < base + bounds[key + 1]; q0 += JR) {
                const uint32_t q1 = std::min(q0 + JR, base + bounds[key + 1]);
                jb[pass].push_back(b);
                jq[pass].push_back(q0);
                je[pass].push_back(q1);
                // a primary job's own cells are its candidates at the same offset
                if (pass == 0) jt0.push_back((q0 - base - bounds[key]) / TC);
                tile_pairs += nct;
                pass_pairs[pass] += nct;
                cells += uint64_t(q1 - q0) * (hc[b + 1] - hc[b]);
            }
        }
    };
    make_jobs(0, hq, 0, 0);
    kg_sec.reset();
    S_.ms_leaves = tm.stop();

    // ── 3. tensor-core shortlist ──
    tm.start();
    const int Ssh = ivf_shortlist(k + 1);        // per entry and column half
    const int Sout = ivf_groups() * Ssh;         // per entry: ivf_groups() ascending runs
    if (Ssh == 0) throw DeviceError{"the tensor-core form supports k <= 31"};
    float* sd = c->get<float>("sl_d", ne * Sout);
    uint32_t* si = c->get<uint32_t>("sl_i", ne * Sout);
    // live length of each run by slot: [position * P + probe rank][run]; a
    // dropped entry's runs stay empty
    uint8_t* sn = c->get<uint8_t>("sl_n", ne * ivf_groups());
    ck(cudaMemsetAsync(sn, 0, ne * ivf_groups(), st), "run lengths");
    float* qthr = c->get<float>("q_thr", ne);
    float* cseed = c->get<float>("cell_seed", n);  // per candidate position
    {
        const bool trace = std::getenv("POLARISEQ_TRACE") != nullptr;
        unsigned long long* tbuf = nullptr;
        if (trace) {
            tbuf = c->get<unsigned long long>("ivf_trace", IVF_TRACE_N);
            ck(cudaMemsetAsync(tbuf, 0, IVF_TRACE_N * 8, st), "trace");
        }
        // the seed: the (k+2)-th best of the primary shortlist.  A candidate of
        // another bucket can reach the cell's k best only by beating it; the two
        // extra places absorb the BF16 ranking error (recall@15 at 4M matches the
        // 2k-th seed to four digits, with 16% fewer tile-kernel cycles)
        // (the E4M3 ranking error is larger: 2k places)
        const int R0 = std::min(Sout, fp8 ? 2 * k : k + 2);
        uint64_t pruned = 0;
        // the timeout test hook applies to this build's two tile passes once
        const uint32_t test_wait = c->test_wait_polls;
        c->test_wait_polls = 0;
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) {
                // the other-probe entries that can admit anything, compacted
                // in order, laid out after the primary ones
                KGScope kg(c, PQ_KG_LAYOUT);
                const size_t m = ne - n;
                uint32_t* keep = c->get<uint32_t>("prune_keep", std::max<size_t>(m, 1));
                uint32_t* kpos = c->get<uint32_t>("prune_pos", std::max<size_t>(m, 1));
                uint64_t* dtot = c->get<uint64_t>("prune_total", 1);
                uint64_t m1 = 0;
                if (m > 0) {
                    k_prune_keep<<<blocks(m, 256), 256, 0, st>>>(ekeys + n, evals + n, m, P, C,
                                                                 pdist, rad2, umax2, wmax2,
                                                                 cdist, cseed, keep);
                    count_launch();
                    ck(scan_exclusive_u32(keep, kpos, m,
                                          c->get<uint8_t>("prune_scan", scan_temp_bytes(m)), dtot,
                                          st),
                       "scan kept");
                    k_compact_entries<<<blocks(m, 256), 256, 0, st>>>(ekeys + n, evals + n, m,
                                                                      keep, kpos, ekeys2 + n,
                                                                      evals2 + n);
                    count_launch();
                    ck(cudaMemcpyAsync(&m1, dtot, 8, cudaMemcpyDeviceToHost, st), "kept");
                    ck(cudaStreamSynchronize(st), "kept");
                }
                pruned = m - m1;
                lay_entries(ekeys2 + n, evals2 + n, uint32_t(n), m1);
                if (m1 > 0) {
                    k_entry_thr<<<blocks(m1, 256), 256, 0, st>>>(eslot + n, m1, P, cseed,
                                                                 qthr + n);
                    count_launch();
                }
                k_key_bounds<<<blocks(m1 + 1, 256), 256, 0, st>>>(ekeys2 + n, m1, C, 2 * C,
                                                                  q_off);
                count_launch();
                ck(cudaMemcpyAsync(hq.data(), q_off, size_t(2 * C + 1) * 4,
                                   cudaMemcpyDeviceToHost, st),
                   "q_off");
                ck(cudaStreamSynchronize(st), "layout");
                make_jobs(1, hq, C, uint32_t(n));
            }
            const uint32_t nj = uint32_t(jb[pass].size());
            if (nj == 0) continue;
            CUtensorMap tq, tcm;
            const bool maps =
                fp8 ? make_fp8_map(&tq, qb8, ne, JR) && make_fp8_map(&tcm, xc8, n, TC)
                    : make_bf16_map(&tq, qb, ne, JR) && make_bf16_map(&tcm, xc, n, TC);
            if (!maps) throw DeviceError{"cuTensorMapEncodeTiled failed"};
            uint32_t* djb = c->get<uint32_t>(pass ? "job_b1" : "job_b0", nj);
            uint32_t* djq = c->get<uint32_t>(pass ? "job_q1" : "job_q0", nj);
            uint32_t* dje = c->get<uint32_t>(pass ? "job_e1" : "job_e0", nj);
            ck(cudaMemcpyAsync(djb, jb[pass].data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
            ck(cudaMemcpyAsync(djq, jq[pass].data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
            ck(cudaMemcpyAsync(dje, je[pass].data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st), "jobs");
            uint32_t* djt = c->get<uint32_t>(pass ? "job_t1" : "job_t0", nj);
            if (pass == 0) {
                ck(cudaMemcpyAsync(djt, jt0.data(), size_t(nj) * 4, cudaMemcpyHostToDevice, st),
                   "jobs");
            } else {
                k_job_tstart<<<blocks(nj, 256), 256, 0, st>>>(djb, djq, nj, ekeys2, C, c_off,
                                                              pair_off, TC, djt);
                count_launch();
            }
            IvfTileArgs a{};
            a.job_bucket = djb;
            a.job_qstart = djq;
            a.job_qend = dje;
            a.job_tstart = djt;
            a.njobs = nj;
            a.c_off = c_off;
            a.qnorm = qbn;
            a.fp8 = fp8 ? 1 : 0;
            a.qscale = qscale;
            a.cscale = cscale;
            a.chalf = xch;
            a.qthr = pass ? qthr : nullptr;
            a.qself = qself;
            a.S = Ssh;
            a.buffered = pass;  // the other probes start from the primary's bound
            a.out_d = sd;
            a.out_i = si;
            a.out_n = sn;
            a.out_slot = eslot;
            a.err = c->d_err;
            a.trace = tbuf;
            a.test_wait_polls = test_wait;
            a.wide = wide_pass;
            {
                KGScope kg(c, PQ_KG_TILES);
                ck(launch_ivf_tiles(tq, tcm, a, std::min<int>(num_sms, int(nj)), st), "ivf tiles");
            }
            if (pass == 0) {  // seed the other probes with the primary shortlist's R-th best
                k_seed_thresholds<<<blocks(n, 256), 256, 0, st>>>(entry_of, n, P, sd, sn, Ssh, R0,
                                                                  cseed);
                count_launch();
            }
            ck(cudaStreamSynchronize(st), "jobs");  // the host job arrays are reused
            if (trace) {
                unsigned long long h[IVF_TRACE_N];
                ck(cudaMemcpy(h, tbuf, sizeof(h), cudaMemcpyDeviceToHost), "trace");
                std::fprintf(stderr,
                             "[chosen] pass %d tiles block 0: jobs %llu tiles %llu | cycles "
                             "epi-wait %llu epi-work %llu epi-end %llu mma-wait-c %llu mma-wait-t "
                             "%llu tma-wait %llu total %llu | warp 0: slow chunks %llu admits %llu "
                             "union bits %llu flagged-chunk cycles %llu tmem-load cycles %llu\n",
                             pass, h[IVF_T_JOBS], h[IVF_T_TILES], h[IVF_T_EPI_WAIT],
                             h[IVF_T_EPI_WORK], h[IVF_T_EPI_END], h[IVF_T_MMA_WAIT_C],
                             h[IVF_T_MMA_WAIT_T], h[IVF_T_TMA_WAIT], h[IVF_T_TOTAL], h[IVF_T_SLOW],
                             h[IVF_T_ADMITS], h[IVF_T_WMBITS], h[IVF_T_SLOW_CYC], h[IVF_T_LD_CYC]);
            }
        }
        S_.shortlist[0] = tile_pairs;
        S_.shortlist[1] = maxb;
        S_.shortlist[2] = C;
        S_.shortlist[3] = cells;
        S_.shortlist[4] = pass_pairs[0];
        S_.shortlist[5] = pass_pairs[1];
        S_.shortlist[7] = pruned;
        if (trace)
            std::fprintf(stderr,
                         "[chosen] %u buckets, largest %llu, %zu + %zu query tiles, %llu tile "
                         "pairs, %llu of %llu other-probe entries dropped\n",
                         C, (unsigned long long)maxb, jb[0].size(), jb[1].size(),
                         (unsigned long long)tile_pairs, (unsigned long long)pruned,
                         (unsigned long long)(ne - n));
    }
    int herr = 0;
    ck(cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, st), "err");
    ck(cudaStreamSynchronize(st), "ivf tiles");
    if (herr) throw DeviceError{"tensor-core tiles: a bounded wait gave up", herr == 2};
    S_.ms_rounds = tm.stop();

    // ── 4. re-rank ──
    tm.start();
    uint32_t* ridx = c->get<uint32_t>("list_idx", size_t(n) * k);
    float* rdist = c->get<float>("list_dist", size_t(n) * k);
    // the exact re-rank list: 2k candidates ("2k-4k shortlist"), at most 64
    // (E4M3: 4k, the wider end of the 2k-4k range, for its cruder ranking)
    const int R = std::min(P * Sout, std::min(64, std::max(fp8 ? 4 * k : 2 * k, k + 1)));
    if (k > 63) throw DeviceError{"the tensor-core form supports k <= 63"};
    ck(cudaMemsetAsync(c->d_acc, 0, 16, st), "acc");
    // auto: no polish round for BF16; for E4M3 one below 2^20 cells (with few
    // buckets its shortlist misses more: recall@15 0.978 at 120k without it,
    // 0.994 at 4M)
    const uint64_t polish = nnd ? resolve(n64, o).n_iters
                            : o.refine_rounds >= 0 ? uint64_t(o.refine_rounds)
                            : (fp8 && n < (1u << 20) ? 1 : 0);
    auto rerank = [&](const uint32_t* by_cell, uint32_t a, uint32_t b) {
        if (d == 50)
            k_rerank<50><<<blocks(b - a, 4), 128, 0, st>>>(X, xp, d, dp, b, k, P, Sout, Ssh, R,
                                                            entry_of, sd, si, sn, perm, by_cell, a,
                                                            ridx, rdist, c->d_acc);
        else
            k_rerank<0><<<blocks(b - a, 4), 128, 0, st>>>(X, xp, d, dp, b, k, P, Sout, Ssh, R,
                                                           entry_of, sd, si, sn, perm, by_cell, a,
                                                           ridx, rdist, c->d_acc);
        count_launch();
    };
    // graph wanted in host memory and no polish: the cells are re-ranked in
    // index order, a chunk at a time, and each chunk's CSR rows (full rows:
    // row i at i * k) are copied to the host on the second stream while the
    // next chunk is re-ranked
    // (only when no row can be short: a short row moves the CSR rows, and the
    // host arrays past nnz must stay untouched)
    bool overlap = host != nullptr && polish == 0 && n >= (1u << 20);
    unsigned* short_rows = reinterpret_cast<unsigned*>(c->d_acc + 1);
    if (overlap) {
        unsigned hshort = 0;
        k_short_rows<<<blocks(n, 256), 256, 0, st>>>(sn, n, P * ivf_groups(), k, short_rows);
        count_launch();
        ck(cudaMemcpyAsync(&hshort, short_rows, 4, cudaMemcpyDeviceToHost, st), "short rows");
        ck(cudaStreamSynchronize(st), "short rows");
        overlap = hshort == 0;
    }
    bool copied = false;
    if (overlap) {
        KGScope kg(c, PQ_KG_RERANK);
        const int NCH = 8;
        EventSet es(NCH);
        cudaEvent_t* evs = es.ev.data();
        for (int j = 0; j < NCH; ++j) {
            const uint32_t a = uint32_t(uint64_t(n) * j / NCH), b = uint32_t(uint64_t(n) * (j + 1) / NCH);
            if (b == a) continue;
            rerank(pos_of, a, b);
            k_list_dense<<<blocks(size_t(b - a) * k, 256), 256, 0, st>>>(ridx, rdist, a, b, k,
                                                                          d_indptr, d_indices,
                                                                          d_dists, short_rows);
            count_launch();
            ck(cudaEventRecord(evs[j], st), "event");
            ck(cudaStreamWaitEvent(c->stream2, evs[j], 0), "event");
            const size_t e0 = size_t(a) * k, ne_ = size_t(b - a) * k;
            ck(cudaMemcpyAsync(host->indices + e0, d_indices + e0, ne_ * 4, cudaMemcpyDeviceToHost,
                               c->stream2), "d2h");
            ck(cudaMemcpyAsync(host->dists + e0, d_dists + e0, ne_ * 4, cudaMemcpyDeviceToHost,
                               c->stream2), "d2h");
            const uint32_t p0 = j == 0 ? 0u : a + 1;
            ck(cudaMemcpyAsync(host->indptr + p0, d_indptr + p0, size_t(b + 1 - p0) * 4,
                               cudaMemcpyDeviceToHost, c->stream2), "d2h");
        }
        unsigned hshort = 0;
        ck(cudaMemcpyAsync(&hshort, short_rows, 4, cudaMemcpyDeviceToHost, st), "short rows");
        ck(cudaStreamSynchronize(st), "re-rank");
        ck(cudaStreamSynchronize(c->stream2), "d2h");
        copied = hshort == 0;  // (checked above; else laid out from the counts below)
    } else {
        KGScope kg(c, PQ_KG_RERANK);
        rerank(nullptr, 0, n);
    }
    unsigned long long fixes = 0;
    ck(cudaMemcpyAsync(&fixes, c->d_acc, 8, cudaMemcpyDeviceToHost, st), "fixes");
    // ── 5. NN-Descent rounds from the shortlist lists, then the extract ──
    const Resolved RR = resolve(n64, o);
    int rounds = 0;
    uint32_t* ecnt = c->get<uint32_t>("ecnt", n);
    uint32_t* eoff = c->get<uint32_t>("eoff", n);
    if (n > 1 && polish > 0) {
        uint32_t* hidx = c->get<uint32_t>("hidx", size_t(n) * k);
        float* hdist = c->get<float>("hdist", size_t(n) * k);
        uint8_t* hflag = c->get<uint8_t>("hflag", size_t(n) * k);
        k_list_to_heap<<<blocks(size_t(n) * k, 256), 256, 0, st>>>(ridx, rdist, n, k, hidx, hdist,
                                                                    hflag); count_launch();
        rounds = run_rounds(c, X, d, dp, n, k, int(RR.max_cand), o.seed, polish, RR.stop_at, hidx,
                            hdist, hflag, perm, 0, nullptr);
        launch_extract_count(hidx, n, k, ecnt, st);
        ck(scan_exclusive_u32(ecnt, eoff, n, stemp, c->d_u64, st), "scan extract");
        launch_extract(hidx, hdist, n, k, eoff, d_indptr, d_indices, d_dists, st);
    } else if (!copied) {
        // the re-ranked lists are already ascending with their entries first
        KGScope kg(c, PQ_KG_EXTRACT);
        k_list_count<<<blocks(n, 256), 256, 0, st>>>(ridx, n, k, ecnt); count_launch();
        ck(scan_exclusive_u32(ecnt, eoff, n, stemp, c->d_u64, st), "scan extract");
        k_list_extract<<<blocks(size_t(n) * k, 256), 256, 0, st>>>(ridx, rdist, n, k, eoff, ecnt,
                                                                    d_indptr, d_indices, d_dists);
        count_launch();
    }
    uint64_t nnz = uint64_t(n) * k;
    if (!copied) ck(cudaMemcpyAsync(&nnz, c->d_u64, 8, cudaMemcpyDeviceToHost, st), "nnz");
    ck(cudaStreamSynchronize(st), "extract");
    if (host) host->copied = copied;
    S_.ms_extract = tm.stop();
    S_.ms_total = tot.stop();
    S_.shortlist[6] = fixes;
    S_.ms_learn_train = ms_train;
    S_.ms_learn_route = ms_route;
    S_.rounds_run = rounds;  // polish rounds after the shortlist
    S_.n_trees = int32_t(C);
    S_.max_candidates = uint64_t(P) << 32 | uint64_t(Ssh);
    S_.launches = g_launches - launches0;
    kg_collect(c);
    return nnz;
}

}  // namespace pqh
