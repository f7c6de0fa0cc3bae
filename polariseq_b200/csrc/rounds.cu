// NN-Descent rounds and extract of the plain form, bit-exact with
// crates/polariseq-core/src/nndescent.rs:848-996.
//
// The reference generates updates in blocks of 4096 source rows and applies
// them per destination bucket in generation order (:307-324, :855-969).
// Candidate lists and the join thresholds are frozen for the whole round, so
// every destination row's final heap is the sequential replay of all updates
// addressed to it, in global generation order.  Here a round's updates are
// generated for all rows at once, written in generation order (per source
// row at an offset from an exclusive scan), stably sorted by destination, and
// replayed by one thread per destination row.
#include "common.cuh"
#include "kernels.cuh"

namespace pq {
namespace {

// Candidate sampling records (nndescent.rs:855-892): slot e = i*k+s makes the
// forward record (i <- j) at 2e and the reverse record (j <- i) at 2e+1, both
// with prio = hash_unit(seed, iter, e) and the slot's new/old flag; value =
// (prio bits | is_new << 31) << 32 | neighbour.  Empty slots get key n.
__global__ void k_cand_gen(const uint32_t* __restrict__ hidx, const uint8_t* __restrict__ hflag,
                           uint32_t n, int k, uint64_t seed, uint32_t iter, uint32_t* keys,
                           uint64_t* vals, uint32_t* dcnt) {
    size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= size_t(n) * k) return;
    uint32_t i = uint32_t(e / k);
    uint32_t j = hidx[e];
    if (j == PQ_EMPTY) {
        keys[2 * e] = n;
        keys[2 * e + 1] = n;
        vals[2 * e] = 0;
        vals[2 * e + 1] = 0;
        return;
    }
    float prio = hash_unit(seed, uint64_t(iter), uint64_t(e));
    uint32_t pb = __float_as_uint(prio) | (hflag[e] ? 0x80000000u : 0u);
    keys[2 * e] = i;
    vals[2 * e] = (uint64_t(pb) << 32) | j;
    keys[2 * e + 1] = j;
    vals[2 * e + 1] = (uint64_t(pb) << 32) | i;
    atomicAdd(&dcnt[i], 1u);
    atomicAdd(&dcnt[j], 1u);
}

// Reset + replay of one row's candidate records into its new and old heaps
// (apply_candidates, nndescent.rs:326-354).
__global__ void k_cand_apply(const uint32_t* __restrict__ keys, const uint64_t* __restrict__ vals,
                             const uint32_t* __restrict__ seg_off,
                             const uint32_t* __restrict__ dcnt, uint32_t n, int m,
                             uint32_t* new_idx, float* new_prio, uint32_t* old_idx,
                             float* old_prio) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint32_t* ni = new_idx + size_t(r) * m;
    float* np = new_prio + size_t(r) * m;
    uint32_t* oi = old_idx + size_t(r) * m;
    float* op = old_prio + size_t(r) * m;
    for (int s = 0; s < m; ++s) {
        ni[s] = PQ_EMPTY;
        np[s] = __int_as_float(0x7f800000);
        oi[s] = PQ_EMPTY;
        op[s] = __int_as_float(0x7f800000);
    }
    uint32_t b = seg_off[r], e = b + dcnt[r];
    for (uint32_t t = b; t < e; ++t) {
        uint64_t v = vals[t];
        uint32_t nbr = uint32_t(v);
        uint32_t pb = uint32_t(v >> 32);
        float prio = __uint_as_float(pb & 0x7fffffffu);
        if (pb >> 31)
            cand_push(ni, np, m, nbr, prio);
        else
            cand_push(oi, op, m, nbr, prio);
    }
}

// Neighbours that made it into the new candidate list become old (:895-909).
__global__ void k_flag_flip(const uint32_t* __restrict__ hidx, uint8_t* hflag,
                            const uint32_t* __restrict__ new_idx, uint32_t n, int k, int m) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t* c = new_idx + size_t(i) * m;
    for (int s = 0; s < k; ++s) {
        size_t e = size_t(i) * k + s;
        uint32_t j = hidx[e];
        if (hflag[e] && j != PQ_EMPTY) {
            for (int t = 0; t < m; ++t)
                if (c[t] == j) {
                    hflag[e] = 0;
                    break;
                }
        }
    }
}

constexpr int JT = 128;  // threads per join CTA

// Loads row i's candidate lists and (when `smem_rows`) their rows.
// Slot (a, b), a < m, b < 2m, numbered a*2m + b, is the reference's pair
// (news[a], news[b]) for b < m, (news[a], olds[b-m]) for b >= m, in its
// generation order (:941-964); invalid slots are skipped exactly as there.
struct JoinSmem {
    uint32_t* cand;  // 2m ids: news then olds
    float* thr;      // 2m thresholds
    float* rows;     // 2m * dp
};

__device__ __forceinline__ void join_load(const float* __restrict__ X, int dp, int k, int m,
                                          const float* __restrict__ hdist,
                                          const uint32_t* __restrict__ new_idx,
                                          const uint32_t* __restrict__ old_idx, uint32_t i,
                                          JoinSmem s, bool smem_rows) {
    for (int t = threadIdx.x; t < 2 * m; t += JT) {
        uint32_t c = t < m ? new_idx[size_t(i) * m + t] : old_idx[size_t(i) * m + (t - m)];
        s.cand[t] = c;
        if (hdist) s.thr[t] = c != PQ_EMPTY ? hdist[size_t(c) * k] : 0.0f;
    }
    __syncthreads();
    if (smem_rows) {
        const int q4 = dp / 4;
        for (int t = threadIdx.x; t < 2 * m * q4; t += JT) {
            int r = t / q4, j = t - r * q4;
            uint32_t c = s.cand[r];
            if (c != PQ_EMPTY)
                reinterpret_cast<float4*>(s.rows)[t] =
                    reinterpret_cast<const float4*>(X + size_t(c) * dp)[j];
        }
    }
    __syncthreads();
}

__device__ __forceinline__ bool join_slot(const JoinSmem& s, int m, int slot, int& a, int& b,
                                          uint32_t& p, uint32_t& q) {
    a = slot / (2 * m);
    b = slot - a * 2 * m;
    p = s.cand[a];
    if (p == PQ_EMPTY) return false;
    if (b < m && b <= a) return false;
    q = s.cand[b];
    return q != PQ_EMPTY && q != p;
}

// Pass 1: distances, the two emit bits per slot (p side: d < thr[p]; q side:
// d < thr[q]) and the row's update count.
__global__ void __launch_bounds__(JT) k_join_count(const float* __restrict__ X, int d, int dp,
                                                   int k, int m, const float* __restrict__ hdist,
                                                   const uint32_t* __restrict__ new_idx,
                                                   const uint32_t* __restrict__ old_idx,
                                                   uint32_t* bits, int words, uint32_t* row_cnt,
                                                   unsigned long long* pairs, bool smem_rows) {
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t i = blockIdx.x;
    JoinSmem s;
    s.rows = reinterpret_cast<float*>(sm);
    size_t rbytes = smem_rows ? size_t(2 * m) * dp * sizeof(float) : 0;
    s.cand = reinterpret_cast<uint32_t*>(sm + rbytes);
    s.thr = reinterpret_cast<float*>(s.cand + 2 * m);
    uint32_t* sbits = reinterpret_cast<uint32_t*>(s.thr + 2 * m);
    __shared__ uint32_t red[JT / 32], redp[JT / 32];
    for (int t = threadIdx.x; t < words; t += JT) sbits[t] = 0;
    join_load(X, dp, k, m, hdist, new_idx, old_idx, i, s, smem_rows);
    const int nslots = 2 * m * m;
    const int per = (nslots + JT - 1) / JT;
    const int s0 = threadIdx.x * per, s1 = min(nslots, s0 + per);
    uint32_t cnt = 0, np = 0;
    for (int slot = s0; slot < s1; ++slot) {
        int a, b;
        uint32_t p, q;
        if (!join_slot(s, m, slot, a, b, p, q)) continue;
        ++np;
        const float* xp = smem_rows ? s.rows + size_t(a) * dp : X + size_t(p) * dp;
        const float* xq = smem_rows ? s.rows + size_t(b) * dp : X + size_t(q) * dp;
        float dd = sq_dist_exact(xp, xq, d);
        uint32_t e1 = dd < s.thr[a], e2 = dd < s.thr[b];
        uint32_t v = e1 | (e2 << 1);
        if (v) {
            atomicOr(&sbits[(2 * slot) >> 5], v << ((2 * slot) & 31));
            cnt += e1 + e2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
        np += __shfl_xor_sync(0xFFFFFFFFu, np, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = cnt;
        redp[threadIdx.x >> 5] = np;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t c = 0, pp = 0;
        for (int w = 0; w < JT / 32; ++w) {
            c += red[w];
            pp += redp[w];
        }
        row_cnt[i] = c;
        if (pp) atomicAdd(pairs, (unsigned long long)pp);
    }
    for (int t = threadIdx.x; t < words; t += JT) bits[size_t(i) * words + t] = sbits[t];
}

// Pass 2: recompute the emitting slots' distances and write their records at
// the row's offset, in slot order, p side before q side (:930-940).
__global__ void __launch_bounds__(JT) k_join_write(const float* __restrict__ X, int d, int dp,
                                                   int m, const uint32_t* __restrict__ new_idx,
                                                   const uint32_t* __restrict__ old_idx,
                                                   const uint32_t* __restrict__ bits, int words,
                                                   const uint32_t* __restrict__ row_off,
                                                   uint32_t* keys, uint64_t* vals,
                                                   uint32_t* dcnt, bool smem_rows) {
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t i = blockIdx.x;
    JoinSmem s;
    s.rows = reinterpret_cast<float*>(sm);
    size_t rbytes = smem_rows ? size_t(2 * m) * dp * sizeof(float) : 0;
    s.cand = reinterpret_cast<uint32_t*>(sm + rbytes);
    s.thr = reinterpret_cast<float*>(s.cand + 2 * m);
    uint32_t* sbits = reinterpret_cast<uint32_t*>(s.thr + 2 * m);
    __shared__ uint32_t ws[JT / 32];
    for (int t = threadIdx.x; t < words; t += JT) sbits[t] = bits[size_t(i) * words + t];
    join_load(X, dp, 0, m, nullptr, new_idx, old_idx, i, s, smem_rows);
    const int nslots = 2 * m * m;
    const int per = (nslots + JT - 1) / JT;
    const int s0 = threadIdx.x * per, s1 = min(nslots, s0 + per);
    uint32_t cnt = 0;
    for (int slot = s0; slot < s1; ++slot) cnt += __popc((sbits[(2 * slot) >> 5] >> ((2 * slot) & 31)) & 3u);
    // exclusive block scan of cnt
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t base = 0;
    for (int ww = 0; ww < w; ++ww) base += ws[ww];
    uint32_t pos = row_off[i] + base + x - cnt;
    if (cnt == 0) return;
    for (int slot = s0; slot < s1; ++slot) {
        uint32_t v = (sbits[(2 * slot) >> 5] >> ((2 * slot) & 31)) & 3u;
        if (!v) continue;
        int a, b;
        uint32_t p, q;
        join_slot(s, m, slot, a, b, p, q);
        const float* xp = smem_rows ? s.rows + size_t(a) * dp : X + size_t(p) * dp;
        const float* xq = smem_rows ? s.rows + size_t(b) * dp : X + size_t(q) * dp;
        float dd = sq_dist_exact(xp, xq, d);
        uint64_t db = uint64_t(__float_as_uint(dd)) << 32;
        if (v & 1u) {
            keys[pos] = p;
            vals[pos] = db | q;
            atomicAdd(&dcnt[p], 1u);
            ++pos;
        }
        if (v & 2u) {
            keys[pos] = q;
            vals[pos] = db | p;
            atomicAdd(&dcnt[q], 1u);
            ++pos;
        }
    }
}

// Replay one destination row's updates in generation order (apply_updates).
__global__ void k_replay(const uint32_t* __restrict__ keys, const uint64_t* __restrict__ vals,
                         const uint32_t* __restrict__ seg_off, const uint32_t* __restrict__ dcnt,
                         uint32_t n, int k, uint32_t* hidx, float* hdist, uint8_t* hflag,
                         unsigned long long* changed) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t chg = 0;
    if (r < n) {
        uint32_t* ri = hidx + size_t(r) * k;
        float* rd = hdist + size_t(r) * k;
        uint8_t* rf = hflag + size_t(r) * k;
        uint32_t b = seg_off[r], e = b + dcnt[r];
        for (uint32_t t = b; t < e; ++t) {
            uint64_t v = vals[t];
            chg += heap_push(ri, rd, rf, k, uint32_t(v), __uint_as_float(uint32_t(v >> 32)), 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) chg += __shfl_xor_sync(0xFFFFFFFFu, chg, o);
    if ((threadIdx.x & 31) == 0 && chg) atomicAdd(changed, (unsigned long long)chg);
}

__global__ void k_extract_count(const uint32_t* __restrict__ hidx, uint32_t n, int k,
                                uint32_t* cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c = 0;
    for (int s = 0; s < k; ++s) c += hidx[size_t(i) * k + s] != PQ_EMPTY;
    cnt[i] = c;
}

// Extract (nndescent.rs:978-996): non-empty entries in heap-array order,
// stable sort by distance, correctly rounded sqrt, CSR at the row's offset.
__global__ void k_extract(const uint32_t* __restrict__ hidx, const float* __restrict__ hdist,
                          uint32_t n, int k, const uint32_t* __restrict__ row_off,
                          uint32_t* indptr, uint32_t* indices, float* dists) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t o = row_off[i];
    uint32_t c = 0;
    // stable insertion sort straight into the output row
    for (int s = 0; s < k; ++s) {
        uint32_t j = hidx[size_t(i) * k + s];
        if (j == PQ_EMPTY) continue;
        float dv = hdist[size_t(i) * k + s];
        uint32_t t = c;
        while (t > 0 && dists[o + t - 1] > dv) {
            dists[o + t] = dists[o + t - 1];
            indices[o + t] = indices[o + t - 1];
            --t;
        }
        dists[o + t] = dv;
        indices[o + t] = j;
        ++c;
    }
    for (uint32_t t = 0; t < c; ++t) dists[o + t] = __fsqrt_rn(dists[o + t]);
    indptr[i + 1] = o + c;
    if (i == 0) indptr[0] = 0;
}

}  // namespace

void launch_cand_gen(const uint32_t* hidx, const uint8_t* hflag, uint32_t n, int k,
                     uint64_t seed, uint32_t iter, uint32_t* keys, uint64_t* vals,
                     uint32_t* dcnt, cudaStream_t st) {
    size_t tot = size_t(n) * k;
    k_cand_gen<<<unsigned((tot + 255) / 256), 256, 0, st>>>(hidx, hflag, n, k, seed, iter, keys,
                                                             vals, dcnt); count_launch();
}
void launch_cand_apply(const uint32_t* keys, const uint64_t* vals, const uint32_t* seg_off,
                       const uint32_t* dcnt, uint32_t n, int m, uint32_t* new_idx,
                       float* new_prio, uint32_t* old_idx, float* old_prio, cudaStream_t st) {
    k_cand_apply<<<(n + 127) / 128, 128, 0, st>>>(keys, vals, seg_off, dcnt, n, m, new_idx,
                                                  new_prio, old_idx, old_prio); count_launch();
}
void launch_flag_flip(const uint32_t* hidx, uint8_t* hflag, const uint32_t* new_idx, uint32_t n,
                      int k, int m, cudaStream_t st) {
    k_flag_flip<<<(n + 127) / 128, 128, 0, st>>>(hidx, hflag, new_idx, n, k, m); count_launch();
}

static size_t join_smem(int m, int dp, int words, bool rows) {
    return (rows ? size_t(2 * m) * dp * sizeof(float) : 0) + size_t(2 * m) * 8 +
           size_t(words) * 4;
}
static bool join_rows_fit(int m, int dp) { return size_t(2 * m) * dp * sizeof(float) <= 96 * 1024; }

void launch_join_count(const float* X, int d, int dp, uint32_t n, int k, int m,
                       const float* hdist, const uint32_t* new_idx, const uint32_t* old_idx,
                       uint32_t* bits, int words, uint32_t* row_cnt,
                       unsigned long long* pairs, cudaStream_t st) {
    bool rows = join_rows_fit(m, dp);
    size_t sm = join_smem(m, dp, words, rows);
    if (sm > 48 * 1024)
        cudaFuncSetAttribute(k_join_count, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    k_join_count<<<n, JT, sm, st>>>(X, d, dp, k, m, hdist, new_idx, old_idx, bits, words,
                                    row_cnt, pairs, rows); count_launch();
}
void launch_join_write(const float* X, int d, int dp, uint32_t n, int m, const uint32_t* new_idx,
                       const uint32_t* old_idx, const uint32_t* bits, int words,
                       const uint32_t* row_off, uint32_t* keys, uint64_t* vals, uint32_t* dcnt,
                       cudaStream_t st) {
    bool rows = join_rows_fit(m, dp);
    size_t sm = join_smem(m, dp, words, rows);
    if (sm > 48 * 1024)
        cudaFuncSetAttribute(k_join_write, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    k_join_write<<<n, JT, sm, st>>>(X, d, dp, m, new_idx, old_idx, bits, words, row_off, keys,
                                    vals, dcnt, rows); count_launch();
}
void launch_replay(const uint32_t* keys, const uint64_t* vals, const uint32_t* seg_off,
                   const uint32_t* dcnt, uint32_t n, int k, uint32_t* hidx, float* hdist,
                   uint8_t* hflag, unsigned long long* changed, cudaStream_t st) {
    k_replay<<<(n + 127) / 128, 128, 0, st>>>(keys, vals, seg_off, dcnt, n, k, hidx, hdist, hflag,
                                              changed); count_launch();
}
void launch_extract_count(const uint32_t* hidx, uint32_t n, int k, uint32_t* cnt,
                          cudaStream_t st) {
    k_extract_count<<<(n + 255) / 256, 256, 0, st>>>(hidx, n, k, cnt); count_launch();
}
void launch_extract(const uint32_t* hidx, const float* hdist, uint32_t n, int k,
                    const uint32_t* row_off, uint32_t* indptr, uint32_t* indices, float* dists,
                    cudaStream_t st) {
    k_extract<<<(n + 127) / 128, 128, 0, st>>>(hidx, hdist, n, k, row_off, indptr, indices,
                                               dists); count_launch();
}

}  // namespace pq
