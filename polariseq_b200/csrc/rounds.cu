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
// (apply_candidates, nndescent.rs:326-354).  One warp per 32 consecutive rows:
// their sorted records are contiguous, so the warp stages them in shared
// memory with coalesced loads (falling back to direct loads past CREC), then
// each lane replays its row into transposed shared-memory heaps ([slot][row])
// that are written back coalesced.
constexpr int CT = 32;      // rows (= threads) per candidate CTA
constexpr int CREC = 2048;  // staged records per CTA

__global__ void __launch_bounds__(CT) k_cand_apply(const uint32_t* __restrict__ keys,
                                                   const uint64_t* __restrict__ vals,
                                                   const uint32_t* __restrict__ seg_off,
                                                   const uint32_t* __restrict__ dcnt, uint32_t n,
                                                   int m, uint32_t* new_idx, float* new_prio,
                                                   uint32_t* old_idx, float* old_prio) {
    extern __shared__ __align__(16) unsigned char csm[];
    uint64_t* rec = reinterpret_cast<uint64_t*>(csm);
    uint32_t* ni = reinterpret_cast<uint32_t*>(rec + CREC);
    float* np = reinterpret_cast<float*>(ni + size_t(m) * CT);
    uint32_t* oi = reinterpret_cast<uint32_t*>(np + size_t(m) * CT);
    float* op = reinterpret_cast<float*>(oi + size_t(m) * CT);
    const uint32_t r0 = blockIdx.x * CT;
    const uint32_t rows = min(uint32_t(CT), n - r0);
    const uint32_t lane = threadIdx.x;
    const uint32_t r = r0 + lane;
    const uint32_t g0 = seg_off[r0];
    const uint32_t last = r0 + rows - 1;
    const uint32_t g1 = seg_off[last] + dcnt[last];
    const bool fits = g1 - g0 <= uint32_t(CREC);
    if (fits)
        for (uint32_t t = lane; t < g1 - g0; t += CT) rec[t] = vals[g0 + t];
    for (int s = 0; s < m; ++s) {
        ni[s * CT + lane] = PQ_EMPTY;
        np[s * CT + lane] = __int_as_float(0x7f800000);
        oi[s * CT + lane] = PQ_EMPTY;
        op[s * CT + lane] = __int_as_float(0x7f800000);
    }
    __syncwarp();
    if (lane < rows) {
        const uint32_t b = seg_off[r], e = b + dcnt[r];
        for (uint32_t t = b; t < e; ++t) {
            const uint64_t v = fits ? rec[t - g0] : vals[t];
            const uint32_t nbr = uint32_t(v);
            const uint32_t pb = uint32_t(v >> 32);
            const float prio = __uint_as_float(pb & 0x7fffffffu);
            if (pb >> 31)
                cand_push_strided(ni + lane, np + lane, m, CT, nbr, prio);
            else
                cand_push_strided(oi + lane, op + lane, m, CT, nbr, prio);
        }
    }
    __syncwarp();
    for (uint32_t o = lane; o < rows * uint32_t(m); o += CT) {
        const uint32_t row = o / m, s = o - row * m;
        const size_t g = size_t(r0) * m + o;
        new_idx[g] = ni[s * CT + row];
        new_prio[g] = np[s * CT + row];
        old_idx[g] = oi[s * CT + row];
        old_prio[g] = op[s * CT + row];
    }
}

// A candidate heap held in registers for a compile-time size M: every index
// of the push is a compile-time constant (the sift-down visits the unrolled
// node list with predicates; the current node only moves to higher indices),
// so the heap never touches memory.  Same rules as cand_push.
template <int M>
struct RHeap {
    uint32_t id[M];
    float pr[M];
};

template <int M>
__device__ __forceinline__ void rheap_init(RHeap<M>& h) {
#pragma unroll
    for (int s = 0; s < M; ++s) {
        h.id[s] = PQ_EMPTY;
        h.pr[s] = __int_as_float(0x7f800000);
    }
}

template <int M>
__device__ __forceinline__ void rheap_push(RHeap<M>& h, uint32_t j, float p) {
    if (p >= h.pr[0]) return;
    bool dup = false;
#pragma unroll
    for (int s = 0; s < M; ++s) dup |= h.id[s] == j;
    if (dup) return;
    int cur = 0;
    bool done = false;
#pragma unroll
    for (int c = 0; c < M; ++c) {
        if (!done && c == cur) {
            constexpr int dummy = 0;
            (void)dummy;
            const int l = 2 * c + 1, r = 2 * c + 2;
            int sw = c;
            float psw = p;
            if (l < M && h.pr[l < M ? l : 0] > psw) {
                sw = l;
                psw = h.pr[l < M ? l : 0];
            }
            if (r < M && h.pr[r < M ? r : 0] > psw) sw = r;
            if (sw == c) {
                h.id[c] = j;
                h.pr[c] = p;
                done = true;
            } else if (sw == l) {
                h.id[c] = h.id[l < M ? l : 0];
                h.pr[c] = h.pr[l < M ? l : 0];
                cur = l;
            } else {
                h.id[c] = h.id[r < M ? r : 0];
                h.pr[c] = h.pr[r < M ? r : 0];
                cur = r;
            }
        }
    }
}

// Register-heap variant of k_cand_apply for max_candidates == M; WHICH: 0 =
// new heap only, 1 = old heap only, 2 = both.
template <int M, int WHICH>
__global__ void __launch_bounds__(128) k_cand_apply_reg(const uint64_t* __restrict__ vals,
                                                        const uint32_t* __restrict__ seg_off,
                                                        const uint32_t* __restrict__ dcnt,
                                                        uint32_t n, uint32_t* new_idx,
                                                        float* new_prio, uint32_t* old_idx,
                                                        float* old_prio) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    RHeap<M> hn, ho;
    if (WHICH != 1) rheap_init(hn);
    if (WHICH != 0) rheap_init(ho);
    const uint32_t b = seg_off[r], e = b + dcnt[r];
    for (uint32_t t = b; t < e; ++t) {
        const uint64_t v = vals[t];
        const uint32_t nbr = uint32_t(v);
        const uint32_t pb = uint32_t(v >> 32);
        const float prio = __uint_as_float(pb & 0x7fffffffu);
        if (pb >> 31) {
            if (WHICH != 1) rheap_push(hn, nbr, prio);
        } else {
            if (WHICH != 0) rheap_push(ho, nbr, prio);
        }
    }
#pragma unroll
    for (int s = 0; s < M; ++s) {
        if (WHICH != 1) {
            new_idx[size_t(r) * M + s] = hn.id[s];
            new_prio[size_t(r) * M + s] = hn.pr[s];
        }
        if (WHICH != 0) {
            old_idx[size_t(r) * M + s] = ho.id[s];
            old_prio[size_t(r) * M + s] = ho.pr[s];
        }
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

// A source row's candidates in shared memory: slot b < m is news[b], slot
// b >= m is olds[b-m].  Pair (a, b) — news[a] with slot b > a — is the
// reference's pair order (nndescent.rs:941-964): a ascending, then the later
// news, then the olds.  Its two emit bits (p side, then q side) sit at bit
// 2*(a*2m + b) of the row's mask, so a record's rank in the row's generation
// order is the number of set bits before its own.  The kernels enumerate
// only the valid pairs (non-empty news x later non-empty news, non-empty news
// x non-empty olds), one per thread.
struct JoinSmem {
    float* rows;      // 2m * dp
    uint32_t* cand;   // 2m
    float* thr;       // 2m
    uint32_t* bits;   // words
    uint32_t* wpre;   // words (write pass: exclusive prefix of popcounts)
    uint16_t* nlist;  // m: slots of the non-empty news, in order
    uint16_t* olist;  // m: slots of the non-empty olds, in order
};

__device__ __forceinline__ JoinSmem join_smem(unsigned char* sm, int m, int dp, int words) {
    JoinSmem s;
    s.rows = reinterpret_cast<float*>(sm);
    s.cand = reinterpret_cast<uint32_t*>(sm + size_t(2 * m) * dp * sizeof(float));
    s.thr = reinterpret_cast<float*>(s.cand + 2 * m);
    s.bits = reinterpret_cast<uint32_t*>(s.thr + 2 * m);
    s.wpre = s.bits + words;
    s.nlist = reinterpret_cast<uint16_t*>(s.wpre + words);
    s.olist = s.nlist + m;
    return s;
}

// Loads the candidate ids, (optionally) thresholds and rows, and compacts the
// non-empty news/olds; returns their counts through nn / no.
__device__ __forceinline__ void join_load(const float* __restrict__ X, int dp, int k, int m,
                                          const float* __restrict__ hdist,
                                          const uint32_t* __restrict__ new_idx,
                                          const uint32_t* __restrict__ old_idx, uint32_t i,
                                          const JoinSmem& s, uint32_t* cnt2) {
    for (int t = threadIdx.x; t < 2 * m; t += JT) {
        uint32_t c = t < m ? new_idx[size_t(i) * m + t] : old_idx[size_t(i) * m + (t - m)];
        s.cand[t] = c;
        if (hdist) s.thr[t] = c != PQ_EMPTY ? hdist[size_t(c) * k] : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // warp 0 compacts both lists with ballots
        const int lane = threadIdx.x;
        uint32_t nn = 0, no = 0;
        for (int b0 = 0; b0 < m; b0 += 32) {
            const int t = b0 + lane;
            const bool vn = t < m && s.cand[t] != PQ_EMPTY;
            const bool vo = t < m && s.cand[m + t] != PQ_EMPTY;
            const unsigned bn = __ballot_sync(0xFFFFFFFFu, vn);
            const unsigned bo = __ballot_sync(0xFFFFFFFFu, vo);
            const unsigned lt = (1u << lane) - 1u;
            if (vn) s.nlist[nn + __popc(bn & lt)] = uint16_t(t);
            if (vo) s.olist[no + __popc(bo & lt)] = uint16_t(t);
            nn += __popc(bn);
            no += __popc(bo);
        }
        if (lane == 0) {
            cnt2[0] = nn;
            cnt2[1] = no;
        }
    }
    const int q4 = dp / 4;
    for (int t = threadIdx.x; t < 2 * m * q4; t += JT) {
        int r = t / q4, j = t - r * q4;
        uint32_t c = s.cand[r];
        if (c != PQ_EMPTY)
            reinterpret_cast<float4*>(s.rows)[t] =
                reinterpret_cast<const float4*>(X + size_t(c) * dp)[j];
    }
    __syncthreads();
}

// Work item t of a row with nn news and no olds -> slots (a, b).  Items
// [0, nn(nn-1)/2) are the news x later-news pairs (a-major), the rest the
// news x olds pairs.
__device__ __forceinline__ void join_item(const JoinSmem& s, int m, uint32_t nn, uint32_t no,
                                          uint32_t t, int& a, int& b) {
    const uint32_t t1 = nn * (nn - 1) / 2;
    if (t < t1) {
        // row ia of the strict upper triangle: S(ia) = ia*nn - ia*(ia+1)/2 <= t
        const float fn = float(2 * nn - 1);
        int ia = int((fn - sqrtf(fn * fn - 8.0f * float(t))) * 0.5f);
        if (ia < 0) ia = 0;
        while (ia > 0 && uint32_t(ia * nn - ia * (ia + 1) / 2) > t) --ia;
        while (uint32_t((ia + 1) * nn - (ia + 1) * (ia + 2) / 2) <= t) ++ia;
        const int ib = ia + 1 + int(t - uint32_t(ia * nn - ia * (ia + 1) / 2));
        a = s.nlist[ia];
        b = s.nlist[ib];
    } else {
        const uint32_t u = t - t1;
        const uint32_t ia = u / no, ib = u - ia * no;
        a = s.nlist[ia];
        b = m + s.olist[ib];
    }
}

// Pass 1: distances, emit bits (p side: d < thr[p]; q side: d < thr[q]) and
// the row's update count.  CTA b handles source row perm[b] (a spatially
// coherent order, so neighbouring CTAs share candidate rows in L2).
template <int D>
__global__ void __launch_bounds__(JT) k_join_count(const float* __restrict__ X, int d, int dp,
                                                   int k, int m, const float* __restrict__ hdist,
                                                   const uint32_t* __restrict__ new_idx,
                                                   const uint32_t* __restrict__ old_idx,
                                                   const uint32_t* __restrict__ perm,
                                                   uint32_t* bits, int words, uint32_t* row_cnt,
                                                   unsigned long long* pairs) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ uint32_t red[JT / 32], redp[JT / 32], cnt2[2];
    const uint32_t i = perm ? perm[blockIdx.x] : blockIdx.x;
    const JoinSmem s = join_smem(sm, m, dp, words);
    for (int t = threadIdx.x; t < words; t += JT) s.bits[t] = 0;
    join_load(X, dp, k, m, hdist, new_idx, old_idx, i, s, cnt2);
    const uint32_t nn = cnt2[0], no = cnt2[1];
    const uint32_t W = nn * (nn - (nn > 0 ? 1 : 0)) / 2 + nn * no;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t cnt = 0, np = 0;
    for (uint32_t t = threadIdx.x; t < W; t += JT) {
        int a, b;
        join_item(s, m, nn, no, t, a, b);
        if (s.cand[a] == s.cand[b]) continue;  // q == p (a news entry also among the olds)
        ++np;
        const float dd = sq_dist_exact_t<D>(s.rows + size_t(a) * dp, s.rows + size_t(b) * dp, d);
        const uint32_t e1 = dd < s.thr[a], e2 = dd < s.thr[b];
        if (e1 | e2) {
            const int bit = 2 * (a * 2 * m + b);
            atomicOr(&s.bits[bit >> 5], (e1 | (e2 << 1)) << (bit & 31));
            cnt += e1 + e2;
        }
    }
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    np = __reduce_add_sync(0xFFFFFFFFu, np);
    if (lane == 0) {
        red[w] = cnt;
        redp[w] = np;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t c = 0, pp = 0;
        for (int ww = 0; ww < JT / 32; ++ww) {
            c += red[ww];
            pp += redp[ww];
        }
        row_cnt[i] = c;
        if (pp) atomicAdd(pairs, (unsigned long long)pp);
    }
    for (int t = threadIdx.x; t < words; t += JT) bits[size_t(i) * words + t] = s.bits[t];
}

// Pass 2: one thread per record (set bit): its rank is its bit's rank in the
// row mask; recompute the pair's distance and write (dest, nbr, dist) at the
// row's offset plus that rank.
template <int D>
__global__ void __launch_bounds__(JT) k_join_write(const float* __restrict__ X, int d, int dp,
                                                   int m, const uint32_t* __restrict__ new_idx,
                                                   const uint32_t* __restrict__ old_idx,
                                                   const uint32_t* __restrict__ perm,
                                                   const uint32_t* __restrict__ bits, int words,
                                                   const uint32_t* __restrict__ row_cnt,
                                                   const uint32_t* __restrict__ row_off,
                                                   uint32_t* keys, uint64_t* vals,
                                                   uint32_t* dcnt) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ uint32_t ws[JT / 32], cnt2[2];
    const uint32_t i = perm ? perm[blockIdx.x] : blockIdx.x;
    const uint32_t R = row_cnt[i];
    if (R == 0) return;
    const JoinSmem s = join_smem(sm, m, dp, words);
    // word popcount prefix: thread t owns a contiguous run of words
    const int per = (words + JT - 1) / JT;
    const int w0 = threadIdx.x * per, w1 = min(words, w0 + per);
    uint32_t c = 0;
    for (int t = w0; t < w1; ++t) {
        uint32_t v = bits[size_t(i) * words + t];
        s.bits[t] = v;
        c += __popc(v);
    }
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        uint32_t x = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        uint32_t run = x - c;
        for (int ww = 0; ww < w; ++ww) run += ws[ww];
        for (int t = w0; t < w1; ++t) {
            s.wpre[t] = run;
            run += __popc(s.bits[t]);
        }
    }
    join_load(X, dp, 0, m, nullptr, new_idx, old_idx, i, s, cnt2);
    const uint32_t base = row_off[i];
    const int m2 = 2 * m;
    for (uint32_t r = threadIdx.x; r < R; r += JT) {
        // word holding the r-th set bit: the last word whose prefix is <= r
        int lo = 0, hi = words - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s.wpre[mid] <= r) lo = mid; else hi = mid - 1;
        }
        const uint32_t bitpos = __fns(s.bits[lo], 0, int(r - s.wpre[lo]) + 1);
        const uint32_t gb = uint32_t(lo) * 32u + bitpos;
        const uint32_t slot = gb >> 1;
        const int a = int(slot / uint32_t(m2)), b = int(slot - uint32_t(a) * m2);
        const uint32_t p = s.cand[a], q = s.cand[b];
        const float dd = sq_dist_exact_t<D>(s.rows + size_t(a) * dp, s.rows + size_t(b) * dp, d);
        const uint64_t db = uint64_t(__float_as_uint(dd)) << 32;
        const uint32_t dest = (gb & 1u) ? q : p, nbr = (gb & 1u) ? p : q;
        keys[base + r] = dest;
        vals[base + r] = db | nbr;
        atomicAdd(&dcnt[dest], 1u);
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
    if (m == 30) {
        k_cand_apply_reg<30, 0><<<(n + 127) / 128, 128, 0, st>>>(vals, seg_off, dcnt, n, new_idx,
                                                                 new_prio, old_idx, old_prio); count_launch();
        k_cand_apply_reg<30, 1><<<(n + 127) / 128, 128, 0, st>>>(vals, seg_off, dcnt, n, new_idx,
                                                                 new_prio, old_idx, old_prio); count_launch();
        return;
    }
    if (m == 60) {
        k_cand_apply_reg<60, 0><<<(n + 127) / 128, 128, 0, st>>>(vals, seg_off, dcnt, n, new_idx,
                                                                 new_prio, old_idx, old_prio); count_launch();
        k_cand_apply_reg<60, 1><<<(n + 127) / 128, 128, 0, st>>>(vals, seg_off, dcnt, n, new_idx,
                                                                 new_prio, old_idx, old_prio); count_launch();
        return;
    }
    size_t sm = size_t(CREC) * 8 + size_t(m) * CT * 16;
    if (sm > 40 * 1024)
        cudaFuncSetAttribute(k_cand_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    k_cand_apply<<<(n + CT - 1) / CT, CT, sm, st>>>(keys, vals, seg_off, dcnt, n, m, new_idx,
                                                    new_prio, old_idx, old_prio); count_launch();
}
void launch_flag_flip(const uint32_t* hidx, uint8_t* hflag, const uint32_t* new_idx, uint32_t n,
                      int k, int m, cudaStream_t st) {
    k_flag_flip<<<(n + 127) / 128, 128, 0, st>>>(hidx, hflag, new_idx, n, k, m); count_launch();
}

static size_t join_smem_bytes(int m, int dp, int words) {
    return size_t(2 * m) * dp * sizeof(float) + size_t(2 * m) * 8 + size_t(words) * 8 +
           size_t(2 * m) * 2 + 16;
}

template <class K>
static void set_smem(K kern, size_t sm) {
    if (sm > 40 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
}

void launch_join_count(const float* X, int d, int dp, uint32_t n, int k, int m,
                       const float* hdist, const uint32_t* new_idx, const uint32_t* old_idx,
                       const uint32_t* perm, uint32_t* bits, int words, uint32_t* row_cnt,
                       unsigned long long* pairs, cudaStream_t st) {
    size_t sm = join_smem_bytes(m, dp, words);
    if (d == 50) {
        set_smem(k_join_count<50>, sm);
        k_join_count<50><<<n, JT, sm, st>>>(X, d, dp, k, m, hdist, new_idx, old_idx, perm, bits,
                                            words, row_cnt, pairs); count_launch();
    } else {
        set_smem(k_join_count<0>, sm);
        k_join_count<0><<<n, JT, sm, st>>>(X, d, dp, k, m, hdist, new_idx, old_idx, perm, bits,
                                           words, row_cnt, pairs); count_launch();
    }
}
void launch_join_write(const float* X, int d, int dp, uint32_t n, int m, const uint32_t* new_idx,
                       const uint32_t* old_idx, const uint32_t* perm, const uint32_t* bits,
                       int words, const uint32_t* row_cnt, const uint32_t* row_off,
                       uint32_t* keys, uint64_t* vals, uint32_t* dcnt, cudaStream_t st) {
    size_t sm = join_smem_bytes(m, dp, words);
    if (d == 50) {
        set_smem(k_join_write<50>, sm);
        k_join_write<50><<<n, JT, sm, st>>>(X, d, dp, m, new_idx, old_idx, perm, bits, words,
                                            row_cnt, row_off, keys, vals, dcnt); count_launch();
    } else {
        set_smem(k_join_write<0>, sm);
        k_join_write<0><<<n, JT, sm, st>>>(X, d, dp, m, new_idx, old_idx, perm, bits, words,
                                           row_cnt, row_off, keys, vals, dcnt); count_launch();
    }
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
