// RP-tree forest of the plain form, bit-exact with the reference's
// build_tree (crates/polariseq-core/src/nndescent.rs:356-646).
//
// Top levels (rp_tree_parallel, :587-641: nodes of >= 8192 points above depth
// 6) are processed level by level for all trees at once: one hyperplane per
// node, one thread per (tree, position) for the margins, and a closed-form
// parallel restatement of the two-pointer partition (:389-405).  Below that
// every subtree is finished by one CTA in depth-first order with one Rng, as
// rp_tree_sequential/rp_tree_leaves (:419-581) draw it.
//
// The two-pointer partition moves, for a node with nL left points:
//   left  point at p <  nL          -> p
//   right point at p <  nL, rank j  -> (j == 1 ? size : B[j-1]) - 1
//   left  point at p >= nL, rank j  -> A[j]          (rank from the top)
//   right point at p >  nL          -> p - 1
//   right point at p == nL          -> (c == 0 ? size : B[c]) - 1
// where A[j] is the position of the j-th right point in [0, nL), B[j] the
// position of the j-th left point in [nL, size) counted from the top, and c
// the number of right points in [0, nL).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "primitives.cuh"

namespace pq {
namespace {

constexpr int FT = 256;             // threads per forest CTA
constexpr int PER = FOREST_CHUNK / FT;  // positions per thread in a chunk
constexpr int STK = 128;            // DFS stack depth (depth > 100 is a leaf)

// Exclusive block scan of one u32 per thread (any multiple of 32 threads, at
// most 1024); *total receives the block sum.
__device__ __forceinline__ uint32_t bscan(uint32_t v, uint32_t* ws, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < nw ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) ws[lane] = s;
    }
    __syncthreads();
    uint32_t r = (w > 0 ? ws[w - 1] : 0) + x - v;
    *total = ws[nw - 1];
    __syncthreads();
    return r;
}

// random_hyperplane (nndescent.rs:367-385) for one top-level node.
__global__ void k_hyper(ForestArgs a, PNode* nodes, float* normals) {
    __shared__ uint32_t sA, sB;
    PNode nd = nodes[blockIdx.x];
    if (threadIdx.x == 0) {
        Rng r{nd.seed};
        const uint32_t* ids = a.ids + size_t(nd.tree) * a.n + nd.start;
        uint32_t A = ids[r.below(nd.size)];
        uint32_t B = ids[r.below(nd.size)];
        int tries = 0;
        while (B == A && tries < 8) {
            B = ids[r.below(nd.size)];
            ++tries;
        }
        sA = A;
        sB = B;
        nodes[blockIdx.x].rng_after = r.s;
    }
    __syncthreads();
    const float* xa = a.X + size_t(sA) * a.dp;
    const float* xb = a.X + size_t(sB) * a.dp;
    float* nv = normals + size_t(blockIdx.x) * a.dp;
    for (int j = threadIdx.x; j < a.dp; j += blockDim.x)
        nv[j] = j < a.d ? __fsub_rn(xa[j], xb[j]) : 0.0f;
    if (threadIdx.x == 0) {
        float s = -0.0f;  // Rust's f32 sum folds from -0.0
        for (int j = 0; j < a.d; ++j) {
            float nvj = __fsub_rn(xa[j], xb[j]);
            s = __fadd_rn(s, __fmul_rn(__fmul_rn(nvj, 0.5f), __fadd_rn(xa[j], xb[j])));
        }
        nodes[blockIdx.x].offset = -s;
    }
}

// Margins of a top-level chunk; ties go by splitmix(seed ^ id) & 1 (:599-607).
__global__ void __launch_bounds__(FT) k_sides(ForestArgs a, const PNode* nodes,
                                              const uint32_t* chunk_node, const float* normals,
                                              uint32_t* chunkL) {
    extern __shared__ __align__(16) float nv[];
    __shared__ uint32_t ws[32];
    const uint32_t ni = chunk_node[blockIdx.x];
    const PNode nd = nodes[ni];
    for (int j = threadIdx.x; j < a.dp; j += FT) nv[j] = normals[size_t(ni) * a.dp + j];
    __syncthreads();
    const uint32_t off = (blockIdx.x - nd.chunk0) * FOREST_CHUNK;
    const uint32_t len = min(uint32_t(FOREST_CHUNK), nd.size - off);
    const size_t tb = size_t(nd.tree) * a.n + nd.start + off;
    uint32_t cnt = 0;
    for (uint32_t i = threadIdx.x; i < len; i += FT) {
        uint32_t id = a.ids[tb + i];
        float m = __fadd_rn(dot_exact(nv, a.X + size_t(id) * a.dp, a.d), nd.offset);
        bool left = fabsf(m) < 1e-8f ? ((splitmix(nd.seed ^ uint64_t(id)) & 1ull) == 0)
                                     : (m > 0.0f);
        a.side[tb + i] = left ? 1 : 0;
        cnt += left;
    }
    uint32_t tot;
    bscan(cnt, ws, &tot);
    if (threadIdx.x == 0) chunkL[blockIdx.x] = tot;
}

// Per node: exclusive prefix of its chunks' left counts; nL = total.
__global__ void k_node_scan(PNode* nodes, uint32_t nn, uint32_t* chunkL) {
    uint32_t ni = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (ni >= nn) return;
    const int lane = threadIdx.x & 31;
    PNode nd = nodes[ni];
    uint32_t nch = (nd.size + FOREST_CHUNK - 1) / FOREST_CHUNK;
    uint32_t run = 0;
    for (uint32_t b = 0; b < nch; b += 32) {
        uint32_t c = b + lane;
        uint32_t v = c < nch ? chunkL[nd.chunk0 + c] : 0;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (c < nch) chunkL[nd.chunk0 + c] = run + x - v;
        run += __shfl_sync(0xFFFFFFFFu, x, 31);
    }
    if (lane == 0) {
        nodes[ni].nL = run;
        nodes[ni].c = 0;
    }
}

// Pass 1 of the partition: rank tables A/B and c (see the file comment).
__global__ void __launch_bounds__(FT) k_part_tables(ForestArgs a, PNode* nodes,
                                                    const uint32_t* chunk_node,
                                                    const uint32_t* chunkPre) {
    __shared__ uint32_t ws[32];
    const uint32_t ni = chunk_node[blockIdx.x];
    const PNode nd = nodes[ni];
    const uint32_t off = (blockIdx.x - nd.chunk0) * FOREST_CHUNK;
    const uint32_t len = min(uint32_t(FOREST_CHUNK), nd.size - off);
    const size_t nb = size_t(nd.tree) * a.n + nd.start;
    uint8_t s[PER];
    uint32_t cnt = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t i = threadIdx.x * PER + j;
        s[j] = i < len ? a.side[nb + off + i] : 0;
        cnt += s[j];
    }
    uint32_t tot;
    uint32_t lp = chunkPre[blockIdx.x] + bscan(cnt, ws, &tot);
    const uint32_t nL = nd.nL;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t i = threadIdx.x * PER + j;
        if (i < len) {
            uint32_t p = off + i;
            if (s[j]) {
                if (p >= nL) a.tabB[nb + (nL - lp) - 1] = p;
            } else {
                if (p < nL) a.tabA[nb + (p - lp)] = p;  // rank p-lp+1, 0-based p-lp
            }
            if (p == nL) nodes[ni].c = nL - lp;
            lp += s[j];
        }
    }
}

// Pass 2: scatter ids to their partitioned positions in tmp.
__global__ void __launch_bounds__(FT) k_part_scatter(ForestArgs a, const PNode* nodes,
                                                     const uint32_t* chunk_node,
                                                     const uint32_t* chunkPre) {
    __shared__ uint32_t ws[32];
    const uint32_t ni = chunk_node[blockIdx.x];
    const PNode nd = nodes[ni];
    const uint32_t off = (blockIdx.x - nd.chunk0) * FOREST_CHUNK;
    const uint32_t len = min(uint32_t(FOREST_CHUNK), nd.size - off);
    const size_t nb = size_t(nd.tree) * a.n + nd.start;
    uint8_t s[PER];
    uint32_t cnt = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t i = threadIdx.x * PER + j;
        s[j] = i < len ? a.side[nb + off + i] : 0;
        cnt += s[j];
    }
    uint32_t tot;
    uint32_t lp = chunkPre[blockIdx.x] + bscan(cnt, ws, &tot);
    const uint32_t nL = nd.nL, size = nd.size, c = nd.c;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        uint32_t i = threadIdx.x * PER + j;
        if (i < len) {
            uint32_t p = off + i, dst;
            if (s[j]) {
                dst = p < nL ? p : a.tabA[nb + (nL - lp) - 1];
            } else if (p < nL) {
                uint32_t r = p - lp + 1;
                dst = (r == 1 ? size : a.tabB[nb + r - 2]) - 1;
            } else if (p > nL) {
                dst = p - 1;
            } else {
                dst = (c == 0 ? size : a.tabB[nb + c - 1]) - 1;
            }
            a.tmp[nb + dst] = a.ids[nb + p];
            lp += s[j];
        }
    }
}

__global__ void __launch_bounds__(FT) k_part_copy(ForestArgs a, const PNode* nodes,
                                                  const uint32_t* chunk_node) {
    const uint32_t ni = chunk_node[blockIdx.x];
    const PNode nd = nodes[ni];
    const uint32_t off = (blockIdx.x - nd.chunk0) * FOREST_CHUNK;
    const uint32_t len = min(uint32_t(FOREST_CHUNK), nd.size - off);
    const size_t nb = size_t(nd.tree) * a.n + nd.start + off;
    for (uint32_t i = threadIdx.x; i < len; i += FT) a.ids[nb + i] = a.tmp[nb + i];
}

// random_split (nndescent.rs:408-415) where the hyperplane separated nothing.
__global__ void k_degenerate(ForestArgs a, PNode* nodes, uint32_t nn) {
    uint32_t ni = blockIdx.x * blockDim.x + threadIdx.x;
    if (ni >= nn) return;
    PNode nd = nodes[ni];
    if (nd.nL != 0 && nd.nL != nd.size) return;
    Rng r{nd.rng_after};
    uint32_t* ids = a.ids + size_t(nd.tree) * a.n + nd.start;
    for (uint32_t i = nd.size - 1; i >= 1; --i) {
        uint32_t j = uint32_t(r.below(uint64_t(i) + 1));
        uint32_t t = ids[i];
        ids[i] = ids[j];
        ids[j] = t;
    }
    nodes[ni].nL = nd.size / 2;
}

// One CTA finishes one subtree depth-first with a single Rng
// (rp_tree_sequential / rp_tree_leaves, nndescent.rs:419-581).
//
// Every thread draws from its own copy of the Rng and sums the hyperplane
// offset itself (the values are identical in all threads), so no node has a
// serial section.  Nodes larger than the staged capacity run in global mode:
// all NT threads compute margins from the rows in HBM and partition through
// the per-tree scratch arrays.  A node of at most SCAP points has its ids and
// rows staged in shared memory once (the reference gathers small subtrees
// for the same reason, :474-491) and warp 0 alone finishes its whole subtree
// with ballots, without block barriers.  The largest subtrees (their
// depth-first chains are the critical path) run with NT = 512.
constexpr int SCAP = 128;   // staged capacity (points): 4 per lane of warp 0
// A node of at most MCAP points in a 512-thread CTA is staged with its whole
// subtree (ids and rows in shared memory): its splits of more than SCAP
// points take one point per thread, the smaller ones go to warp 0.
constexpr int MCAP = 512;

// Shared state of one subtree CTA; CAP staged points (MCAP in 512-thread
// CTAs, which stage whole subtrees of up to 512 points, SCAP otherwise: the
// smaller CTAs never stage more, and hold 7 KB instead of 17 KB).
template <int CAP>
struct SeqShared {
    uint32_t stS[STK], stN[STK];
    uint16_t stD[STK];
    uint32_t lS[STK], lN[STK];
    uint16_t lD[STK];
    uint32_t mS[STK], mN[STK];
    uint16_t mD[STK];
    uint32_t sid[CAP], sslot[CAP], sid2[CAP], sslot2[CAP];
    uint8_t code[CAP];
    uint32_t tabA[CAP], tabB[CAP];
    uint32_t ws[32];
    uint64_t rng;
    float off;
    uint32_t cntL, sc;
    int sp, anytie;
};

// The global nanosecond timer (comparable across SMs; trace only).
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// 16-byte asynchronous global -> shared copies (both addresses 16-byte
// aligned), bypassing L1.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// Draws of random_hyperplane (nndescent.rs:369-375) as positions: ids within
// a node are distinct, so the reference's `b == a` is a position test.
// x mod n for n < 2^16 in 32-bit arithmetic: (hi * 2^32 + lo) mod n =
// ((hi mod n) * t32 + lo mod n) mod n with t32 = 2^32 mod n (every product and
// sum stays below n^2 + n < 2^32).
__device__ __forceinline__ uint32_t mod_u64_small(uint64_t x, uint32_t n, uint32_t t32) {
    const uint32_t hi = uint32_t(x >> 32) % n, lo = uint32_t(x) % n;
    return (hi * t32 + lo) % n;
}

// The draws of one node share their divisor's constants (below(n) is
// next_u64() % n): 32-bit steps for n < 2^16 (staged nodes), a shared
// reciprocal above.
__device__ __forceinline__ void draw_pair(Rng& r, uint32_t n, uint32_t& pa, uint32_t& pb) {
    int tries = 0;
    if (n < 65536u) {
        const uint32_t t32 = (0xFFFFFFFFu % n + 1u) % n;
        pa = mod_u64_small(r.next_u64(), n, t32);
        pb = mod_u64_small(r.next_u64(), n, t32);
        while (pb == pa && tries < 8) {
            pb = mod_u64_small(r.next_u64(), n, t32);
            ++tries;
        }
        return;
    }
    const double rn = __drcp_rn(double(n));
    pa = mod_u64_u32_r(r.next_u64(), n, rn);
    pb = mod_u64_u32_r(r.next_u64(), n, rn);
    while (pb == pa && tries < 8) {
        pb = mod_u64_u32_r(r.next_u64(), n, rn);
        ++tries;
    }
}

// The normal nv = xa - xb in registers and the hyperplane offset in one pass
// over the two rows (16-byte loads), in hyper_offset_t's sequential order.
template <int D>
__device__ __forceinline__ float normal_offset_reg(const float* __restrict__ xa,
                                                   const float* __restrict__ xb, float (&nvr)[D]) {
    float s = -0.0f;
    const float4* a4 = reinterpret_cast<const float4*>(xa);
    const float4* b4 = reinterpret_cast<const float4*>(xb);
#pragma unroll
    for (int q = 0; q < D / 4; ++q) {
        const float4 x = a4[q], y = b4[q];
        const float av[4] = {x.x, x.y, x.z, x.w}, bv[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float t = __fsub_rn(av[u], bv[u]);
            nvr[4 * q + u] = t;
            s = __fadd_rn(s, __fmul_rn(__fmul_rn(t, 0.5f), __fadd_rn(av[u], bv[u])));
        }
    }
#pragma unroll
    for (int j = D / 4 * 4; j < D; ++j) {
        const float t = __fsub_rn(xa[j], xb[j]);
        nvr[j] = t;
        s = __fadd_rn(s, __fmul_rn(__fmul_rn(t, 0.5f), __fadd_rn(xa[j], xb[j])));
    }
    return -s;
}

// dot_exact_t<D>(nv, x) with the normal in registers (the same lanes, order
// and rounding; a product is the same either way round).
template <int D>
__device__ __forceinline__ float dot_reg(const float (&nvr)[D], const float* __restrict__ x) {
    constexpr int FULL = D / 8;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float4* x4 = reinterpret_cast<const float4*>(x);
#pragma unroll
    for (int c = 0; c < FULL; ++c) {
        const float4 y0 = x4[2 * c], y1 = x4[2 * c + 1];
        const float y[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
        for (int l = 0; l < 8; ++l) acc[l] = __fadd_rn(acc[l], __fmul_rn(nvr[8 * c + l], y[l]));
    }
    float tail = 0.0f;
#pragma unroll
    for (int j = FULL * 8; j < D; ++j) tail = __fadd_rn(tail, __fmul_rn(nvr[j], x[j]));
    const float r = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[4]), __fadd_rn(acc[1], acc[5])),
                              __fadd_rn(__fadd_rn(acc[2], acc[6]), __fadd_rn(acc[3], acc[7])));
    return __fadd_rn(r, tail);
}

// x mod n for a 32-bit x from m = floor((2^32 - 1) / n): m >= (2^32 - n) / n,
// so q = floor(x m / 2^32) > x / n - 2, i.e. q is floor(x / n) or one below,
// and one conditional subtraction of n finishes the remainder.
__device__ __forceinline__ uint32_t mod_magic(uint32_t x, uint32_t n, uint32_t m) {
    const uint32_t r = x - __umulhi(x, m) * n;
    return r >= n ? r - n : r;
}
// mod_u64_small with the node's one division shared by all its draws.
__device__ __forceinline__ uint32_t mod_u64_magic(uint64_t x, uint32_t n, uint32_t m,
                                                  uint32_t t32) {
    const uint32_t hi = mod_magic(uint32_t(x >> 32), n, m), lo = mod_magic(uint32_t(x), n, m);
    return mod_magic(hi * t32 + lo, n, m);
}

// draw_pair with the next two Rng states already computed (la1 =
// splitmix(r.s), la2 = splitmix(la1)), for n < 2^16; the caller recomputes the
// look-ahead after every other draw, off the critical path.
__device__ __forceinline__ void draw_pair_la(Rng& r, uint64_t la1, uint64_t la2, uint32_t n,
                                             uint32_t& pa, uint32_t& pb) {
    const uint32_t m = 0xFFFFFFFFu / n;
    const uint32_t r1 = 0xFFFFFFFFu - m * n + 1u;  // (2^32 - 1) mod n, plus one
    const uint32_t t32 = r1 == n ? 0u : r1;        // 2^32 mod n
    pa = mod_u64_magic(la1, n, m, t32);
    pb = mod_u64_magic(la2, n, m, t32);
    r.s = la2;
    int tries = 0;
    while (pb == pa && tries < 8) {
        pb = mod_u64_magic(r.next_u64(), n, m, t32);
        ++tries;
    }
}

// Warp 0 finishes a staged subtree: local positions [0, n0) of the staged
// ids/slots, rows in `rows` (slot-indexed), normal in `nv`.
template <int D, class SS>
__device__ uint32_t warp_subtree(const ForestArgs& a, SS& S, uint32_t* sid, uint32_t* sslot,
                                 float* rows, float* nv, uint32_t st, uint32_t n0, uint32_t dep0,
                                 Rng& rng, uint8_t* leaf, bool tb0 = false) {
    const int lane = threadIdx.x & 31;
    uint32_t nodes = 0;
    unsigned long long* tr = a.trace;
    long long tc = tb0 ? clock64() : 0;
    auto phase = [&](int slot) {
        if (tb0) {
            const long long t1 = clock64();
            tr[slot] += t1 - tc;
            tc = t1;
        }
    };
    const int d = a.d, dp = a.dp;
    const unsigned lt = (1u << lane) - 1u;
    // the next two Rng states, computed while the previous split works
    uint64_t la1 = splitmix(rng.s), la2 = splitmix(la1);
    int lsp = 1;
    if (lane == 0) {
        S.lS[0] = 0;
        S.lN[0] = n0;
        S.lD[0] = uint16_t(dep0);
    }
    __syncwarp();
    while (lsp > 0) {
        const uint32_t ls = S.lS[lsp - 1], ln = S.lN[lsp - 1], ld = S.lD[lsp - 1];
        __syncwarp();
        lsp -= 1;
        if (ln <= a.leaf_size || ld > 100) {
            if (lane == 0) leaf[st + ls] = 1;
            phase(SEQ_T_W_LEAF);
            continue;
        }
        if (a.trace && lane == 0) atomicAdd(&a.trace[SEQ_T_STAGED_NODES], 1ull);
        ++nodes;
        uint32_t pa, pb;
        draw_pair_la(rng, la1, la2, ln, pa, pb);
        la1 = splitmix(rng.s);
        la2 = splitmix(la1);
        phase(SEQ_T_W_DRAW);
        const float* xa = rows + size_t(sslot[ls + pa]) * dp;
        const float* xb = rows + size_t(sslot[ls + pb]) * dp;
        // margins of the positions this lane owns (lane + 32*i): the offset's
        // sequential sum and the dot products are independent chains, issued
        // together: the first group always, the second for nodes above 32
        // points (a position past the node reads its last row, whose product
        // is ignored), the next two only for nodes above 64 points
        float dots[SCAP / 32];
        float off;
        const uint32_t last = ln - 1;
        if constexpr (D > 0) {
            // every lane holds the normal in registers (no shared-memory round
            // trip), built in the same pass as the offset
            float nvr[D];
            off = normal_offset_reg<D>(xa, xb, nvr);
            dots[1] = dots[2] = dots[3] = 0.f;
            if (ln > 32u) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const uint32_t p = min(uint32_t(lane + 32 * i), last);
                    dots[i] = dot_reg<D>(nvr, rows + size_t(sslot[ls + p]) * dp);
                }
            } else {
                dots[0] = dot_reg<D>(nvr, rows + size_t(sslot[ls + min(uint32_t(lane), last)]) * dp);
            }
            if (ln > 64u) {
#pragma unroll
                for (int i = 2; i < SCAP / 32; ++i) {
                    const uint32_t p = min(uint32_t(lane + 32 * i), last);
                    dots[i] = dot_reg<D>(nvr, rows + size_t(sslot[ls + p]) * dp);
                }
            }
        } else {
            for (int j = lane; j < dp; j += 32) nv[j] = j < d ? __fsub_rn(xa[j], xb[j]) : 0.0f;
            __syncwarp();
            off = hyper_offset_t<D>(xa, xb, d);
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t p = min(uint32_t(lane + 32 * i), last);
                dots[i] = dot_exact_t<D>(nv, rows + size_t(sslot[ls + p]) * dp, d);
            }
            dots[2] = dots[3] = 0.f;
            if (ln > 64u) {
#pragma unroll
                for (int i = 2; i < SCAP / 32; ++i) {
                    const uint32_t p = min(uint32_t(lane + 32 * i), last);
                    dots[i] = dot_exact_t<D>(nv, rows + size_t(sslot[ls + p]) * dp, d);
                }
            }
        }
        // sides in registers; through shared memory only when a tie draws
        unsigned any_tie = 0;
        uint8_t code[SCAP / 32];
#pragma unroll
        for (int i = 0; i < SCAP / 32; ++i) {
            const uint32_t p = lane + 32 * i;
            code[i] = 0;
            if (p < ln) {
                const float m = __fadd_rn(dots[i], off);
                code[i] = fabsf(m) < 1e-8f ? 2 : (m > 0.0f ? 1 : 0);
                any_tie |= code[i] == 2;
            }
        }
        if (__any_sync(0xFFFFFFFFu, any_tie)) {
            // ties draw from the Rng in position order (every lane replays the
            // same draws so that all copies of the Rng stay equal)
            if (a.trace && lane == 0) atomicAdd(&a.trace[SEQ_T_TIES], 1ull);
#pragma unroll
            for (int i = 0; i < SCAP / 32; ++i) {
                const uint32_t p = lane + 32 * i;
                if (p < ln) S.code[p] = code[i];
            }
            __syncwarp();
            for (uint32_t p = 0; p < ln; ++p)
                if (S.code[p] == 2) {
                    uint8_t v = (rng.next_u64() & 1ull) == 0 ? 1 : 0;
                    __syncwarp();
                    if (lane == 0) S.code[p] = v;
                    __syncwarp();
                }
#pragma unroll
            for (int i = 0; i < SCAP / 32; ++i) {
                const uint32_t p = lane + 32 * i;
                if (p < ln) code[i] = S.code[p];
            }
            la1 = splitmix(rng.s);  // the tie draws moved the Rng on
            la2 = splitmix(la1);
        }
        phase(SEQ_T_W_MARGIN);
        // groups of 32 positions past the node's size are skipped by the whole
        // warp; the ids and slots this lane moves are read ahead of the tables
        unsigned mask[SCAP / 32];
        uint32_t mid[SCAP / 32], msl[SCAP / 32];
        uint32_t nL = 0;
#pragma unroll
        for (int i = 0; i < SCAP / 32; ++i) {
            const uint32_t p = lane + 32 * i;
            mask[i] = 0;
            mid[i] = msl[i] = 0;
            if (32u * i < ln) {
                mask[i] = __ballot_sync(0xFFFFFFFFu, p < ln && code[i] == 1);
                nL += __popc(mask[i]);
                if (p < ln) {
                    mid[i] = sid[ls + p];
                    msl[i] = sslot[ls + p];
                }
            }
        }
        uint32_t c = 0;
        uint32_t pre = 0;
#pragma unroll
        for (int i = 0; i < SCAP / 32; ++i) {
            if (32u * i >= ln) break;
            const uint32_t p = lane + 32 * i;
            const uint32_t lp = pre + __popc(mask[i] & lt);
            const bool isL = (mask[i] >> lane) & 1u;
            if (p < ln) {
                if (isL) {
                    if (p >= nL) S.tabB[(nL - lp) - 1] = p;
                } else if (p < nL) {
                    S.tabA[p - lp] = p;
                }
            }
            // c = right points in [0, nL) = nL - (left points in [0, nL))
            if (nL >= 32u * i && nL < 32u * i + 32u)
                c = nL - (pre + __popc(mask[i] & ((1u << (nL - 32u * i)) - 1u)));
            pre += __popc(mask[i]);
        }
        __syncwarp();
        pre = 0;
#pragma unroll
        for (int i = 0; i < SCAP / 32; ++i) {
            if (32u * i >= ln) break;
            const uint32_t p = lane + 32 * i;
            const uint32_t lp = pre + __popc(mask[i] & lt);
            const bool isL = (mask[i] >> lane) & 1u;
            if (p < ln) {
                uint32_t dst;
                if (isL) {
                    dst = p < nL ? p : S.tabA[(nL - lp) - 1];
                } else if (p < nL) {
                    uint32_t rr = p - lp + 1;
                    dst = (rr == 1 ? ln : S.tabB[rr - 2]) - 1;
                } else if (p > nL) {
                    dst = p - 1;
                } else {
                    dst = (c == 0 ? ln : S.tabB[c - 1]) - 1;
                }
                // in place: every lane read its ids and slots before the
                // barrier after the tables
                sid[ls + dst] = mid[i];
                sslot[ls + dst] = msl[i];
            }
            pre += __popc(mask[i]);
        }
        __syncwarp();
        uint32_t split = nL;
        if (nL == 0 || nL == ln) {
            if (a.trace && lane == 0) atomicAdd(&a.trace[SEQ_T_DEGENERATE], 1ull);
            for (uint32_t i = ln - 1; i >= 1; --i) {
                uint32_t j = uint32_t(rng.below(uint64_t(i) + 1));
                if (lane == 0) {
                    uint32_t t1 = sid[ls + i], t2 = sslot[ls + i];
                    sid[ls + i] = sid[ls + j];
                    sslot[ls + i] = sslot[ls + j];
                    sid[ls + j] = t1;
                    sslot[ls + j] = t2;
                }
                __syncwarp();
            }
            split = ln / 2;
            la1 = splitmix(rng.s);  // the random split moved the Rng on
            la2 = splitmix(la1);
        }
        if (lsp + 2 > STK) {
            if (lane == 0) atomicExch(a.err, 1);
            return nodes;
        }
        if (lane == 0) {
            S.lS[lsp] = ls + split;
            S.lN[lsp] = ln - split;
            S.lD[lsp] = uint16_t(ld + 1);
            S.lS[lsp + 1] = ls;
            S.lN[lsp + 1] = split;
            S.lD[lsp + 1] = uint16_t(ld + 1);
        }
        lsp += 2;
        __syncwarp();
        phase(SEQ_T_W_PART);
    }
    return nodes;
}

// One node split in global mode (random_hyperplane, margins with tie draws
// in position order, the two-pointer partition in its closed form,
// random_split when the hyperplane separates nothing) of positions
// [st, st + sz) of `ids`, with the per-tree scratch arrays tmp / side / tabA /
// tabB at the same positions.  Every thread holds the same Rng.  Returns the
// split point.
template <int NT, int D, class SS>
__device__ uint32_t split_node(const ForestArgs& a, SS& S, uint32_t* ids, uint32_t* tmp,
                               uint8_t* side, uint32_t* tabA, uint32_t* tabB, uint32_t st,
                               uint32_t sz, Rng& rng, float* nv, float* xab, bool tb0,
                               long long& tclk) {
    constexpr int PERT = 8;  // positions per thread per partition tile
    const int tid = threadIdx.x, lane = tid & 31;
    const int d = a.d, dp = a.dp;
    unsigned long long* tr = a.trace;
    if (tr && tid == 0) {
        atomicAdd(&tr[SEQ_T_GLOBAL_NODES], 1ull);
        atomicAdd(&tr[SEQ_T_GLOBAL_POINTS], (unsigned long long)sz);
    }
    uint32_t pa, pb;
    draw_pair(rng, sz, pa, pb);
    {
        const uint32_t A = ids[st + pa], B = ids[st + pb];
        for (int j = tid; j < 2 * dp; j += NT)
            xab[j] = j < dp ? a.X[size_t(A) * dp + j] : a.X[size_t(B) * dp + (j - dp)];
    }
    if (tid == 0) {
        S.anytie = 0;
        S.cntL = 0;
        S.sc = 0;
    }
    __syncthreads();
    for (int j = tid; j < dp; j += NT) nv[j] = j < d ? __fsub_rn(xab[j], xab[dp + j]) : 0.0f;
    const float off = hyper_offset_t<D>(xab, xab + dp, d);
    __syncthreads();
    if (tb0) {
        long long t1 = clock64();
        tr[SEQ_T_CYC_DRAW] += t1 - tclk;
        tclk = t1;
    }
    uint32_t cnt = 0;
    bool tie = false;
    {
        // margins: each thread reads its rows directly, U in flight
        constexpr int U = NT >= 512 ? 2 : 4;  // rows in flight per thread
        for (uint32_t p0 = tid; p0 < sz; p0 += U * NT) {
            uint32_t id[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t p = p0 + u * NT;
                id[u] = ids[st + (p < sz ? p : p0)];
            }
            float m[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                m[u] = __fadd_rn(dot_exact_t<D>(nv, a.X + size_t(id[u]) * dp, d), off);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t p = p0 + u * NT;
                if (p < sz) {
                    const uint8_t c = fabsf(m[u]) < 1e-8f ? 2 : (m[u] > 0.0f ? 1 : 0);
                    side[st + p] = c;
                    tie |= c == 2;
                    cnt += c == 1;
                }
            }
        }
    }
    if (tie) S.anytie = 1;
    cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
    if (lane == 0) atomicAdd(&S.cntL, cnt);
    __syncthreads();
    if (tb0) {
        long long t1 = clock64();
        tr[SEQ_T_CYC_MARGIN] += t1 - tclk;
        tclk = t1;
    }
    if (S.anytie) {
        if (tr && tid == 0) atomicAdd(&tr[SEQ_T_TIES], 1ull);
        // every thread replays the tie draws; thread 0 writes the sides
        uint32_t add = 0;
        for (uint32_t p = 0; p < sz; ++p)
            if (side[st + p] == 2) {
                uint8_t v = (rng.next_u64() & 1ull) == 0 ? 1 : 0;
                add += v;
                __syncthreads();
                if (tid == 0) side[st + p] = v;
                __syncthreads();
            }
        if (tid == 0) S.cntL += add;
        __syncthreads();
    }
    const uint32_t nL = S.cntL;
    uint32_t carry = 0;
    for (uint32_t t0 = 0; t0 < sz; t0 += NT * PERT) {
        uint8_t sd[PERT];
        uint32_t c2 = 0;
#pragma unroll
        for (int j = 0; j < PERT; ++j) {
            uint32_t p = t0 + tid * PERT + j;
            sd[j] = p < sz ? side[st + p] : 0;
            c2 += sd[j];
        }
        uint32_t tt;
        uint32_t lp = carry + bscan(c2, S.ws, &tt);
#pragma unroll
        for (int j = 0; j < PERT; ++j) {
            uint32_t p = t0 + tid * PERT + j;
            if (p < sz) {
                if (sd[j]) {
                    if (p >= nL) tabB[st + (nL - lp) - 1] = p;
                } else if (p < nL) {
                    tabA[st + (p - lp)] = p;
                }
                if (p == nL) S.sc = nL - lp;
                lp += sd[j];
            }
        }
        carry += tt;
    }
    __syncthreads();
    const uint32_t c = S.sc;
    carry = 0;
    for (uint32_t t0 = 0; t0 < sz; t0 += NT * PERT) {
        uint8_t sd[PERT];
        uint32_t c2 = 0;
#pragma unroll
        for (int j = 0; j < PERT; ++j) {
            uint32_t p = t0 + tid * PERT + j;
            sd[j] = p < sz ? side[st + p] : 0;
            c2 += sd[j];
        }
        uint32_t tt;
        uint32_t lp = carry + bscan(c2, S.ws, &tt);
#pragma unroll
        for (int j = 0; j < PERT; ++j) {
            uint32_t p = t0 + tid * PERT + j;
            if (p < sz) {
                uint32_t dst;
                if (sd[j]) {
                    dst = p < nL ? p : tabA[st + (nL - lp) - 1];
                } else if (p < nL) {
                    uint32_t rr = p - lp + 1;
                    dst = (rr == 1 ? sz : tabB[st + rr - 2]) - 1;
                } else if (p > nL) {
                    dst = p - 1;
                } else {
                    dst = (c == 0 ? sz : tabB[st + c - 1]) - 1;
                }
                tmp[st + dst] = ids[st + p];
                lp += sd[j];
            }
        }
        carry += tt;
    }
    __syncthreads();
    for (uint32_t p = tid; p < sz; p += NT) ids[st + p] = tmp[st + p];
    __syncthreads();
    uint32_t split = nL;
    if (nL == 0 || nL == sz) {
        if (tr && tid == 0) atomicAdd(&tr[SEQ_T_DEGENERATE], 1ull);
        for (uint32_t i = sz - 1; i >= 1; --i) {
            uint32_t j = uint32_t(rng.below(uint64_t(i) + 1));
            if (tid == 0) {
                uint32_t t = ids[st + i];
                ids[st + i] = ids[st + j];
                ids[st + j] = t;
            }
            __syncthreads();
        }
        split = sz / 2;
    }
    if (tb0) {
        long long t1 = clock64();
        tr[SEQ_T_CYC_PART] += t1 - tclk;
        tclk = t1;
    }
    return split;
}

// One split of a staged node of m <= NT points (positions [0, m) of
// sid/sslot, rows in shared memory), one point per thread: the same draws,
// margins, tie draws, closed-form partition and random split as the
// global-mode split.  Returns the split point.
template <int NT, int D, class SS>
__device__ uint32_t cta_split(const ForestArgs& a, SS& S, uint32_t* sid, uint32_t* sslot,
                              uint32_t m, Rng& rng, float* rows, float* nv, bool tb0) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int d = a.d, dp = a.dp;
    const uint32_t p = uint32_t(tid);
    unsigned long long* tr = a.trace;
    long long tc = tb0 ? clock64() : 0;
    auto phase = [&](int slot) {
        if (tb0) {
            const long long t1 = clock64();
            tr[slot] += t1 - tc;
            tc = t1;
        }
    };
    uint32_t pa, pb;
    draw_pair(rng, m, pa, pb);
    phase(SEQ_T_M_DRAW);
    const float* xa = rows + size_t(sslot[pa]) * dp;
    const float* xb = rows + size_t(sslot[pb]) * dp;
    for (int j = tid; j < dp; j += NT) nv[j] = j < d ? __fsub_rn(xa[j], xb[j]) : 0.0f;
    __syncthreads();
    // the offset's sequential sum in warp 0 alone (beside its dot products)
    float dt = 0.0f;
    if (p < m) dt = dot_exact_t<D>(nv, rows + size_t(sslot[p]) * dp, d);
    if (w == 0) {
        const float o = hyper_offset_t<D>(xa, xb, d);
        if (lane == 0) S.off = o;
    }
    __syncthreads();
    uint8_t c = 0;
    if (p < m) {
        const float mg = __fadd_rn(dt, S.off);
        c = fabsf(mg) < 1e-8f ? 2 : (mg > 0.0f ? 1 : 0);
        S.code[p] = c;
    }
    if (__syncthreads_or(c == 2)) {
        // ties draw from the Rng in position order (every thread replays the
        // same draws; thread 0 writes the sides)
        if (a.trace && tid == 0) atomicAdd(&a.trace[SEQ_T_TIES], 1ull);
        for (uint32_t q = 0; q < m; ++q)
            if (S.code[q] == 2) {
                const uint8_t v = (rng.next_u64() & 1ull) == 0 ? 1 : 0;
                __syncthreads();
                if (tid == 0) S.code[q] = v;
                __syncthreads();
            }
        c = p < m ? S.code[p] : 0;
    }
    phase(SEQ_T_M_MARGIN);
    // left points before each position: warp ballots, then a scan of the
    // warp counts
    const bool isL = p < m && c == 1;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, isL);
    if (lane == 0) S.ws[w] = __popc(bal);
    __syncthreads();
    if (w == 0) {
        uint32_t v = lane < NT / 32 ? S.ws[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
            if (lane >= o) v += y;
        }
        if (lane < NT / 32) S.ws[lane] = v;  // inclusive
    }
    __syncthreads();
    const uint32_t nL = S.ws[NT / 32 - 1];
    const uint32_t lp = (w > 0 ? S.ws[w - 1] : 0u) + __popc(bal & ((1u << lane) - 1u));
    if (p < m) {
        if (isL) {
            if (p >= nL) S.tabB[(nL - lp) - 1] = p;
        } else if (p < nL) {
            S.tabA[p - lp] = p;
        }
        if (p == nL) S.sc = nL - lp;  // right points in [0, nL)
    }
    __syncthreads();
    if (p < m) {
        uint32_t dst;
        if (isL) {
            dst = p < nL ? p : S.tabA[(nL - lp) - 1];
        } else if (p < nL) {
            const uint32_t rr = p - lp + 1;
            dst = (rr == 1 ? m : S.tabB[rr - 2]) - 1;
        } else if (p > nL) {
            dst = p - 1;
        } else {
            const uint32_t cr = S.sc;
            dst = (cr == 0 ? m : S.tabB[cr - 1]) - 1;
        }
        S.sid2[dst] = sid[p];
        S.sslot2[dst] = sslot[p];
    }
    __syncthreads();
    if (p < m) {
        sid[p] = S.sid2[p];
        sslot[p] = S.sslot2[p];
    }
    __syncthreads();
    uint32_t split = nL;
    if (nL == 0 || nL == m) {
        if (a.trace && tid == 0) atomicAdd(&a.trace[SEQ_T_DEGENERATE], 1ull);
        for (uint32_t i = m - 1; i >= 1; --i) {
            const uint32_t j = uint32_t(rng.below(uint64_t(i) + 1));
            if (tid == 0) {
                const uint32_t t1 = sid[i], t2 = sslot[i];
                sid[i] = sid[j];
                sslot[i] = sslot[j];
                sid[j] = t1;
                sslot[j] = t2;
            }
            __syncthreads();
        }
        split = m / 2;
    }
    phase(SEQ_T_M_PART);
    return split;
}

// A staged subtree of at most MCAP points (NT = 512): ids[0, sz) and their
// rows are staged once; its nodes of more than SCAP points are split by the
// whole CTA (cta_split), the smaller ones finished by warp 0; the ids come
// back in tree order.  `gpos` is its first position in the tree.
template <int NT, int D, class SS>
__device__ void mid_subtree(const ForestArgs& a, SS& S, uint32_t* ids, uint32_t gpos,
                            uint32_t sz, uint32_t dep, Rng& rng, float* rows, float* nv,
                            uint8_t* leaf, bool tb0) {
    const int tid = threadIdx.x;
    const int dp = a.dp, q4 = dp / 4;
    for (uint32_t p = tid; p < sz; p += NT) {
        S.sid[p] = ids[p];
        S.sslot[p] = p;
    }
    __syncthreads();
    for (uint32_t t = tid; t < sz * q4; t += NT) {
        const uint32_t r = t / q4, c4 = t - r * q4;
        cp_async16(rows + size_t(r) * dp + 4 * c4, a.X + size_t(S.sid[r]) * dp + 4 * c4);
    }
    cp_async_wait_all();
    const long long cst = tb0 ? clock64() : 0;
    if (tid == 0) {
        S.mS[0] = 0;
        S.mN[0] = sz;
        S.mD[0] = uint16_t(dep);
    }
    int msp = 1;  // every thread tracks the same stack depth
    __syncthreads();
    if (tb0) a.trace[SEQ_T_M_STAGE] += clock64() - cst;
    while (msp > 0) {
        const uint32_t ls = S.mS[msp - 1], ln = S.mN[msp - 1], ld = S.mD[msp - 1];
        __syncthreads();  // the top is read before it is overwritten
        msp -= 1;
        if (ln <= a.leaf_size || ld > 100) {
            if (tid == 0) leaf[gpos + ls] = 1;
            continue;
        }
        if (ln <= uint32_t(SCAP)) {
            if (tid < 32) {
                const long long c0 = tb0 ? clock64() : 0;
                const uint32_t nodes = warp_subtree<D>(a, S, S.sid + ls, S.sslot + ls, rows, nv,
                                                       gpos + ls, ln, ld, rng, leaf, tb0);
                if (tid == 0) S.rng = rng.s;
                if (tb0) {
                    a.trace[SEQ_T_R0_CYC_WARP] += clock64() - c0;
                    a.trace[SEQ_T_R0_SNODES] += nodes;
                    a.trace[SEQ_T_R0_STAGED] += 1;
                }
            }
            __syncthreads();
            rng.s = S.rng;  // the other warps adopt warp 0's Rng state
            continue;
        }
        if (a.trace && tid == 0) {
            atomicAdd(&a.trace[SEQ_T_MID_NODES], 1ull);
            if (tb0) a.trace[SEQ_T_R0_MNODES] += 1;
        }
        const uint32_t split =
            cta_split<NT, D>(a, S, S.sid + ls, S.sslot + ls, ln, rng, rows, nv, tb0);
        if (msp + 2 > STK) {
            if (tid == 0) atomicExch(a.err, 1);
            break;
        }
        if (tid == 0) {
            S.mS[msp] = ls + split;  // right, popped after the whole left subtree
            S.mN[msp] = ln - split;
            S.mD[msp] = uint16_t(ld + 1);
            S.mS[msp + 1] = ls;
            S.mN[msp + 1] = split;
            S.mD[msp + 1] = uint16_t(ld + 1);
        }
        msp += 2;
        __syncthreads();
    }
    for (uint32_t p = tid; p < sz; p += NT) ids[p] = S.sid[p];
    __syncthreads();
    if (a.trace && tid == 0) atomicAdd(&a.trace[SEQ_T_MID_TREES], 1ull);
}

// A staged subtree of at most smax points: ids[0, sz) with their rows in
// shared memory, finished by warp 0; the ids come back in tree order.  `gpos`
// is its first position in the tree (for the leaf flags).
template <int NT, int D, class SS>
__device__ void staged_subtree(const ForestArgs& a, SS& S, uint32_t* ids, uint32_t gpos,
                               uint32_t sz, uint32_t dep, Rng& rng, float* rows, float* nv,
                               uint8_t* leaf, bool tb0) {
    const int tid = threadIdx.x;
    const int dp = a.dp;
    for (uint32_t p = tid; p < sz; p += NT) {
        S.sid[p] = ids[p];
        S.sslot[p] = p;
    }
    __syncthreads();
    const int q4 = dp / 4;
    for (uint32_t t = tid; t < sz * q4; t += NT) {
        uint32_t r = t / q4, j = t - r * q4;
        reinterpret_cast<float4*>(rows)[t] =
            reinterpret_cast<const float4*>(a.X + size_t(S.sid[r]) * dp)[j];
    }
    __syncthreads();
    if (tid < 32) {
        const long long c0 = tb0 ? clock64() : 0;
        const uint32_t nodes =
            warp_subtree<D>(a, S, S.sid, S.sslot, rows, nv, gpos, sz, dep, rng, leaf, tb0);
        if (tid == 0) S.rng = rng.s;
        if (tb0) {
            a.trace[SEQ_T_R0_CYC_WARP] += clock64() - c0;
            a.trace[SEQ_T_R0_SNODES] += nodes;
            a.trace[SEQ_T_R0_STAGED] += 1;
        }
    }
    __syncthreads();
    rng.s = S.rng;  // the other warps adopt warp 0's Rng state
    for (uint32_t p = tid; p < sz; p += NT) ids[p] = S.sid[p];
    __syncthreads();
    if (a.trace && tid == 0) atomicAdd(&a.trace[SEQ_T_STAGED_TREES], 1ull);
}

template <int NT, int D>
__global__ void __launch_bounds__(NT) k_seqtree(ForestArgs a, const SRoot* roots, int smax,
                                                int trows) {
    extern __shared__ __align__(16) float dyn[];
    __shared__ SeqShared<NT == MCAP ? MCAP : SCAP> S;
    float* nv = dyn;                 // dp
    float* xab = dyn + a.dp;         // 2 * dp: the two hyperplane rows
    float* rows = dyn + 3 * a.dp;    // max(smax, trows) * dp: staged subtrees
    const int tid = threadIdx.x;
    const SRoot rt = roots[blockIdx.x];
    const size_t tb = size_t(rt.tree) * a.n;
    uint32_t* ids = a.ids + tb;
    uint32_t* tmp = a.tmp + tb;
    uint8_t* side = a.side + tb;
    uint32_t* tabA = a.tabA + tb;
    uint32_t* tabB = a.tabB + tb;
    uint8_t* leaf = a.leafflag + tb;
    Rng rng{rt.seed};  // every thread holds the same state
    unsigned long long* tr = a.trace;
    const bool tb0 = tr && rt.size == tr[SEQ_T_ROOT0] && tid == 0;
    long long t_start = clock64(), tclk = 0;
    const unsigned long long g_start = a.tl ? globaltimer_ns() : 0ull;
    if (tid == 0) {
        S.sp = 1;
        S.stS[0] = rt.start;
        S.stN[0] = rt.size;
        S.stD[0] = uint16_t(rt.depth);
    }
    __syncthreads();
    while (S.sp > 0) {
        const uint32_t st = S.stS[S.sp - 1], sz = S.stN[S.sp - 1], dep = S.stD[S.sp - 1];
        __syncthreads();
        if (tid == 0) S.sp -= 1;
        if (sz <= a.leaf_size || dep > 100) {
            if (tid == 0) leaf[st] = 1;
            __syncthreads();
            continue;
        }
        if constexpr (NT == MCAP) {
            if (trows >= MCAP && sz > uint32_t(smax) && sz <= uint32_t(MCAP)) {
                if (tb0) tclk = clock64();
                mid_subtree<NT, D>(a, S, ids + st, st, sz, dep, rng, rows, nv, leaf, tb0);
                if (tb0) tr[SEQ_T_CYC_STAGED] += clock64() - tclk;
                continue;
            }
        }
        if (sz <= uint32_t(smax)) {
            if (tb0) tclk = clock64();
            staged_subtree<NT, D>(a, S, ids + st, st, sz, dep, rng, rows, nv, leaf, tb0);
            if (tb0) tr[SEQ_T_CYC_STAGED] += clock64() - tclk;
            continue;
        }
        // ── global mode ──
        if (tb0) {
            tclk = clock64();
            tr[SEQ_T_R0_GNODES] += 1;
        }
        const uint32_t split =
            split_node<NT, D>(a, S, ids, tmp, side, tabA, tabB, st, sz, rng, nv, xab, tb0, tclk);
        if (tid == 0) {
            if (S.sp + 2 > STK) {
                atomicExch(a.err, 1);
                S.sp = 0;
            } else {
                S.stS[S.sp] = st + split;  // right, popped after the whole left subtree
                S.stN[S.sp] = sz - split;
                S.stD[S.sp] = uint16_t(dep + 1);
                S.stS[S.sp + 1] = st;
                S.stN[S.sp + 1] = split;
                S.stD[S.sp + 1] = uint16_t(dep + 1);
                S.sp += 2;
            }
        }
        __syncthreads();
    }
    if (tb0) tr[SEQ_T_CYC_TOTAL] = clock64() - t_start;
    if (a.tl && tid == 0) {
        unsigned long long* tl = a.tl;
        const unsigned long long g_end = globaltimer_ns();
        if (NT == MCAP) {
            if (blockIdx.x < unsigned(SEQ_T_BIG_N)) {
                tl[SEQ_T_BIG + 2 * blockIdx.x] = g_start;
                tl[SEQ_T_BIG + 2 * blockIdx.x + 1] = g_end;
            }
        } else {
            atomicMax(&tl[SEQ_T_SMALL_T0], ~g_start);  // the earliest start, complemented
            atomicMax(&tl[SEQ_T_SMALL_T1], g_end);
        }
    }
}

// Compact leaf starts of one tree: flags (u8) -> u32 -> exclusive scan -> positions.
__global__ void k_flags_u32(const uint8_t* f, uint32_t n, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = f[i];
}
__global__ void k_leaf_scatter(const uint8_t* f, const uint32_t* pre, uint32_t n,
                               uint32_t* leaf_start) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && f[i]) leaf_start[pre[i]] = i;
}

// Leaf all-pairs of one tree (nndescent.rs:785-815).  The member at a
// position receives every other member of its leaf in leaf order, which is
// the order the reference's (i<j, p-then-q) generation addresses it.
//
// A CTA takes lpb consecutive leaves (as many as fit LCAP positions at the
// tree's leaf size, at most LPB): it stages their ids, rows and their
// members' heap rows in shared memory once (the heap rows column-major, one
// column per position, so that the pushes of a warp hit distinct banks),
// computes each pair's distance once into a per-position table, and then each
// thread replays its own member's pushes on the staged row; the changed rows
// go back.  The heap rows move between global and shared memory in position x
// slot order (consecutive threads on one row's slots: coalesced), the staged
// columns LCAP + 1 apart so that those accesses spread over the banks.  A push whose distance is not below the row's root (its
// current worst) is rejected unchanged (nndescent.rs:176).  Tiles whose span
// exceeds LCAP or whose leaves exceed LMAX members take the direct path.
constexpr int LPB = 8;      // leaves per CTA, at most
constexpr int LCAP = 128;   // staged positions per CTA (= threads)
constexpr int LMAXC = 64;   // largest leaf of the staged path
constexpr int HS = LCAP + 1;  // column stride of the staged heap rows

size_t leaf_pairs_smem(int dp, int lmax, int k) {
    return size_t(LCAP) * dp * 4 + size_t(LCAP) * lmax * 4 + size_t(HS) * k * 9;
}

template <int D>
__global__ void __launch_bounds__(LCAP) k_leaf_pairs(
    const float* __restrict__ X, int d, int dp, const uint32_t* __restrict__ ids,
    const uint32_t* __restrict__ leaf_start, uint32_t nleaves, uint32_t n, int k, uint32_t* hidx,
    float* hdist, uint8_t* hflag, int LMAX, int lpb) {
    extern __shared__ __align__(16) float lsm[];
    __shared__ uint32_t sls[LPB + 1];
    __shared__ int staged;
    float* R = lsm;                               // LCAP * dp
    float* Dt = lsm + size_t(LCAP) * dp;          // LCAP * LMAX (LMAX: 16 or 32)
    uint32_t* hI = reinterpret_cast<uint32_t*>(Dt + size_t(LCAP) * LMAX);  // k x HS
    float* hD = reinterpret_cast<float*>(hI + size_t(k) * HS);             // k x HS
    uint8_t* hF = reinterpret_cast<uint8_t*>(hD + size_t(k) * HS);         // k x HS
    __shared__ uint32_t sid[LCAP];
    __shared__ uint8_t chg[LCAP];  // the staged heap row changed
    __shared__ uint16_t sl0[LCAP], sl1[LCAP];     // leaf bounds of each staged position
    const uint32_t L0 = blockIdx.x * uint32_t(lpb);
    const uint32_t L1 = min(nleaves, L0 + uint32_t(lpb));
    const int tid = threadIdx.x;
    if (tid <= int(L1 - L0)) {
        const uint32_t li = L0 + tid;
        sls[tid] = li < nleaves ? leaf_start[li] : n;
    }
    __syncthreads();
    const uint32_t P0 = sls[0], P1 = sls[L1 - L0];
    const uint32_t span = P1 - P0;
    if (tid == 0) {
        bool ok = span <= uint32_t(LCAP);
        for (uint32_t l = 0; l < L1 - L0; ++l) ok &= sls[l + 1] - sls[l] <= uint32_t(LMAX);
        staged = ok;
    }
    __syncthreads();
    if (!staged) {
        for (uint32_t pos = P0 + tid; pos < P1; pos += LCAP) {
            uint32_t l = 0;
            while (sls[l + 1] <= pos) ++l;
            const uint32_t ls = sls[l], le = sls[l + 1];
            const uint32_t p = ids[pos];
            const float* xp = X + size_t(p) * dp;
            for (uint32_t qp = ls; qp < le; ++qp) {
                if (qp == pos) continue;
                const uint32_t q = ids[qp];
                heap_push(hidx + size_t(p) * k, hdist + size_t(p) * k, hflag + size_t(p) * k, k,
                          q, sq_dist_exact_t<D>(xp, X + size_t(q) * dp, d), 1);
            }
        }
        return;
    }
    const bool own = uint32_t(tid) < span;
    uint32_t p = 0;
    if (own) {
        p = ids[P0 + tid];
        sid[tid] = p;
        uint32_t l = 0;
        while (sls[l + 1] <= P0 + tid) ++l;
        sl0[tid] = uint16_t(sls[l] - P0);
        sl1[tid] = uint16_t(sls[l + 1] - P0);
    }
    __syncthreads();
    // rows and heap rows, all loads in flight together
    const int q4 = dp / 4;
    for (uint32_t t = tid; t < span * q4; t += LCAP) {
        const uint32_t r = t / q4, j = t - r * q4;
        reinterpret_cast<float4*>(R)[t] = reinterpret_cast<const float4*>(X + size_t(sid[r]) * dp)[j];
    }
    for (uint32_t t = tid; t < span * uint32_t(k); t += LCAP) {
        const uint32_t r = t / uint32_t(k), sl = t - r * uint32_t(k);
        const size_t g = size_t(sid[r]) * k + sl;
        hI[sl * HS + r] = hidx[g];
        hD[sl * HS + r] = hdist[g];
        hF[sl * HS + r] = hflag[g];
    }
    __syncthreads();
    if (own) {  // each pair once: this position with its later mates
        const uint32_t l0 = sl0[tid], l1 = sl1[tid];
        for (uint32_t j = tid + 1; j < l1; ++j) {
            const float dd = sq_dist_exact_t<D>(R + size_t(tid) * dp, R + size_t(j) * dp, d);
            Dt[size_t(tid) * LMAX + (j - l0)] = dd;
            Dt[size_t(j) * LMAX + (tid - l0)] = dd;
        }
    }
    __syncthreads();
    if (own) {
        const uint32_t l0 = sl0[tid], l1 = sl1[tid];
        uint32_t* ri = hI + tid;
        float* rd = hD + tid;
        uint8_t* rf = hF + tid;
        bool changed = false;
        for (uint32_t j = l0; j < l1; ++j) {
            if (j == uint32_t(tid)) continue;
            const float dd = Dt[size_t(tid) * LMAX + (j - l0)];
            if (dd >= rd[0]) continue;  // heap_push would reject it unchanged
            changed |= heap_push_strided(ri, rd, rf, k, HS, sid[j], dd, 1);
        }
        chg[tid] = changed ? 1 : 0;
    }
    __syncthreads();
    for (uint32_t t = tid; t < span * uint32_t(k); t += LCAP) {
        const uint32_t r = t / uint32_t(k), sl = t - r * uint32_t(k);
        if (!chg[r]) continue;
        const size_t g = size_t(sid[r]) * k + sl;
        hidx[g] = hI[sl * HS + r];
        hdist[g] = hD[sl * HS + r];
        hflag[g] = hF[sl * HS + r];
    }
}

__global__ void k_random_fill(const float* __restrict__ X, int d, int dp, uint32_t n, int k,
                              uint64_t seed, uint32_t* hidx, float* hdist, uint8_t* hflag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t* ri = hidx + size_t(i) * k;
    float* rd = hdist + size_t(i) * k;
    uint8_t* rf = hflag + size_t(i) * k;
    for (uint64_t attempt = 0; attempt < 64; ++attempt) {
        bool empty = false;
        for (int s = 0; s < k; ++s) empty |= ri[s] == PQ_EMPTY;
        if (!empty) break;
        uint64_t j = hash_index(seed, uint64_t(i), attempt, n);
        if (j == i) j = (j + 1) % n;
        float dd = sq_dist_exact(X + size_t(i) * dp, X + size_t(j) * dp, d);
        heap_push(ri, rd, rf, k, uint32_t(j), dd, 1);
    }
}

}  // namespace

void launch_hyperplanes(const ForestArgs& a, PNode* nodes, uint32_t nn, float* normals,
                        cudaStream_t st) {
    k_hyper<<<nn, 64, 0, st>>>(a, nodes, normals); count_launch();
}
void launch_sides(const ForestArgs& a, const PNode* nodes, const uint32_t* chunk_node,
                  uint32_t nchunks, const float* normals, uint32_t* chunkL, cudaStream_t st) {
    k_sides<<<nchunks, FT, size_t(a.dp) * sizeof(float), st>>>(a, nodes, chunk_node, normals,
                                                               chunkL); count_launch();
}
void launch_node_scan(PNode* nodes, uint32_t nn, uint32_t* chunkL, cudaStream_t st) {
    k_node_scan<<<(nn + 3) / 4, 128, 0, st>>>(nodes, nn, chunkL); count_launch();
}
void launch_partition(const ForestArgs& a, PNode* nodes, const uint32_t* chunk_node,
                      uint32_t nchunks, const uint32_t* chunkPre, cudaStream_t st) {
    k_part_tables<<<nchunks, FT, 0, st>>>(a, nodes, chunk_node, chunkPre); count_launch();
    k_part_scatter<<<nchunks, FT, 0, st>>>(a, nodes, chunk_node, chunkPre); count_launch();
    k_part_copy<<<nchunks, FT, 0, st>>>(a, nodes, chunk_node); count_launch();
}
void launch_degenerate(const ForestArgs& a, PNode* nodes, uint32_t nn, cudaStream_t st) {
    k_degenerate<<<(nn + 63) / 64, 64, 0, st>>>(a, nodes, nn); count_launch();
}
template <int NT, int D>
static void seqtree_launch(const ForestArgs& a, const SRoot* roots, uint32_t nr, int smax,
                           cudaStream_t st) {
    if (nr == 0) return;
    // shared rows: the two hyperplane rows, the normal, and max(smax, tr) rows
    // for staged subtrees (tr = NT rows, the CTA-staged subtrees of 512-thread
    // CTAs, when they fit in 200 KB)
    const size_t row = size_t(a.dp) * sizeof(float);
    const size_t fit = (200 * 1024) / row;
    int tr = int(std::min<size_t>(NT, fit > 3 ? fit - 3 : 0));
    if (tr < 32) tr = 0;
    const size_t dyn = row * (3 + size_t(std::max(smax, tr)));
    // (with the static staged arrays the total passes 48 KB well before dyn does)
    cudaFuncSetAttribute(k_seqtree<NT, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn));
    k_seqtree<NT, D><<<nr, NT, dyn, st>>>(a, roots, smax, tr); count_launch();
}

void launch_seqtrees(const ForestArgs& a, const SRoot* roots, uint32_t n_big, uint32_t nr,
                     cudaStream_t st, cudaStream_t st_big) {
    if (nr == 0) return;
    // staged capacity: as many rows as fit beside the hyperplane rows in ~28 KB
    size_t row = size_t(a.dp) * sizeof(float);
    int smax = int(std::min<size_t>(SCAP, (28 * 1024) / row));
    if (smax < 2) smax = 0;
    // roots[0, n_big) are the largest subtrees: 512 threads each, own stream
    // (64-thread CTAs for the rest, six per SM instead of four, took 1065
    // instead of 926 ms per 4M build: their global-mode nodes slow down more
    // than the extra CTAs gain)
    if (a.d == 50) {
        seqtree_launch<512, 50>(a, roots, n_big, smax, st_big);
        seqtree_launch<128, 50>(a, roots + n_big, nr - n_big, smax, st);
    } else {
        seqtree_launch<512, 0>(a, roots, n_big, smax, st_big);
        seqtree_launch<128, 0>(a, roots + n_big, nr - n_big, smax, st);
    }
}
void launch_leaf_compact(const uint8_t* leafflag_t, uint32_t n, uint32_t* leaf_start,
                         uint32_t* scan_buf, void* scan_temp, uint64_t* count_dev,
                         cudaStream_t st) {
    k_flags_u32<<<(n + 255) / 256, 256, 0, st>>>(leafflag_t, n, scan_buf); count_launch();
    scan_exclusive_u32(scan_buf, scan_buf, n, scan_temp, count_dev, st);
    k_leaf_scatter<<<(n + 255) / 256, 256, 0, st>>>(leafflag_t, scan_buf, n, leaf_start); count_launch();
}
void launch_leaf_pairs(const float* X, int d, int dp, const uint32_t* ids_t,
                       const uint32_t* leaf_start, uint32_t nleaves, uint32_t n, int k,
                       uint32_t leaf_cap, uint32_t* hidx, float* hdist, uint8_t* hflag,
                       cudaStream_t st) {
    if (nleaves == 0) return;
    // leaves never exceed leaf_size (or come from depth > 100); the mate table
    // is as wide as the leaf size allows (16, 32 or 64), and a CTA takes as
    // many leaves as fit its LCAP positions at that size
    int lmax = leaf_cap <= 16 ? 16 : leaf_cap <= 32 ? 32 : LMAXC;
    const int lpb = int(std::max<uint32_t>(1, std::min<uint32_t>(LPB, LCAP / std::max(leaf_cap, 1u))));
    size_t sm = leaf_pairs_smem(dp, lmax, k);
    if (sm > 200 * 1024 || leaf_cap > uint32_t(LMAXC)) {
        // wide rows, large k or large leaves: every tile takes the direct path
        lmax = 0;
        sm = 0;
    }
    const unsigned grid = (nleaves + lpb - 1) / lpb;
    if (d == 50) {
        if (sm > 40 * 1024)
            cudaFuncSetAttribute(k_leaf_pairs<50>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sm));
        k_leaf_pairs<50><<<grid, LCAP, sm, st>>>(X, d, dp, ids_t, leaf_start, nleaves, n, k,
                                                 hidx, hdist, hflag, lmax, lpb); count_launch();
    } else {
        if (sm > 40 * 1024)
            cudaFuncSetAttribute(k_leaf_pairs<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sm));
        k_leaf_pairs<0><<<grid, LCAP, sm, st>>>(X, d, dp, ids_t, leaf_start, nleaves, n, k,
                                                hidx, hdist, hflag, lmax, lpb); count_launch();
    }
}
void launch_random_fill(const float* X, int d, int dp, uint32_t n, int k, uint64_t seed,
                        uint32_t* hidx, float* hdist, uint8_t* hflag, cudaStream_t st) {
    k_random_fill<<<(n + 127) / 128, 128, 0, st>>>(X, d, dp, n, k, seed, hidx, hdist, hflag); count_launch();
}

}  // namespace pq
