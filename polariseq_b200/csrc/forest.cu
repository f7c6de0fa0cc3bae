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
#include "common.cuh"
#include "kernels.cuh"
#include "primitives.cuh"

namespace pq {
namespace {

constexpr int FT = 256;             // threads per forest CTA
constexpr int PER = FOREST_CHUNK / FT;  // positions per thread in a chunk
constexpr int STK = 128;            // DFS stack depth (depth > 100 is a leaf)

// Exclusive block scan of one u32 per thread (FT threads).
__device__ __forceinline__ uint32_t bscan(uint32_t v, uint32_t* ws, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (FT / 32) ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < FT / 32) ws[lane] = s;
    }
    __syncthreads();
    uint32_t r = (w > 0 ? ws[w - 1] : 0) + x - v;
    *total = ws[FT / 32 - 1];
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
__global__ void __launch_bounds__(FT) k_seqtree(ForestArgs a, const SRoot* roots) {
    extern __shared__ __align__(16) float nv[];
    __shared__ uint32_t stS[STK], stN[STK];
    __shared__ uint16_t stD[STK];
    __shared__ int sp;
    __shared__ uint64_t rng;
    __shared__ uint32_t sA, sB, snL, sc;
    __shared__ float soff;
    __shared__ int anytie;
    __shared__ uint32_t ws[32];
    const SRoot rt = roots[blockIdx.x];
    const size_t tb = size_t(rt.tree) * a.n;
    uint32_t* ids = a.ids + tb;
    uint32_t* tmp = a.tmp + tb;
    uint8_t* side = a.side + tb;
    uint32_t* tabA = a.tabA + tb;
    uint32_t* tabB = a.tabB + tb;
    if (threadIdx.x == 0) {
        sp = 1;
        stS[0] = rt.start;
        stN[0] = rt.size;
        stD[0] = uint16_t(rt.depth);
        rng = rt.seed;
    }
    __syncthreads();
    for (;;) {
        if (sp == 0) break;
        const uint32_t st = stS[sp - 1], sz = stN[sp - 1], dep = stD[sp - 1];
        __syncthreads();
        if (threadIdx.x == 0) sp -= 1;
        if (sz <= a.leaf_size || dep > 100) {
            if (threadIdx.x == 0) a.leafflag[tb + st] = 1;
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) {
            Rng r{rng};
            uint32_t A = ids[st + r.below(sz)];
            uint32_t B = ids[st + r.below(sz)];
            int tries = 0;
            while (B == A && tries < 8) {
                B = ids[st + r.below(sz)];
                ++tries;
            }
            rng = r.s;
            sA = A;
            sB = B;
            anytie = 0;
        }
        __syncthreads();
        {
            const float* xa = a.X + size_t(sA) * a.dp;
            const float* xb = a.X + size_t(sB) * a.dp;
            for (int j = threadIdx.x; j < a.dp; j += FT)
                nv[j] = j < a.d ? __fsub_rn(xa[j], xb[j]) : 0.0f;
            if (threadIdx.x == 0) {
                float s = -0.0f;
                for (int j = 0; j < a.d; ++j) {
                    float nvj = __fsub_rn(xa[j], xb[j]);
                    s = __fadd_rn(s, __fmul_rn(__fmul_rn(nvj, 0.5f), __fadd_rn(xa[j], xb[j])));
                }
                soff = -s;
            }
        }
        __syncthreads();
        const float off = soff;
        for (uint32_t p = threadIdx.x; p < sz; p += FT) {
            uint32_t id = ids[st + p];
            float m = __fadd_rn(dot_exact(nv, a.X + size_t(id) * a.dp, a.d), off);
            uint8_t code;
            if (fabsf(m) < 1e-8f) {
                code = 2;
                anytie = 1;
            } else {
                code = m > 0.0f ? 1 : 0;
            }
            side[st + p] = code;
        }
        __syncthreads();
        if (anytie) {  // ties draw from the Rng in position order
            if (threadIdx.x == 0) {
                Rng r{rng};
                for (uint32_t p = 0; p < sz; ++p)
                    if (side[st + p] == 2) side[st + p] = (r.next_u64() & 1ull) == 0 ? 1 : 0;
                rng = r.s;
            }
            __syncthreads();
        }
        // nL
        uint32_t cnt = 0;
        for (uint32_t p = threadIdx.x; p < sz; p += FT) cnt += side[st + p];
        uint32_t tot;
        bscan(cnt, ws, &tot);
        if (threadIdx.x == 0) {
            snL = tot;
            sc = 0;
        }
        __syncthreads();
        const uint32_t nL = snL;
        // pass 1: tables and c; positions in tiles of FT*PER, PER consecutive per thread
        uint32_t carry = 0;
        for (uint32_t t0 = 0; t0 < sz; t0 += FT * PER) {
            uint8_t s[PER];
            uint32_t c2 = 0;
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                uint32_t p = t0 + threadIdx.x * PER + j;
                s[j] = p < sz ? side[st + p] : 0;
                c2 += s[j];
            }
            uint32_t tt;
            uint32_t lp = carry + bscan(c2, ws, &tt);
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                uint32_t p = t0 + threadIdx.x * PER + j;
                if (p < sz) {
                    if (s[j]) {
                        if (p >= nL) tabB[st + (nL - lp) - 1] = p;
                    } else if (p < nL) {
                        tabA[st + (p - lp)] = p;
                    }
                    if (p == nL) sc = nL - lp;
                    lp += s[j];
                }
            }
            carry += tt;
        }
        __syncthreads();
        const uint32_t c = sc;
        carry = 0;
        for (uint32_t t0 = 0; t0 < sz; t0 += FT * PER) {
            uint8_t s[PER];
            uint32_t c2 = 0;
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                uint32_t p = t0 + threadIdx.x * PER + j;
                s[j] = p < sz ? side[st + p] : 0;
                c2 += s[j];
            }
            uint32_t tt;
            uint32_t lp = carry + bscan(c2, ws, &tt);
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                uint32_t p = t0 + threadIdx.x * PER + j;
                if (p < sz) {
                    uint32_t dst;
                    if (s[j]) {
                        dst = p < nL ? p : tabA[st + (nL - lp) - 1];
                    } else if (p < nL) {
                        uint32_t r = p - lp + 1;
                        dst = (r == 1 ? sz : tabB[st + r - 2]) - 1;
                    } else if (p > nL) {
                        dst = p - 1;
                    } else {
                        dst = (c == 0 ? sz : tabB[st + c - 1]) - 1;
                    }
                    tmp[st + dst] = ids[st + p];
                    lp += s[j];
                }
            }
            carry += tt;
        }
        __syncthreads();
        for (uint32_t p = threadIdx.x; p < sz; p += FT) ids[st + p] = tmp[st + p];
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t split = nL;
            if (nL == 0 || nL == sz) {
                Rng r{rng};
                for (uint32_t i = sz - 1; i >= 1; --i) {
                    uint32_t j = uint32_t(r.below(uint64_t(i) + 1));
                    uint32_t t = ids[st + i];
                    ids[st + i] = ids[st + j];
                    ids[st + j] = t;
                }
                rng = r.s;
                split = sz / 2;
            }
            if (sp + 2 > STK) {
                atomicExch(a.err, 1);
                sp = 0;
            } else {
                stS[sp] = st + split;  // right, popped after the whole left subtree
                stN[sp] = sz - split;
                stD[sp] = uint16_t(dep + 1);
                stS[sp + 1] = st;
                stN[sp + 1] = split;
                stD[sp + 1] = uint16_t(dep + 1);
                sp += 2;
            }
        }
        __syncthreads();
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

// Leaf all-pairs: a warp per leaf; each member receives every other member
// in leaf order, which is the order the reference's (i<j, p-then-q)
// generation addresses it (nndescent.rs:793-810).
__global__ void __launch_bounds__(256) k_leaf_pairs(const float* __restrict__ X, int d, int dp,
                                                    const uint32_t* __restrict__ ids,
                                                    const uint32_t* __restrict__ leaf_start,
                                                    uint32_t nleaves, uint32_t n, int k,
                                                    uint32_t* hidx, float* hdist,
                                                    uint8_t* hflag) {
    uint32_t li = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (li >= nleaves) return;
    const int lane = threadIdx.x & 31;
    uint32_t ls = leaf_start[li];
    uint32_t le = li + 1 < nleaves ? leaf_start[li + 1] : n;
    uint32_t L = le - ls;
    for (uint32_t mi = lane; mi < L; mi += 32) {
        uint32_t p = ids[ls + mi];
        const float* xp = X + size_t(p) * dp;
        uint32_t* ri = hidx + size_t(p) * k;
        float* rd = hdist + size_t(p) * k;
        uint8_t* rf = hflag + size_t(p) * k;
        for (uint32_t qi = 0; qi < L; ++qi) {
            if (qi == mi) continue;
            uint32_t q = ids[ls + qi];
            float dd = sq_dist_exact(xp, X + size_t(q) * dp, d);
            heap_push(ri, rd, rf, k, q, dd, 1);
        }
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
void launch_seqtrees(const ForestArgs& a, const SRoot* roots, uint32_t nr, cudaStream_t st) {
    if (nr == 0) return;
    k_seqtree<<<nr, FT, size_t(a.dp) * sizeof(float), st>>>(a, roots); count_launch();
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
                       uint32_t* hidx, float* hdist, uint8_t* hflag, cudaStream_t st) {
    if (nleaves == 0) return;
    k_leaf_pairs<<<(nleaves + 7) / 8, 256, 0, st>>>(X, d, dp, ids_t, leaf_start, nleaves, n, k,
                                                    hidx, hdist, hflag); count_launch();
}
void launch_random_fill(const float* X, int d, int dp, uint32_t n, int k, uint64_t seed,
                        uint32_t* hidx, float* hdist, uint8_t* hflag, cudaStream_t st) {
    k_random_fill<<<(n + 127) / 128, 128, 0, st>>>(X, d, dp, n, k, seed, hidx, hdist, hflag); count_launch();
}

}  // namespace pq
