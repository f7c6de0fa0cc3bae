// Kernel entry points of the plain (bit-exact) NN-Descent, shared between the
// phase drivers.  All device arrays are described where they are declared in
// the host driver (api.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pq {

// A node of the level-parallel top of a tree (rp_tree_parallel,
// nndescent.rs:587-641): rows [start, start+size) of tree `tree`'s id array.
struct PNode {
    uint32_t tree, start, size, depth;
    uint64_t seed;       // the node's seed (tree seed, or splitmix(parent ^ 1|2))
    uint64_t rng_after;  // Rng state after the hyperplane draws (for random_split)
    float offset;
    uint32_t nL;         // out: points on the left side (or size/2 after a random split)
    uint32_t c;          // out: right-side points in the left segment
    uint32_t chunk0;     // first chunk of this node
};

// A subtree finished by sequential depth-first recursion with one Rng
// (rp_tree_sequential, nndescent.rs:474-581).
struct SRoot {
    uint32_t tree, start, size, depth;
    uint64_t seed;
};

struct ForestArgs {
    const float* X;      // n x dp padded rows
    int d, dp;
    uint32_t n;
    uint32_t leaf_size;
    uint32_t* ids;       // T x n permutations
    uint32_t* tmp;       // T x n scratch
    uint8_t* side;       // T x n per-position side (1 = left)
    uint32_t* tabA;      // T x n: positions of right points in the left segment, by rank
    uint32_t* tabB;      // T x n: positions of left points in the right segment, by rank from the top
    uint8_t* leafflag;   // T x n: 1 where a leaf starts
    int* err;            // device error flag
    unsigned long long* trace;  // optional: SEQ_TRACE_N counters (POLARISEQ_TRACE)
    unsigned long long* tl;     // optional: the same buffer, for the CTA timeline stamps only
};

// Trace counters of the depth-first subtree kernel.
enum {
    SEQ_T_GLOBAL_NODES = 0,   // nodes split in global mode
    SEQ_T_GLOBAL_POINTS = 1,  // margins evaluated in global mode
    SEQ_T_STAGED_TREES = 2,   // staged subtrees
    SEQ_T_STAGED_NODES = 3,   // nodes split in staged subtrees
    SEQ_T_TIES = 4,           // nodes with tie draws
    SEQ_T_DEGENERATE = 5,     // random splits
    SEQ_T_CYC_DRAW = 6,       // block 0 cycles: draws + hyperplane rows
    SEQ_T_CYC_MARGIN = 7,     // block 0 cycles: global-mode margins
    SEQ_T_CYC_PART = 8,       // block 0 cycles: global-mode partition
    SEQ_T_CYC_STAGED = 9,     // block 0 cycles: staged subtrees
    SEQ_T_CYC_TOTAL = 10,     // block 0 cycles: whole kernel
    SEQ_T_ROOT0 = 11,         // block 0 root size
    SEQ_T_R0_STAGED = 12,     // block 0: staged subtrees
    SEQ_T_R0_SNODES = 13,     // block 0: nodes split in staged subtrees
    SEQ_T_R0_GNODES = 14,     // block 0: nodes split in global mode
    SEQ_T_R0_CYC_WARP = 15,   // block 0 cycles: warp 0's splits of staged subtrees
    SEQ_T_MID_TREES = 16,     // staged subtrees of up to 512 points (512-thread CTAs)
    SEQ_T_MID_NODES = 17,     // their nodes split by the whole CTA
    SEQ_T_R0_MNODES = 18,     // block 0: the same
    SEQ_T_W_LEAF = 20,        // block 0 cycles, warp 0's staged splits: leaf pops
    SEQ_T_W_DRAW = 21,        //   draws
    SEQ_T_W_MARGIN = 22,      //   normal, offset, margins, sides
    SEQ_T_W_PART = 23,        //   partition and pushes
    SEQ_T_M_DRAW = 24,        // block 0 cycles, CTA-staged splits: draws
    SEQ_T_M_MARGIN = 25,      //   normal, offset, margins, sides
    SEQ_T_M_PART = 26,        //   partition
    SEQ_T_M_STAGE = 27,       //   staging ids and rows
    SEQ_T_SMALL_T0 = 28,      // 128-thread CTAs: earliest start (globaltimer ns)
    SEQ_T_SMALL_T1 = 29,      //   latest end
    SEQ_T_BIG = 32,           // 512-thread CTAs: start and end (globaltimer ns) of each of
                              // the first SEQ_T_BIG_N, slots SEQ_T_BIG + 2 * block (+ 1)
    SEQ_T_BIG_N = 148,
    SEQ_TRACE_N = SEQ_T_BIG + 2 * SEQ_T_BIG_N
};

constexpr int FOREST_CHUNK = 2048;

void launch_hyperplanes(const ForestArgs& a, PNode* nodes, uint32_t nn, float* normals,
                        cudaStream_t st);
void launch_sides(const ForestArgs& a, const PNode* nodes, const uint32_t* chunk_node,
                  uint32_t nchunks, const float* normals, uint32_t* chunkL, cudaStream_t st);
void launch_node_scan(PNode* nodes, uint32_t nn, uint32_t* chunkL, cudaStream_t st);
void launch_partition(const ForestArgs& a, PNode* nodes, const uint32_t* chunk_node,
                      uint32_t nchunks, const uint32_t* chunkPre, cudaStream_t st);
void launch_degenerate(const ForestArgs& a, PNode* nodes, uint32_t nn, cudaStream_t st);
// roots sorted by size, descending; the first n_big run with 512 threads on st_big.
void launch_seqtrees(const ForestArgs& a, const SRoot* roots, uint32_t n_big, uint32_t nr,
                     cudaStream_t st, cudaStream_t st_big);

// Leaf all-pairs of one tree into the heaps (nndescent.rs:785-815).
// leaf_cap: the largest leaf the forest can produce below depth 101 (leaf_size).
void launch_leaf_pairs(const float* X, int d, int dp, const uint32_t* ids_t,
                       const uint32_t* leaf_start, uint32_t nleaves, uint32_t n, int k,
                       uint32_t leaf_cap, uint32_t* hidx, float* hdist, uint8_t* hflag,
                       cudaStream_t st);
void launch_leaf_compact(const uint8_t* leafflag_t, uint32_t n, uint32_t* leaf_start,
                         uint32_t* scan_buf, void* scan_temp, uint64_t* count_dev,
                         cudaStream_t st);
// Random fill of empty slots (nndescent.rs:820-845).
void launch_random_fill(const float* X, int d, int dp, uint32_t n, int k, uint64_t seed,
                        uint32_t* hidx, float* hdist, uint8_t* hflag, cudaStream_t st);

// ── rounds ──
void launch_cand_gen(const uint32_t* hidx, const uint8_t* hflag, uint32_t n, int k,
                     uint64_t seed, uint32_t iter, uint32_t* keys, uint64_t* vals,
                     uint32_t* dcnt, cudaStream_t st);
void launch_cand_apply(const uint32_t* keys, const uint64_t* vals, const uint32_t* seg_off,
                       const uint32_t* dcnt, uint32_t n, int m, uint32_t* new_idx,
                       float* new_prio, uint32_t* old_idx, float* old_prio, cudaStream_t st);
void launch_flag_flip(const uint32_t* hidx, uint8_t* hflag, const uint32_t* new_idx, uint32_t n,
                      int k, int m, cudaStream_t st);
// perm (may be null): the order in which CTAs visit source rows.
void launch_join_count(const float* X, int d, int dp, uint32_t n, int k, int m,
                       const float* hdist, const uint32_t* new_idx, const uint32_t* old_idx,
                       const uint32_t* perm, uint32_t* bits, int words, uint32_t* row_cnt,
                       unsigned long long* pairs, cudaStream_t st);
void launch_join_write(const float* X, int d, int dp, uint32_t n, int m, const uint32_t* new_idx,
                       const uint32_t* old_idx, const uint32_t* perm, const uint32_t* bits,
                       int words, const uint32_t* row_cnt, const uint32_t* row_off,
                       uint32_t* keys, uint64_t* vals, uint32_t* dcnt, cudaStream_t st);
void launch_replay(const uint32_t* keys, const uint64_t* vals, const uint32_t* seg_off,
                   const uint32_t* dcnt, uint32_t n, int k, uint32_t* hidx, float* hdist,
                   uint8_t* hflag, unsigned long long* changed, cudaStream_t st);
void launch_extract_count(const uint32_t* hidx, uint32_t n, int k, uint32_t* cnt,
                          cudaStream_t st);
void launch_extract(const uint32_t* hidx, const float* hdist, uint32_t n, int k,
                    const uint32_t* row_off, uint32_t* indptr, uint32_t* indices, float* dists,
                    cudaStream_t st);

}  // namespace pq
