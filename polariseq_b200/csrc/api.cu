// C ABI and host driver of the kNN-graph builder (include/polariseq_knn.h).
//
// The driver resolves NndescentOptions exactly as the reference does
// (crates/polariseq-core/src/nndescent.rs:708-752), pads the embedding to
// 16-byte rows in HBM, then runs the plain form's phases on the context's
// stream: RP forest, leaf pairs, random fill, rounds, extract.
#include <cstdio>
#include <cstring>
#include <functional>

#include "ctx.cuh"
#include "exact.cuh"
#include "batched.cuh"
#include "mlp.cuh"
#include "fuzzy.cuh"
#include "kernels.cuh"
#include "primitives.cuh"

namespace pq {
unsigned long long g_launches = 0;
}

using namespace pqh;

namespace {

// Padded copy of row-major n x d rows: dst[i][j] = src[i][j] for j < d, 0 up to dp.
__global__ void k_pad_rows(const float* __restrict__ src, size_t n, int d, int dp,
                           float* __restrict__ dst) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * size_t(dp)) return;
    const size_t i = t / dp;
    const int j = int(t - i * dp);
    dst[t] = j < d ? src[i * d + j] : 0.0f;
}

__global__ void k_fill_u32(uint32_t* p, size_t n, uint32_t v) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
__global__ void k_fill_f32(float* p, size_t n, float v) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
__global__ void k_iota_trees(uint32_t* ids, uint32_t n, uint32_t T) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < size_t(n) * T) ids[i] = uint32_t(i % n);
}

// Records of one round's join beyond which the round is replayed in
// source-row chunks (a memory bound: 24 bytes of sort buffers per record).
// POLARISEQ_JOIN_CHUNK overrides it (tests force many small chunks).
uint64_t join_chunk_records() {
    if (const char* e = std::getenv("POLARISEQ_JOIN_CHUNK")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v >= 2) return v;
    }
    return uint64_t(1) << 30;
}

__global__ void k_widen_u32(const uint32_t* __restrict__ in, uint32_t n, uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}
__global__ void k_low_u32(const uint64_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = uint32_t(in[i]);
}
// bnd[j] = the first row whose exclusive record prefix reaches j * half
// (bnd[0] = 0, bnd[J] = n): every chunk holds less than half + one row's
// records.
__global__ void k_chunk_bounds(const uint64_t* __restrict__ pre, uint32_t n, uint64_t half,
                               uint32_t J, uint32_t* __restrict__ bnd) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > J) return;
    if (j == 0 || j == J) {
        bnd[j] = j == 0 ? 0u : n;
        return;
    }
    const uint64_t target = uint64_t(j) * half;
    uint32_t lo = 0, hi = n;  // first i in [0, n) with pre[i] >= target, else n
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (pre[mid] >= target) hi = mid; else lo = mid + 1;
    }
    bnd[j] = lo;
}
// (chunk of row perm[t], perm[t]): sorted stably by chunk, the rows of each
// chunk in perm order.
__global__ void k_chunk_keys(const uint32_t* __restrict__ perm, uint32_t n,
                             const uint32_t* __restrict__ bnd, uint32_t J,
                             uint32_t* __restrict__ keys, uint64_t* __restrict__ vals) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t i = perm ? perm[t] : t;
    uint32_t lo = 0, hi = J;  // the last j with bnd[j] <= i
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (bnd[mid] <= i) lo = mid; else hi = mid;
    }
    keys[t] = lo;
    vals[t] = i;
}

// Host-side probe destinations.
struct Probe {
    int32_t stop_after = -2;
    uint32_t* heap_idx = nullptr;
    float* heap_dist = nullptr;
    uint8_t* heap_flag = nullptr;
    uint32_t* cand_new = nullptr;
    uint32_t* cand_old = nullptr;
    int32_t tree = -1;  // pq_debug_tree: stop after the forest and copy this tree
    uint32_t* tree_ids = nullptr;
    uint32_t* tree_leaves = nullptr;
    uint64_t leaves_cap = 0;
    uint64_t* n_leaves = nullptr;
    bool done = false;
};

// NN-Descent rounds (nndescent.rs:853-975) on the heaps in place: candidate
// sampling, flag flip, ordered join and per-destination replay, until a round
// changes at most stop_at entries.  Round statistics go to stats slots
// [stats_offset, ...).  `perm` orders the join CTAs (spatially coherent rows
// share candidate rows in L2).  Returns the rounds run (negative if
// after_round asked to stop).
}  // namespace

namespace pqh {
float* load_embedding(pq_ctx* c, const float* data, bool on_host, uint32_t n, int d, int dp,
                      cudaStream_t st) {
    if (!st) st = c->stream;
    float* X = c->get<float>("X", size_t(n) * dp);
    const size_t bytes = size_t(n) * d * sizeof(float);
    if (dp == d) {
        ck(cudaMemcpyAsync(X, data, bytes,
                           on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st),
           "copy embedding");
        return X;
    }
    const float* src = data;
    if (on_host) {  // one contiguous transfer, then the padding on the device
        float* stage = c->get<float>("X_stage", size_t(n) * d);
        ck(cudaMemcpyAsync(stage, data, bytes, cudaMemcpyHostToDevice, st), "copy embedding");
        src = stage;
    }
    k_pad_rows<<<blocks(size_t(n) * dp, 256), 256, 0, st>>>(src, n, d, dp, X);
    pq::count_launch();
    ck(cudaGetLastError(), "pad embedding");
    return X;
}

float* load_embedding_rows(pq_ctx* c, const float* data, uint32_t n, int d, int dp, uint32_t r0,
                           uint32_t r1, cudaStream_t st) {
    float* X = c->get<float>("X", size_t(n) * dp);
    if (r1 <= r0) return X;
    const size_t rows = r1 - r0;
    if (dp == d) {
        ck(cudaMemcpyAsync(X + size_t(r0) * dp, data + size_t(r0) * d, rows * d * sizeof(float),
                           cudaMemcpyHostToDevice, st),
           "copy embedding");
        return X;
    }
    float* stage = c->get<float>("X_stage", size_t(n) * d);
    ck(cudaMemcpyAsync(stage + size_t(r0) * d, data + size_t(r0) * d, rows * d * sizeof(float),
                       cudaMemcpyHostToDevice, st),
       "copy embedding");
    k_pad_rows<<<blocks(rows * dp, 256), 256, 0, st>>>(stage + size_t(r0) * d, rows, d, dp,
                                                        X + size_t(r0) * dp);
    pq::count_launch();
    ck(cudaGetLastError(), "pad embedding");
    return X;
}

// The records of source rows [a, b) (offsets row_off[a..b) local to the
// chunk, `total` of them): written in generation order, sorted stably by
// destination and replayed into the heaps.  `rows` lists the chunk's rows in
// the order the CTAs take them.
void replay_join_chunk(pq_ctx* c, const float* X, int d, int dp, uint32_t n, int k, int m,
                       const uint32_t* new_idx, const uint32_t* old_idx, const uint32_t* rows,
                       const uint32_t* bits, int words, const uint32_t* row_cnt,
                       const uint32_t* row_off, uint32_t a, uint32_t b, uint64_t total,
                       uint32_t* dcnt, uint32_t* seg_off, void* stemp, uint32_t* hidx,
                       float* hdist, uint8_t* hflag) {
    using namespace pq;
    cudaStream_t st = c->stream;
    uint32_t* jk = c->get<uint32_t>("jkeys", total);
    uint64_t* jv = c->get<uint64_t>("jvals", total);
    uint32_t* jk2 = c->get<uint32_t>("jkeys2", total);
    uint64_t* jv2 = c->get<uint64_t>("jvals2", total);
    void* rtj = c->get<uint8_t>("radix_temp_j", radix_temp_bytes(total));
    ck(cudaMemsetAsync(dcnt, 0, size_t(n) * 4, st), "memset dcnt");
    {
        KGScope kg(c, PQ_KG_JOIN_WRITE);
        launch_join_write(X, d, dp, b - a, m, new_idx, old_idx, rows, bits, words, row_cnt,
                          row_off, jk, jv, dcnt, st);
    }
    {
        KGScope kg(c, PQ_KG_SORT);
        ck(radix_sort_pairs(jk, jv, jk2, jv2, total, key_bits(n > 1 ? n - 1 : 1), rtj, st),
           "sort join");
        ck(scan_exclusive_u32(dcnt, seg_off, n, stemp, nullptr, st), "scan replay");
    }
    {
        KGScope kg(c, PQ_KG_REPLAY);
        launch_replay(jk, jv, seg_off, dcnt, n, k, hidx, hdist, hflag, c->d_acc + 1, st);
    }
}

int run_rounds(pq_ctx* c, const float* X, int d, int dp, uint32_t n, int k, int m, uint64_t seed,
               uint64_t n_iters, uint64_t stop_at, uint32_t* hidx, float* hdist, uint8_t* hflag,
               const uint32_t* perm, int stats_offset,
               const std::function<bool(int, const uint32_t*, const uint32_t*)>& after_round) {
    using namespace pq;
    cudaStream_t st = c->stream;
    pq_nnd_stats& S = c->stats;
    uint32_t* new_idx = c->get<uint32_t>("new_idx", size_t(n) * m);
    float* new_prio = c->get<float>("new_prio", size_t(n) * m);
    uint32_t* old_idx = c->get<uint32_t>("old_idx", size_t(n) * m);
    float* old_prio = c->get<float>("old_prio", size_t(n) * m);
    uint32_t* dcnt = c->get<uint32_t>("dcnt", n);
    uint32_t* seg_off = c->get<uint32_t>("seg_off", n);
    uint32_t* row_cnt = c->get<uint32_t>("row_cnt", n);
    const int words = (4 * m * m + 31) / 32;
    uint32_t* bits = c->get<uint32_t>("bits", size_t(n) * words);
    void* stemp = c->get<uint8_t>("scan_temp", scan_temp_bytes(n));
    const size_t nrec_c = 2 * size_t(n) * k;
    int rounds = 0;
    for (uint64_t iter = 0; iter < n_iters; ++iter) {
        // candidates
        uint32_t* ck_ = c->get<uint32_t>("ckeys", nrec_c);
        uint64_t* cv = c->get<uint64_t>("cvals", nrec_c);
        uint32_t* ck2 = c->get<uint32_t>("ckeys2", nrec_c);
        uint64_t* cv2 = c->get<uint64_t>("cvals2", nrec_c);
        void* rtemp = c->get<uint8_t>("radix_temp_c", radix_temp_bytes(nrec_c));
        {
            KGScope kg(c, PQ_KG_CANDIDATES);
            ck(cudaMemsetAsync(dcnt, 0, size_t(n) * 4, st), "memset dcnt");
            launch_cand_gen(hidx, hflag, n, k, seed, uint32_t(iter), ck_, cv, dcnt, st);
            ck(radix_sort_pairs(ck_, cv, ck2, cv2, nrec_c, key_bits(n), rtemp, st), "sort cand");
            ck(scan_exclusive_u32(dcnt, seg_off, n, stemp, nullptr, st), "scan cand");
            launch_cand_apply(ck_, cv, seg_off, dcnt, n, m, new_idx, new_prio, old_idx, old_prio,
                              st);
            launch_flag_flip(hidx, hflag, new_idx, n, k, m, st);
        }
        // join
        ck(cudaMemsetAsync(c->d_acc, 0, 2 * sizeof(unsigned long long), st), "memset acc");
        {
            KGScope kg(c, PQ_KG_JOIN_COUNT);
            launch_join_count(X, d, dp, n, k, m, hdist, new_idx, old_idx, perm, bits, words,
                              row_cnt, c->d_acc, st);
        }
        uint32_t* row_off = seg_off;  // free until the replay's segments are computed
        ck(scan_exclusive_u32(row_cnt, row_off, n, stemp, c->d_u64, st), "scan join");
        uint64_t total = 0;
        ck(cudaMemcpyAsync(&total, c->d_u64, 8, cudaMemcpyDeviceToHost, st), "total");
        ck(cudaStreamSynchronize(st), "join count");
        const uint64_t cap = join_chunk_records();
        if (total > 0 && total <= cap) {
            replay_join_chunk(c, X, d, dp, n, k, m, new_idx, old_idx, perm, bits, words, row_cnt,
                              row_off, 0, n, total, dcnt, seg_off, stemp, hidx, hdist, hflag);
        } else if (total > cap) {
            // source-row chunks [b_j, b_j+1) in index order, each holding at
            // most cap records: replaying them one after another keeps every
            // destination's updates in generation order (the reference applies
            // its 4096-row blocks the same way, nndescent.rs:916-969)
            uint64_t* pre = c->get<uint64_t>("join_pre", size_t(n) + 1);
            const uint64_t half = cap / 2;
            const uint32_t J = uint32_t((total + half - 1) / half);
            uint32_t* bnd = c->get<uint32_t>("join_bounds", size_t(J) + 1);
            k_widen_u32<<<blocks(n, 256), 256, 0, st>>>(row_cnt, n, pre); count_launch();
            ck(scan_exclusive_u64(pre, pre, n, c->get<uint8_t>("scan_temp64", scan_temp_bytes(n)),
                                  nullptr, st),
               "scan join 64");
            k_chunk_bounds<<<blocks(size_t(J) + 1, 256), 256, 0, st>>>(pre, n, half, J, bnd);
            count_launch();
            std::vector<uint32_t> hb(size_t(J) + 1);
            ck(cudaMemcpyAsync(hb.data(), bnd, (size_t(J) + 1) * 4, cudaMemcpyDeviceToHost, st),
               "bounds");
            // the join CTAs of each chunk keep the spatially coherent order:
            // the rows in perm order, stably grouped by chunk
            uint32_t* ck_k = c->get<uint32_t>("join_ck", n);
            uint64_t* ck_v = c->get<uint64_t>("join_cv", n);
            uint32_t* ck_k2 = c->get<uint32_t>("join_ck2", n);
            uint64_t* ck_v2 = c->get<uint64_t>("join_cv2", n);
            k_chunk_keys<<<blocks(n, 256), 256, 0, st>>>(perm, n, bnd, J, ck_k, ck_v);
            count_launch();
            ck(radix_sort_pairs(ck_k, ck_v, ck_k2, ck_v2, n, key_bits(J > 1 ? J - 1 : 1),
                                c->get<uint8_t>("radix_temp_ck", radix_temp_bytes(n)), st),
               "sort chunks");
            uint32_t* cperm = c->get<uint32_t>("join_cperm", n);
            k_low_u32<<<blocks(n, 256), 256, 0, st>>>(ck_v, n, cperm); count_launch();
            ck(cudaStreamSynchronize(st), "bounds");
            for (uint32_t j = 0; j < J; ++j) {
                const uint32_t a = hb[j], b = hb[j + 1];
                if (b <= a) continue;
                ck(scan_exclusive_u32(row_cnt + a, row_off + a, b - a, stemp, c->d_u64, st),
                   "scan chunk");
                uint64_t tj = 0;
                ck(cudaMemcpyAsync(&tj, c->d_u64, 8, cudaMemcpyDeviceToHost, st), "chunk total");
                ck(cudaStreamSynchronize(st), "chunk total");
                if (tj == 0) continue;  // (tj < cap / 2 + one row's records)
                replay_join_chunk(c, X, d, dp, n, k, m, new_idx, old_idx, cperm + a, bits, words,
                                  row_cnt, row_off, a, b, tj, dcnt, seg_off, stemp, hidx, hdist,
                                  hflag);
            }
        }
        unsigned long long acc[2];
        ck(cudaMemcpyAsync(acc, c->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, st), "acc");
        ck(cudaStreamSynchronize(st), "round");
        const uint64_t changed = acc[1];
        const uint64_t slot = stats_offset + iter;
        if (slot < 64) {
            S.changed[slot] = changed;
            S.emitted[slot] = total;
            S.pairs[slot] = acc[0];
        }
        rounds = int(iter + 1);
        if (after_round && after_round(int(iter), new_idx, old_idx)) return -rounds;
        if (changed <= stop_at) break;
    }
    return rounds;
}
}  // namespace pqh

namespace {

// The plain form on device data.  Returns nnz (outputs written) unless the
// probe stopped early.
uint64_t build_plain(pq_ctx* c, const float* data, bool data_on_host, uint64_t n64, uint64_t d64,
                     const pq_nnd_opts& o, uint32_t* d_indptr, uint32_t* d_indices,
                     float* d_dists, Probe* probe) {
    using namespace pq;
    cudaStream_t st = c->stream;
    const Resolved R = resolve(n64, o);
    const uint32_t n = uint32_t(n64);
    const int d = int(d64), dp = int((d64 + 3) / 4 * 4);
    const int k = int(R.k), m = int(R.max_cand);
    const uint32_t T = uint32_t(R.n_trees);
    const uint64_t seed = o.seed;
    pq_nnd_stats& S = c->stats;
    std::memset(&S, 0, sizeof(S));
    S.n_trees = int32_t(T);
    S.k = R.k;
    S.max_candidates = R.max_cand;
    S.n_iters = R.n_iters;
    S.leaf_size = R.leaf_size;
    S.stop_at = R.stop_at;
    Timer tm(st), tot(st);
    tot.start();
    const unsigned long long launches0 = g_launches;

    // padded rows
    float* X = load_embedding(c, data, data_on_host, n, d, dp);

    // heaps
    uint32_t* hidx = c->get<uint32_t>("hidx", size_t(n) * k);
    float* hdist = c->get<float>("hdist", size_t(n) * k);
    uint8_t* hflag = c->get<uint8_t>("hflag", size_t(n) * k);
    k_fill_u32<<<blocks(size_t(n) * k, 256), 256, 0, st>>>(hidx, size_t(n) * k, PQ_EMPTY); count_launch();
    k_fill_f32<<<blocks(size_t(n) * k, 256), 256, 0, st>>>(hdist, size_t(n) * k,
                                                           __builtin_huge_valf()); count_launch();
    ck(cudaMemsetAsync(hflag, 0, size_t(n) * k, st), "memset flags");
    ck(cudaMemsetAsync(c->d_err, 0, sizeof(int), st), "memset err");

    // ── forest ──
    tm.start();
    const size_t TN = size_t(T) * n;
    ForestArgs fa;
    fa.X = X;
    fa.d = d;
    fa.dp = dp;
    fa.n = n;
    fa.leaf_size = uint32_t(std::min<uint64_t>(R.leaf_size, 0xFFFFFFFFull));
    fa.ids = c->get<uint32_t>("ids", TN);
    fa.tmp = c->get<uint32_t>("tmp", TN);
    fa.side = c->get<uint8_t>("side", TN);
    fa.tabA = c->get<uint32_t>("tabA", TN);
    fa.tabB = c->get<uint32_t>("tabB", TN);
    fa.leafflag = c->get<uint8_t>("leafflag", TN);
    fa.err = c->d_err;
    // POLARISEQ_TRACE=timeline keeps only the subtree CTAs' start and end
    // stamps (no counters, so the kernels run at their untraced speed)
    const char* tv = std::getenv("POLARISEQ_TRACE");
    const bool trace = tv != nullptr;
    const bool timeline_only = trace && std::strcmp(tv, "timeline") == 0;
    fa.trace = nullptr;
    fa.tl = nullptr;
    unsigned long long* tbuf = nullptr;
    if (trace) {
        tbuf = c->get<unsigned long long>("seq_trace", SEQ_TRACE_N);
        ck(cudaMemsetAsync(tbuf, 0, SEQ_TRACE_N * 8, st), "trace");
        fa.tl = tbuf;
        if (!timeline_only) fa.trace = tbuf;
    }
    k_iota_trees<<<blocks(TN, 256), 256, 0, st>>>(fa.ids, n, T); count_launch();
    ck(cudaMemsetAsync(fa.leafflag, 0, TN, st), "memset leafflag");

    std::vector<PNode> cur;
    for (uint32_t t = 0; t < T; ++t) {
        PNode nd{};
        nd.tree = t;
        nd.start = 0;
        nd.size = n;
        nd.depth = 0;
        nd.seed = splitmix(seed ^ (uint64_t(t) + 1));
        cur.push_back(nd);
    }
    std::vector<SRoot> roots;
    while (!cur.empty()) {
        std::vector<PNode> act;
        for (const PNode& nd : cur) {
            if (nd.size < 8192 || nd.depth >= 6)
                roots.push_back(SRoot{nd.tree, nd.start, nd.size, nd.depth, nd.seed});
            else
                act.push_back(nd);
        }
        if (act.empty()) break;
        std::vector<uint32_t> chunk_node;
        for (uint32_t i = 0; i < act.size(); ++i) {
            act[i].chunk0 = uint32_t(chunk_node.size());
            uint32_t nch = (act[i].size + FOREST_CHUNK - 1) / FOREST_CHUNK;
            for (uint32_t q = 0; q < nch; ++q) chunk_node.push_back(i);
        }
        const uint32_t nn = uint32_t(act.size()), nch = uint32_t(chunk_node.size());
        PNode* d_nodes = c->get<PNode>("pnodes", nn);
        uint32_t* d_cn = c->get<uint32_t>("chunk_node", nch);
        uint32_t* d_cl = c->get<uint32_t>("chunkL", nch);
        float* d_norm = c->get<float>("normals", size_t(nn) * dp);
        ck(cudaMemcpyAsync(d_nodes, act.data(), nn * sizeof(PNode), cudaMemcpyHostToDevice, st),
           "upload nodes");
        ck(cudaMemcpyAsync(d_cn, chunk_node.data(), nch * sizeof(uint32_t),
                           cudaMemcpyHostToDevice, st),
           "upload chunks");
        {
            KGScope kg(c, PQ_KG_FOREST_TOP);
            launch_hyperplanes(fa, d_nodes, nn, d_norm, st);
            launch_sides(fa, d_nodes, d_cn, nch, d_norm, d_cl, st);
            launch_node_scan(d_nodes, nn, d_cl, st);
            launch_partition(fa, d_nodes, d_cn, nch, d_cl, st);
            launch_degenerate(fa, d_nodes, nn, st);
        }
        ck(cudaMemcpyAsync(act.data(), d_nodes, nn * sizeof(PNode), cudaMemcpyDeviceToHost, st),
           "download nodes");
        ck(cudaStreamSynchronize(st), "forest level");
        cur.clear();
        for (const PNode& nd : act) {
            PNode l{}, r{};
            l.tree = r.tree = nd.tree;
            l.depth = r.depth = nd.depth + 1;
            l.start = nd.start;
            l.size = nd.nL;
            l.seed = splitmix(nd.seed ^ 1ull);
            r.start = nd.start + nd.nL;
            r.size = nd.size - nd.nL;
            r.seed = splitmix(nd.seed ^ 2ull);
            cur.push_back(l);
            cur.push_back(r);
        }
    }
    {
        // largest subtrees first: their depth-first chains are the critical path
        std::stable_sort(roots.begin(), roots.end(),
                         [](const SRoot& x, const SRoot& y) { return x.size > y.size; });
        SRoot* d_roots = c->get<SRoot>("sroots", roots.size());
        ck(cudaMemcpyAsync(d_roots, roots.data(), roots.size() * sizeof(SRoot),
                           cudaMemcpyHostToDevice, st),
           "upload roots");
        KGScope kg(c, PQ_KG_SEQTREE);
        uint32_t n_big = 0;
        while (n_big < roots.size() && n_big < 148 && roots[n_big].size > 65536) ++n_big;
        if (fa.trace) {
            uint64_t r0 = roots.empty() ? 0 : roots[0].size;
            ck(cudaMemcpyAsync(fa.trace + SEQ_T_ROOT0, &r0, 8, cudaMemcpyHostToDevice, st), "tr");
        }
        // the big-root stream starts after everything queued so far and the
        // main stream waits for it before the leaf pairs
        ck(cudaEventRecord(c->ev_fork, st), "fork");
        ck(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0), "fork");
        launch_seqtrees(fa, d_roots, n_big, uint32_t(roots.size()), st, c->stream2);
        ck(cudaEventRecord(c->ev_join, c->stream2), "join");
        ck(cudaStreamWaitEvent(st, c->ev_join, 0), "join");
        ck(cudaGetLastError(), "seqtrees");
    }
    int herr = 0;
    ck(cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "err");
    S.ms_forest = tm.stop();
    if (trace) {
        unsigned long long h[SEQ_TRACE_N];
        ck(cudaMemcpy(h, tbuf, sizeof(h), cudaMemcpyDeviceToHost), "trace");
        std::fprintf(stderr,
                     "[nndescent] rp-forest build (%u trees, leaf %llu): %.2f ms; %zu subtree "
                     "roots, largest %llu\n",
                     T, (unsigned long long)R.leaf_size, S.ms_forest, roots.size(), h[SEQ_T_ROOT0]);
        std::fprintf(stderr,
                     "[nndescent]   subtrees: global nodes %llu (points %llu), staged subtrees "
                     "%llu (nodes %llu), tie nodes %llu, random splits %llu\n",
                     h[0], h[1], h[2], h[3], h[4], h[5]);
        std::fprintf(stderr,
                     "[nndescent]   largest subtree cycles: draw %llu margin %llu partition %llu "
                     "staged %llu total %llu\n",
                     h[6], h[7], h[8], h[9], h[10]);
        std::fprintf(stderr,
                     "[nndescent]   largest subtree: global nodes %llu, CTA-staged nodes %llu, "
                     "staged subtrees %llu (nodes %llu, warp cycles %llu); CTA-staged subtrees "
                     "%llu (nodes %llu) in all\n",
                     h[SEQ_T_R0_GNODES], h[SEQ_T_R0_MNODES], h[SEQ_T_R0_STAGED],
                     h[SEQ_T_R0_SNODES], h[SEQ_T_R0_CYC_WARP], h[SEQ_T_MID_TREES],
                     h[SEQ_T_MID_NODES]);
        std::fprintf(stderr,
                     "[nndescent]   largest subtree, warp splits: leaf pops %llu draws %llu "
                     "margins %llu partition %llu; CTA splits: staging %llu draws %llu margins "
                     "%llu partition %llu cycles\n",
                     h[SEQ_T_W_LEAF], h[SEQ_T_W_DRAW], h[SEQ_T_W_MARGIN], h[SEQ_T_W_PART],
                     h[SEQ_T_M_STAGE], h[SEQ_T_M_DRAW], h[SEQ_T_M_MARGIN], h[SEQ_T_M_PART]);
        // timeline of the two subtree kernels (globaltimer): each large root's
        // CTA against the span of the 128-thread kernel
        uint32_t nb = 0;
        while (nb < roots.size() && nb < 148 && roots[nb].size > 65536) ++nb;
        unsigned long long t0 = ~h[SEQ_T_SMALL_T0], t1s = h[SEQ_T_SMALL_T1];
        for (uint32_t b = 0; b < nb && b < uint32_t(SEQ_T_BIG_N); ++b)
            t0 = std::min(t0, h[SEQ_T_BIG + 2 * b]);
        std::fprintf(stderr,
                     "[nndescent]   subtree timeline: %u roots above 65536 points, %zu below; "
                     "128-thread kernel ends at %.2f ms\n",
                     nb, roots.size() - nb, (t1s - t0) * 1e-6);
        for (uint32_t b = 0; b < nb && b < uint32_t(SEQ_T_BIG_N); ++b) {
            if (b >= 24 && b % 16 != 0 && b + 1 != nb) continue;
            std::fprintf(stderr, "[nndescent]     root %u: %u points, %.2f .. %.2f ms\n", b,
                         roots[b].size, (h[SEQ_T_BIG + 2 * b] - t0) * 1e-6,
                         (h[SEQ_T_BIG + 2 * b + 1] - t0) * 1e-6);
        }
    }
    if (herr) throw DeviceError{"forest: a subtree exceeded the depth-first stack"};

    if (probe && probe->tree >= 0) {
        uint32_t t = uint32_t(probe->tree);
        std::vector<uint8_t> lf(n);
        ck(cudaMemcpy(probe->tree_ids, fa.ids + size_t(t) * n, size_t(n) * 4,
                      cudaMemcpyDeviceToHost),
           "tree ids");
        ck(cudaMemcpy(lf.data(), fa.leafflag + size_t(t) * n, n, cudaMemcpyDeviceToHost),
           "tree leaves");
        uint64_t nl = 0;
        std::vector<uint32_t> starts;
        for (uint32_t i = 0; i < n; ++i)
            if (lf[i]) starts.push_back(i);
        nl = starts.size();
        if (nl <= probe->leaves_cap)
            for (uint64_t q = 0; q < nl; ++q) {
                probe->tree_leaves[2 * q] = starts[q];
                probe->tree_leaves[2 * q + 1] = q + 1 < nl ? starts[q + 1] : n;
            }
        *probe->n_leaves = nl;
        probe->done = true;
        return 0;
    }

    // ── leaf pairs, one tree after another ──
    tm.start();
    {
        uint32_t* leaf_start = fa.tabA;  // reused: the forest scratch is free now
        uint32_t* scanbuf = fa.tabB;
        void* stemp = c->get<uint8_t>("scan_temp", scan_temp_bytes(n));
        uint64_t* cnts = c->get<uint64_t>("leaf_counts", T);
        for (uint32_t t = 0; t < T; ++t)
            launch_leaf_compact(fa.leafflag + size_t(t) * n, n, leaf_start + size_t(t) * n,
                                scanbuf + size_t(t) * n, stemp, cnts + t, st);
        std::vector<uint64_t> hc(T);
        ck(cudaMemcpyAsync(hc.data(), cnts, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, st),
           "leaf counts");
        ck(cudaStreamSynchronize(st), "leaf compact");
        KGScope kg(c, PQ_KG_LEAF_PAIRS);
        for (uint32_t t = 0; t < T; ++t)
            launch_leaf_pairs(X, d, dp, fa.ids + size_t(t) * n, leaf_start + size_t(t) * n,
                              uint32_t(hc[t]), n, k, fa.leaf_size, hidx, hdist, hflag, st);
        launch_random_fill(X, d, dp, n, k, seed, hidx, hdist, hflag, st);
        ck(cudaGetLastError(), "leaf pairs");
    }
    S.ms_leaves = tm.stop();

    auto copy_heaps = [&]() {
        if (probe->heap_idx)
            ck(cudaMemcpy(probe->heap_idx, hidx, size_t(n) * k * 4, cudaMemcpyDeviceToHost), "p");
        if (probe->heap_dist)
            ck(cudaMemcpy(probe->heap_dist, hdist, size_t(n) * k * 4, cudaMemcpyDeviceToHost), "p");
        if (probe->heap_flag)
            ck(cudaMemcpy(probe->heap_flag, hflag, size_t(n) * k, cudaMemcpyDeviceToHost), "p");
    };
    if (probe && probe->stop_after == -1) {
        ck(cudaStreamSynchronize(st), "probe");
        copy_heaps();
        probe->done = true;
        return 0;
    }

    // ── rounds ──
    tm.start();
    {
        // join CTAs visit source rows in tree 0's leaf order (spatially coherent)
        const int r = run_rounds(
            c, X, d, dp, n, k, m, seed, R.n_iters, R.stop_at, hidx, hdist, hflag, fa.ids, 0,
            [&](int iter, const uint32_t* new_idx, const uint32_t* old_idx) {
                if (!probe || probe->stop_after != iter) return false;
                copy_heaps();
                if (probe->cand_new)
                    ck(cudaMemcpy(probe->cand_new, new_idx, size_t(n) * m * 4,
                                  cudaMemcpyDeviceToHost),
                       "p");
                if (probe->cand_old)
                    ck(cudaMemcpy(probe->cand_old, old_idx, size_t(n) * m * 4,
                                  cudaMemcpyDeviceToHost),
                       "p");
                probe->done = true;
                return true;
            });
        S.rounds_run = r < 0 ? -r : r;
        if (r < 0) return 0;
    }
    S.ms_rounds = tm.stop();

    // ── extract ──
    tm.start();
    void* stemp = c->get<uint8_t>("scan_temp", scan_temp_bytes(n));
    uint32_t* ecnt = c->get<uint32_t>("ecnt", n);
    uint32_t* eoff = c->get<uint32_t>("eoff", n);
    {
        KGScope kg(c, PQ_KG_EXTRACT);
        launch_extract_count(hidx, n, k, ecnt, st);
        ck(scan_exclusive_u32(ecnt, eoff, n, stemp, c->d_u64, st), "scan extract");
        launch_extract(hidx, hdist, n, k, eoff, d_indptr, d_indices, d_dists, st);
    }
    uint64_t nnz = 0;
    ck(cudaMemcpyAsync(&nnz, c->d_u64, 8, cudaMemcpyDeviceToHost, st), "nnz");
    ck(cudaStreamSynchronize(st), "extract");
    S.ms_extract = tm.stop();
    S.ms_total = tot.stop();
    S.launches = g_launches - launches0;
    kg_collect(c);
    if (probe) {
        copy_heaps();
        probe->done = true;
    }
    return nnz;
}

// Learned-init NN-Descent: the initial lists from the learned buckets, the
// reference's rounds to convergence (build_chosen with PQ_MODE_PLAIN), then
// the recall estimate on sampled cells; below the target the RP-initialised
// build runs too and the graph with the higher estimate is kept.
// POLARISEQ_LEARNED_MIN_RECALL overrides the 0.99 target (tests force the
// fallback with a target above 1).
uint64_t build_learned_nnd(pq_ctx* c, const float* data, bool data_on_host, uint64_t n64,
                           uint64_t d64, const pq_nnd_opts& o, uint32_t* d_indptr,
                           uint32_t* d_indices, float* d_dists) {
    cudaStream_t st = c->stream;
    const uint32_t n = uint32_t(n64);
    const int d = int(d64), dp = int((d64 + 3) / 4 * 4);
    const int k = int(effective_k(n64, o.k));
    double target = 0.99;
    if (const char* e = std::getenv("POLARISEQ_LEARNED_MIN_RECALL")) target = std::atof(e);
    const uint32_t Q = 1024;
    uint64_t nnz = build_chosen(c, data, data_on_host, n64, d64, o, d_indptr, d_indices, d_dists);
    const float* X = c->get<float>("X", size_t(n) * dp);  // the padded rows of this build
    Timer tm(st);
    tm.start();
    const double rl = pq::sampled_recall(c, X, d, dp, n, k, d_indptr, d_indices, Q, o.seed);
    const double ms_check = tm.stop();
    if (std::getenv("POLARISEQ_TRACE"))
        std::fprintf(stderr, "[learned] sampled recall %.4f (%u queries): %.2f ms; build %.2f ms\n",
                     rl, Q, ms_check, c->stats.ms_total);
    pq_nnd_stats learned = c->stats;
    learned.est_recall = learned.est_recall_learned = rl;
    learned.learned_rounds = learned.rounds_run;
    if (rl >= target) {
        c->stats = learned;
        return nnz;
    }
    // the fallback: keep the learned graph aside, build with the RP forest
    uint32_t* sip = c->get<uint32_t>("lf_ip", n64 + 1);
    uint32_t* six = c->get<uint32_t>("lf_ix", std::max<uint64_t>(nnz, 1));
    float* sdx = c->get<float>("lf_dx", std::max<uint64_t>(nnz, 1));
    ck(cudaMemcpyAsync(sip, d_indptr, (n64 + 1) * 4, cudaMemcpyDeviceToDevice, st), "keep");
    ck(cudaMemcpyAsync(six, d_indices, nnz * 4, cudaMemcpyDeviceToDevice, st), "keep");
    ck(cudaMemcpyAsync(sdx, d_dists, nnz * 4, cudaMemcpyDeviceToDevice, st), "keep");
    pq_nnd_opts po = o;
    po.init = PQ_INIT_RP;
    const uint64_t nnz_rp =
        build_plain(c, data, data_on_host, n64, d64, po, d_indptr, d_indices, d_dists, nullptr);
    const float* X2 = c->get<float>("X", size_t(n) * dp);
    const double rr = pq::sampled_recall(c, X2, d, dp, n, k, d_indptr, d_indices, Q, o.seed);
    pq_nnd_stats& S = c->stats;  // the RP build's statistics
    const double ms_rp = S.ms_total;
    if (rr >= rl) {
        S.est_recall = rr;
        S.fell_back = 2;
        nnz = nnz_rp;
    } else {
        ck(cudaMemcpyAsync(d_indptr, sip, (n64 + 1) * 4, cudaMemcpyDeviceToDevice, st), "back");
        ck(cudaMemcpyAsync(d_indices, six, nnz * 4, cudaMemcpyDeviceToDevice, st), "back");
        ck(cudaMemcpyAsync(d_dists, sdx, nnz * 4, cudaMemcpyDeviceToDevice, st), "back");
        ck(cudaStreamSynchronize(st), "back");
        S = learned;
        S.est_recall = rl;
        S.fell_back = 1;
        S.ms_total += ms_rp;
    }
    S.est_recall_learned = rl;
    S.est_recall_rp = rr;
    S.learned_rounds = learned.rounds_run;
    return nnz;
}

int fail(pq_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int check_args(pq_ctx* c, uint64_t n, uint64_t d, const pq_nnd_opts* o) {
    if (!c) return PQ_EINVAL;
    if (!o) return fail(c, PQ_EINVAL, "options pointer is null");
    if (n == 0 || d == 0) return fail(c, PQ_EINVAL, "empty data");  // nndescent.rs:708
    if (o->k == 0) return fail(c, PQ_EINVAL, "k must be >= 1");      // nndescent.rs:709
    if (n >= 0xFFFFFFFEull) return fail(c, PQ_EINVAL, "n_obs must be below 2^32 - 1");
    if (d > 65536) return fail(c, PQ_EINVAL, "n_dim above 65536 is not supported");
    Resolved R = resolve(n, *o);
    if (2 * n * R.k >= 0xFFFFFFFFull)
        return fail(c, PQ_EINVAL, "n_obs * k must be below 2^31");
    if (R.n_trees * n > (uint64_t(1) << 36))
        return fail(c, PQ_EINVAL, "n_trees * n_obs is too large");
    if (2 * R.max_cand * ((d + 3) / 4 * 4) * 4 > 200 * 1024 || R.max_cand > 200)
        return fail(c, PQ_ENOTSUP,
                    "n_dim * max_candidates exceeds the join's shared-memory tile "
                    "(2 * max_candidates * n_dim * 4 bytes must stay under 200 KiB, "
                    "max_candidates <= 200)");
    if (o->mode != PQ_MODE_PLAIN && o->mode != PQ_MODE_BF16 && o->mode != PQ_MODE_FP8)
        return fail(c, PQ_ENOTSUP, "mode not available in this build");
    if (o->init != PQ_INIT_RP && o->init != PQ_INIT_LEARNED)
        return fail(c, PQ_ENOTSUP, "init not available in this build");
    if (o->init == PQ_INIT_LEARNED && n < 65536)
        return fail(c, PQ_ENOTSUP, "learned buckets need at least 65,536 cells");
    const bool tiles = o->mode != PQ_MODE_PLAIN || o->init == PQ_INIT_LEARNED;
    if (tiles && d > 62)
        return fail(c, PQ_ENOTSUP, "the tensor-core tiles support n_dim <= 62");
    if (tiles && R.k > 31) return fail(c, PQ_ENOTSUP, "the tensor-core tiles support k <= 31");
    return PQ_OK;
}

// neighbors::neighbors argument rules (neighbors.rs:106-117) and the limits of
// the exact kernel.
int check_neighbors(pq_ctx* c, uint64_t n, uint64_t d, uint64_t nn, int32_t metric) {
    if (!c) return PQ_EINVAL;
    if (n == 0 || d == 0)
        return fail(c, PQ_EINVAL, "embedding has zero rows (" + std::to_string(n) + ") or dims (" +
                                      std::to_string(d) + ")");
    if (nn == 0) return fail(c, PQ_EINVAL, "n_neighbors must be >= 1, got 0");
    if (metric != PQ_METRIC_EUCLIDEAN && metric != PQ_METRIC_COSINE)
        return fail(c, PQ_EINVAL, "unknown metric");
    if (n >= 0xFFFFFFFEull) return fail(c, PQ_EINVAL, "n_obs must be below 2^32 - 1");
    const uint64_t kws = std::min(nn, n);
    if (kws > uint64_t(pq::EXACT_MAX_K))
        return fail(c, PQ_ENOTSUP, "the exact search supports n_neighbors <= " +
                                       std::to_string(pq::EXACT_MAX_K));
    if (d > uint64_t(pq::EXACT_MAX_DIM))
        return fail(c, PQ_ENOTSUP, "the exact search supports n_dim <= " +
                                       std::to_string(pq::EXACT_MAX_DIM));
    if (n * (kws - 1) >= 0xFFFFFFFFull)
        return fail(c, PQ_EINVAL, "n_obs * (n_neighbors - 1) must be below 2^32");
    return PQ_OK;
}

// Runs f, mapping its exceptions to status codes.  On an error both of the
// context's streams are drained before returning, so no copy into the
// caller's buffers is still in flight when the caller sees the status.
template <class F>
int guarded(pq_ctx* c, F&& f) {
    auto drain = [c]() {
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->stream2);
        cudaGetLastError();
    };
    try {
        if (cudaSetDevice(c->device) != cudaSuccess)
            return fail(c, PQ_EDEVICE, "cudaSetDevice failed");
        return f();
    } catch (const DeviceError& e) {
        drain();
        return fail(c, e.timeout ? PQ_ETIMEOUT : PQ_EDEVICE, e.msg);
    } catch (const std::string& s) {
        drain();
        return fail(c, PQ_ENOMEM, s);
    } catch (const std::exception& e) {  // host-side failures (allocation, sizes)
        drain();
        return fail(c, PQ_EDEVICE, std::string("host error: ") + e.what());
    }
}

}  // namespace

extern "C" {

void pq_nnd_opts_default(pq_nnd_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->k = 15;
    o->delta = 0.001;
    o->mode = PQ_MODE_PLAIN;
    o->init = PQ_INIT_RP;
    o->probes = 0;
    o->refine_rounds = -1;
}

uint64_t pq_effective_k(uint64_t n_obs, uint64_t k) { return effective_k(n_obs, k); }

int pq_ctx_create(int device, pq_ctx** out) {
    if (!out) return PQ_EINVAL;
    *out = nullptr;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
        cudaGetLastError();
        return PQ_EDEVICE;
    }
    if (device < 0 || device >= nd) return PQ_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return PQ_EDEVICE;
    pq_ctx* c = new pq_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->d_u64, 8 * sizeof(uint64_t)) != cudaSuccess ||
        cudaMalloc(&c->d_acc, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        pq_ctx_destroy(c);
        return PQ_EDEVICE;
    }
    *out = c;
    return PQ_OK;
}

void pq_ctx_destroy(pq_ctx* c) {
    if (!c) return;
    if (c->sub) pq_ctx_destroy(c->sub);
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& kv : c->bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    if (c->d_err) cudaFree(c->d_err);
    if (c->d_u64) cudaFree(c->d_u64);
    if (c->d_acc) cudaFree(c->d_acc);
    if (c->stream2) cudaStreamSynchronize(c->stream2);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* pq_ctx_last_error(const pq_ctx* c) { return c ? c->err.c_str() : "null context"; }

int pq_ctx_set_profiling(pq_ctx* c, int on) {
    if (!c) return PQ_EINVAL;
    c->profile = on ? 1 : 0;
    return PQ_OK;
}

int pq_ctx_set_test_wait(pq_ctx* c, uint32_t polls) {
    if (!c) return PQ_EINVAL;
    c->test_wait_polls = polls;
    return PQ_OK;
}

int pq_ctx_stats(const pq_ctx* c, pq_nnd_stats* out) {
    if (!c || !out) return PQ_EINVAL;
    *out = c->stats;
    return PQ_OK;
}

int pq_nndescent_into(pq_ctx* c, const float* data, uint64_t n, uint64_t d,
                      const pq_nnd_opts* o, uint32_t* indptr, uint64_t indptr_len,
                      uint32_t* indices, uint64_t indices_len, float* dists,
                      uint64_t dists_len, uint64_t* nnz_out) {
    int rc = check_args(c, n, d, o);
    if (rc != PQ_OK) return rc;
    if (!data || !indptr || !indices || !dists || !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    if (indptr_len != n + 1) return fail(c, PQ_EINVAL, "indptr must have n_obs + 1 entries");
    uint64_t cap = n * effective_k(n, o->k);
    if (indices_len < cap || dists_len < cap)
        return fail(c, PQ_EINVAL, "the graph arrays are too short");
    return guarded(c, [&]() -> int {
        uint32_t* dip = c->get<uint32_t>("out_indptr", n + 1);
        uint32_t* dix = c->get<uint32_t>("out_indices", cap);
        float* ddx = c->get<float>("out_dists", cap);
        HostGraph hg{indptr, indices, dists, false};
        uint64_t nnz = o->mode != PQ_MODE_PLAIN
                           ? build_chosen(c, data, true, n, d, *o, dip, dix, ddx, &hg)
                       : o->init == PQ_INIT_LEARNED
                           ? build_learned_nnd(c, data, true, n, d, *o, dip, dix, ddx)
                           : build_plain(c, data, true, n, d, *o, dip, dix, ddx, nullptr);
        if (!hg.copied) {
            ck(cudaMemcpyAsync(indptr, dip, (n + 1) * 4, cudaMemcpyDeviceToHost, c->stream), "d2h");
            ck(cudaMemcpyAsync(indices, dix, nnz * 4, cudaMemcpyDeviceToHost, c->stream), "d2h");
            ck(cudaMemcpyAsync(dists, ddx, nnz * 4, cudaMemcpyDeviceToHost, c->stream), "d2h");
            ck(cudaStreamSynchronize(c->stream), "d2h");
        }
        *nnz_out = nnz;
        return PQ_OK;
    });
}

int pq_nndescent_into_device(pq_ctx* c, const float* d_data, uint64_t n, uint64_t d,
                             const pq_nnd_opts* o, uint32_t* d_indptr, uint32_t* d_indices,
                             float* d_dists, uint64_t* nnz_out, void* stream) {
    int rc = check_args(c, n, d, o);
    if (rc != PQ_OK) return rc;
    if (!d_data || !d_indptr || !d_indices || !d_dists || !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    return guarded(c, [&]() -> int {
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        cudaEvent_t ev;
        ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ev, user), "event");
        ck(cudaStreamWaitEvent(c->stream, ev, 0), "event");
        uint64_t nnz =
            o->mode != PQ_MODE_PLAIN
                ? build_chosen(c, d_data, false, n, d, *o, d_indptr, d_indices, d_dists)
            : o->init == PQ_INIT_LEARNED
                ? build_learned_nnd(c, d_data, false, n, d, *o, d_indptr, d_indices, d_dists)
                : build_plain(c, d_data, false, n, d, *o, d_indptr, d_indices, d_dists, nullptr);
        ck(cudaEventRecord(ev, c->stream), "event");
        ck(cudaStreamWaitEvent(user, ev, 0), "event");
        cudaEventDestroy(ev);
        *nnz_out = nnz;
        return PQ_OK;
    });
}

int pq_nndescent_probe(pq_ctx* c, const float* data, uint64_t n, uint64_t d,
                       const pq_nnd_opts* o, int32_t stop_after, uint32_t* heap_idx,
                       float* heap_dist, uint8_t* heap_flag, uint32_t* cand_new,
                       uint32_t* cand_old) {
    int rc = check_args(c, n, d, o);
    if (rc != PQ_OK) return rc;
    return guarded(c, [&]() -> int {
        uint64_t cap = n * effective_k(n, o->k);
        uint32_t* dip = c->get<uint32_t>("out_indptr", n + 1);
        uint32_t* dix = c->get<uint32_t>("out_indices", cap);
        float* ddx = c->get<float>("out_dists", cap);
        Probe p;
        p.stop_after = stop_after;
        p.heap_idx = heap_idx;
        p.heap_dist = heap_dist;
        p.heap_flag = heap_flag;
        p.cand_new = cand_new;
        p.cand_old = cand_old;
        build_plain(c, data, true, n, d, *o, dip, dix, ddx, &p);
        return PQ_OK;
    });
}

int pq_debug_tree(pq_ctx* c, const float* data, uint64_t n, uint64_t d, const pq_nnd_opts* o,
                  uint32_t tree, uint32_t* ids, uint32_t* leaves, uint64_t leaves_cap,
                  uint64_t* n_leaves) {
    int rc = check_args(c, n, d, o);
    if (rc != PQ_OK) return rc;
    if (!ids || !leaves || !n_leaves) return fail(c, PQ_EINVAL, "null buffer");
    Resolved R = resolve(n, *o);
    if (tree >= R.n_trees) return fail(c, PQ_EINVAL, "tree index out of range");
    return guarded(c, [&]() -> int {
        Probe p;
        p.tree = int32_t(tree);
        p.tree_ids = ids;
        p.tree_leaves = leaves;
        p.leaves_cap = leaves_cap;
        p.n_leaves = n_leaves;
        build_plain(c, data, true, n, d, *o, nullptr, nullptr, nullptr, &p);
        return PQ_OK;
    });
}

int pq_neighbors_into(pq_ctx* c, const float* data, uint64_t n, uint64_t d,
                      uint64_t n_neighbors, int32_t metric, uint32_t* indptr,
                      uint64_t indptr_len, uint32_t* indices, uint64_t indices_len,
                      float* dists, uint64_t dists_len, uint64_t* nnz_out) {
    int rc = check_neighbors(c, n, d, n_neighbors, metric);
    if (rc != PQ_OK) return rc;
    if (!data || !indptr || !indices || !dists || !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    const uint64_t kws = std::min(n_neighbors, n), nnz = n * (kws - 1);
    if (indptr_len != n + 1) return fail(c, PQ_EINVAL, "indptr must have n_obs + 1 entries");
    if (indices_len < nnz || dists_len < nnz)
        return fail(c, PQ_EINVAL, "the graph arrays are too short");
    return guarded(c, [&]() -> int {
        cudaStream_t st = c->stream;
        float* X = c->get<float>("ex_X", n * d);
        float* norms = c->get<float>("ex_norms", n);
        uint32_t* dip = c->get<uint32_t>("out_indptr", n + 1);
        uint32_t* dix = c->get<uint32_t>("out_indices", std::max<uint64_t>(nnz, 1));
        float* ddx = c->get<float>("out_dists", std::max<uint64_t>(nnz, 1));
        ck(cudaMemcpyAsync(X, data, n * d * 4, cudaMemcpyHostToDevice, st), "h2d");
        ck(pq::exact_knn_prepare(), "exact kNN set-up");
        ck(pq::launch_exact_knn(X, n, int(d), int(kws), metric == PQ_METRIC_COSINE, norms, dip, dix,
                            ddx, st),
           "exact kNN");
        ck(cudaMemcpyAsync(indptr, dip, (n + 1) * 4, cudaMemcpyDeviceToHost, st), "d2h");
        if (nnz) {
            ck(cudaMemcpyAsync(indices, dix, nnz * 4, cudaMemcpyDeviceToHost, st), "d2h");
            ck(cudaMemcpyAsync(dists, ddx, nnz * 4, cudaMemcpyDeviceToHost, st), "d2h");
        }
        ck(cudaStreamSynchronize(st), "d2h");
        *nnz_out = nnz;
        return PQ_OK;
    });
}

int pq_neighbors_into_device(pq_ctx* c, const float* d_data, uint64_t n, uint64_t d,
                             uint64_t n_neighbors, int32_t metric, uint32_t* d_indptr,
                             uint32_t* d_indices, float* d_dists, uint64_t* nnz_out,
                             void* stream) {
    int rc = check_neighbors(c, n, d, n_neighbors, metric);
    if (rc != PQ_OK) return rc;
    if (!d_data || !d_indptr || !d_indices || !d_dists || !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    const uint64_t kws = std::min(n_neighbors, n);
    return guarded(c, [&]() -> int {
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        float* norms = c->get<float>("ex_norms", n);
        cudaEvent_t ev;
        ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ev, user), "event");
        ck(cudaStreamWaitEvent(c->stream, ev, 0), "event");
        ck(pq::exact_knn_prepare(), "exact kNN set-up");
        ck(pq::launch_exact_knn(d_data, n, int(d), int(kws), metric == PQ_METRIC_COSINE, norms,
                            d_indptr, d_indices, d_dists, c->stream),
           "exact kNN");
        ck(cudaEventRecord(ev, c->stream), "event");
        ck(cudaStreamWaitEvent(user, ev, 0), "event");
        cudaEventDestroy(ev);
        *nnz_out = n * (kws - 1);
        return PQ_OK;
    });
}

int pq_knn_batched_into_device(pq_ctx* c, const float* d_data, uint64_t d, uint32_t n_samples,
                               const uint64_t* offsets, const uint32_t* ks, uint32_t* d_indices,
                               float* d_dists, int32_t flags, int32_t* shape_out, void* stream) {
    if (!c) return PQ_EINVAL;
    if (!d_data || !offsets || !ks || !d_indices || !d_dists)
        return fail(c, PQ_EINVAL, "null buffer");
    if (d == 0 || d > 64) return fail(c, PQ_ENOTSUP, "the batched search supports 1 <= n_dim <= 64");
    if (n_samples == 0) return fail(c, PQ_EINVAL, "no samples");
    if (offsets[0] != 0) return fail(c, PQ_EINVAL, "offsets[0] must be 0");
    uint32_t kmax = 1;
    uint64_t total_out = 0;
    std::vector<uint64_t> s_out(n_samples);
    for (uint32_t s = 0; s < n_samples; ++s) {
        if (offsets[s + 1] < offsets[s]) return fail(c, PQ_EINVAL, "offsets must not decrease");
        const uint64_t ns = offsets[s + 1] - offsets[s];
        if (ns >= 0xFFFFFFFFull) return fail(c, PQ_EINVAL, "a sample has 2^32 rows or more");
        if (ns > 0 && (ks[s] == 0 || ks[s] >= ns))
            return fail(c, PQ_EINVAL, "sample " + std::to_string(s) + ": k must be in [1, n)");
        if (ks[s] > 512) return fail(c, PQ_ENOTSUP, "the batched search supports k <= 512");
        kmax = std::max(kmax, ks[s]);
        s_out[s] = total_out;
        total_out += ns * ks[s];
    }
    int kp = 32;
    while (kp < int(kmax)) kp <<= 1;
    return guarded(c, [&]() -> int {
        cudaStream_t st = c->stream;
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        cudaEvent_t ev;
        ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ev, user), "event");
        ck(cudaStreamWaitEvent(st, ev, 0), "event");
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        uint64_t* ds_off = c->get<uint64_t>("bt_off", n_samples + 1);
        uint32_t* ds_k = c->get<uint32_t>("bt_k", n_samples);
        uint64_t* ds_out = c->get<uint64_t>("bt_out", n_samples);
        uint32_t* counter = c->get<uint32_t>("bt_counter", 1);
        ck(cudaMemcpyAsync(ds_off, offsets, (n_samples + 1) * 8ull, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(ds_k, ks, n_samples * 4ull, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(ds_out, s_out.data(), n_samples * 8ull, cudaMemcpyHostToDevice, st), "h2d");
        // samples largest first, then their query blocks
        std::vector<uint32_t> order(n_samples);
        for (uint32_t s = 0; s < n_samples; ++s) order[s] = s;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
            return offsets[x + 1] - offsets[x] > offsets[y + 1] - offsets[y];
        });
        auto items_for = [&](int shape, std::vector<uint32_t>& is, std::vector<uint32_t>& iq) {
            const uint32_t qpi = uint32_t(pq::batched_queries_per_item(shape));
            is.clear();
            iq.clear();
            for (uint32_t s : order)
                for (uint64_t q = 0; q < offsets[s + 1] - offsets[s]; q += qpi) {
                    is.push_back(s);
                    iq.push_back(uint32_t(q));
                }
        };
        pq::BatchLaunch b{};
        b.X = d_data;
        b.d = int(d);
        b.s_off = ds_off;
        b.s_k = ds_k;
        b.s_out = ds_out;
        b.counter = counter;
        b.kp = kp;
        b.sms = sms;
        b.out_idx = d_indices;
        b.out_dist = d_dists;
        std::vector<uint32_t> is, iq;
        auto upload_items = [&](uint32_t count) {
            uint32_t* di_s = c->get<uint32_t>("bt_item_s", std::max<size_t>(is.size(), 1));
            uint32_t* di_q = c->get<uint32_t>("bt_item_q", std::max<size_t>(iq.size(), 1));
            ck(cudaMemcpyAsync(di_s, is.data(), is.size() * 4, cudaMemcpyHostToDevice, st), "h2d");
            ck(cudaMemcpyAsync(di_q, iq.data(), iq.size() * 4, cudaMemcpyHostToDevice, st), "h2d");
            b.item_s = di_s;
            b.item_q = di_q;
            b.n_items = count;
        };
        // ── autotune: each fitting shape on the largest work items ──
        const uint64_t key = (d <= 32 ? 32ull : 64ull) << 32 | uint64_t(kp);
        auto it = c->batch_shape.find(key);
        int shape = -1;
        if (it != c->batch_shape.end() && !(flags & PQ_BATCH_AUTOTUNE)) {
            shape = it->second;
        } else {
            float best = 0.f;
            cudaEvent_t e0, e1;
            ck(cudaEventCreate(&e0), "event");
            ck(cudaEventCreate(&e1), "event");
            for (int sh = 0; sh < pq::batched_shapes(); ++sh) {
                if (!pq::batched_shape_fits(sh, int(d), kp)) continue;
                items_for(sh, is, iq);
                // about four waves of the heaviest items, at equal query count per shape
                const uint64_t want_q = uint64_t(4) * sms * 32;
                const uint32_t qpi = uint32_t(pq::batched_queries_per_item(sh));
                const uint32_t cnt = uint32_t(std::min<uint64_t>(is.size(), (want_q + qpi - 1) / qpi));
                upload_items(cnt);
                float ms = 0.f;
                for (int rep = 0; rep < 2; ++rep) {  // the first run loads the kernel
                    ck(cudaMemsetAsync(counter, 0, 4, st), "counter");
                    ck(cudaEventRecord(e0, st), "event");
                    ck(pq::launch_batched_knn(b, sh, st), "batched kNN (autotune)");
                    ck(cudaEventRecord(e1, st), "event");
                    ck(cudaEventSynchronize(e1), "event");
                    ck(cudaEventElapsedTime(&ms, e0, e1), "event");
                }
                if (shape < 0 || ms < best) {
                    shape = sh;
                    best = ms;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            if (shape < 0) throw DeviceError{"no tile shape fits this k and n_dim"};
            c->batch_shape[key] = shape;
        }
        items_for(shape, is, iq);
        upload_items(uint32_t(is.size()));
        if (flags & PQ_BATCH_GRAPH) {
            cudaStream_t cs;
            ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            ck(cudaStreamSynchronize(st), "items");
            ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "capture");
            cudaMemsetAsync(counter, 0, 4, cs);
            pq::launch_batched_knn(b, shape, cs);
            const cudaError_t ce = cudaStreamEndCapture(cs, &g);
            if (ce != cudaSuccess) {
                cudaStreamDestroy(cs);
                ck(ce, "capture");
            }
            ck(cudaGraphInstantiate(&ge, g, 0), "graph");
            ck(cudaGraphLaunch(ge, st), "graph launch");
            ck(cudaStreamSynchronize(st), "graph");
            cudaGraphExecDestroy(ge);
            cudaGraphDestroy(g);
            cudaStreamDestroy(cs);
        } else {
            ck(cudaMemsetAsync(counter, 0, 4, st), "counter");
            ck(pq::launch_batched_knn(b, shape, st), "batched kNN");
        }
        ck(cudaEventRecord(ev, st), "event");
        ck(cudaStreamWaitEvent(user, ev, 0), "event");
        ck(cudaStreamSynchronize(st), "batched kNN");  // the host item arrays are reused
        cudaEventDestroy(ev);
        if (shape_out) *shape_out = shape;
        return PQ_OK;
    });
}

uint64_t pq_mlp_params(uint64_t n_dim) { return pq::mlp_params(int(n_dim)); }

int pq_mlp_grad(pq_ctx* c, uint64_t d, const float* params, const float* X, uint64_t rows,
                const uint32_t* tb, const float* tw, uint32_t T, float* grad_out,
                float* loss_out, float* logits_out) {
    if (!c) return PQ_EINVAL;
    if (!params || !X || !tb || !tw || !grad_out || !loss_out)
        return fail(c, PQ_EINVAL, "null buffer");
    if (d == 0 || d > 4096 || rows == 0 || rows > (1u << 20) || T == 0 || T > 32)
        return fail(c, PQ_EINVAL, "bad sizes");
    return guarded(c, [&]() -> int {
        cudaStream_t st = c->stream;
        const size_t np = pq::mlp_params(int(d));
        ck(cudaMemsetAsync(c->d_err, 0, sizeof(int), st), "err");
        pq::MlpView net{int(d), c->get<float>("mg_w", np),
                        c->get<__nv_bfloat16>("mg_wt", pq::mlp_wt_elems()), c->d_err};
        const pq::MlpBufs b16 = pq::mlp_bufs(
            c->get<uint8_t>("mg_b16", pq::mlp_bufs_bytes(int(rows), true)), int(rows), true);
        float* dx = c->get<float>("mg_x", rows * d);
        uint32_t* dtb = c->get<uint32_t>("mg_tb", rows * T);
        float* dtw = c->get<float>("mg_tw", rows * T);
        float* h1 = c->get<float>("mg_h1", rows * pq::MLP_H);
        float* h2 = c->get<float>("mg_h2", rows * pq::MLP_H);
        float* z = c->get<float>("mg_z", rows * pq::MLP_OUT);
        float* dh1 = c->get<float>("mg_dh1", rows * pq::MLP_H);
        float* dh2 = c->get<float>("mg_dh2", rows * pq::MLP_H);
        float* g = c->get<float>("mg_g", np);
        float* loss = c->get<float>("mg_loss", rows);
        float* scratch = c->get<float>("mg_scratch", pq::mlp_scratch_floats());
        ck(cudaMemcpyAsync(net.w, params, np * 4, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dx, X, rows * d * 4, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dtb, tb, rows * T * 4, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dtw, tw, rows * T * 4, cudaMemcpyHostToDevice, st), "h2d");
        pq::mlp_sync_bf16(net, st);
        ck(pq::mlp_forward(net, dx, int(rows), h1, h2, z, b16, true, st), "mlp forward");
        if (logits_out)
            ck(cudaMemcpyAsync(logits_out, z, rows * pq::MLP_OUT * 4, cudaMemcpyDeviceToHost, st),
               "d2h");
        ck(pq::mlp_backward(net, int(rows), h1, h2, z, b16, dtb, dtw, int(T), loss, dh1, dh2, g,
                            scratch, st),
           "mlp backward");
        ck(cudaMemcpyAsync(grad_out, g, np * 4, cudaMemcpyDeviceToHost, st), "d2h");
        ck(cudaMemcpyAsync(loss_out, loss, rows * 4, cudaMemcpyDeviceToHost, st), "d2h");
        int herr = 0;
        ck(cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "err");
        ck(cudaStreamSynchronize(st), "mlp");
        if (herr) throw DeviceError{"mlp tensor-core products: a bounded wait gave up", herr == 2};
        return PQ_OK;
    });
}

namespace {
int fuzzy_run(pq_ctx* c, uint64_t n, uint64_t nnz, const uint32_t* d_ip, const uint32_t* d_ix,
              const float* d_dx, uint32_t* d_oip, uint32_t* d_oix, float* d_ow, uint64_t out_cap,
              uint64_t* nnz_out, cudaStream_t st) {
    uint8_t* temp = c->get<uint8_t>("fz_temp", pq::fuzzy_temp_bytes(n, nnz));
    uint64_t h = 0;
    const cudaError_t e = pq::launch_fuzzy(n, nnz, d_ip, d_ix, d_dx, temp, d_oip, d_oix, d_ow,
                                           out_cap, c->d_u64, c->d_err, &h, st);
    if (e == cudaErrorNotSupported)
        return fail(c, PQ_ENOTSUP, "a row of the graph has more than 256 entries");
    if (e == cudaErrorInvalidValue)
        return fail(c, PQ_EINVAL, "the connectivity arrays are too short");
    ck(e, "fuzzy connectivities");
    *nnz_out = h;
    return PQ_OK;
}
}  // namespace

int pq_fuzzy_connectivities(pq_ctx* c, uint64_t n, const uint32_t* indptr,
                            const uint32_t* indices, const float* data, uint32_t* out_indptr,
                            uint32_t* out_indices, float* out_weights, uint64_t out_cap,
                            uint64_t* nnz_out) {
    if (!c) return PQ_EINVAL;
    if (!indptr || !indices || !data || !out_indptr || !out_indices || !out_weights || !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    if (n == 0 || n >= 0xFFFFFFFFull) return fail(c, PQ_EINVAL, "n_obs must be in [1, 2^32 - 1)");
    const uint64_t nnz = indptr[n];
    return guarded(c, [&]() -> int {
        cudaStream_t st = c->stream;
        uint32_t* ip = c->get<uint32_t>("fz_ip", n + 1);
        uint32_t* ix = c->get<uint32_t>("fz_ix", std::max<uint64_t>(nnz, 1));
        float* dx = c->get<float>("fz_dx", std::max<uint64_t>(nnz, 1));
        const uint64_t cap = std::max<uint64_t>(2 * nnz, 1);
        uint32_t* oip = c->get<uint32_t>("fz_oip", n + 1);
        uint32_t* oix = c->get<uint32_t>("fz_oix", cap);
        float* ow = c->get<float>("fz_ow", cap);
        ck(cudaMemcpyAsync(ip, indptr, (n + 1) * 4, cudaMemcpyHostToDevice, st), "h2d");
        if (nnz) {
            ck(cudaMemcpyAsync(ix, indices, nnz * 4, cudaMemcpyHostToDevice, st), "h2d");
            ck(cudaMemcpyAsync(dx, data, nnz * 4, cudaMemcpyHostToDevice, st), "h2d");
        }
        uint64_t m = 0;
        const int rc = fuzzy_run(c, n, nnz, ip, ix, dx, oip, oix, ow, cap, &m, st);
        if (rc != PQ_OK) return rc;
        if (m > out_cap) return fail(c, PQ_EINVAL, "the connectivity arrays are too short");
        ck(cudaMemcpyAsync(out_indptr, oip, (n + 1) * 4, cudaMemcpyDeviceToHost, st), "d2h");
        if (m) {
            ck(cudaMemcpyAsync(out_indices, oix, m * 4, cudaMemcpyDeviceToHost, st), "d2h");
            ck(cudaMemcpyAsync(out_weights, ow, m * 4, cudaMemcpyDeviceToHost, st), "d2h");
        }
        ck(cudaStreamSynchronize(st), "d2h");
        *nnz_out = m;
        return PQ_OK;
    });
}

int pq_fuzzy_connectivities_device(pq_ctx* c, uint64_t n, const uint32_t* d_indptr,
                                   const uint32_t* d_indices, const float* d_data, uint64_t nnz,
                                   uint32_t* d_out_indptr, uint32_t* d_out_indices,
                                   float* d_out_weights, uint64_t out_cap, uint64_t* nnz_out,
                                   void* stream) {
    if (!c) return PQ_EINVAL;
    if (!d_indptr || !d_indices || !d_data || !d_out_indptr || !d_out_indices || !d_out_weights ||
        !nnz_out)
        return fail(c, PQ_EINVAL, "null buffer");
    if (n == 0 || n >= 0xFFFFFFFFull) return fail(c, PQ_EINVAL, "n_obs must be in [1, 2^32 - 1)");
    return guarded(c, [&]() -> int {
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        cudaEvent_t ev;
        ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ev, user), "event");
        ck(cudaStreamWaitEvent(c->stream, ev, 0), "event");
        const int rc = fuzzy_run(c, n, nnz, d_indptr, d_indices, d_data, d_out_indptr,
                                 d_out_indices, d_out_weights, out_cap, nnz_out, c->stream);
        ck(cudaEventRecord(ev, c->stream), "event");
        ck(cudaStreamWaitEvent(user, ev, 0), "event");
        cudaEventDestroy(ev);
        return rc;
    });
}

}  // extern "C"
