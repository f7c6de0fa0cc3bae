/*
 * polariseq-knn-b200: C ABI of the B200 (sm_100a) kNN-graph builder.
 *
 * Drop-in for the reference's NN-Descent entry points:
 *   - Rust  polariseq_core::nndescent::nndescent_into
 *           (crates/polariseq-core/src/nndescent.rs:688-707)
 *   - Rust  polariseq_core::nndescent::nndescent / effective_k
 *           (nndescent.rs:648-686)
 *   - PyO3  _polariseq.nndescent_dense(embedding, k, max_iterations=0, seed=0,
 *           max_candidates=0, n_trees=0, delta=0.001, out=None)
 *           (crates/polariseq-python/src/lib.rs:503-566)
 * A Rust `CudaBackend` (the ComputeBackend slot, crates/polariseq-core/src/
 * backend.rs:68-94) binds these symbols through `extern "C"`; the Python
 * package `polariseq_b200` binds them through ctypes.
 *
 * Plain pointers and sizes only; every function returns a pq_status.  Errors
 * that the reference raises as panics (empty data, k == 0, short output
 * arrays) come back as PQ_EINVAL with a message from pq_ctx_last_error().
 */
#ifndef POLARISEQ_KNN_H
#define POLARISEQ_KNN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pq_status {
    PQ_OK = 0,
    PQ_EINVAL = 1,   /* bad shape / option / output size (reference: panic or ValueError) */
    PQ_ENOMEM = 2,   /* device allocation failed */
    PQ_EDEVICE = 3,  /* CUDA error, no device, or a kernel reported an error flag */
    PQ_ETIMEOUT = 4, /* a bounded device-side wait gave up */
    PQ_ENOTSUP = 5,  /* option combination not supported by this build */
    PQ_ETOOBIG = 6   /* input beyond the fixed capacity of an allocation-free entry point */
} pq_status;

/* Metric of the exact search (neighbors.rs:16-39). */
enum { PQ_METRIC_EUCLIDEAN = 0, PQ_METRIC_COSINE = 1 };

/* Search form.  PLAIN reproduces the reference graph bit for bit; BF16 and
 * FP8 are the tensor-core shortlist forms (FP8: E4M3 tiles, every query and
 * candidate row with its own power-of-two scale); both take k <= 31. */
enum { PQ_MODE_PLAIN = 0, PQ_MODE_BF16 = 1, PQ_MODE_FP8 = 2 };
/* Initial neighbour lists: the reference's RP-tree forest, or learned buckets
 * (n_obs >= 65,536, n_dim <= 62, k <= 31): an MLP trained on a subsample's
 * plain graph routes each cell to the buckets its neighbours live in.
 *   - with PQ_MODE_BF16 / PQ_MODE_FP8 the router chooses the buckets each
 *     cell's shortlist searches;
 *   - with PQ_MODE_PLAIN it is the learned-init NN-Descent: each cell's
 *     initial list is its k nearest within its `probes` (default 12) most
 *     likely buckets (BF16 tensor-core tiles, exact FP32 re-rank), in place
 *     of the RP forest + random fill (nndescent.rs:768-845); the reference's
 *     rounds (max_iterations, delta, max_candidates) then run to
 *     convergence.  Its recall is estimated on 1,024 sampled cells against
 *     their exact FP32 neighbours; below 0.99 the RP-initialised build runs
 *     too (the fallback) and the graph with the higher estimate is kept
 *     (pq_nnd_stats.fell_back / est_recall*).  Not bit-exact with the
 *     RP-initialised graph. */
enum { PQ_INIT_RP = 0, PQ_INIT_LEARNED = 1 };

/* Mirrors NndescentOptions (nndescent.rs:42-76): zero = auto for the sized
 * fields, resolved exactly as nndescent.rs:722-752 does. */
typedef struct pq_nnd_opts {
    uint64_t k;              /* neighbours per cell (reference default 15) */
    uint64_t max_candidates; /* 0 -> min(60, 2k) */
    uint64_t max_iterations; /* 0 -> max(5, round(log2 n)) */
    double delta;            /* stop when changed <= delta*n*k (default 0.001) */
    uint64_t n_trees;        /* 0 -> min(48, 8 + round(sqrt(n)/10)) */
    uint64_t leaf_size;      /* 0 -> max(10, k) */
    uint64_t gather_max;     /* accepted for API parity; never changes the graph */
    uint64_t seed;
    int32_t mode;            /* PQ_MODE_* */
    int32_t init;            /* PQ_INIT_* */
    /* Tensor-core forms only (ignored by PQ_MODE_PLAIN): */
    int32_t probes;          /* buckets each cell searches (<= 16); 0 -> min(13, buckets)
                              * (14 for k > 15, 16 from 6M cells), 6 with PQ_INIT_LEARNED (1024 buckets,
                              * own bucket + MLP), 12 for the learned-init NN-Descent */
    int32_t refine_rounds;   /* NN-Descent rounds after the shortlist; -1 -> auto (none; one
                              * for FP8 below 2^20 cells) */
    int32_t buckets;         /* k-means buckets; 0 -> round(n / 4096), 1024 with PQ_INIT_LEARNED */
} pq_nnd_opts;

/* Per-call statistics of the last build on a context. */
typedef struct pq_nnd_stats {
    int32_t rounds_run;
    int32_t n_trees;
    uint64_t k, max_candidates, n_iters, leaf_size, stop_at;
    uint64_t changed[64];    /* heap entries changed per round */
    uint64_t emitted[64];    /* join updates that passed a threshold per round */
    uint64_t pairs[64];      /* join distances evaluated per round */
    double ms_forest, ms_leaves, ms_rounds, ms_extract, ms_total;
    uint64_t launches;       /* kernels launched by the last build */
    /* With profiling on (pq_ctx_set_profiling): CUDA-event time and launch
     * count per kernel group, indexed by PQ_KG_*. */
    double kg_ms[16];
    uint64_t kg_launches[16];
    /* Tensor-core form: [0] 128x256 tile pairs, [1] largest bucket, [2] buckets,
     * [3] (query entry, candidate) distances contracted, [4] / [5] tile pairs of
     * the primary pass / the other probes, [6] FP64 boundary resolutions,
     * [7] other-probe entries dropped (a lower bound shows they can admit no
     * candidate). */
    uint64_t shortlist[8];
    /* PQ_INIT_LEARNED: mean training loss of the first and of the last epoch
     * (the untrained router is the nearest-centroid prior), and the time of
     * the subsample graph + training, and of routing every cell, in ms. */
    double learn_loss_first, learn_loss_last, ms_learn_train, ms_learn_route;
    /* Learned-init NN-Descent (PQ_MODE_PLAIN + PQ_INIT_LEARNED): recall@k
     * estimated on sampled cells for the returned graph, for the learned-init
     * graph and for the RP-initialised fallback (0 when it did not run);
     * fell_back = 1 when the fallback ran, 2 when its graph was kept. */
    double est_recall, est_recall_learned, est_recall_rp;
    int32_t fell_back;
    int32_t learned_rounds;  /* rounds the learned-init build ran */
} pq_nnd_stats;

/* Kernel groups timed by the profiling mode. */
enum {
    PQ_KG_FOREST_TOP = 0,  /* top-level hyperplanes, margins and partition */
    PQ_KG_SEQTREE = 1,     /* depth-first subtrees */
    PQ_KG_LEAF_PAIRS = 2,  /* leaf all-pairs replay + random fill */
    PQ_KG_CANDIDATES = 3,  /* candidate records, their sort and replay, flag flip */
    PQ_KG_JOIN_COUNT = 4,  /* join pass 1: distances and emit bits */
    PQ_KG_JOIN_WRITE = 5,  /* join pass 2: records in generation order */
    PQ_KG_SORT = 6,        /* stable sort of join records by destination */
    PQ_KG_REPLAY = 7,      /* per-destination replay of join records */
    PQ_KG_EXTRACT = 8,     /* sorted CSR extract */
    PQ_KG_BUCKETS = 9,     /* tensor-core form: k-means buckets and every cell's probes */
    PQ_KG_LAYOUT = 10,     /* tensor-core form: bucket-ordered BF16 rows and query entries */
    PQ_KG_TILES = 11,      /* tensor-core form: the shortlist tile kernel (one launch per pass) */
    PQ_KG_RERANK = 12,     /* tensor-core form: exact re-rank with the FP64 boundary step */
    PQ_KG_COUNT = 13
};

typedef struct pq_ctx pq_ctx;

/* Fills the reference defaults (NndescentOptions::default, nndescent.rs:64-76). */
void pq_nnd_opts_default(pq_nnd_opts* opts);

/* effective_k (nndescent.rs:648-650): k.min(n_obs - 1).max(1). */
uint64_t pq_effective_k(uint64_t n_obs, uint64_t k);

/* One context per device and caller thread; owns a stream and a device
 * workspace that grows on demand and is reused across calls. */
int pq_ctx_create(int device, pq_ctx** out);
void pq_ctx_destroy(pq_ctx* ctx);
const char* pq_ctx_last_error(const pq_ctx* ctx);
int pq_ctx_stats(const pq_ctx* ctx, pq_nnd_stats* out);
/* Measurement hook: when on, each kernel group of a build is bracketed by
 * CUDA events on the context's stream (pq_nnd_stats.kg_ms / kg_launches). */
int pq_ctx_set_profiling(pq_ctx* ctx, int on);

/* Test hook of the bounded device waits (no counterpart in the reference):
 * with polls > 0, the next tensor-core build's shortlist tile kernels first
 * wait `polls` polls on an mbarrier that nothing arrives at, before issuing
 * any copy or MMA; the wait gives up, the kernels exit with nothing in
 * flight and the build returns PQ_ETIMEOUT.  Applies to one build, after
 * which the context is usable as before. */
int pq_ctx_set_test_wait(pq_ctx* ctx, uint32_t polls);

/* nndescent_into (nndescent.rs:688-707) with HOST buffers: data is n_obs x
 * n_dim row-major f32; indptr holds n_obs+1 entries; indices/dists hold at
 * least n_obs * effective_k(n_obs, k).  Writes the CSR graph (Euclidean
 * distances, ascending per row) and *nnz_out; entries past nnz untouched. */
int pq_nndescent_into(pq_ctx* ctx, const float* data, uint64_t n_obs, uint64_t n_dim,
                      const pq_nnd_opts* opts, uint32_t* indptr, uint64_t indptr_len,
                      uint32_t* indices, uint64_t indices_len, float* dists,
                      uint64_t dists_len, uint64_t* nnz_out);

/* The same with DEVICE buffers on the context's device; `stream` (a
 * cudaStream_t, may be null) is ordered before and after the build. */
int pq_nndescent_into_device(pq_ctx* ctx, const float* d_data, uint64_t n_obs, uint64_t n_dim,
                             const pq_nnd_opts* opts, uint32_t* d_indptr, uint32_t* d_indices,
                             float* d_dists, uint64_t* nnz_out, void* stream);

/* Parity probe (test hook): runs the plain form up to `stop_after` (-1: after
 * forest + random fill; r >= 0: after round r's apply) and copies the neighbour
 * heaps (n*k idx/dist/flag) and, for r >= 0, that round's candidate heaps
 * (n*m new/old), to HOST buffers; any pointer may be null. */
int pq_nndescent_probe(pq_ctx* ctx, const float* data, uint64_t n_obs, uint64_t n_dim,
                       const pq_nnd_opts* opts, int32_t stop_after, uint32_t* heap_idx,
                       float* heap_dist, uint8_t* heap_flag, uint32_t* cand_new,
                       uint32_t* cand_old);

/* One RP tree of the forest (test hook): tree t's permutation ids (n) and its
 * leaf ranges (2 * n_leaves, DFS order) to HOST buffers, as build_tree
 * (nndescent.rs:643-646) with seed splitmix(opts.seed ^ (t + 1)). */
int pq_debug_tree(pq_ctx* ctx, const float* data, uint64_t n_obs, uint64_t n_dim,
                  const pq_nnd_opts* opts, uint32_t tree, uint32_t* ids, uint32_t* leaves,
                  uint64_t leaves_cap, uint64_t* n_leaves);

/* neighbors::neighbors (crates/polariseq-core/src/neighbors.rs:101-147), the
 * exact brute-force kNN behind PyO3 neighbors_dense (crates/polariseq-python/
 * src/lib.rs:474-501), bit for bit: each cell's k_with_self = min(n_neighbors,
 * n_obs) nearest are searched including itself and the closest is dropped, so
 * every row has k_with_self - 1 entries; distances are Euclidean (sqrt of the
 * reference's squared distance) or cosine (1 - cos).  HOST buffers: indptr
 * n_obs+1, indices/dists at least n_obs * (k_with_self - 1).  Errors follow
 * NeighborsError (neighbors.rs:62-84): PQ_EINVAL for empty input, zero
 * neighbours or an unknown metric; PQ_ENOTSUP above n_dim 512 or
 * k_with_self 256. */
int pq_neighbors_into(pq_ctx* ctx, const float* data, uint64_t n_obs, uint64_t n_dim,
                      uint64_t n_neighbors, int32_t metric, uint32_t* indptr,
                      uint64_t indptr_len, uint32_t* indices, uint64_t indices_len,
                      float* dists, uint64_t dists_len, uint64_t* nnz_out);

/* The same with DEVICE buffers (data n_obs x n_dim row-major f32, any
 * alignment); `stream` (a cudaStream_t, may be null) is ordered before and
 * after the search.  The context's workspace holds the cosine row norms. */
int pq_neighbors_into_device(pq_ctx* ctx, const float* d_data, uint64_t n_obs, uint64_t n_dim,
                             uint64_t n_neighbors, int32_t metric, uint32_t* d_indptr,
                             uint32_t* d_indices, float* d_dists, uint64_t* nnz_out,
                             void* stream);

/* umap::fuzzy_connectivities_from (crates/polariseq-core/src/umap.rs:122-138,
 * 283-620; PyO3 fuzzy_connectivities, crates/polariseq-python/src/lib.rs:
 * 568-589): the symmetrised fuzzy simplicial set of a kNN distance graph —
 * per-row membership strengths (smooth_knn_dist), their transpose, and the
 * fuzzy union a + b - a*b per pair, pruned at 1e-5 — as a symmetric CSR with
 * both directions stored, rows sorted by column, no self-loops.  HOST
 * buffers: the distance graph (indptr n_obs+1, indices/data indptr[n_obs]);
 * the result needs at most 2 * indptr[n_obs] entries (out_cap).  Rows of the
 * input may hold at most 256 entries (PQ_ENOTSUP beyond). */
int pq_fuzzy_connectivities(pq_ctx* ctx, uint64_t n_obs, const uint32_t* indptr,
                            const uint32_t* indices, const float* data, uint32_t* out_indptr,
                            uint32_t* out_indices, float* out_weights, uint64_t out_cap,
                            uint64_t* nnz_out);

/* The same on DEVICE buffers (nnz = the input's entry count), so the graph of
 * pq_nndescent_into_device / pq_neighbors_into_device is used where it is;
 * synchronises the context's stream once (to size the result). */
int pq_fuzzy_connectivities_device(pq_ctx* ctx, uint64_t n_obs, const uint32_t* d_indptr,
                                   const uint32_t* d_indices, const float* d_data, uint64_t nnz,
                                   uint32_t* d_out_indptr, uint32_t* d_out_indices,
                                   float* d_out_weights, uint64_t out_cap, uint64_t* nnz_out,
                                   void* stream);

/* Learned bucket routing (PQ_INIT_LEARNED), test hooks: the parameter count
 * of the d -> 256 -> 256 -> 1024 MLP (layout W1 [d x 256], b1, W2 [256 x 256],
 * b2, W3 [256 x 1024], b3, row-major f32), and one forward + backward pass on
 * HOST buffers: weights used in BF16 (rounded from `params`), biases in FP32,
 * softmax cross-entropy against T sparse (bucket, weight) targets per row
 * (bucket 0xFFFFFFFF unused); writes the gradients of the mean loss, the
 * per-row losses and (if not null) the logits (rows x 1024). */
uint64_t pq_mlp_params(uint64_t n_dim);
int pq_mlp_grad(pq_ctx* ctx, uint64_t n_dim, const float* params, const float* X, uint64_t rows,
                const uint32_t* tb, const float* tw, uint32_t T, float* grad_out,
                float* loss_out, float* logits_out);

/* Flags of pq_knn_batched_into_device. */
enum { PQ_BATCH_AUTOTUNE = 1, PQ_BATCH_GRAPH = 2 };

/* Batched exact kNN: every point's k_s nearest other points within its own
 * sample, for n_samples samples of uneven size in ONE persistent,
 * work-queued launch — the per-sample searches of doublet scoring
 * (crates/polariseq-core/src/doublets.rs:544-650 knn_exact: exact, itself
 * excluded, ties by index, ascending).  d_data holds all samples' rows back
 * to back (row-major f32, n_dim <= 64); offsets (HOST, n_samples + 1, rows)
 * delimit the samples; ks (HOST) gives each sample's k (1 <= k < its size,
 * k <= 512).  Sample s's rows write k_s entries each, back to back from
 * sum_{t<s} n_t * k_t: indices local to the sample, Euclidean distances.
 * PQ_BATCH_AUTOTUNE re-times the tile shapes (otherwise the context's choice
 * for this n_dim and k range is reused, timing them on first use);
 * PQ_BATCH_GRAPH captures the launch in a CUDA graph and replays it.
 * *shape_out (may be null) receives the tile shape used. */
int pq_knn_batched_into_device(pq_ctx* ctx, const float* d_data, uint64_t n_dim,
                               uint32_t n_samples, const uint64_t* offsets, const uint32_t* ks,
                               uint32_t* d_indices, float* d_dists, int32_t flags,
                               int32_t* shape_out, void* stream);

/* Doublet scoring of many samples after their PCA (the steps of Scrublet's
 * score_batch in crates/polariseq-core/src/doublets.rs:1040-1127), on the
 * GPU.  Sample s has n_cells[s] cells and n_sim[s] simulated doublets, p <= 64
 * components.  DEVICE inputs, samples back to back: d_u (f64, cells x p:
 * each cell's counts over the gene deviations, projected), d_w and d_totals
 * (f64 per cell: 1e6 / total and the total), d_mv (f64, n_samples x p: the
 * projected gene means), d_pairs (u32, 2 per doublet: its two parents, cell
 * indices local to the sample).  Each sample's points are its cells
 * (w u - mv) and doublets (1e6 / (total_x + total_y) (u_x + u_y) - mv) in f32
 * from f64 arithmetic in the reference's order; the exact kNN of every point
 * within its sample runs in one persistent launch (pq_knn_batched_into_device)
 * with k_adj = round_half_even(k (1 + n_sim / n)) neighbours; every point's
 * score is the reference's Bayesian score from its simulated neighbours
 * (q = (n_d + 1) / (k_adj + 2), rho the expected doublet rate), f64 into
 * d_score_obs (cells) and d_score_sim (doublets), back to back.  Optional
 * outputs (may be null): k_adj_out (HOST, per sample), d_pts_out (f32, all
 * points x p) and d_knn_out (u32, each point's k_adj neighbours).  The
 * threshold between the score modes (threshold_from_simulated) stays with the
 * caller. */
int pq_scrublet_scores_device(pq_ctx* ctx, uint32_t n_samples, uint64_t p,
                              const uint64_t* n_cells, const uint64_t* n_sim, const uint32_t* k,
                              const double* d_u, const double* d_w, const double* d_totals,
                              const double* d_mv, const uint32_t* d_pairs, double rho,
                              double* d_score_obs, double* d_score_sim, uint32_t* k_adj_out,
                              float* d_pts_out, uint32_t* d_knn_out, void* stream);

/* Allocation-free exact kNN.  No counterpart in the reference: it is an
 * addition of this library for callers that must not allocate device memory,
 * such as a host framework that owns the whole device budget through its own
 * pool (a cudaMalloc outside it can push the framework out of memory), or a
 * serving loop where cudaMalloc / cudaFree would synchronise the device and
 * stall the work of other streams.  It computes exactly what
 * pq_neighbors_into_device computes, with DEVICE buffers the caller passes,
 * enqueued on `stream` (a cudaStream_t, may be null) of the current device; it
 * needs no context, calls no allocator and does not wait for the GPU.
 *
 * Limit: n_obs <= 262144 (PQ_ETOOBIG beyond), n_dim <= 512 and
 * min(n_neighbors, n_obs) <= 256 (PQ_ENOTSUP beyond).  The cosine metric keeps
 * per-row norms in one fixed 1 MiB device array inside the library, shared by
 * every call on that device: nothing in it needs to start at zero (each call
 * writes the norms it reads before reading them), but calls whose work
 * overlaps on the GPU (other streams, other host threads) race on it, so
 * order them.  The first call on each device does a one-time set-up (looks up
 * that array's device address and loads the kernels): make it before any
 * stream capture.  Errors: PQ_EINVAL (null buffer, empty data, zero
 * neighbours, unknown metric), PQ_ETOOBIG, PQ_ENOTSUP, PQ_EDEVICE. */
int pq_neighbors_into_device_noalloc(const float* d_data, uint64_t n_obs, uint64_t n_dim,
                                     uint64_t n_neighbors, int32_t metric, uint32_t* d_indptr,
                                     uint32_t* d_indices, float* d_dists, uint64_t* nnz_out,
                                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* POLARISEQ_KNN_H */
