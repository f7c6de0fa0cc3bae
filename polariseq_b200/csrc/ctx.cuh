// Host-side context and helpers shared by the plain and chosen forms.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/polariseq_knn.h"
#include "common.cuh"

namespace pqh {

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Resolved {
    uint64_t k, max_cand, n_iters, n_trees, leaf_size, stop_at;
};

struct DeviceError {
    std::string msg;
    bool timeout = false;  // a bounded device-side wait gave up (PQ_ETIMEOUT)
};

inline void ck(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw DeviceError{std::string(where) + ": " + cudaGetErrorString(e)};
}

inline uint64_t effective_k(uint64_t n, uint64_t k) {
    uint64_t m = n > 0 ? n - 1 : 0;
    uint64_t e = k < m ? k : m;
    return e > 0 ? e : 1;
}

// NndescentOptions resolution (nndescent.rs:722-752) and stop_at (:850).
inline Resolved resolve(uint64_t n, const pq_nnd_opts& o) {
    Resolved r;
    r.k = effective_k(n, o.k);
    uint64_t mc = o.max_candidates > 0 ? o.max_candidates : std::min<uint64_t>(2 * r.k, 60);
    r.max_cand = mc > 0 ? mc : 1;
    if (o.max_iterations > 0) {
        r.n_iters = o.max_iterations;
    } else {
        double lg = std::round(std::log2(double(n)));
        uint64_t it = lg > 0 ? uint64_t(lg) : 0;
        r.n_iters = it > 5 ? it : 5;
    }
    if (o.n_trees > 0) {
        r.n_trees = o.n_trees;
    } else {
        double t = std::round(std::sqrt(double(n)) / 10.0);
        r.n_trees = std::min<uint64_t>(8 + uint64_t(t), 48);
    }
    r.leaf_size = o.leaf_size > 0 ? o.leaf_size : std::max<uint64_t>(r.k, 10);
    double sa = o.delta * double(n) * double(r.k);
    r.stop_at = (sa > 0 && sa == sa) ? (sa >= 1.8e19 ? UINT64_MAX : uint64_t(sa)) : 0;
    return r;
}

inline int key_bits(uint64_t maxkey) {
    int b = 0;
    while (b < 32 && (maxkey >> b) != 0) ++b;
    return b > 0 ? b : 1;
}

inline unsigned blocks(size_t n, int t) { return unsigned((n + t - 1) / t); }

struct Timer {
    cudaEvent_t a, b;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void start() { cudaEventRecord(a, s); }
    double stop() {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

}  // namespace pqh

struct pq_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    pq_nnd_stats stats{};
    std::map<std::string, pqh::Buf> bufs;
    int* d_err = nullptr;
    uint64_t* d_u64 = nullptr;            // small device scalars
    unsigned long long* d_acc = nullptr;  // device accumulators
    cudaStream_t stream2 = nullptr;  // the largest subtrees run here, concurrently
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int profile = 0;
    uint32_t test_wait_polls = 0;  // pq_ctx_set_test_wait: the next tile passes give up
    struct KGRec {
        cudaEvent_t a, b;
        int group;
        unsigned long long launches;
    };
    std::vector<KGRec> kg_pending;
    std::map<uint64_t, int> batch_shape;  // autotuned tile shape per (dims, heap size)
    // the learned-init subsample's plain graph is built on this context, kept
    // from build to build (its workspace is not reallocated each time)
    pq_ctx* sub = nullptr;

    template <class T>
    T* get(const std::string& name, size_t count) {
        size_t need = count * sizeof(T);
        if (need == 0) need = 16;
        pqh::Buf& b = bufs[name];
        if (b.bytes < need) {
            if (b.p) {
                cudaStreamSynchronize(stream);
                cudaFree(b.p);
                b.p = nullptr;
                b.bytes = 0;
            }
            size_t alloc = need + need / 8;  // headroom for slightly larger calls
            if (cudaMalloc(&b.p, alloc) != cudaSuccess) {
                cudaGetLastError();
                throw std::string("device allocation of ") + std::to_string(alloc) +
                    " bytes failed (" + name + ")";
            }
            b.bytes = alloc;
        }
        return static_cast<T*>(b.p);
    }
};

namespace pqh {

// Brackets one kernel group with CUDA events on the context's stream when
// profiling is on; the records are summed into the stats at the end.
struct KGScope {
    pq_ctx* c;
    int g;
    cudaEvent_t a{}, b{};
    unsigned long long l0;
    KGScope(pq_ctx* c_, int g_) : c(c_), g(g_), l0(pq::g_launches) {
        if (c->profile) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, c->stream);
        }
    }
    ~KGScope() {
        if (c->profile) {
            cudaEventRecord(b, c->stream);
            c->kg_pending.push_back({a, b, g, pq::g_launches - l0});
        }
    }
};

inline void kg_collect(pq_ctx* c) {
    cudaStreamSynchronize(c->stream);
    for (auto& r : c->kg_pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        c->stats.kg_ms[r.group] += ms;
        c->stats.kg_launches[r.group] += r.launches;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    c->kg_pending.clear();
}

// The caller's row-major n x d f32 embedding (host or device) as padded rows
// X[n][dp] in the context's workspace, 16-byte aligned and zero padded, on
// stream st (null: the context's stream) (api.cu).
float* load_embedding(pq_ctx* c, const float* data, bool on_host, uint32_t n, int d, int dp,
                      cudaStream_t st = nullptr);
// Host rows [r0, r1) of the caller's n x d embedding into the padded rows X
// (the same workspace as load_embedding), on stream st; returns X.
float* load_embedding_rows(pq_ctx* c, const float* data, uint32_t n, int d, int dp, uint32_t r0,
                           uint32_t r1, cudaStream_t st);

// NN-Descent rounds on heaps in place (api.cu).
int run_rounds(pq_ctx* c, const float* X, int d, int dp, uint32_t n, int k, int m, uint64_t seed,
               uint64_t n_iters, uint64_t stop_at, uint32_t* hidx, float* hdist, uint8_t* hflag,
               const uint32_t* perm, int stats_offset,
               const std::function<bool(int, const uint32_t*, const uint32_t*)>& after_round);

// Learned probes (learned.cu): probes[i * P] = primary[i], then the MLP's P - 1
// most likely other buckets; trains the MLP on a subsample's plain graph.
// Returns the routing (inference) time in ms; *ms_train gets the training time.
double learned_probes(pq_ctx* c, const float* X, int d, int dp, uint32_t n, uint32_t C,
                      const uint32_t* primary, const float* primary_d, const float* cent, int P,
                      uint64_t seed, uint32_t* probes, double* ms_train, double* loss_first,
                      double* loss_last);

// Host destinations of the graph: a build may copy its CSR there itself,
// overlapping the copy with its last stage (copied = true), else the caller
// copies the device arrays.
struct HostGraph {
    uint32_t* indptr;
    uint32_t* indices;
    float* dists;
    bool copied;
};

}  // namespace pqh

namespace pq {
// recall@k of the graph (device CSR) on Q seeded sampled cells against their
// exact FP32 k nearest (recall.cu).
double sampled_recall(pq_ctx* c, const float* X, int d, int dp, uint32_t n, int k,
                      const uint32_t* d_indptr, const uint32_t* d_indices, uint32_t Q,
                      uint64_t seed);
}  // namespace pq

namespace pqh {

// The chosen form (tensor-core shortlist), chosen.cu.
uint64_t build_chosen(pq_ctx* c, const float* data, bool data_on_host, uint64_t n64,
                      uint64_t d64, const pq_nnd_opts& o, uint32_t* d_indptr,
                      uint32_t* d_indices, float* d_dists, HostGraph* host = nullptr);

}  // namespace pqh
