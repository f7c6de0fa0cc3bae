// ORACLE — test infrastructure only, never shipped and never on the product path.
//
// 1. An FP64 exact brute-force kNN over sampled queries: distances are
//    sum((double)x - (double)y)^2, self excluded, ties broken by
//    (distance, index) as the reference's exact Scrublet search orders them
//    (crates/polariseq-core/src/doublets.rs:544-546).  Recall@k is
//    |approx ∩ exact| / k averaged over queries, the definition of
//    nndescent.rs:1038-1056 and python/polariseq/tests/test_neighbors.py:26-29.
// 2. A restatement of the reference's exact f32 search `neighbors::neighbors`
//    (crates/polariseq-core/src/neighbors.rs:101-241): per-query bounded
//    max-heap over all points in index order, sort, sqrt, self dropped.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline float reduce8(const float* a) {
    return ((a[0] + a[4]) + (a[1] + a[5])) + ((a[2] + a[6]) + (a[3] + a[7]));
}

inline float sq_dist(const float* a, const float* b, size_t d) {  // simd.rs:43-62
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t full = d / 8 * 8;
    for (size_t c = 0; c < full; c += 8)
        for (int l = 0; l < 8; ++l) {
            float t = a[c + l] - b[c + l];
            acc[l] = acc[l] + t * t;
        }
    float tail = 0.0f;
    for (size_t j = full; j < d; ++j) {
        float t = a[j] - b[j];
        tail = tail + t * t;
    }
    return reduce8(acc) + tail;
}

inline float dot(const float* a, const float* b, size_t d) {  // simd.rs:20-36
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t full = d / 8 * 8;
    for (size_t c = 0; c < full; c += 8)
        for (int l = 0; l < 8; ++l) acc[l] = acc[l] + a[c + l] * b[c + l];
    float tail = 0.0f;
    for (size_t j = full; j < d; ++j) tail = tail + a[j] * b[j];
    return reduce8(acc) + tail;
}

struct Nb {
    float dist;
    uint32_t idx;
};

// knn_for_one (neighbors.rs:151-223).
void knn_for_one(const float* emb, size_t n, size_t d, size_t query, size_t k, int cosine,
                 std::vector<Nb>& heap) {
    const float* qv = emb + query * d;
    heap.clear();
    auto sift_down = [&](size_t p) {
        size_t len = heap.size();
        for (;;) {
            size_t l = 2 * p + 1, r = 2 * p + 2, m = p;
            if (l < len && heap[l].dist > heap[m].dist) m = l;
            if (r < len && heap[r].dist > heap[m].dist) m = r;
            if (m == p) break;
            std::swap(heap[p], heap[m]);
            p = m;
        }
    };
    for (size_t j = 0; j < n; ++j) {
        const float* o = emb + j * d;
        float dd;
        if (!cosine) {
            dd = sq_dist(qv, o, d);
        } else {  // cosine_dist (neighbors.rs:231-241)
            float dt = dot(qv, o, d), na = dot(qv, qv, d), nb = dot(o, o, d);
            float den = std::sqrt(na) * std::sqrt(nb);
            dd = den > 0.0f ? 1.0f - dt / den : 1.0f;
        }
        if (heap.size() < k) {
            heap.push_back({dd, uint32_t(j)});
            size_t c = heap.size() - 1;
            while (c > 0) {
                size_t parent = (c - 1) / 2;
                if (heap[c].dist > heap[parent].dist) {
                    std::swap(heap[c], heap[parent]);
                    c = parent;
                } else {
                    break;
                }
            }
        } else if (dd < heap[0].dist) {
            heap[0] = {dd, uint32_t(j)};
            sift_down(0);
        }
    }
    std::stable_sort(heap.begin(), heap.end(),
                     [](const Nb& a, const Nb& b) { return a.dist < b.dist; });
    if (!cosine)
        for (Nb& e : heap) e.dist = std::sqrt(e.dist);
}

}  // namespace

extern "C" {

// FP64 exact kNN of `nq` query rows against all n rows, self excluded,
// (distance, index) order.  out_idx/out_dist are nq*k (squared distances).
void oracle_exact_knn_f64(const float* data, uint64_t n, uint64_t d, const uint32_t* queries,
                          uint64_t nq, uint64_t k, uint32_t* out_idx, double* out_dist) {
#pragma omp parallel
    {
        std::vector<std::pair<double, uint32_t>> buf;
#pragma omp for schedule(dynamic, 4)
        for (uint64_t qi = 0; qi < nq; ++qi) {
            uint32_t q = queries[qi];
            const float* xq = data + size_t(q) * d;
            buf.clear();
            buf.reserve(n);
            for (uint64_t j = 0; j < n; ++j) {
                if (j == q) continue;
                const float* xj = data + size_t(j) * d;
                double s = 0.0;
                for (uint64_t t = 0; t < d; ++t) {
                    double df = double(xq[t]) - double(xj[t]);
                    s += df * df;
                }
                buf.emplace_back(s, uint32_t(j));
            }
            size_t kk = std::min<size_t>(k, buf.size());
            std::partial_sort(buf.begin(), buf.begin() + kk, buf.end());
            for (size_t t = 0; t < k; ++t) {
                out_idx[qi * k + t] = t < kk ? buf[t].second : 0xFFFFFFFFu;
                out_dist[qi * k + t] = t < kk ? buf[t].first : INFINITY;
            }
        }
    }
}

// neighbors::neighbors (neighbors.rs:101-147): returns 0, or the error the
// reference raises: -1 empty input, -3 zero neighbours.
int oracle_neighbors_exact(const float* emb, uint64_t n, uint64_t d, uint64_t n_neighbors,
                           int cosine, uint32_t* indptr, uint32_t* indices, float* dists) {
    if (n == 0 || d == 0) return -1;
    if (n_neighbors == 0) return -3;
    size_t kws = std::min<uint64_t>(n_neighbors, n);
    size_t per = kws - 1;
    std::vector<std::vector<Nb>> rows(n);
#pragma omp parallel
    {
        std::vector<Nb> heap;
#pragma omp for schedule(dynamic, 16)
        for (uint64_t i = 0; i < n; ++i) {
            knn_for_one(emb, n, d, i, kws, cosine, heap);
            rows[i] = heap;
        }
    }
    indptr[0] = 0;
    size_t pos = 0;
    for (uint64_t i = 0; i < n; ++i) {
        for (size_t t = 1; t < rows[i].size(); ++t) {  // skip(1) drops the closest (self)
            indices[pos] = rows[i][t].idx;
            dists[pos] = rows[i][t].dist;
            ++pos;
        }
        indptr[i + 1] = uint32_t(pos);
    }
    (void)per;
    return 0;
}

}  // extern "C"
