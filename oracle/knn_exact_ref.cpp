// ORACLE (test infrastructure and CPU baseline only; never linked by the
// product): a restatement of the reference's exact per-sample kNN of doublet
// scoring, `knn_exact` (crates/polariseq-core/src/doublets.rs:544-650), and of
// the way scoring runs samples (doublets.rs:1369-1374: samples in parallel,
// largest first; inside a sample, query tiles in parallel).
//
// Per query tile of 128 rows, the points are walked in blocks of 2,048; a
// block's squared distances are |q|^2 + |p|^2 - 2 p.q from one dot-product
// block (the reference takes p.q from a faer matmul, whose FP32 summation
// order is a third-party detail: the results here are exact sets, not bits).
// Each query keeps the candidates within its current k-th distance in a
// buffer of 2k (+ one run of slack); a run of 16 candidates is turned away at
// once when none is within reach; a full buffer is cut to its k nearest by
// one selection, ordered by (distance, index) (doublets.rs:540-545).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>

namespace {

using Cand = std::pair<float, uint32_t>;

inline bool by_distance(const Cand& a, const Cand& b) {
    if (a.first != b.first) return a.first < b.first;
    return a.second < b.second;
}

// One tile of queries [q0, q0 + rows) of a sample with n points.
void knn_tile(const float* p, const float* norms, size_t n, int d, int k, size_t q0, int rows,
              uint32_t* out) {
    constexpr size_t BLOCK = 2048;
    constexpr int RUN = 16;
    const int cap = 2 * k + RUN;
    std::vector<Cand> bufs(size_t(rows) * cap);
    std::vector<int> used(rows, 0);
    std::vector<float> reach(rows, INFINITY);
    std::vector<float> dots(BLOCK * size_t(rows));
    std::vector<float> xt(BLOCK * size_t(d));  // the block's points, dimension-major
    auto shrink = [k](Cand* buf, int len) -> float {
        std::nth_element(buf, buf + (k - 1), buf + len, by_distance);
        return buf[k - 1].first;
    };
    for (size_t b0 = 0; b0 < n; b0 += BLOCK) {
        const size_t len = std::min(BLOCK, n - b0);
        // dots[t][j] = p[b0 + j] . q[q0 + t], summed over the dimensions in
        // order; the block is laid out dimension-major so that the loop over
        // its points vectorises (one lane per point)
        for (size_t j = 0; j < len; ++j)
            for (int c = 0; c < d; ++c) xt[size_t(c) * BLOCK + j] = p[(b0 + j) * size_t(d) + c];
        for (int t = 0; t < rows; ++t) {
            const float* q = p + (q0 + t) * size_t(d);
            float* col = dots.data() + size_t(t) * BLOCK;
            for (size_t j = 0; j < len; ++j) col[j] = 0.f;
            for (int c = 0; c < d; ++c) {
                const float qc = q[c];
                const float* xc = xt.data() + size_t(c) * BLOCK;
                for (size_t j = 0; j < len; ++j) col[j] += xc[j] * qc;
            }
        }
        for (int t = 0; t < rows; ++t) {
            const size_t i = q0 + t;
            const float ni = norms[i];
            const float* col = dots.data() + size_t(t) * BLOCK;
            Cand* buf = bufs.data() + size_t(t) * cap;
            int& fill = used[t];
            float& tau = reach[t];
            float dist[RUN];
            for (size_t j0 = 0; j0 < len; j0 += RUN) {
                const int run = int(std::min<size_t>(RUN, len - j0));
                float nearest = INFINITY;
                for (int r = 0; r < run; ++r) {
                    const float x = ni + norms[b0 + j0 + r] - 2.0f * col[j0 + r];
                    dist[r] = x;
                    nearest = x < nearest ? x : nearest;
                }
                if (nearest <= tau) {
                    for (int r = 0; r < run; ++r) {
                        const size_t j = b0 + j0 + r;
                        buf[fill] = Cand(dist[r], uint32_t(j));
                        fill += (dist[r] <= tau && j != i) ? 1 : 0;
                    }
                    if (fill >= 2 * k) {
                        tau = shrink(buf, fill);
                        fill = k;
                    }
                }
            }
        }
    }
    for (int t = 0; t < rows; ++t) {
        Cand* buf = bufs.data() + size_t(t) * cap;
        int len = used[t];
        if (len > k) {
            shrink(buf, len);
            len = k;
        }
        std::sort(buf, buf + len, by_distance);
        for (int s = 0; s < len; ++s) out[(q0 + t) * size_t(k) + s] = buf[s].second;
    }
}

}  // namespace

extern "C" {

// Exact kNN of every point of each sample within that sample, itself
// excluded: samples back to back in `p` (offsets[s] .. offsets[s + 1] rows of
// d f32), ks[s] neighbours each (1 <= k < n_s), written back to back from
// sum_{t<s} n_t k_t (indices local to the sample).  Samples largest first,
// every (sample, tile) task spread over the OpenMP threads.
void oracle_knn_exact_batched(const float* p, int d, uint32_t n_samples, const uint64_t* offsets,
                              const uint32_t* ks, uint32_t* out) {
    std::vector<uint32_t> order(n_samples);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return offsets[a + 1] - offsets[a] > offsets[b + 1] - offsets[b];
    });
    std::vector<uint64_t> out_off(n_samples + 1, 0);
    for (uint32_t s = 0; s < n_samples; ++s)
        out_off[s + 1] = out_off[s] + (offsets[s + 1] - offsets[s]) * ks[s];
    std::vector<std::vector<float>> norms(n_samples);
    struct Task {
        uint32_t s;
        size_t q0;
        int rows;
    };
    std::vector<Task> tasks;
    for (uint32_t s : order) {
        const size_t n = offsets[s + 1] - offsets[s];
        for (size_t q0 = 0; q0 < n; q0 += 128) tasks.push_back({s, q0, int(std::min<size_t>(128, n - q0))});
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (long long s = 0; s < (long long)n_samples; ++s) {
        const size_t n = offsets[s + 1] - offsets[s];
        const float* ps = p + offsets[s] * size_t(d);
        norms[s].resize(n);
        for (size_t i = 0; i < n; ++i) {
            float acc = 0.f;
            for (int c = 0; c < d; ++c) acc += ps[i * d + c] * ps[i * d + c];
            norms[s][i] = acc;
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (long long t = 0; t < (long long)tasks.size(); ++t) {
        const Task& tk = tasks[t];
        const size_t n = offsets[tk.s + 1] - offsets[tk.s];
        knn_tile(p + offsets[tk.s] * size_t(d), norms[tk.s].data(), n, d, int(ks[tk.s]), tk.q0,
                 tk.rows, out + out_off[tk.s]);
    }
}

}  // extern "C"
