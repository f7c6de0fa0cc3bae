// ORACLE — test infrastructure only, never shipped and never on the product path.
//
// A C++17 restatement of the reference's fuzzy simplicial set
// (crates/polariseq-core/src/umap.rs:283-620): per-row membership strengths
// (smooth_knn_dist, umap.rs:551-620: rho = nearest non-zero distance, 64-step
// bisection of sigma in f64 to sum exp(-max(0, d - rho) / sigma) = log2(k),
// floored at 1e-3 x the mean distance including the self distance), the
// counting-sort transpose (umap.rs:342-385), and the row merge with the fuzzy
// union acc + w - acc * w in f32, own entries first, pruned at 1e-5
// (umap.rs:488-545).  Pinned by the reference's known answer for
// smooth_knn_dist (umap.rs:2260-2276, umap-learn 0.5.12 values) and its
// structure tests (umap.rs:1937-2001), restated in tests/.
// Compiled with -ffp-contract=off: every f32 operation rounds as Rust's.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

void smooth_knn_dist(const float* dists, size_t len, float* out) {
    const int N_ITER = 64;
    const double TOLERANCE = 1e-5, MIN_K_DIST_SCALE = 1e-3;
    if (len == 0) return;
    const size_t kws = len + 1;
    const double target = std::log2(double(kws));
    std::vector<double> d64(dists, dists + len);
    double rho = 0.0;
    for (double d : d64)
        if (d > 0.0) {
            rho = d;
            break;
        }
    double lo = 0.0, hi = INFINITY, mid = 1.0;
    for (int it = 0; it < N_ITER; ++it) {
        double psum = 0.0;
        for (double d : d64) {
            const double x = d - rho;
            psum += x > 0.0 ? std::exp(-(x / mid)) : 1.0;
        }
        if (std::fabs(psum - target) < TOLERANCE) break;
        if (psum > target) {
            hi = mid;
            mid = (lo + hi) / 2.0;
        } else {
            lo = mid;
            mid = std::isinf(hi) ? mid * 2.0 : (lo + hi) / 2.0;
        }
    }
    double sum = 0.0;
    for (double d : d64) sum += d;
    const double mean = sum / double(kws);
    const double sigma = rho > 0.0 ? std::max(mid, MIN_K_DIST_SCALE * mean) : mid;
    for (size_t t = 0; t < len; ++t) {
        const double x = d64[t] - rho;
        out[t] = (x <= 0.0 || sigma == 0.0) ? 1.0f : float(std::exp(-(x / sigma)));
    }
}

}  // namespace

extern "C" {

void oracle_smooth_knn_dist(const float* dists, uint64_t len, float* out) {
    smooth_knn_dist(dists, len, out);
}

// Returns nnz of the symmetric graph, or ~0 when out_cap is too small.
uint64_t oracle_fuzzy(uint64_t n, const uint32_t* indptr, const uint32_t* indices,
                      const float* data, uint32_t* out_indptr, uint32_t* out_indices,
                      float* out_weights, uint64_t out_cap) {
    const size_t nnz = indptr[n];
    std::vector<float> strengths(nnz);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < int64_t(n); ++i)
        smooth_knn_dist(data + indptr[i], indptr[i + 1] - indptr[i], strengths.data() + indptr[i]);
    std::vector<uint32_t> t_indptr(n + 1, 0), t_cols(nnz);
    std::vector<float> t_vals(nnz);
    for (size_t e = 0; e < nnz; ++e) t_indptr[indices[e] + 1] += 1;
    for (uint64_t j = 0; j < n; ++j) t_indptr[j + 1] += t_indptr[j];
    std::vector<uint32_t> cursor(t_indptr.begin(), t_indptr.end() - 1);
    for (uint64_t i = 0; i < n; ++i)
        for (uint32_t e = indptr[i]; e < indptr[i + 1]; ++e) {
            const uint32_t c = cursor[indices[e]]++;
            t_cols[c] = uint32_t(i);
            t_vals[c] = strengths[e];
        }
    uint64_t o = 0;
    out_indptr[0] = 0;
    std::vector<std::pair<uint32_t, float>> w, t;
    for (uint64_t i = 0; i < n; ++i) {
        w.clear();
        for (uint32_t e = indptr[i]; e < indptr[i + 1]; ++e) w.push_back({indices[e], strengths[e]});
        std::stable_sort(w.begin(), w.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        t.clear();
        for (uint32_t e = t_indptr[i]; e < t_indptr[i + 1]; ++e) t.push_back({t_cols[e], t_vals[e]});
        std::stable_sort(t.begin(), t.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        size_t a = 0, b = 0;
        while (a < w.size() || b < t.size()) {
            const uint32_t col =
                (a < w.size() && (b >= t.size() || w[a].first <= t[b].first)) ? w[a].first : t[b].first;
            float acc = 0.0f;
            while (a < w.size() && w[a].first == col) {
                acc = (acc + w[a].second) - acc * w[a].second;
                ++a;
            }
            while (b < t.size() && t[b].first == col) {
                acc = (acc + t[b].second) - acc * t[b].second;
                ++b;
            }
            if (acc > 1e-5f) {
                if (o >= out_cap) return ~uint64_t(0);
                out_indices[o] = col;
                out_weights[o] = acc;
                ++o;
            }
        }
        out_indptr[i + 1] = uint32_t(o);
    }
    return o;
}

}  // extern "C"
