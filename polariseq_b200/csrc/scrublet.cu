// Doublet scoring of many samples on the GPU (the steps of the reference's
// score_batch after its PCA, crates/polariseq-core/src/doublets.rs:1040-1127):
//
//   1. k_scrublet_points: each sample's point set, its cells then its
//      simulated doublets, in f32 from f64 arithmetic in the reference's
//      order (no fused multiply-add): cell i -> w_i u_i - mv, doublet (x, y)
//      -> s (u_x + u_y) - mv with s = 1e6 / (totals_x + totals_y);
//   2. the exact kNN of every point within its sample, all samples in one
//      persistent launch (pq_knn_batched_into_device; (distance, index)
//      order, as knn_exact), k_adj = round_half_even(k (1 + r)), r = n_sim/n;
//   3. k_scrublet_score: the Bayesian score from the count of simulated
//      neighbours, q = (n_d + 1) / (k_adj + 2),
//      score = q rho / r / (1 - rho - q (1 - rho - rho / r)), in f64.
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace pq {
namespace {

// One thread per (point, component): sample s's points are rows
// [pt_off[s], pt_off[s + 1]); its first n_s rows are its cells (rows
// [cell_off[s], ...) of u, w, totals), the rest its doublets (pairs from
// pair_off[s], sample-local cell indices).
__global__ void k_scrublet_points(const double* __restrict__ u, const double* __restrict__ w,
                                  const double* __restrict__ totals, const double* __restrict__ mv,
                                  const uint32_t* __restrict__ pairs,
                                  const uint64_t* __restrict__ cell_off,
                                  const uint64_t* __restrict__ pt_off,
                                  const uint64_t* __restrict__ pair_off, uint32_t n_samples,
                                  int p, float* __restrict__ pts) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t row = t / uint64_t(p);
    const int j = int(t - row * uint64_t(p));
    if (row >= pt_off[n_samples]) return;
    uint32_t lo = 0, hi = n_samples;  // the sample holding this row
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (pt_off[mid] <= row) lo = mid; else hi = mid;
    }
    const uint32_t s = lo;
    const uint64_t c0 = cell_off[s], n = cell_off[s + 1] - c0;
    const uint64_t r = row - pt_off[s];
    const double m = mv[uint64_t(s) * p + j];
    double v;
    if (r < n) {
        v = __dsub_rn(__dmul_rn(w[c0 + r], u[(c0 + r) * p + j]), m);
    } else {
        const uint64_t e = pair_off[s] + (r - n);
        const uint64_t x = c0 + pairs[2 * e], y = c0 + pairs[2 * e + 1];
        const double sc = __ddiv_rn(1e6, __dadd_rn(totals[x], totals[y]));
        v = __dsub_rn(__dmul_rn(sc, __dadd_rn(u[x * p + j], u[y * p + j])), m);
    }
    pts[t] = __double2float_rn(v);
}

// One thread per point: the number of its k_adj neighbours that are simulated
// doublets (local index >= n_s) and its score.
__global__ void k_scrublet_score(const uint32_t* __restrict__ knn,
                                 const uint64_t* __restrict__ pt_off,
                                 const uint64_t* __restrict__ cell_off,
                                 const uint64_t* __restrict__ knn_off,
                                 const uint32_t* __restrict__ kadj, const double* __restrict__ ratio,
                                 uint32_t n_samples, double rho, double* __restrict__ score_obs,
                                 double* __restrict__ score_sim,
                                 const uint64_t* __restrict__ pair_off) {
    const uint64_t row = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (row >= pt_off[n_samples]) return;
    uint32_t lo = 0, hi = n_samples;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (pt_off[mid] <= row) lo = mid; else hi = mid;
    }
    const uint32_t s = lo;
    const uint64_t n = cell_off[s + 1] - cell_off[s], r = row - pt_off[s];
    const uint32_t k = kadj[s];
    const uint32_t* nb = knn + knn_off[s] + r * k;
    uint32_t nd = 0;
    for (uint32_t t = 0; t < k; ++t) nd += nb[t] >= n ? 1u : 0u;
    const double rr = ratio[s];
    const double q = __ddiv_rn(double(nd) + 1.0, double(k) + 2.0);
    const double a = __dsub_rn(1.0, rho);
    const double den = __dsub_rn(a, __dmul_rn(q, __dsub_rn(a, __ddiv_rn(rho, rr))));
    const double sc = __ddiv_rn(__ddiv_rn(__dmul_rn(q, rho), rr), den);
    if (r < n) score_obs[cell_off[s] + r] = sc;
    else score_sim[pair_off[s] + (r - n)] = sc;
}

// numpy's round (half to even) of a non-negative value, as doublets.rs:477-485.
uint64_t round_half_even(double x) {
    double r = std::round(x);
    if (std::fabs(x - std::trunc(x)) == 0.5 && std::fmod(r, 2.0) != 0.0) r -= x > 0 ? 1.0 : -1.0;
    return r > 0 ? uint64_t(r) : 0;
}

}  // namespace
}  // namespace pq

using namespace pqh;

extern "C" int pq_scrublet_scores_device(pq_ctx* c, uint32_t n_samples, uint64_t p,
                                         const uint64_t* n_cells, const uint64_t* n_sim,
                                         const uint32_t* k, const double* d_u,
                                         const double* d_w, const double* d_totals,
                                         const double* d_mv, const uint32_t* d_pairs,
                                         double rho, double* d_score_obs, double* d_score_sim,
                                         uint32_t* k_adj_out, float* d_pts_out,
                                         uint32_t* d_knn_out, void* stream) {
    if (!c) return PQ_EINVAL;
    auto fail = [&](int code, const char* msg) {
        c->err = msg;
        return code;
    };
    if (!n_cells || !n_sim || !k || !d_u || !d_w || !d_totals || !d_mv || !d_score_obs ||
        !d_score_sim)
        return fail(PQ_EINVAL, "null buffer");
    if (n_samples == 0) return fail(PQ_EINVAL, "no samples");
    if (p == 0 || p > 64) return fail(PQ_ENOTSUP, "doublet scoring supports 1 <= p <= 64");
    if (!(rho > 0.0 && rho < 1.0)) return fail(PQ_EINVAL, "the expected doublet rate must be in (0, 1)");
    std::vector<uint64_t> cell_off(n_samples + 1, 0), pt_off(n_samples + 1, 0),
        pair_off(n_samples + 1, 0), knn_off(n_samples + 1, 0);
    std::vector<uint32_t> kadj(n_samples);
    std::vector<double> ratio(n_samples);
    for (uint32_t s = 0; s < n_samples; ++s) {
        const uint64_t n = n_cells[s], m = n_sim[s], total = n + m;
        if (n == 0 || m == 0) return fail(PQ_EINVAL, "every sample needs cells and simulated doublets");
        if (total >= 0xFFFFFFFFull) return fail(PQ_EINVAL, "a sample has 2^32 points or more");
        if (k[s] == 0) return fail(PQ_EINVAL, "k must be >= 1");
        ratio[s] = double(m) / double(n);
        uint64_t ka = pq::round_half_even(double(k[s]) * (1.0 + ratio[s]));
        ka = std::min<uint64_t>(std::max<uint64_t>(ka, 1), total - 1);
        if (ka > 512) return fail(PQ_ENOTSUP, "doublet scoring supports k_adj <= 512");
        kadj[s] = uint32_t(ka);
        cell_off[s + 1] = cell_off[s] + n;
        pair_off[s + 1] = pair_off[s] + m;
        pt_off[s + 1] = pt_off[s] + total;
        knn_off[s + 1] = knn_off[s] + total * ka;
    }
    if (pair_off[n_samples] > 0 && !d_pairs) return fail(PQ_EINVAL, "null buffer");
    try {
        if (cudaSetDevice(c->device) != cudaSuccess) return fail(PQ_EDEVICE, "cudaSetDevice failed");
        cudaStream_t st = c->stream;
        cudaStream_t user = static_cast<cudaStream_t>(stream);
        cudaEvent_t ev;
        ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(ev, user), "event");
        ck(cudaStreamWaitEvent(st, ev, 0), "event");
        const uint64_t npt = pt_off[n_samples];
        float* pts = c->get<float>("sc_pts", npt * p);
        uint32_t* knn = c->get<uint32_t>("sc_knn", knn_off[n_samples]);
        float* kd = c->get<float>("sc_kd", knn_off[n_samples]);
        uint64_t* dco = c->get<uint64_t>("sc_cell_off", n_samples + 1);
        uint64_t* dpo = c->get<uint64_t>("sc_pt_off", n_samples + 1);
        uint64_t* dpr = c->get<uint64_t>("sc_pair_off", n_samples + 1);
        uint64_t* dko = c->get<uint64_t>("sc_knn_off", n_samples + 1);
        uint32_t* dka = c->get<uint32_t>("sc_kadj", n_samples);
        double* dra = c->get<double>("sc_ratio", n_samples);
        const size_t o8 = (n_samples + 1) * 8ull;
        ck(cudaMemcpyAsync(dco, cell_off.data(), o8, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dpo, pt_off.data(), o8, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dpr, pair_off.data(), o8, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dko, knn_off.data(), o8, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dka, kadj.data(), n_samples * 4ull, cudaMemcpyHostToDevice, st), "h2d");
        ck(cudaMemcpyAsync(dra, ratio.data(), n_samples * 8ull, cudaMemcpyHostToDevice, st), "h2d");
        const uint64_t nt = npt * p;
        pq::k_scrublet_points<<<unsigned((nt + 255) / 256), 256, 0, st>>>(
            d_u, d_w, d_totals, d_mv, d_pairs, dco, dpo, dpr, n_samples, int(p), pts);
        pq::count_launch();
        ck(cudaGetLastError(), "scrublet points");
        const int rc = pq_knn_batched_into_device(c, pts, p, n_samples, pt_off.data(), kadj.data(),
                                                  knn, kd, PQ_BATCH_GRAPH, nullptr, st);
        if (rc != PQ_OK) {
            cudaEventDestroy(ev);
            return rc;
        }
        pq::k_scrublet_score<<<unsigned((npt + 255) / 256), 256, 0, st>>>(
            knn, dpo, dco, dko, dka, dra, n_samples, rho, d_score_obs, d_score_sim, dpr);
        pq::count_launch();
        ck(cudaGetLastError(), "scrublet score");
        if (d_pts_out)
            ck(cudaMemcpyAsync(d_pts_out, pts, npt * p * 4, cudaMemcpyDeviceToDevice, st), "pts");
        if (d_knn_out)
            ck(cudaMemcpyAsync(d_knn_out, knn, knn_off[n_samples] * 4, cudaMemcpyDeviceToDevice, st),
               "knn");
        ck(cudaEventRecord(ev, st), "event");
        ck(cudaStreamWaitEvent(user, ev, 0), "event");
        ck(cudaStreamSynchronize(st), "scrublet");  // the host offset arrays go out of scope
        cudaEventDestroy(ev);
        if (k_adj_out)
            for (uint32_t s = 0; s < n_samples; ++s) k_adj_out[s] = kadj[s];
        return PQ_OK;
    } catch (const DeviceError& e) {
        cudaStreamSynchronize(c->stream);
        cudaGetLastError();
        return fail(PQ_EDEVICE, e.msg.c_str());
    } catch (const std::string& s) {
        cudaStreamSynchronize(c->stream);
        cudaGetLastError();
        c->err = s;
        return PQ_ENOMEM;
    }
}
