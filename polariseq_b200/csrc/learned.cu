// Learned probes for the tensor-core form (PQ_INIT_LEARNED).
//
// 1. an evenly strided subsample of the cells (at most 262,144) gets its plain
//    NN-Descent graph (k = 15, the bit-exact form, on a separate context);
// 2. each subsample cell's target is the distribution of the k-means buckets
//    of itself and its neighbours (at most 16 distinct buckets);
// 3. the MLP (mlp.cu) is trained on those targets with Adam, batches of 8192,
//    a fixed number of epochs, a seeded initialisation and seeded shuffles
//    (every epoch's order from one device sort of hashed keys);
// 4. every cell's probes are its own bucket followed by the P - 1 most likely
//    other buckets.
// The logits are the MLP's output plus a nearest-centroid prior,
// -|x - c_b|^2 / (mean squared distance to the own centroid): untrained, the
// router ranks buckets as the centroid distances do, and training learns where
// the neighbours are beyond that.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <vector>

#include "ctx.cuh"
#include "mlp.cuh"
#include "primitives.cuh"

namespace pq {
namespace {

constexpr int T_MAX = 16;  // target buckets per training cell

// Shuffle keys of one epoch: 32 hashed bits per subsample cell, the cell's
// index as the value; a stable sort gives the epoch's order.
__global__ void k_shuffle_keys(uint32_t ns, uint32_t ep, uint64_t seed, uint32_t* __restrict__ keys,
                               uint64_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const uint64_t h = splitmix(seed ^ splitmix(0x5348554646ull + ep) ^ splitmix(uint64_t(i) << 3));
    keys[i] = uint32_t(h >> 32);
    vals[i] = i;
}

// Rows i * n / ns of the padded embedding, d columns each, contiguous.
__global__ void k_take_rows(const float* __restrict__ X, int d, int dp, uint64_t n, uint32_t ns,
                            float* __restrict__ out) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(ns) * d) return;
    const uint32_t r = uint32_t(t / d);
    const int j = int(t - size_t(r) * d);
    out[t] = X[(uint64_t(r) * n / ns) * dp + j];
}

// Targets: the buckets of the cell and of its graph neighbours, merged, with
// weights = count / total.
__global__ void k_targets(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                          uint32_t ns, uint64_t n, const uint32_t* __restrict__ primary,
                          uint32_t* __restrict__ tb, float* __restrict__ tw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    uint32_t b[T_MAX];
    float w[T_MAX];
    int m = 0, total = 0;
    auto add = [&](uint32_t bucket) {
        for (int t = 0; t < m; ++t)
            if (b[t] == bucket) {
                w[t] += 1.f;
                return;
            }
        if (m < T_MAX) {
            b[m] = bucket;
            w[m] = 1.f;
            ++m;
        }
    };
    add(primary[uint64_t(i) * n / ns]);
    ++total;
    for (uint32_t e = indptr[i]; e < indptr[i + 1] && total < T_MAX; ++e) {
        add(primary[uint64_t(indices[e]) * n / ns]);
        ++total;
    }
    for (int t = 0; t < T_MAX; ++t) {
        tb[size_t(i) * T_MAX + t] = t < m ? b[t] : 0xFFFFFFFFu;
        tw[size_t(i) * T_MAX + t] = t < m ? w[t] / float(total) : 0.f;
    }
}

__global__ void k_gather_batch(const float* __restrict__ Xs, int d, const uint64_t* __restrict__ perm,
                               uint32_t rows, const uint32_t* __restrict__ tb,
                               const float* __restrict__ tw, float* __restrict__ xb,
                               uint32_t* __restrict__ bb, float* __restrict__ wbt) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < size_t(rows) * d) {
        const uint32_t r = uint32_t(t / d);
        xb[t] = Xs[size_t(perm[r]) * d + (t - size_t(r) * d)];
    }
    if (t < size_t(rows) * T_MAX) {
        const uint32_t r = uint32_t(t / T_MAX);
        const size_t s = size_t(perm[r]) * T_MAX + (t - size_t(r) * T_MAX);
        bb[t] = tb[s];
        wbt[t] = tw[s];
    }
}

// Seeded uniform(-a, a) weights for the hidden layers; the output layer and
// the biases start at zero, so that the untrained router is the prior.
__global__ void k_init_params(float* __restrict__ w, size_t n, MlpLayout L, int d,
                              uint64_t seed) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float fan_in, fan_out;
    if (i < L.b1) {
        fan_in = float(d);
        fan_out = float(MLP_H);
    } else if (i >= L.w2 && i < L.b2) {
        fan_in = fan_out = float(MLP_H);
    } else {
        w[i] = 0.f;
        return;
    }
    const float a = sqrtf(6.f / (fan_in + fan_out));
    w[i] = (2.f * hash_unit(seed, 0x4d4c50ull, i) - 1.f) * a;
}

// Prior terms: cs = 2 beta c (d columns of the padded centroid rows) and
// cb = -beta |c|^2, beta = 1 / the mean squared distance of a cell to its
// own centroid (sum_d / count).
__global__ void k_prior(const float* __restrict__ cent, int d, int dp, uint32_t C,
                        const double* __restrict__ sum_d, double count, float* __restrict__ cs,
                        float* __restrict__ cb) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= C) return;
    const float beta = float(count / fmax(*sum_d, 1e-30));
    float s = 0.f;
    for (int j = 0; j < d; ++j) {
        const float v = cent[size_t(b) * dp + j];
        cs[size_t(b) * d + j] = 2.f * beta * v;
        s = fmaf(v, v, s);
    }
    cb[b] = -beta * s;
}

__global__ void k_sum_f32(const float* __restrict__ a, size_t n, double* __restrict__ out) {
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += size_t(gridDim.x) * blockDim.x)
        s += double(a[i]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void k_rows_of(const float* __restrict__ X, int d, int dp, uint64_t r0, uint32_t rows,
                          float* __restrict__ out) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * d) return;
    const uint32_t r = uint32_t(t / d);
    out[t] = X[(r0 + r) * dp + (t - size_t(r) * d)];
}

__global__ void k_assemble_probes(const uint32_t* __restrict__ primary, const uint32_t* __restrict__ top,
                                  uint64_t r0, uint32_t rows, int P, uint32_t* __restrict__ probes) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * P) return;
    const uint32_t r = uint32_t(t / P);
    const int p = int(t - size_t(r) * P);
    probes[(r0 + r) * P + p] = p == 0 ? primary[r0 + r] : top[size_t(r) * (P - 1) + (p - 1)];
}

}  // namespace
}  // namespace pq

namespace pqh {

using namespace pq;

double learned_probes(pq_ctx* c, const float* X, int d, int dp, uint32_t n, uint32_t C,
                      const uint32_t* primary, const float* primary_d, const float* cent, int P,
                      uint64_t seed, uint32_t* probes, double* ms_train, double* loss_first,
                      double* loss_last) {
    cudaStream_t st = c->stream;
    if (C != uint32_t(MLP_OUT)) throw DeviceError{"learned probes need 1024 buckets"};
    const auto t0 = std::chrono::steady_clock::now();
    // the nearest-centroid prior of the logits
    double* dsum = c->get<double>("ml_dsum", 1);
    ck(cudaMemsetAsync(dsum, 0, 8, st), "prior");
    k_sum_f32<<<256, 256, 0, st>>>(primary_d, n, dsum); count_launch();
    MlpPrior prior;
    float* pcs = c->get<float>("ml_pcs", size_t(C) * d);
    float* pcb = c->get<float>("ml_pcb", C);
    k_prior<<<blocks(C, 256), 256, 0, st>>>(cent, d, dp, C, dsum, double(n), pcs, pcb); count_launch();
    prior.cs = pcs;
    prior.ld = d;
    prior.cb = pcb;
    // ── 1. the subsample and its plain graph ──
    const uint32_t ns = std::min<uint32_t>(n, 1u << 18);
    float* xs = c->get<float>("ml_xs", size_t(ns) * d);
    k_take_rows<<<blocks(size_t(ns) * d, 256), 256, 0, st>>>(X, d, dp, n, ns, xs); count_launch();
    ck(cudaStreamSynchronize(st), "subsample");
    const int gk = int(std::min<uint64_t>(15, ns > 1 ? ns - 1 : 1));
    uint32_t* gip = c->get<uint32_t>("ml_ip", size_t(ns) + 1);
    uint32_t* gix = c->get<uint32_t>("ml_ix", size_t(ns) * gk);
    float* gdx = c->get<float>("ml_dx", size_t(ns) * gk);
    {
        if (!c->sub && pq_ctx_create(c->device, &c->sub) != PQ_OK) {
            c->sub = nullptr;
            throw DeviceError{"graph context"};
        }
        pq_ctx* g = c->sub;
        pq_nnd_opts go;
        pq_nnd_opts_default(&go);
        go.k = uint64_t(gk);
        go.seed = seed;
        uint64_t nnz = 0;
        const int rc = pq_nndescent_into_device(g, xs, ns, uint64_t(d), &go, gip, gix, gdx, &nnz, st);
        cudaSetDevice(c->device);
        if (rc != PQ_OK) throw DeviceError{"subsample graph: " + std::string(pq_ctx_last_error(g))};
    }
    const bool trace = std::getenv("POLARISEQ_TRACE") != nullptr;
    auto since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a)
            .count();
    };
    if (trace) {
        ck(cudaStreamSynchronize(st), "trace");
        std::fprintf(stderr, "[learned] subsample of %u cells and its plain graph: %.1f ms\n", ns,
                     since(t0));
    }
    // ── 2. targets ──
    uint32_t* tb = c->get<uint32_t>("ml_tb", size_t(ns) * T_MAX);
    float* tw = c->get<float>("ml_tw", size_t(ns) * T_MAX);
    k_targets<<<blocks(ns, 256), 256, 0, st>>>(gip, gix, ns, n, primary, tb, tw); count_launch();
    // ── 3. training ──
    const size_t np = mlp_params(d);
    ck(cudaMemsetAsync(c->d_err, 0, sizeof(int), st), "err");
    MlpView net{d, c->get<float>("ml_w", np), c->get<__nv_bfloat16>("ml_wt", mlp_wt_elems()),
                c->d_err};
    float* am = c->get<float>("ml_m", np);
    float* av = c->get<float>("ml_v", np);
    float* grad = c->get<float>("ml_g", np);
    ck(cudaMemsetAsync(am, 0, np * 4, st), "adam");
    ck(cudaMemsetAsync(av, 0, np * 4, st), "adam");
    k_init_params<<<blocks(np, 256), 256, 0, st>>>(net.w, np, mlp_layout(d), d, seed); count_launch();
    mlp_sync_bf16(net, st);
    mlp_set_prior(net, prior, st);
    // batches of 8192 at learning rate 2e-3: at 4M x 50 the same recall as
    // 4096 at 1e-3 (0.994) in half the steps; 16384 at 2e-3 or 3e-3 needs a
    // third round
    const int B = 8192, epochs = 8;
    const float lr = 2e-3f;
    float* xb = c->get<float>("ml_xb", size_t(B) * d);
    uint32_t* bb = c->get<uint32_t>("ml_bb", size_t(B) * T_MAX);
    float* bw = c->get<float>("ml_bw", size_t(B) * T_MAX);
    float* h1 = c->get<float>("ml_h1", size_t(B) * MLP_H);
    float* h2 = c->get<float>("ml_h2", size_t(B) * MLP_H);
    float* z = c->get<float>("ml_z", size_t(B) * MLP_OUT);
    float* dh1 = c->get<float>("ml_dh1", size_t(B) * MLP_H);
    float* dh2 = c->get<float>("ml_dh2", size_t(B) * MLP_H);
    float* loss = c->get<float>("ml_loss", B);
    float* scratch = c->get<float>("ml_scratch", mlp_scratch_floats());
    const MlpBufs tb16 = mlp_bufs(c->get<uint8_t>("ml_b16", mlp_bufs_bytes(B, true)), B, true);
    // every epoch's seeded order, on the device (no host round trip between
    // epochs)
    const size_t ne = size_t(ns) * epochs;
    uint32_t* skeys = c->get<uint32_t>("ml_skeys", ns);
    uint32_t* skeys2 = c->get<uint32_t>("ml_skeys2", ns);
    uint64_t* dperm = c->get<uint64_t>("ml_perm", ne);  // the sorted values: the orders
    uint64_t* svals2 = c->get<uint64_t>("ml_svals2", ns);
    void* stemp = c->get<uint8_t>("ml_sort_temp", radix_temp_bytes(ns));
    for (int ep = 0; ep < epochs; ++ep) {
        uint64_t* order = dperm + size_t(ep) * ns;
        k_shuffle_keys<<<blocks(ns, 256), 256, 0, st>>>(ns, uint32_t(ep), seed, skeys, order);
        count_launch();
        ck(radix_sort_pairs(skeys, order, skeys2, svals2, ns, 32, stemp, st), "shuffle");
    }
    int step = 0;
    double* eloss = c->get<double>("ml_eloss", epochs);
    ck(cudaMemsetAsync(eloss, 0, epochs * 8, st), "loss");
    std::vector<uint64_t> erows(epochs, 0);
    for (int ep = 0; ep < epochs; ++ep) {
        for (uint32_t b0 = 0; b0 + B <= ns || (b0 == 0 && ns > 0); b0 += B) {
            const uint32_t rows = std::min<uint32_t>(B, ns - b0);
            k_gather_batch<<<blocks(size_t(rows) * std::max(d, T_MAX), 256), 256, 0, st>>>(
                xs, d, dperm + size_t(ep) * ns + b0, rows, tb, tw, xb, bb, bw);
            count_launch();
            ck(mlp_forward(net, xb, int(rows), h1, h2, z, tb16, true, st, &prior), "mlp forward");
            ck(mlp_backward(net, int(rows), h1, h2, z, tb16, bb, bw, T_MAX, loss, dh1, dh2, grad,
                            scratch, st),
               "mlp backward");
            mlp_adam(net, am, av, grad, ++step, lr, st);
            k_sum_f32<<<8, 256, 0, st>>>(loss, rows, eloss + ep); count_launch();
            erows[ep] += rows;
            if (rows < uint32_t(B)) break;
        }
    }
    ck(cudaGetLastError(), "training");
    std::vector<double> hl(epochs);
    // on the training stream: the losses are complete only when it is
    ck(cudaMemcpyAsync(hl.data(), eloss, epochs * 8, cudaMemcpyDeviceToHost, st), "loss");
    ck(cudaStreamSynchronize(st), "loss");
    *loss_first = hl[0] / double(std::max<uint64_t>(erows[0], 1));
    *loss_last = hl[epochs - 1] / double(std::max<uint64_t>(erows[epochs - 1], 1));
    const auto t1 = std::chrono::steady_clock::now();
    *ms_train = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (trace) {
        std::fprintf(stderr, "[learned] %d epochs of %u cells (batches of %d): done at %.1f ms; "
                     "loss per epoch", epochs, ns, B, *ms_train);
        for (int e = 0; e < epochs; ++e)
            std::fprintf(stderr, " %.4f", hl[e] / double(std::max<uint64_t>(erows[e], 1)));
        std::fprintf(stderr, "\n");
    }
    // ── 4. probes of every cell ──
    const uint32_t R = 65536;
    float* xr = c->get<float>("ml_xr", size_t(R) * d);
    float* ih1 = c->get<float>("ml_ih1", size_t(R) * MLP_H);
    float* ih2 = c->get<float>("ml_ih2", size_t(R) * MLP_H);
    float* iz = c->get<float>("ml_iz", size_t(R) * MLP_OUT);
    uint32_t* top = c->get<uint32_t>("ml_top", size_t(R) * std::max(P - 1, 1));
    const MlpBufs ib16 = mlp_bufs(c->get<uint8_t>("ml_i16", mlp_bufs_bytes(R, false)), R, false);
    for (uint64_t r0 = 0; r0 < n; r0 += R) {
        const uint32_t rows = uint32_t(std::min<uint64_t>(R, n - r0));
        k_rows_of<<<blocks(size_t(rows) * d, 256), 256, 0, st>>>(X, d, dp, r0, rows, xr); count_launch();
        ck(mlp_forward(net, xr, int(rows), ih1, ih2, iz, ib16, false, st, &prior), "mlp routing");
        if (P > 1) mlp_topp(iz, int(rows), P - 1, primary + r0, top, st);
        k_assemble_probes<<<blocks(size_t(rows) * P, 256), 256, 0, st>>>(primary, top, r0, rows, P,
                                                                        probes);
        count_launch();
    }
    ck(cudaStreamSynchronize(st), "learned probes");
    int herr = 0;
    ck(cudaMemcpy(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost), "err");
    if (herr) throw DeviceError{"mlp tensor-core products: a bounded wait gave up", herr == 2};
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
}

}  // namespace pqh
