// Learned bucket routing: a small MLP d -> 256 -> 256 -> 1024 (ReLU) maps a
// cell's embedding to logits over the 1024 k-means buckets; trained so that
// a cell puts its probability where its neighbours (in a plain NN-Descent
// graph of a subsample) live.  Its top buckets replace the nearest-centroid
// probes of the tensor-core form.
//
// Hand-written kernels, no library calls: a tiled GEMM (64 x 64 output tile
// per 256-thread block, 4 x 4 per thread, 16-deep K steps through shared
// memory) with BF16 weights and FP32 activations / accumulation, used for the
// forward pass and both backward products; a softmax cross-entropy against
// sparse soft targets; column sums for the bias gradients; ReLU masks; Adam
// on FP32 master weights that refreshes the BF16 copies; and a per-row top-P
// of the logits.
#include <cuda_bf16.h>

#include "common.cuh"
#include "mlp.cuh"

namespace pq {
namespace {

constexpr int GT = 64;   // output tile (rows and columns)
constexpr int GK = 16;   // K step

__device__ __forceinline__ float ld(const float* p, size_t i) { return p[i]; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p, size_t i) {
    return __bfloat162float(p[i]);
}

// C[M x N] (= or +=) op(A)[M x K] . op(B)[K x N] (+ bias[n]) (ReLU).  A is
// M x K row-major (lda) or, transposed, K x M; B is K x N row-major (ldb) or,
// transposed, N x K.
template <typename TA, typename TB, bool TRA, bool TRB>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const TA* __restrict__ A,
                                              int lda, const TB* __restrict__ B, int ldb,
                                              float* __restrict__ C, int ldc,
                                              const float* __restrict__ bias, int relu,
                                              int accumulate) {
    __shared__ float As[GK][GT + 4];
    __shared__ float Bs[GK][GT + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int t = threadIdx.x; t < GT * GK; t += 256) {
            // A tile: As[kk][mm] = op(A)[m0 + mm][k0 + kk]
            const int mm = TRA ? t % GT : t / GK, kk = TRA ? t / GT : t % GK;
            const int m = m0 + mm, k = k0 + kk;
            float va = 0.f;
            if (m < M && k < K) va = TRA ? ld(A, size_t(k) * lda + m) : ld(A, size_t(m) * lda + k);
            As[kk][mm] = va;
            // B tile: Bs[kk][nn] = op(B)[k0 + kk][n0 + nn]
            const int nn = TRB ? t / GK : t % GT, kb = TRB ? t % GK : t / GT;
            const int n = n0 + nn, kq = k0 + kb;
            float vb = 0.f;
            if (n < N && kq < K) vb = TRB ? ld(B, size_t(n) * ldb + kq) : ld(B, size_t(kq) * ldb + n);
            Bs[kb][nn] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[n];
            if (relu) v = fmaxf(v, 0.f);
            float* c = C + size_t(m) * ldc + n;
            *c = accumulate ? *c + v : v;
        }
    }
}

template <typename TA, typename TB, bool TRA, bool TRB>
void gemm(int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* C, int ldc,
          const float* bias, bool relu, bool accumulate, cudaStream_t st) {
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    k_gemm<TA, TB, TRA, TRB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias,
                                                   relu ? 1 : 0, accumulate ? 1 : 0);
    count_launch();
}

// Softmax cross-entropy of each row's logits against its sparse soft target
// (T (bucket, weight) pairs, bucket ~0 = unused; weights sum to 1): writes
// the loss per row and dlogits = (softmax - target) / rows.  One warp per row.
__global__ void k_softmax_xent(float* __restrict__ Z, int rows, int N,
                               const uint32_t* __restrict__ tb, const float* __restrict__ tw,
                               int T, float* __restrict__ loss) {
    const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float* z = Z + size_t(r) * N;
    float mx = -__int_as_float(0x7f800000);
    for (int j = lane; j < N; j += 32) mx = fmaxf(mx, z[j]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    float se = 0.f;
    for (int j = lane; j < N; j += 32) se += expf(z[j] - mx);
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
    const float lse = mx + logf(se);
    float tl = 0.f;  // sum of w_t * z[b_t]
    if (lane < T) {
        const uint32_t b = tb[size_t(r) * T + lane];
        if (b != 0xFFFFFFFFu) tl = tw[size_t(r) * T + lane] * z[b];
    }
    for (int o = 16; o > 0; o >>= 1) tl += __shfl_xor_sync(0xFFFFFFFFu, tl, o);
    __syncwarp();
    const float inv = 1.0f / float(rows);
    for (int j = lane; j < N; j += 32) z[j] = expf(z[j] - lse) * inv;
    __syncwarp();
    if (lane < T) {
        const uint32_t b = tb[size_t(r) * T + lane];
        if (b != 0xFFFFFFFFu) z[b] -= tw[size_t(r) * T + lane] * inv;
    }
    if (lane == 0) loss[r] = lse - tl;
}

// dH *= (H > 0)
__global__ void k_relu_back(float* __restrict__ dH, const float* __restrict__ H, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && !(H[i] > 0.f)) dH[i] = 0.f;
}

// Column sums in two deterministic stages: part[c][n] = sum of rows
// c*chunk.. of column n, then db[n] = sum over c of part[c][n].
constexpr int CS_CHUNKS = 64;
__global__ void k_col_partial(const float* __restrict__ dY, int rows, int N,
                              float* __restrict__ part) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (n >= N) return;
    const int chunk = (rows + CS_CHUNKS - 1) / CS_CHUNKS;
    const int r1 = min(rows, (c + 1) * chunk);
    float s = 0.f;
    for (int r = c * chunk; r < r1; ++r) s += dY[size_t(r) * N + n];
    part[size_t(c) * N + n] = s;
}
__global__ void k_col_final(const float* __restrict__ part, int N, float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int c = 0; c < CS_CHUNKS; ++c) s += part[size_t(c) * N + n];
    db[n] = s;
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, size_t n, float lr, float b1, float b2,
                       float c1, float c2, float eps, __nv_bfloat16* __restrict__ wb) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, size_t n, __nv_bfloat16* __restrict__ b) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

// The P largest logits of each row (ties by index), descending, skipping the
// bucket `skip[r]` (the row's own primary, probed anyway).  One warp per row.
__global__ void k_topp(const float* __restrict__ Z, int rows, int N, int P,
                       const uint32_t* __restrict__ skip, uint32_t* __restrict__ out) {
    const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    const float* z = Z + size_t(r) * N;
    const uint32_t sk = skip ? skip[r] : 0xFFFFFFFFu;
    uint32_t taken = 0;  // bits of this lane's columns already chosen (N <= 1024)
    for (int p = 0; p < P; ++p) {
        float bv = -__int_as_float(0x7f800000);
        int bj = 0x7FFFFFFF;
        for (int t = 0; t * 32 + lane < N; ++t) {
            const int j = t * 32 + lane;
            if ((taken >> t) & 1u || uint32_t(j) == sk) continue;
            const float v = z[j];
            if (v > bv || (v == bv && j < bj)) {
                bv = v;
                bj = j;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
            const int oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
            if (ov > bv || (ov == bv && oj < bj)) {
                bv = ov;
                bj = oj;
            }
        }
        if (lane == (bj & 31)) taken |= 1u << (bj >> 5);
        if (lane == 0) out[size_t(r) * P + p] = uint32_t(bj);
    }
}

void col_sums(const float* dY, int rows, int N, float* part, float* db, cudaStream_t st) {
    k_col_partial<<<dim3((N + 255) / 256, CS_CHUNKS), 256, 0, st>>>(dY, rows, N, part);
    count_launch();
    k_col_final<<<(N + 255) / 256, 256, 0, st>>>(part, N, db);
    count_launch();
}

}  // namespace

size_t mlp_scratch_floats() { return size_t(CS_CHUNKS) * MLP_OUT; }

size_t mlp_params(int d) { return size_t(d) * MLP_H + MLP_H + size_t(MLP_H) * MLP_H + MLP_H +
                                  size_t(MLP_H) * MLP_OUT + MLP_OUT; }

MlpLayout mlp_layout(int d) {
    MlpLayout L;
    L.w1 = 0;
    L.b1 = L.w1 + size_t(d) * MLP_H;
    L.w2 = L.b1 + MLP_H;
    L.b2 = L.w2 + size_t(MLP_H) * MLP_H;
    L.w3 = L.b2 + MLP_H;
    L.b3 = L.w3 + size_t(MLP_H) * MLP_OUT;
    return L;
}

void mlp_forward(const MlpView& net, const float* X, int rows, float* H1, float* H2, float* Z,
                 cudaStream_t st, const MlpPrior* prior) {
    const MlpLayout L = mlp_layout(net.d);
    gemm<float, __nv_bfloat16, false, false>(rows, MLP_H, net.d, X, net.d, net.wb + L.w1, MLP_H,
                                             H1, MLP_H, net.w + L.b1, true, false, st);
    gemm<float, __nv_bfloat16, false, false>(rows, MLP_H, MLP_H, H1, MLP_H, net.wb + L.w2, MLP_H,
                                             H2, MLP_H, net.w + L.b2, true, false, st);
    gemm<float, __nv_bfloat16, false, false>(rows, MLP_OUT, MLP_H, H2, MLP_H, net.wb + L.w3,
                                             MLP_OUT, Z, MLP_OUT, net.w + L.b3, false, false, st);
    if (prior && prior->cs)
        gemm<float, float, false, true>(rows, MLP_OUT, net.d, X, net.d, prior->cs, prior->ld, Z,
                                        MLP_OUT, prior->cb, false, true, st);
}

void mlp_backward(const MlpView& net, const float* X, int rows, float* H1, float* H2, float* Z,
                  const uint32_t* tb, const float* tw, int T, float* loss, float* dH1,
                  float* dH2, float* grad, float* scratch, cudaStream_t st) {
    const MlpLayout L = mlp_layout(net.d);
    // Z becomes dZ
    k_softmax_xent<<<(rows + 7) / 8, 256, 0, st>>>(Z, rows, MLP_OUT, tb, tw, T, loss);
    count_launch();
    // layer 3: dW3 = H2^T dZ, db3, dH2 = dZ W3^T, masked by ReLU
    gemm<float, float, true, false>(MLP_H, MLP_OUT, rows, H2, MLP_H, Z, MLP_OUT, grad + L.w3,
                                    MLP_OUT, nullptr, false, false, st);
    col_sums(Z, rows, MLP_OUT, scratch, grad + L.b3, st);
    gemm<float, __nv_bfloat16, false, true>(rows, MLP_H, MLP_OUT, Z, MLP_OUT, net.wb + L.w3,
                                            MLP_OUT, dH2, MLP_H, nullptr, false, false, st);
    k_relu_back<<<unsigned((size_t(rows) * MLP_H + 255) / 256), 256, 0, st>>>(dH2, H2,
                                                                            size_t(rows) * MLP_H);
    count_launch();
    // layer 2
    gemm<float, float, true, false>(MLP_H, MLP_H, rows, H1, MLP_H, dH2, MLP_H, grad + L.w2, MLP_H,
                                    nullptr, false, false, st);
    col_sums(dH2, rows, MLP_H, scratch, grad + L.b2, st);
    gemm<float, __nv_bfloat16, false, true>(rows, MLP_H, MLP_H, dH2, MLP_H, net.wb + L.w2, MLP_H,
                                            dH1, MLP_H, nullptr, false, false, st);
    k_relu_back<<<unsigned((size_t(rows) * MLP_H + 255) / 256), 256, 0, st>>>(dH1, H1,
                                                                            size_t(rows) * MLP_H);
    count_launch();
    // layer 1
    gemm<float, float, true, false>(net.d, MLP_H, rows, X, net.d, dH1, MLP_H, grad + L.w1, MLP_H,
                                    nullptr, false, false, st);
    col_sums(dH1, rows, MLP_H, scratch, grad + L.b1, st);
}

void mlp_adam(MlpView& net, float* m, float* v, const float* grad, int step, float lr,
              cudaStream_t st) {
    const size_t np = mlp_params(net.d);
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    k_adam<<<unsigned((np + 255) / 256), 256, 0, st>>>(net.w, m, v, grad, np, lr, b1, b2, c1, c2,
                                                       1e-8f, net.wb);
    count_launch();
}

void mlp_sync_bf16(MlpView& net, cudaStream_t st) {
    const size_t np = mlp_params(net.d);
    k_f32_to_bf16<<<unsigned((np + 255) / 256), 256, 0, st>>>(net.w, np, net.wb);
    count_launch();
}

void mlp_topp(const float* Z, int rows, int P, const uint32_t* skip, uint32_t* out,
              cudaStream_t st) {
    k_topp<<<(rows + 7) / 8, 256, 0, st>>>(Z, rows, MLP_OUT, P, skip, out);
    count_launch();
}

}  // namespace pq
