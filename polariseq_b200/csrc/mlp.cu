// Learned bucket routing: a small MLP d -> 256 -> 256 -> 1024 (ReLU) maps a
// cell's embedding to logits over the 1024 k-means buckets; trained so that
// a cell puts its probability where its neighbours (in a plain NN-Descent
// graph of a subsample) live.
//
// Hand-written kernels, no library calls.  Every product of the forward and
// backward pass runs on the tcgen05 tensor cores: one 128 x 256 output tile
// per CTA, BF16 operands staged K-major in shared memory by TMA (128-byte
// swizzle, four stages), FP32 accumulation in TMEM, and an epilogue that adds
// the bias, applies ReLU or the ReLU-backward mask and writes FP32 and BF16
// (row-major and transposed) copies, so that each product's output is the
// next one's operand without another pass.  Weights are BF16 copies of FP32
// master weights (both orientations); activations and output gradients are
// rounded to BF16 where they feed a product.  The nearest-centroid prior of
// the routing logits rides in the output product as 192 extra K columns:
// x.cs = x_hi.cs_hi + x_lo.cs_hi + x_hi.cs_lo with BF16 hi / lo splits of
// both sides (about 16 bits of each).  The softmax cross-entropy, the
// bias-gradient column sums, Adam and the per-row top-P run on CUDA cores.
#include <cuda_bf16.h>

#include "common.cuh"
#include "ivf.cuh"
#include "mlp.cuh"
#include "tc.cuh"

namespace pq {
namespace {

// ── tensor-core GEMM: C[M x N] = A[M x K] . B[N x K]^T ─────────────────────
constexpr int TM = 128;   // output rows per CTA (TMEM lanes)
constexpr int TN = 256;   // output columns per CTA (TMEM columns)
constexpr int GS = 4;     // pipeline stages
constexpr int G_THREADS = 192;  // TMA warp, MMA warp, four epilogue warps
constexpr uint32_t G_WAIT = 1u << 24;
constexpr int A_BYTES = TM * 128, B_BYTES = TN * 128;  // one 64-deep K block

struct TcOut {
    const float* bias;    // [N] or null
    const float* bias2;   // a second [N] added, or null
    int relu;             // max(0, .)
    const float* mask;    // optional ReLU-backward mask: out *= (mask[m][n] > 0)
    int ldm;
    float* C;             // optional FP32 [M x N], ldc
    int ldc;
    __nv_bfloat16* Cb;    // optional BF16 row-major, ldcb
    int ldcb;
    __nv_bfloat16* Ct;    // optional BF16 transposed: Ct[n * ldct + m]
    int ldct;
    int M, N, K;
    int* err;
};

struct __align__(8) GemmBars {
    uint64_t full[GS], empty[GS], done;
    uint32_t tmem;
    int abort;
};

__global__ void __launch_bounds__(G_THREADS, 1) k_tc_gemm(const __grid_constant__ CUtensorMap tA,
                                                          const __grid_constant__ CUtensorMap tB,
                                                          TcOut o) {
    extern __shared__ __align__(1024) uint8_t graw[];
    uint8_t* smem = graw + ((1024u - (tc::smem_u32(graw) & 1023u)) & 1023u);
    uint8_t* sA = smem;
    uint8_t* sB = smem + GS * A_BYTES;
    __shared__ GemmBars Bb;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    volatile int* abort_flag = &Bb.abort;
    if (w == 0) {
        tc::tmem_alloc(&Bb.tmem, TN);
        tc::tmem_relinquish();
    }
    if (tid == 32) {
        for (int s = 0; s < GS; ++s) {
            tc::mbar_init(&Bb.full[s], 1);
            tc::mbar_init(&Bb.empty[s], 1);
        }
        tc::mbar_init(&Bb.done, 1);
        tc::fence_barrier_init();
        Bb.abort = 0;
        tc::prefetch_tmap(&tA);
        tc::prefetch_tmap(&tB);
    }
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = Bb.tmem;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int nk = (o.K + 63) / 64;
    if (w == 0) {
        // ── TMA producer ──
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < nk && !*abort_flag; ++kb) {
                const int s = kb % GS;
                if (!tc::mbar_wait(&Bb.empty[s], ((kb / GS) & 1) ^ 1, G_WAIT)) {
                    *abort_flag = 1;
                    break;
                }
                tc::mbar_expect_tx(&Bb.full[s], A_BYTES + B_BYTES);
                tc::tma_load_2d(sA + s * A_BYTES, &tA, &Bb.full[s], kb * 64, m0);
                tc::tma_load_2d(sB + s * B_BYTES, &tB, &Bb.full[s], kb * 64, n0);
                ++issued;
            }
            // every issued copy has landed before the CTA may exit
            for (int s = 0; s < GS; ++s) {
                const int uses = issued / GS + (s < issued % GS ? 1 : 0);
                if (uses > 0 && !tc::mbar_wait(&Bb.full[s], (uses - 1) & 1, G_WAIT))
                    *abort_flag = 1;
            }
        }
        __syncwarp();
    } else if (w == 1) {
        // ── MMA issuer ──
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(TM, TN);
            for (int kb = 0; kb < nk && !*abort_flag; ++kb) {
                const int s = kb % GS;
                if (!tc::mbar_wait(&Bb.full[s], (kb / GS) & 1, G_WAIT)) {
                    *abort_flag = 1;
                    break;
                }
                tc::tc_fence_after();
                const uint64_t dA = tc::desc_k_sw128(tc::smem_u32(sA + s * A_BYTES));
                const uint64_t dB = tc::desc_k_sw128(tc::smem_u32(sB + s * B_BYTES));
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)  // K = 64 as four K = 16 steps (32 B each)
                    tc::umma_f16(taddr, dA + uint64_t(2 * kk), dB + uint64_t(2 * kk), idesc,
                                 (kb | kk) > 0 ? 1u : 0u);
                tc::umma_commit(&Bb.empty[s]);
            }
            // every issued MMA has completed before the epilogue reads TMEM
            tc::umma_commit(&Bb.done);
        }
        __syncwarp();
    } else {
        // ── epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 32 ──
        const int quarter = w & 3;
        const int m = m0 + quarter * 32 + lane;
        const uint32_t lane_base = uint32_t(quarter * 32) << 16;
        const bool ok = __all_sync(0xFFFFFFFFu, tc::mbar_wait(&Bb.done, 0, G_WAIT));
        if (!ok) {
            if (lane == 0) *abort_flag = 1;
        } else {
            tc::tc_fence_after();
            for (int c = 0; c < TN / 32; ++c) {
                uint32_t r[32];
                tc::tmem_ld32(taddr + lane_base + uint32_t(c * 32), r);
                tc::tmem_ld_wait();
                const int nb = n0 + c * 32;
                if (nb >= o.N) break;
                float v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float x = __uint_as_float(r[j]);
                    if (o.bias) x += o.bias[nb + j];
                    if (o.bias2) x += o.bias2[nb + j];
                    if (o.relu) x = fmaxf(x, 0.f);
                    v[j] = x;
                }
                if (m < o.M) {
                    if (o.mask) {
                        const float4* mk = reinterpret_cast<const float4*>(o.mask + size_t(m) * o.ldm + nb);
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const float4 t = mk[q];
                            v[4 * q] = t.x > 0.f ? v[4 * q] : 0.f;
                            v[4 * q + 1] = t.y > 0.f ? v[4 * q + 1] : 0.f;
                            v[4 * q + 2] = t.z > 0.f ? v[4 * q + 2] : 0.f;
                            v[4 * q + 3] = t.w > 0.f ? v[4 * q + 3] : 0.f;
                        }
                    }
                    if (o.C) {
                        float4* cp = reinterpret_cast<float4*>(o.C + size_t(m) * o.ldc + nb);
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            cp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                    }
                    if (o.Cb) {
                        uint4* bp = reinterpret_cast<uint4*>(o.Cb + size_t(m) * o.ldcb + nb);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            uint32_t pk[4];
#pragma unroll
                            for (int h = 0; h < 4; ++h) {
                                const __nv_bfloat162 b2 =
                                    __floats2bfloat162_rn(v[8 * q + 2 * h], v[8 * q + 2 * h + 1]);
                                pk[h] = *reinterpret_cast<const uint32_t*>(&b2);
                            }
                            bp[q] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                        }
                    }
                    if (o.Ct) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            o.Ct[size_t(nb + j) * o.ldct + m] = __float2bfloat16_rn(v[j]);
                    }
                }
            }
        }
    }
    __syncthreads();
    if (*abort_flag && tid == 0 && o.err) atomicExch(o.err, 2);
    tc::tc_fence_after();
    if (w == 0) tc::tmem_dealloc(taddr, TN);
}

size_t tc_gemm_smem() { return 1024 + size_t(GS) * (A_BYTES + B_BYTES); }

// out = A[M x K] . B[N x K]^T (A, B BF16 with leading dimensions lda, ldb;
// K need not be a multiple of 64: reads past K are zeros).
bool tc_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, const TcOut& o,
             cudaStream_t st) {
    CUtensorMap ta, tb;
    if (!make_bf16_map_ld(&ta, A, uint64_t(o.M), uint64_t(o.K), uint64_t(lda), TM) ||
        !make_bf16_map_ld(&tb, B, uint64_t(o.N), uint64_t(o.K), uint64_t(ldb), TN))
        return false;
    if (cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(tc_gemm_smem())) != cudaSuccess)
        return false;
    dim3 grid((o.N + TN - 1) / TN, (o.M + TM - 1) / TM);
    k_tc_gemm<<<grid, G_THREADS, tc_gemm_smem(), st>>>(ta, tb, o);
    count_launch();
    return true;
}

TcOut tc_out(int M, int N, int K, int* err) {
    TcOut o{};
    o.M = M;
    o.N = N;
    o.K = K;
    o.err = err;
    return o;
}

// X [rows x d] FP32 -> BF16 rows padded to 64 columns (zeros) and the
// transposed copy [64 x ldt] (rows d..63 zero).
// (ext, if not null: the prior's columns [x_hi | x_lo | x_hi] of the output
// product's A operand, 192 columns from ext + r * ldext.)
__global__ void k_x_bf16(const float* __restrict__ X, int rows, int d, __nv_bfloat16* __restrict__ xb,
                         __nv_bfloat16* __restrict__ xt, int ldt, __nv_bfloat16* __restrict__ ext,
                         int ldext) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * 64) return;
    const int r = int(t / 64), c = int(t % 64);
    const float x = c < d ? X[size_t(r) * d + c] : 0.f;
    const __nv_bfloat16 v = __float2bfloat16_rn(x);
    xb[t] = v;
    if (xt) xt[size_t(c) * ldt + r] = v;
    if (ext) {
        const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(v));
        __nv_bfloat16* e = ext + size_t(r) * ldext;
        e[c] = v;
        e[64 + c] = lo;
        e[128 + c] = v;
    }
}

// The prior's columns of the output product's B operand: row n (bucket) of
// W3t gets [cs_hi | cs_hi | cs_lo] of cs[n] (d values, zeros to 64 each) in
// columns MLP_H .. MLP_H + 191.
__global__ void k_prior_cols(const float* __restrict__ cs, int ld, int d,
                             __nv_bfloat16* __restrict__ w3t, int ldw) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(MLP_OUT) * 64) return;
    const int n = int(t / 64), c = int(t % 64);
    const float x = c < d ? cs[size_t(n) * ld + c] : 0.f;
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
    __nv_bfloat16* e = w3t + size_t(n) * ldw + MLP_H;
    e[c] = hi;
    e[64 + c] = hi;
    e[128 + c] = lo;
}

// Y [rows x N] FP32 -> BF16 row-major (may be null) and transposed [N x ldt],
// through 32 x 32 shared-memory tiles.
__global__ void k_bf16_both(const float* __restrict__ Y, int rows, int N,
                            __nv_bfloat16* __restrict__ yb, __nv_bfloat16* __restrict__ yt,
                            int ldt) {
    __shared__ float tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads: 8 rows a pass
    for (int i = ty; i < 32; i += 8) {
        const int r = r0 + i, c = c0 + tx;
        float v = 0.f;
        if (r < rows && c < N) {
            v = Y[size_t(r) * N + c];
            if (yb) yb[size_t(r) * N + c] = __float2bfloat16_rn(v);
        }
        tile[i][tx] = v;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        const int c = c0 + i, r = r0 + tx;
        if (c < N && r < rows) yt[size_t(c) * ldt + r] = __float2bfloat16_rn(tile[tx][i]);
    }
}

// BF16 transposed weights: W1t [256 x 64] (columns >= d zero), W2t [256 x 256],
// W3t [1024 x 256] (leading dimension MLP_K3: its prior columns are left as
// they are), from the FP32 masters W1 [d x 256], W2 [256 x 256], W3 [256 x 1024].
__global__ void k_w_transpose(const float* __restrict__ w, MlpLayout L, int d,
                              __nv_bfloat16* __restrict__ wt) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n1 = size_t(MLP_H) * 64, n2 = size_t(MLP_H) * MLP_H, n3 = size_t(MLP_OUT) * MLP_H;
    if (t < n1) {
        const int n = int(t / 64), k = int(t % 64);
        wt[t] = __float2bfloat16_rn(k < d ? w[L.w1 + size_t(k) * MLP_H + n] : 0.f);
    } else if (t < n1 + n2) {
        const size_t u = t - n1;
        const int n = int(u / MLP_H), k = int(u % MLP_H);
        wt[t] = __float2bfloat16_rn(w[L.w2 + size_t(k) * MLP_H + n]);
    } else if (t < n1 + n2 + n3) {
        const size_t u = t - n1 - n2;
        const int n = int(u / MLP_H), k = int(u % MLP_H);
        wt[n1 + n2 + size_t(n) * MLP_K3 + k] = __float2bfloat16_rn(w[L.w3 + size_t(k) * MLP_OUT + n]);
    }
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
                       float c1, float c2, float eps) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
}


// The P largest logits of each row (ties by index), descending, skipping the
// bucket `skip[r]` (the row's own primary, probed anyway).  One warp per row:
// each lane holds its 32 columns (j = 32 t + lane) in registers, and each of
// the P picks is a register scan and a warp argmax.
__global__ void k_topp(const float* __restrict__ Z, int rows, int P,
                       const uint32_t* __restrict__ skip, uint32_t* __restrict__ out) {
    const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    constexpr int PER = MLP_OUT / 32;
    const float* z = Z + size_t(r) * MLP_OUT;
    const uint32_t sk = skip ? skip[r] : 0xFFFFFFFFu;
    float v[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int j = t * 32 + lane;
        v[t] = uint32_t(j) == sk ? -__int_as_float(0x7f800000) : z[j];
    }
    for (int p = 0; p < P; ++p) {
        float bv = -__int_as_float(0x7f800000);
        int bt = 0;
#pragma unroll
        for (int t = 0; t < PER; ++t)
            if (v[t] > bv) {  // strict: the lowest column wins a tie within the lane
                bv = v[t];
                bt = t;
            }
        int bj = bv == -__int_as_float(0x7f800000) ? 0x7FFFFFFF : bt * 32 + lane;
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
            const int oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
            if (ov > bv || (ov == bv && oj < bj)) {
                bv = ov;
                bj = oj;
            }
        }
        if (bj != 0x7FFFFFFF && lane == (bj & 31)) {
#pragma unroll
            for (int t = 0; t < PER; ++t)
                if (t == (bj >> 5)) v[t] = -__int_as_float(0x7f800000);
        }
        if (lane == 0) out[size_t(r) * P + p] = bj == 0x7FFFFFFF ? 0u : uint32_t(bj);
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

size_t mlp_wt_elems() {
    return size_t(MLP_H) * 64 + 2 * size_t(MLP_H) * MLP_H + size_t(MLP_OUT) * MLP_K3 +
           size_t(MLP_OUT) * MLP_H;
}

namespace {
// Offsets (elements) of the BF16 weight copies in `wt`; all 256-byte aligned.
struct WtLayout {
    size_t w1t, w2t, w3t, w2, w3;
};
WtLayout wt_layout() {
    WtLayout L;
    L.w1t = 0;
    L.w2t = L.w1t + size_t(MLP_H) * 64;
    L.w3t = L.w2t + size_t(MLP_H) * MLP_H;
    L.w2 = L.w3t + size_t(MLP_OUT) * MLP_K3;
    L.w3 = L.w2 + size_t(MLP_H) * MLP_H;
    return L;
}

// Row-major BF16 copies of W2 [256 x 256] and W3 [256 x 1024] (the B operands
// of the backward products).
__global__ void k_w_rowmajor(const float* __restrict__ w, MlpLayout L,
                             __nv_bfloat16* __restrict__ w2, __nv_bfloat16* __restrict__ w3) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t n2 = size_t(MLP_H) * MLP_H, n3 = size_t(MLP_H) * MLP_OUT;
    if (t < n2) w2[t] = __float2bfloat16_rn(w[L.w2 + t]);
    else if (t < n2 + n3) w3[t - n2] = __float2bfloat16_rn(w[L.w3 + (t - n2)]);
}

void refresh_wt(const MlpView& net, cudaStream_t st) {
    const MlpLayout L = mlp_layout(net.d);
    const WtLayout W = wt_layout();
    const size_t nt = size_t(MLP_H) * 64 + size_t(MLP_H) * MLP_H + size_t(MLP_OUT) * MLP_H;
    k_w_transpose<<<unsigned((nt + 255) / 256), 256, 0, st>>>(net.w, L, net.d, net.wt);
    count_launch();
    const size_t nr = size_t(MLP_H) * MLP_H + size_t(MLP_H) * MLP_OUT;
    k_w_rowmajor<<<unsigned((nr + 255) / 256), 256, 0, st>>>(net.w, L, net.wt + W.w2,
                                                             net.wt + W.w3);
    count_launch();
}

size_t up64(size_t x) { return (x + 63) / 64 * 64; }
}  // namespace

size_t mlp_bufs_bytes(int rows, bool train) {
    const size_t R = up64(size_t(rows));
    size_t e = R * (64 + MLP_H + MLP_K3);                         // xb, h1b, h2b
    if (train) e += R * (MLP_OUT + MLP_H) + R * (64 + 4 * MLP_H + MLP_OUT);  // dzb, dh2b; transposes
    return e * sizeof(__nv_bfloat16) + 16 * 256;
}

MlpBufs mlp_bufs(void* base, int rows, bool train) {
    MlpBufs b{};
    const size_t R = up64(size_t(rows));
    b.ldt = int(R);
    __nv_bfloat16* p = static_cast<__nv_bfloat16*>(base);
    auto take = [&](size_t elems) {
        __nv_bfloat16* q = p;
        p += (elems + 127) / 128 * 128;  // 256-byte aligned pieces
        return q;
    };
    b.xb = take(R * 64);
    b.h1b = take(R * MLP_H);
    b.h2b = take(R * MLP_K3);
    if (train) {
        b.dzb = take(R * MLP_OUT);
        b.dh2b = take(R * MLP_H);
        b.xt = take(R * 64);
        b.h1t = take(R * MLP_H);
        b.h2t = take(R * MLP_H);
        b.dzt = take(R * MLP_OUT);
        b.dh2t = take(R * MLP_H);
        b.dh1t = take(R * MLP_H);
    }
    return b;
}

cudaError_t mlp_forward(const MlpView& net, const float* X, int rows, float* H1, float* H2,
                        float* Z, const MlpBufs& b, bool train, cudaStream_t st,
                        const MlpPrior* prior) {
    const MlpLayout L = mlp_layout(net.d);
    const WtLayout W = wt_layout();
    const bool pr = prior && prior->cs;
    k_x_bf16<<<unsigned((size_t(rows) * 64 + 255) / 256), 256, 0, st>>>(
        X, rows, net.d, b.xb, train ? b.xt : nullptr, b.ldt, pr ? b.h2b + MLP_H : nullptr,
        MLP_K3);
    count_launch();
    TcOut o = tc_out(rows, MLP_H, 64, net.err);
    o.bias = net.w + L.b1;
    o.relu = 1;
    o.C = H1;
    o.ldc = MLP_H;
    o.Cb = b.h1b;
    o.ldcb = MLP_H;
    if (train) {
        o.Ct = b.h1t;
        o.ldct = b.ldt;
    }
    if (!tc_gemm(b.xb, 64, net.wt + W.w1t, 64, o, st)) return cudaErrorInvalidValue;
    o = tc_out(rows, MLP_H, MLP_H, net.err);
    o.bias = net.w + L.b2;
    o.relu = 1;
    o.C = H2;
    o.ldc = MLP_H;
    o.Cb = b.h2b;
    o.ldcb = MLP_K3;
    if (train) {
        o.Ct = b.h2t;
        o.ldct = b.ldt;
    }
    if (!tc_gemm(b.h1b, MLP_H, net.wt + W.w2t, MLP_H, o, st)) return cudaErrorInvalidValue;
    // the output product, with the prior's 192 columns when there is one
    o = tc_out(rows, MLP_OUT, pr ? MLP_K3 : MLP_H, net.err);
    o.bias = net.w + L.b3;
    o.bias2 = pr ? prior->cb : nullptr;
    o.C = Z;
    o.ldc = MLP_OUT;
    if (!tc_gemm(b.h2b, MLP_K3, net.wt + W.w3t, MLP_K3, o, st)) return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t mlp_backward(const MlpView& net, int rows, float* H1, float* H2, float* Z,
                         const MlpBufs& b, const uint32_t* tb, const float* tw, int T,
                         float* loss, float* dH1, float* dH2, float* grad, float* scratch,
                         cudaStream_t st) {
    const MlpLayout L = mlp_layout(net.d);
    const WtLayout W = wt_layout();
    // Z becomes dZ, and its BF16 copies
    k_softmax_xent<<<(rows + 7) / 8, 256, 0, st>>>(Z, rows, MLP_OUT, tb, tw, T, loss);
    count_launch();
    k_bf16_both<<<dim3(MLP_OUT / 32, (rows + 31) / 32), 256, 0, st>>>(Z, rows, MLP_OUT, b.dzb,
                                                                      b.dzt, b.ldt);
    count_launch();
    // layer 3: dW3 = H2^T dZ, db3, dH2 = (dZ W3^T) * (H2 > 0)
    TcOut o = tc_out(MLP_H, MLP_OUT, rows, net.err);
    o.C = grad + L.w3;
    o.ldc = MLP_OUT;
    if (!tc_gemm(b.h2t, b.ldt, b.dzt, b.ldt, o, st)) return cudaErrorInvalidValue;
    col_sums(Z, rows, MLP_OUT, scratch, grad + L.b3, st);
    o = tc_out(rows, MLP_H, MLP_OUT, net.err);
    o.mask = H2;
    o.ldm = MLP_H;
    o.C = dH2;
    o.ldc = MLP_H;
    o.Cb = b.dh2b;
    o.ldcb = MLP_H;
    o.Ct = b.dh2t;
    o.ldct = b.ldt;
    if (!tc_gemm(b.dzb, MLP_OUT, net.wt + W.w3, MLP_OUT, o, st)) return cudaErrorInvalidValue;
    // layer 2: dW2 = H1^T dH2, db2, dH1 = (dH2 W2^T) * (H1 > 0)
    o = tc_out(MLP_H, MLP_H, rows, net.err);
    o.C = grad + L.w2;
    o.ldc = MLP_H;
    if (!tc_gemm(b.h1t, b.ldt, b.dh2t, b.ldt, o, st)) return cudaErrorInvalidValue;
    col_sums(dH2, rows, MLP_H, scratch, grad + L.b2, st);
    o = tc_out(rows, MLP_H, MLP_H, net.err);
    o.mask = H1;
    o.ldm = MLP_H;
    o.C = dH1;
    o.ldc = MLP_H;
    o.Ct = b.dh1t;
    o.ldct = b.ldt;
    if (!tc_gemm(b.dh2b, MLP_H, net.wt + W.w2, MLP_H, o, st)) return cudaErrorInvalidValue;
    // layer 1: dW1 = X^T dH1, db1
    o = tc_out(net.d, MLP_H, rows, net.err);
    o.C = grad + L.w1;
    o.ldc = MLP_H;
    if (!tc_gemm(b.xt, b.ldt, b.dh1t, b.ldt, o, st)) return cudaErrorInvalidValue;
    col_sums(dH1, rows, MLP_H, scratch, grad + L.b1, st);
    return cudaGetLastError();
}

void mlp_adam(MlpView& net, float* m, float* v, const float* grad, int step, float lr,
              cudaStream_t st) {
    const size_t np = mlp_params(net.d);
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    k_adam<<<unsigned((np + 255) / 256), 256, 0, st>>>(net.w, m, v, grad, np, lr, b1, b2, c1, c2,
                                                       1e-8f);
    count_launch();
    refresh_wt(net, st);
}

void mlp_sync_bf16(MlpView& net, cudaStream_t st) { refresh_wt(net, st); }

void mlp_set_prior(MlpView& net, const MlpPrior& prior, cudaStream_t st) {
    const WtLayout W = wt_layout();
    k_prior_cols<<<unsigned((size_t(MLP_OUT) * 64 + 255) / 256), 256, 0, st>>>(
        prior.cs, prior.ld, net.d, net.wt + W.w3t, MLP_K3);
    count_launch();
}

void mlp_topp(const float* Z, int rows, int P, const uint32_t* skip, uint32_t* out,
              cudaStream_t st) {
    k_topp<<<(rows + 7) / 8, 256, 0, st>>>(Z, rows, P, skip, out);
    count_launch();
}

}  // namespace pq
