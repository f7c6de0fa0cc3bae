// Learned bucket routing MLP (mlp.cu): d -> 256 -> 256 -> 1024, ReLU.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pq {

constexpr int MLP_H = 256;     // hidden width
constexpr int MLP_OUT = 1024;  // bucket logits
constexpr int MLP_K3 = MLP_H + 192;  // the output product's K with the prior's columns

// Offsets (in parameters) of W1 [d x H], b1 [H], W2 [H x H], b2, W3 [H x OUT], b3.
struct MlpLayout {
    size_t w1, b1, w2, b2, w3, b3;
};
MlpLayout mlp_layout(int d);
size_t mlp_params(int d);
size_t mlp_scratch_floats();

// FP32 master parameters `w`; `wt` (mlp_wt_elems) holds the BF16 copies the
// tensor-core products read (mlp_sync_bf16 / mlp_adam refresh them): W1^T
// [256 x 64], W2^T, W3^T [1024 x MLP_K3: 256 weights + the prior's 192
// columns], W2 and W3 row-major; `err` (device int) receives 2 if a bounded
// wait of a product gave up.
struct MlpView {
    int d;
    float* w;
    __nv_bfloat16* wt;
    int* err;
};
size_t mlp_wt_elems();

// BF16 operand copies of one batch of at most `rows` rows: X (padded to 64
// columns), H1, H2, dZ, dH2 row-major and X, H1, H2, dZ, dH2, dH1 transposed
// (leading dimension ldt = rows rounded up to 64).  Inference needs only the
// row-major X, H1, H2.
struct MlpBufs {
    __nv_bfloat16 *xb, *h1b, *h2b, *dzb, *dh2b;
    __nv_bfloat16 *xt, *h1t, *h2t, *dzt, *dh2t, *dh1t;
    int ldt;
};
size_t mlp_bufs_bytes(int rows, bool train);
MlpBufs mlp_bufs(void* base, int rows, bool train);

// The nearest-centroid prior added to the logits: -beta |x - c_b|^2 up to a
// per-row constant, i.e. X . cs_b^T + cb_b with cs = 2 beta c (1024 x d rows,
// stride ld) and cb = -beta |c_b|^2.  The MLP learns a correction to it.
struct MlpPrior {
    const float* cs = nullptr;
    int ld = 0;
    const float* cb = nullptr;
};

// H1 = relu(X W1 + b1), H2 = relu(H1 W2 + b2), Z = H2 W3 + b3 (+ prior)
// (rows x 1024); `train` also writes the transposed copies the backward pass
// reads.  Returns cudaErrorInvalidValue if a tensor map cannot be made.
cudaError_t mlp_forward(const MlpView& net, const float* X, int rows, float* H1, float* H2,
                        float* Z, const MlpBufs& b, bool train, cudaStream_t st,
                        const MlpPrior* prior = nullptr);
// Softmax cross-entropy against sparse soft targets (T pairs per row, bucket
// ~0 unused) and the parameter gradients of the mean loss into `grad`
// (overwritten); Z is overwritten with dZ, loss gets the per-row loss.
cudaError_t mlp_backward(const MlpView& net, int rows, float* H1, float* H2, float* Z,
                         const MlpBufs& b, const uint32_t* tb, const float* tw, int T,
                         float* loss, float* dH1, float* dH2, float* grad, float* scratch,
                         cudaStream_t st);
// One Adam step (step >= 1) on the master weights; refreshes the BF16 copies.
void mlp_adam(MlpView& net, float* m, float* v, const float* grad, int step, float lr,
              cudaStream_t st);
void mlp_sync_bf16(MlpView& net, cudaStream_t st);
// Writes the prior's columns of the output product's BF16 weights once (they
// survive the Adam steps' refreshes); a forward pass given the prior uses them.
void mlp_set_prior(MlpView& net, const MlpPrior& prior, cudaStream_t st);
// The P largest logits of each row, skipping skip[r] (may be null).
void mlp_topp(const float* Z, int rows, int P, const uint32_t* skip, uint32_t* out,
              cudaStream_t st);

}  // namespace pq
