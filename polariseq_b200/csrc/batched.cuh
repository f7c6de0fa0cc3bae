// Batched exact kNN over many samples in one persistent launch (batched.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pq {

struct BatchLaunch {
    const float* X;          // all samples' rows, row-major, d floats each
    int d;                   // <= 64
    const uint64_t* s_off;   // device: sample row offsets (n_samples + 1)
    const uint32_t* s_k;     // device: neighbours per point, per sample
    const uint64_t* s_out;   // device: output offset of each sample's first row
    const uint32_t* item_s;  // device: work item -> sample
    const uint32_t* item_q;  // device: work item -> first local query
    uint32_t n_items;
    uint32_t* counter;       // device: zero before the launch
    int kp;                  // power of two >= the largest k
    int sms;
    uint32_t* out_idx;
    float* out_dist;
};

// Tile shapes (queries per warp x warps per CTA) the autotuner chooses from.
int batched_shapes();
int batched_queries_per_item(int shape);
bool batched_shape_fits(int shape, int d, int kp);
cudaError_t launch_batched_knn(const BatchLaunch& b, int shape, cudaStream_t st);

}  // namespace pq
