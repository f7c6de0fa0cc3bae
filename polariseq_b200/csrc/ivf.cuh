// Chosen form (tensor-core shortlist) interfaces.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pq {

// One tensor-core tile job list: job j covers query entries
// [job_qstart[j], job_qend[j]) (at most 128) against the candidates
// [c_off[b], c_off[b + 1]) of bucket b = job_bucket[j].  Query rows are
// [q~, -1/2, -1/2, 0...] and candidate rows [x~, hi, lo, 0...] (BF16, 64
// columns) with hi + lo = |x~|^2.
struct IvfTileArgs {
    const uint32_t* job_bucket;  // the job's candidate bucket
    const uint32_t* job_qstart;  // the job's query entries [qstart, qend)
    const uint32_t* job_qend;
    const uint32_t* job_tstart;  // optional: the candidate tile each job starts from
    uint32_t njobs;
    const uint32_t* c_off;   // buckets + 1
    const float* qnorm;      // per query entry: |q~|^2 of its BF16 row
    const float* qthr;       // optional per query entry: initial admission bound
    const uint32_t* qself;   // per query entry: its own candidate position, or ~0
    int S;                   // shortlist length per entry and column half: 1, 16 or 32
    // 1: admitted entries are staged in a shared-memory buffer and merged
    // into the shortlist when it fills and at job end (for launches whose
    // bound starts tight, qthr, so that admissions are rare); 0: each is
    // inserted at once, tightening the bound (launches that start unbounded)
    int buffered;
    // E4M3 tiles (the maps hold 128 one-byte columns per row, no norm
    // columns): the accumulator times qscale[entry] * cscale[candidate] (each
    // row's own inverse scale) is the dot product, and chalf[candidate] =
    // |x~|^2 / 2 is subtracted in FP32
    int fp8;
    const float* qscale;
    const float* cscale;
    const float* chalf;
    float* out_d;            // entries x (ivf_groups() x S): ascending runs of S
    uint32_t* out_i;         // the candidate positions (~0 = none)
    // optional: the number of finite entries of each run (a prefix), written
    // to out_n[out_slot[entry] * ivf_groups() + half] (out_slot null: entry);
    // when given, only that prefix of the run is written
    uint8_t* out_n;
    const uint32_t* out_slot;
    int* err;
    unsigned long long* trace;  // optional: block 0 cycle counters (IVF_T_*)
    // test hook: when non-zero, thread 0 of every CTA first waits this many
    // polls on a barrier that nothing arrives at, before any copy or MMA is
    // issued; the wait gives up, every role skips its jobs and the kernel
    // reports error 2 (a bounded wait gave up) with nothing in flight
    uint32_t test_wait_polls;
    // BF16 with S = 16: jobs of ivf_job_rows(1) = 256 query entries against
    // candidate tiles of ivf_tile_cols(1) = 128 (16 epilogue warps); else 128
    // entries against tiles of 256
    int wide;
};

enum { IVF_T_EPI_WAIT = 0, IVF_T_EPI_WORK = 1, IVF_T_EPI_END = 2, IVF_T_MMA_WAIT_C = 3,
       IVF_T_MMA_WAIT_T = 4, IVF_T_TMA_WAIT = 5, IVF_T_TILES = 6, IVF_T_TOTAL = 7,
       IVF_T_JOBS = 8, IVF_T_SLOW = 9, IVF_T_ADMITS = 10, IVF_T_WMBITS = 11,
       IVF_T_SLOW_CYC = 12, IVF_T_LD_CYC = 13, IVF_TRACE_N = 16 };

bool make_bf16_map(CUtensorMap* map, const void* base, uint64_t rows, uint32_t box_rows);
// A [rows x cols] BF16 matrix with leading dimension ld (elements, a multiple
// of 8; base 16-byte aligned) as 128-byte-swizzled boxes of box_rows x 64;
// reads beyond rows or cols fill zeros.
bool make_bf16_map_ld(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                      uint64_t ld, uint32_t box_rows);
// A [rows x 128] one-byte (E4M3) matrix as 128-byte-swizzled boxes of box_rows x 128.
bool make_fp8_map(CUtensorMap* map, const void* base, uint64_t rows, uint32_t box_rows);
// Runs of one entry's output row.
int ivf_groups();
// The shortlist length the kernel supports for `want` entries (0 = too many).
int ivf_shortlist(int want);
// Job and tile geometry: query entries per job and candidates per tile (the
// maps' box rows), for the wide (BF16, S = 16) or the standard kernel.
inline int ivf_job_rows(int wide) { return wide ? 256 : 128; }
inline int ivf_tile_cols(int wide) { return wide ? 128 : 256; }
cudaError_t launch_ivf_tiles(const CUtensorMap& tmQ, const CUtensorMap& tmC,
                             const IvfTileArgs& a, int grid, cudaStream_t st);

}  // namespace pq
