// Chosen form, stage 1: bucketed distance tiles on tcgen05 tensor cores.
//
// The cells are split into buckets (k-means centroids); every cell is a
// candidate of exactly one bucket (its primary) and probes P buckets as a
// query.  Within a bucket, coordinates are centred on the bucket's centroid
// before rounding to BF16 (squared distances are shift invariant, and centring
// keeps BF16's 8-bit mantissa accurate at the scale of neighbour distances).
//
// Rows are augmented so that one product gives the ranking quantity: a query
// row is [q~, -1/2, -1/2, 0...] and a candidate row [x~, hi, lo, 0...] with
// hi + lo = |x~|^2 (hi = BF16(|x~|^2), lo = BF16 of the remainder, 2^-17
// relative), so the accumulator holds a = q~.x~ - |x~|^2 / 2 and the
// approximate squared distance is |q~|^2 - 2a.  An entry with admission bound
// thr keeps a candidate only if a > (|q~|^2 - thr) / 2: the hot loop is one
// three-input max per two accumulators and a warp vote per 32 columns; only
// the columns some row of the warp admits are visited after that.
//
// One CTA per SM runs a persistent job loop (job = 128 query entries of one
// bucket against all of the bucket's candidates, 256 per tile) with
// warp-specialised roles and mbarrier hand-offs, no CTA-wide barrier inside
// the loop:
//   warp 8 (one lane)  TMA loads: the job's Q tile (2 stages) and candidate
//                      tiles (3 stages, 128-byte swizzled, K-major);
//   warp 9 (one lane)  tcgen05.mma M=128 N=256 K=16 x4 into one of two TMEM
//                      accumulator buffers (256 columns each); commits free
//                      the candidate stage and fill the TMEM buffer;
//   warps 0-7          epilogue: warp w reads TMEM lanes 32(w%4).. (its query
//                      rows) for column half w/4 (tcgen05.ld 32x32b), 32
//                      columns at a time, and filters; in a chunk that some
//                      row admits, each lane takes its admitted columns, then
//                      the TMEM buffer is freed.
// Each thread keeps its row's shortlist for its column half in registers: S
// (distance, candidate) pairs in ascending order, a new entry shifting the
// worse ones up by one place (S - 1 compare-and-selects, no memory traffic).
// Launches that start unbounded insert every admitted column at once, so the
// bound tightens with each insertion; seeded launches (few admissions) stage
// them in a shared-memory buffer merged when it fills and at job end.  At job
// end the shortlist is written as it stands: the output row of an entry is NG
// ascending runs of S (and, when asked, the number of finite entries of each
// run).
//
// BF16 launches with 16-entry shortlists run k_ivf_wide (further down), the
// same scheme with jobs of 256 query entries, 128-candidate tiles and 16
// epilogue warps.
//
// Every wait is bounded: a wait that gives up raises the CTA's abort flag,
// every role leaves its loop, in-flight copies and MMAs are waited for (again
// bounded), TMEM is freed and the kernel reports error 2.
#include <cuda.h>

#include "common.cuh"
#include "ivf.cuh"
#include "tc.cuh"

namespace pq {
namespace {

constexpr int TQ = 128;   // query rows per tile (TMEM lanes)
constexpr int TCN = 256;  // candidate rows per tile (TMEM columns per buffer)
constexpr int ROWB = 128; // bytes per BF16 row (64 dims)
constexpr int NG = 2;     // epilogue warpgroups: each owns half of a tile's columns
constexpr int NEPI = TQ * NG;   // epilogue threads
constexpr int NT = NEPI + 64;   // + TMA warp + MMA warp
constexpr int CPG = TCN / NG;   // columns per warpgroup
constexpr int BUF = 32;         // staged admissions per (row, column half), buffered mode
                                // (at least the 32 one chunk can admit)
constexpr int STASH = 32;       // BF16: floats per epilogue thread, a flagged chunk's values
constexpr int QST = 2;          // Q tile stages
constexpr int MAXCS = 3;        // candidate tile stages (at most)
constexpr uint32_t WAIT_LIMIT = 1u << 24;
constexpr uint32_t FULL = 0xFFFFFFFFu;

struct __align__(8) IvfBars {
    uint64_t q_full[QST], q_empty[QST];
    uint64_t c_full[MAXCS], c_empty[MAXCS];
    uint64_t t_full[2], t_empty[2];
    uint64_t done;
    uint64_t never;  // nothing arrives here: the target of the timeout test hook
    uint32_t tmem;
    int abort;
};

__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
// Maximum of 32 values as a tree of three-input maxes.
__device__ __forceinline__ float max32(const float (&v)[32]) {
    float m[11];
#pragma unroll
    for (int i = 0; i < 10; ++i) m[i] = max3f(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    m[10] = fmaxf(v[30], v[31]);
    const float a = max3f(m[0], m[1], m[2]), b = max3f(m[3], m[4], m[5]),
                c = max3f(m[6], m[7], m[8]), d = fmaxf(m[9], m[10]);
    return fmaxf(max3f(a, b, c), d);
}

// x[j] for a per-lane j in [0, 32): a five-level select tree over the
// registers (no local-memory indexing).
__device__ __forceinline__ uint32_t select32(const uint32_t (&x)[32], int j) {
    uint32_t a[16], b[8], c[4], d[2];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = (j & 16) ? x[i + 16] : x[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) b[i] = (j & 8) ? a[i + 8] : a[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) c[i] = (j & 4) ? b[i + 4] : b[i];
#pragma unroll
    for (int i = 0; i < 2; ++i) d[i] = (j & 2) ? c[i + 2] : c[i];
    return (j & 1) ? d[1] : d[0];
}

// Inserts (d, id) into an ascending register shortlist of S entries (the
// caller checked d < v[S - 1]): the entries after it move up one place and
// the last one drops out.  Equal distances keep their arrival order.
template <int S>
__device__ __forceinline__ void shortlist_push(float (&v)[S], uint32_t (&x)[S], float d,
                                               uint32_t id) {
#pragma unroll
    for (int j = S - 1; j > 0; --j) {
        const bool up = d < v[j - 1];
        const bool here = !up && d < v[j];
        v[j] = up ? v[j - 1] : (here ? d : v[j]);
        x[j] = up ? x[j - 1] : (here ? id : x[j]);
    }
    if (d < v[0]) {
        v[0] = d;
        x[0] = id;
    }
}

__host__ __device__ constexpr int cand_stages(int, bool) { return 3; }

template <int S, bool F8>
__global__ void __launch_bounds__(NT, 1) k_ivf_tiles(const __grid_constant__ CUtensorMap tmQ,
                                                     const __grid_constant__ CUtensorMap tmC,
                                                     IvfTileArgs a) {
    constexpr int NCS = cand_stages(S, F8);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-align the dynamic region (the swizzle pattern follows address bits)
    uint8_t* smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* sQ = smem;                                          // QST x 16 KB
    uint8_t* sC = sQ + QST * TQ * ROWB;                          // NCS x 32 KB
    float* bdall = reinterpret_cast<float*>(sC + NCS * TCN * ROWB);        // NG x BUF x TQ
    uint32_t* biall = reinterpret_cast<uint32_t*>(bdall + NG * BUF * TQ);  // NG x BUF x TQ
    // E4M3 only: |x~|^2 / 2 and the inverse scale of the tile's columns, per
    // TMEM buffer parity and column half (the four warps of a half write the
    // same values)
    float* hsall = reinterpret_cast<float*>(biall + NG * BUF * TQ);        // 2 x NG x CPG
    float* hkall = hsall + 2 * NG * CPG;                                   // 2 x NG x CPG
    // BF16: each epilogue thread's stash row for a flagged chunk (its 16-byte
    // groups XOR-swizzled by lane so that a warp's stores hit every bank);
    // E4M3 (whose scale slots take the room) selects from registers instead
    float* stash = hsall;                                                  // NEPI x STASH
    __shared__ IvfBars B;
    __shared__ unsigned long long ld_cyc;  // tracing: block 0 warp 0's TMEM load waits
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    volatile int* abort_flag = &B.abort;

    if (w == 0) {
        tc::tmem_alloc(&B.tmem, 512);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < QST; ++s) {
            tc::mbar_init(&B.q_full[s], 1);
            tc::mbar_init(&B.q_empty[s], 1);
        }
        for (int s = 0; s < MAXCS; ++s) {
            tc::mbar_init(&B.c_full[s], 1);
            tc::mbar_init(&B.c_empty[s], 1);
        }
        for (int s = 0; s < 2; ++s) {
            tc::mbar_init(&B.t_full[s], 1);
            tc::mbar_init(&B.t_empty[s], NEPI / 32);
        }
        tc::mbar_init(&B.done, 1);
        tc::mbar_init(&B.never, 1);
        tc::fence_barrier_init();
        B.abort = 0;
        ld_cyc = 0;
        // the timeout test hook: a bounded wait that runs out before any work
        if (a.test_wait_polls && !tc::mbar_wait(&B.never, 0, a.test_wait_polls)) B.abort = 1;
    }
    if (tid == NEPI) {
        tc::prefetch_tmap(&tmQ);
        tc::prefetch_tmap(&tmC);
    }
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = B.tmem;
    const bool tracing = a.trace && blockIdx.x == 0;
    const long long c_start = clock64();

    if (w == NEPI / 32) {
        // ── TMA producer ──
        if (lane == 0) {
            uint32_t qi = 0, ci = 0;
            long long c_wait = 0;
            for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
                const uint32_t b = a.job_bucket[job], qs = a.job_qstart[job];
                const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
                const uint32_t nct = (ce - cs + TCN - 1) / TCN;
                // tiles run from the job's start tile, wrapping around
                const uint32_t tfirst =
                    (a.job_tstart && a.job_tstart[job] < nct) ? a.job_tstart[job] : 0u;
                if (nct == 0) continue;
                const int qsd = int(qi % QST);
                long long c0 = clock64();
                if (!tc::mbar_wait(&B.q_empty[qsd], ((qi / QST) & 1) ^ 1, WAIT_LIMIT)) {
                    *abort_flag = 1;
                    break;
                }
                c_wait += clock64() - c0;
                tc::mbar_expect_tx(&B.q_full[qsd], TQ * ROWB);
                tc::tma_load_2d(sQ + qsd * TQ * ROWB, &tmQ, &B.q_full[qsd], 0, int(qs));
                ++qi;
                for (uint32_t t = 0; t < nct; ++t) {
                    const int s = int(ci % NCS);
                    c0 = clock64();
                    if (!tc::mbar_wait(&B.c_empty[s], ((ci / NCS) & 1) ^ 1, WAIT_LIMIT)) {
                        *abort_flag = 1;
                        break;
                    }
                    c_wait += clock64() - c0;
                    tc::mbar_expect_tx(&B.c_full[s], TCN * ROWB);
                    const uint32_t tt = tfirst + t >= nct ? tfirst + t - nct : tfirst + t;
                    tc::tma_load_2d(sC + s * TCN * ROWB, &tmC, &B.c_full[s], 0, int(cs + tt * TCN));
                    ++ci;
                }
            }
            // every issued copy has landed before the CTA may exit
            for (int s = 0; s < NCS; ++s) {
                const uint32_t uses = ci / NCS + (uint32_t(s) < ci % NCS ? 1u : 0u);
                if (uses > 0 && !tc::mbar_wait(&B.c_full[s], (uses - 1) & 1, WAIT_LIMIT))
                    *abort_flag = 1;
            }
            for (int s = 0; s < QST; ++s) {
                const uint32_t uses = qi / QST + (uint32_t(s) < qi % QST ? 1u : 0u);
                if (uses > 0 && !tc::mbar_wait(&B.q_full[s], (uses - 1) & 1, WAIT_LIMIT))
                    *abort_flag = 1;
            }
            if (tracing) a.trace[IVF_T_TMA_WAIT] = (unsigned long long)c_wait;
        }
        __syncwarp();
    } else if (w == NEPI / 32 + 1) {
        // ── MMA issuer ──
        if (lane == 0) {
            const uint32_t idesc = F8 ? tc::idesc_e4m3_f32(TQ, TCN) : tc::idesc_bf16_f32(TQ, TCN);
            uint32_t qi = 0, ci = 0, ti = 0;
            long long c_wait_c = 0, c_wait_t = 0;
            for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
                const uint32_t b = a.job_bucket[job];
                const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
                const uint32_t nct = (ce - cs + TCN - 1) / TCN;
                if (nct == 0) continue;
                const int qsd = int(qi % QST);
                if (!tc::mbar_wait(&B.q_full[qsd], (qi / QST) & 1, WAIT_LIMIT)) {
                    *abort_flag = 1;
                    break;
                }
                const uint64_t dQ = tc::desc_k_sw128(tc::smem_u32(sQ + qsd * TQ * ROWB));
                bool ok = true;
                for (uint32_t t = 0; t < nct && ok; ++t) {
                    const int s = int(ci % NCS), tb = int(ti & 1);
                    long long c0 = clock64();
                    ok = tc::mbar_wait(&B.c_full[s], (ci / NCS) & 1, WAIT_LIMIT);
                    long long c1 = clock64();
                    ok = ok && tc::mbar_wait(&B.t_empty[tb], ((ti >> 1) & 1) ^ 1, WAIT_LIMIT);
                    c_wait_c += c1 - c0;
                    c_wait_t += clock64() - c1;
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint64_t dC = tc::desc_k_sw128(tc::smem_u32(sC + s * TCN * ROWB));
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)  // K = 64 as four K = 16 steps (32 B each)
                        if constexpr (F8)  // K = 128 one-byte columns as four K = 32 steps
                            tc::umma_f8(taddr + uint32_t(tb * TCN), dQ + uint64_t(2 * kk),
                                        dC + uint64_t(2 * kk), idesc, kk > 0 ? 1u : 0u);
                        else
                            tc::umma_f16(taddr + uint32_t(tb * TCN), dQ + uint64_t(2 * kk),
                                         dC + uint64_t(2 * kk), idesc, kk > 0 ? 1u : 0u);
                    tc::umma_commit(&B.c_empty[s]);
                    tc::umma_commit(&B.t_full[tb]);
                    ++ci;
                    ++ti;
                }
                tc::umma_commit(&B.q_empty[qsd]);
                ++qi;
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
            }
            // every issued MMA has completed before TMEM is freed
            tc::umma_commit(&B.done);
            if (!tc::mbar_wait(&B.done, 0, WAIT_LIMIT)) *abort_flag = 1;
            if (tracing) {
                a.trace[IVF_T_MMA_WAIT_C] = (unsigned long long)c_wait_c;
                a.trace[IVF_T_MMA_WAIT_T] = (unsigned long long)c_wait_t;
                a.trace[IVF_T_TILES] = ti;
            }
        }
        __syncwarp();
    } else {
        // ── epilogue ──
        const int g = w >> 2;
        const int row = (w & 3) * 32 + lane;
        const uint32_t lane_base = uint32_t((w & 3) * 32) << 16;
        const bool t0 = tracing && tid == 0;
        const bool buffered = a.buffered != 0;
        float* bd = bdall + size_t(g) * BUF * TQ + row;
        uint32_t* bi = biall + size_t(g) * BUF * TQ + row;
        long long c_wait = 0, c_work = 0, c_end = 0, c_slow = 0;
        unsigned long long jobs = 0, slow = 0, admits = 0, wmbits = 0;
        uint32_t ti = 0;
        // each job's descriptor is loaded one job ahead, so that a job's start
        // waits for one dependent load (the bucket's bounds), not two
        uint32_t nb = 0, nqs = 0, nqe = 0, nts = 0;
        auto load_job = [&](uint32_t j) {
            if (j < a.njobs) {
                nb = a.job_bucket[j];
                nqs = a.job_qstart[j];
                nqe = a.job_qend[j];
                nts = a.job_tstart ? a.job_tstart[j] : 0u;
            }
        };
        load_job(blockIdx.x);
        for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
            const uint32_t b = nb, qs = nqs, qe = nqe, ts = nts;
            load_job(job + gridDim.x);
            const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
            const uint32_t nct = (ce - cs + TCN - 1) / TCN;
            // tiles run from the job's start tile, wrapping around
            const uint32_t tfirst = ts < nct ? ts : 0u;
            const uint32_t entry = qs + row;
            const bool valid = entry < qe;
            // an invalid row's infinite |q|^2 makes its bound +inf or NaN: it
            // admits nothing
            const float qn = valid ? a.qnorm[entry] : __int_as_float(0x7f800000);
            const uint32_t qself = valid ? a.qself[entry] : 0xFFFFFFFFu;
            const float thr0 = (valid && a.qthr) ? a.qthr[entry] : __int_as_float(0x7f800000);
            // where the run length goes, loaded with the row's other inputs
            const uint32_t slot = (valid && a.out_slot) ? a.out_slot[entry] : entry;
            float thr = thr0;
            float ath = (qn - thr) * 0.5f;
            // E4M3: the query row's part of the accumulator's scale back to
            // the dot product (the candidate's part is per column)
            const float rq = F8 && valid ? a.qscale[entry] : 1.0f;
            // the shortlist: S ascending (distance, candidate) pairs in registers
            float sv[S];
            uint32_t sx[S];
#pragma unroll
            for (int j = 0; j < S; ++j) {
                sv[j] = __int_as_float(0x7f800000);
                sx[j] = 0xFFFFFFFFu;
            }
            int cnt = 0;  // staged entries (buffered mode)
            // merge the staged entries into the shortlist
            auto flush = [&]() {
                for (int u = 0; u < cnt; ++u) {
                    const float d = bd[u * TQ];
                    if (d < thr) {
                        shortlist_push<S>(sv, sx, d, bi[u * TQ]);
                        thr = fminf(thr0, sv[S - 1]);
                    }
                }
                cnt = 0;
                ath = (qn - thr) * 0.5f;
            };
            bool ok = true;
            for (uint32_t t = 0; t < nct; ++t) {
                const int tb = int(ti & 1);
                long long c0 = t0 ? clock64() : 0;
                ok = tc::mbar_wait(&B.t_full[tb], (ti >> 1) & 1, WAIT_LIMIT);
                ok = __all_sync(FULL, ok);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t tcol = taddr + lane_base + uint32_t(tb * TCN + g * CPG);
                // columns of this slice that belong to the bucket
                const uint32_t tt = tfirst + t >= nct ? tfirst + t - nct : tfirst + t;
                const int lim = int(ce) - int(cs + tt * TCN + g * CPG);
                const uint32_t cbase = cs + tt * TCN + g * CPG;
                long long c1 = t0 ? clock64() : 0;
                float* hs = hsall + (tb * NG + g) * CPG;
                float* hk = hkall + (tb * NG + g) * CPG;
                if constexpr (F8) {
#pragma unroll
                    for (int i = 0; i < CPG / 32; ++i) {
                        const int col = i * 32 + lane;
                        hs[col] = col < lim ? a.chalf[cbase + col] : 0.0f;
                        hk[col] = col < lim ? a.cscale[cbase + col] : 0.0f;
                    }
                    __syncwarp();
                }
                // the slice's four 32-column chunks, one at a time: one max and
                // one vote each; a chunk some row admits is handled on the spot
#pragma unroll 1
                for (int q = 0; q < CPG / 32; ++q) {
                    uint32_t r[32];
                    const long long cl = t0 ? clock64() : 0;
                    tc::tmem_ld32(tcol + uint32_t(q * 32), r);
                    tc::tmem_ld_wait();
                    if (t0) ld_cyc += clock64() - cl;
                    float v[32];
                    if constexpr (F8) {
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            const float4 h4 = *reinterpret_cast<const float4*>(hs + q * 32 + j);
                            const float4 k4 = *reinterpret_cast<const float4*>(hk + q * 32 + j);
                            v[j] = fmaf(__uint_as_float(r[j]) * k4.x, rq, -h4.x);
                            v[j + 1] = fmaf(__uint_as_float(r[j + 1]) * k4.y, rq, -h4.y);
                            v[j + 2] = fmaf(__uint_as_float(r[j + 2]) * k4.z, rq, -h4.z);
                            v[j + 3] = fmaf(__uint_as_float(r[j + 3]) * k4.w, rq, -h4.w);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
                    }
                    if (lim < (q + 1) * 32) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (q * 32 + j >= lim) v[j] = __int_as_float(0xff800000);
                    }
                    if (!__any_sync(FULL, max32(v) > ath)) continue;
                    const long long cs0 = t0 ? clock64() : 0;
                    uint32_t lm = 0;  // this lane's admitted columns
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (v[j] > ath) lm |= 1u << j;
                    // BF16: the chunk's values go to this thread's stash row, read
                    // back by column below (no register select per admission)
                    float* srow = stash + size_t(tid) * STASH;
                    const int swz = (lane & 7) << 2;
                    if constexpr (!F8) {
#pragma unroll
                        for (int j = 0; j < 32; j += 4)
                            *reinterpret_cast<float4*>(srow + (j ^ swz)) =
                                make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    }
                    if (tracing) {
                        const uint32_t na = __reduce_add_sync(FULL, uint32_t(__popc(lm)));
                        const uint32_t wm = __reduce_or_sync(FULL, lm);
                        if (t0) {
                            ++slow;
                            admits += na;
                            wmbits += __popc(wm);
                        }
                    }
                    // each lane takes its admitted columns, lowest first: into
                    // the shortlist at once (each checked against the bound its
                    // predecessors tightened), or staged (buffered mode; the
                    // buffer is merged first when this chunk could overflow it)
                    if (buffered &&
                        __reduce_max_sync(FULL, uint32_t(cnt + __popc(lm))) > uint32_t(BUF))
                        flush();
                    const uint32_t cb0 = cbase + q * 32;
                    while (__any_sync(FULL, lm != 0)) {
                        if (lm) {
                            const int j = __ffs(lm) - 1;
                            lm &= lm - 1;
                            float vj;
                            if constexpr (F8)
                                vj = fmaf(__uint_as_float(select32(r, j)) * hk[q * 32 + j], rq,
                                          -hs[q * 32 + j]);
                            else
                                vj = srow[j ^ swz];
                            const float dj = fmaf(-2.0f, vj, qn);
                            if (dj < thr && cb0 + j != qself) {
                                if (buffered) {
                                    bd[cnt * TQ] = dj;
                                    bi[cnt * TQ] = cb0 + j;
                                    ++cnt;
                                } else {
                                    shortlist_push<S>(sv, sx, dj, cb0 + j);
                                    thr = fminf(thr0, sv[S - 1]);
                                    ath = (qn - thr) * 0.5f;
                                }
                            }
                        }
                    }
                    if (t0) c_slow += clock64() - cs0;
                }
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&B.t_empty[tb]);
                ++ti;
                if (t0) {  // epi-wait: wait; epi-work: filter and admissions
                    const long long c2 = clock64();
                    c_wait += c1 - c0;
                    c_work += c2 - c1;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                break;
            }
            // job end: the shortlist (staged entries merged) is one ascending
            // run of S
            long long c3 = t0 ? clock64() : 0;
            if (cnt > 0) flush();
            if (valid) {
                // with run lengths asked for, only the live prefix is written
                int live = S;
                if (a.out_n) {
                    live = 0;
#pragma unroll
                    for (int j = 0; j < S; ++j)
                        live += sv[j] < __int_as_float(0x7f800000) ? 1 : 0;
                    a.out_n[size_t(slot) * NG + g] = uint8_t(live);
                }
                if constexpr (S % 4 == 0) {
                    float4* od = reinterpret_cast<float4*>(a.out_d + (size_t(entry) * NG + g) * S);
                    uint4* oi = reinterpret_cast<uint4*>(a.out_i + (size_t(entry) * NG + g) * S);
#pragma unroll
                    for (int j = 0; j < S / 4; ++j)
                        if (4 * j < live) {
                            od[j] = make_float4(sv[4 * j], sv[4 * j + 1], sv[4 * j + 2],
                                                sv[4 * j + 3]);
                            oi[j] = make_uint4(sx[4 * j], sx[4 * j + 1], sx[4 * j + 2],
                                               sx[4 * j + 3]);
                        }
                } else {
#pragma unroll
                    for (int j = 0; j < S; ++j)
                        if (j < live) {
                            a.out_d[(size_t(entry) * NG + g) * S + j] = sv[j];
                            a.out_i[(size_t(entry) * NG + g) * S + j] = sx[j];
                        }
                }
            }
            ++jobs;
            if (t0) c_end += clock64() - c3;
        }
        if (t0) {
            a.trace[IVF_T_EPI_WAIT] = (unsigned long long)c_wait;
            a.trace[IVF_T_EPI_WORK] = (unsigned long long)c_work;
            a.trace[IVF_T_EPI_END] = (unsigned long long)c_end;
            a.trace[IVF_T_JOBS] = jobs;
            a.trace[IVF_T_SLOW] = slow;
            a.trace[IVF_T_ADMITS] = admits;
            a.trace[IVF_T_WMBITS] = wmbits;
            a.trace[IVF_T_SLOW_CYC] = (unsigned long long)c_slow;
            a.trace[IVF_T_LD_CYC] = ld_cyc;
        }
    }
    __syncthreads();
    if (tracing && tid == 0) a.trace[IVF_T_TOTAL] = (unsigned long long)(clock64() - c_start);
    if (*abort_flag && tid == 0) atomicExch(a.err, 2);
    tc::tc_fence_after();
    if (w == 0) tc::tmem_dealloc(taddr, 512);
}

// ── wide variant (BF16, S = 16) ─────────────────────────────────────────
// Jobs of 256 query entries against candidate tiles of 128: each tile is two
// M = 128, N = 128 products (query rows 0-127 and 128-255) into the two
// halves of one TMEM buffer (256 columns, two buffers), and 16 epilogue warps
// (four per scheduler) take them: warp w reads TMEM lanes 32(w%4).. of row
// half w/8 for column half (w/4)%2 (64 columns), 16 columns per load.  Each
// (entry, column half) keeps one shortlist as in the standard kernel, so the
// output runs are the same; twice the warps hide the epilogue's dependency
// chains.
enum { ET_WAIT, ET_WORK, ET_END, ET_SLOW_CYC, ET_JOBS, ET_SLOW, ET_ADMITS, ET_WMBITS };
constexpr int WQ = 256;            // query entries per job
constexpr int WCN = 128;           // candidates per tile
constexpr int WEPI = 512;          // epilogue threads
constexpr int WNT = WEPI + 64;     // + TMA warp + MMA warp
constexpr int WCPG = WCN / NG;     // columns per warp and tile (64)
constexpr int WBUF = 16;           // staged admissions per (entry, half): one 16-column chunk's
constexpr int WSTASH = 16;         // floats per epilogue thread: a flagged chunk's values
constexpr int WCS = 3;             // candidate tile stages

__device__ __forceinline__ float max16(const float (&v)[16]) {
    const float a = max3f(v[0], v[1], v[2]), b = max3f(v[3], v[4], v[5]),
                c = max3f(v[6], v[7], v[8]), e = max3f(v[9], v[10], v[11]),
                f = max3f(v[12], v[13], v[14]);
    return fmaxf(max3f(a, b, c), max3f(e, f, v[15]));
}

size_t wide_smem() {
    return 1024 + size_t(QST) * WQ * ROWB + size_t(WCS) * WCN * ROWB +
           size_t(NG) * WBUF * WQ * 8 + size_t(WEPI) * WSTASH * 4;
}

__global__ void __launch_bounds__(WNT, 1) k_ivf_wide(const __grid_constant__ CUtensorMap tmQ,
                                                     const __grid_constant__ CUtensorMap tmC,
                                                     IvfTileArgs a) {
    constexpr int S = 16;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* sQ = smem;                                                    // QST x 32 KB
    uint8_t* sC = sQ + QST * WQ * ROWB;                                    // WCS x 16 KB
    float* bdall = reinterpret_cast<float*>(sC + WCS * WCN * ROWB);        // NG x WBUF x WQ
    uint32_t* biall = reinterpret_cast<uint32_t*>(bdall + NG * WBUF * WQ); // NG x WBUF x WQ
    float* stash = reinterpret_cast<float*>(biall + NG * WBUF * WQ);       // WEPI x WSTASH
    __shared__ IvfBars B;
    __shared__ unsigned long long et[8];  // tracing: block 0 thread 0's counters
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    volatile int* abort_flag = &B.abort;

    if (w == 0) {
        tc::tmem_alloc(&B.tmem, 512);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < QST; ++s) {
            tc::mbar_init(&B.q_full[s], 1);
            tc::mbar_init(&B.q_empty[s], 1);
        }
        for (int s = 0; s < MAXCS; ++s) {
            tc::mbar_init(&B.c_full[s], 1);
            tc::mbar_init(&B.c_empty[s], 1);
        }
        for (int s = 0; s < 2; ++s) {
            tc::mbar_init(&B.t_full[s], 1);
            tc::mbar_init(&B.t_empty[s], WEPI / 32);
        }
        tc::mbar_init(&B.done, 1);
        tc::mbar_init(&B.never, 1);
        tc::fence_barrier_init();
        B.abort = 0;
        for (int i = 0; i < 8; ++i) et[i] = 0;
        if (a.test_wait_polls && !tc::mbar_wait(&B.never, 0, a.test_wait_polls)) B.abort = 1;
    }
    if (tid == WEPI) {
        tc::prefetch_tmap(&tmQ);
        tc::prefetch_tmap(&tmC);
    }
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = B.tmem;
    const bool tracing = a.trace && blockIdx.x == 0;
    const long long c_start = clock64();

    if (w == WEPI / 32) {
        // ── TMA producer ──
        if (lane == 0) {
            uint32_t qi = 0, ci = 0;
            long long c_wait = 0;
            for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
                const uint32_t b = a.job_bucket[job], qs = a.job_qstart[job];
                const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
                const uint32_t nct = (ce - cs + WCN - 1) / WCN;
                const uint32_t tfirst =
                    (a.job_tstart && a.job_tstart[job] < nct) ? a.job_tstart[job] : 0u;
                if (nct == 0) continue;
                const int qsd = int(qi % QST);
                long long c0 = clock64();
                if (!tc::mbar_wait(&B.q_empty[qsd], ((qi / QST) & 1) ^ 1, WAIT_LIMIT)) {
                    *abort_flag = 1;
                    break;
                }
                c_wait += clock64() - c0;
                tc::mbar_expect_tx(&B.q_full[qsd], WQ * ROWB);
                tc::tma_load_2d(sQ + qsd * WQ * ROWB, &tmQ, &B.q_full[qsd], 0, int(qs));
                ++qi;
                for (uint32_t t = 0; t < nct; ++t) {
                    const int s = int(ci % WCS);
                    c0 = clock64();
                    if (!tc::mbar_wait(&B.c_empty[s], ((ci / WCS) & 1) ^ 1, WAIT_LIMIT)) {
                        *abort_flag = 1;
                        break;
                    }
                    c_wait += clock64() - c0;
                    tc::mbar_expect_tx(&B.c_full[s], WCN * ROWB);
                    const uint32_t tt = tfirst + t >= nct ? tfirst + t - nct : tfirst + t;
                    tc::tma_load_2d(sC + s * WCN * ROWB, &tmC, &B.c_full[s], 0, int(cs + tt * WCN));
                    ++ci;
                }
            }
            for (int s = 0; s < WCS; ++s) {
                const uint32_t uses = ci / WCS + (uint32_t(s) < ci % WCS ? 1u : 0u);
                if (uses > 0 && !tc::mbar_wait(&B.c_full[s], (uses - 1) & 1, WAIT_LIMIT))
                    *abort_flag = 1;
            }
            for (int s = 0; s < QST; ++s) {
                const uint32_t uses = qi / QST + (uint32_t(s) < qi % QST ? 1u : 0u);
                if (uses > 0 && !tc::mbar_wait(&B.q_full[s], (uses - 1) & 1, WAIT_LIMIT))
                    *abort_flag = 1;
            }
            if (tracing) a.trace[IVF_T_TMA_WAIT] = (unsigned long long)c_wait;
        }
        __syncwarp();
    } else if (w == WEPI / 32 + 1) {
        // ── MMA issuer: two M = 128 products per tile ──
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16_f32(128, WCN);
            uint32_t qi = 0, ci = 0, ti = 0;
            long long c_wait_c = 0, c_wait_t = 0;
            for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
                const uint32_t b = a.job_bucket[job];
                const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
                const uint32_t nct = (ce - cs + WCN - 1) / WCN;
                if (nct == 0) continue;
                const int qsd = int(qi % QST);
                if (!tc::mbar_wait(&B.q_full[qsd], (qi / QST) & 1, WAIT_LIMIT)) {
                    *abort_flag = 1;
                    break;
                }
                // the query tile's row halves: 128 rows of 128 B each, 16 KB apart
                const uint64_t dQ0 = tc::desc_k_sw128(tc::smem_u32(sQ + qsd * WQ * ROWB));
                const uint64_t dQ1 =
                    tc::desc_k_sw128(tc::smem_u32(sQ + qsd * WQ * ROWB + 128 * ROWB));
                bool ok = true;
                for (uint32_t t = 0; t < nct && ok; ++t) {
                    const int s = int(ci % WCS), tb = int(ti & 1);
                    long long c0 = clock64();
                    ok = tc::mbar_wait(&B.c_full[s], (ci / WCS) & 1, WAIT_LIMIT);
                    long long c1 = clock64();
                    ok = ok && tc::mbar_wait(&B.t_empty[tb], ((ti >> 1) & 1) ^ 1, WAIT_LIMIT);
                    c_wait_c += c1 - c0;
                    c_wait_t += clock64() - c1;
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint64_t dC = tc::desc_k_sw128(tc::smem_u32(sC + s * WCN * ROWB));
                    const uint32_t d0 = taddr + uint32_t(tb * 2 * WCN);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        tc::umma_f16(d0, dQ0 + uint64_t(2 * kk), dC + uint64_t(2 * kk), idesc,
                                     kk > 0 ? 1u : 0u);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        tc::umma_f16(d0 + uint32_t(WCN), dQ1 + uint64_t(2 * kk),
                                     dC + uint64_t(2 * kk), idesc, kk > 0 ? 1u : 0u);
                    tc::umma_commit(&B.c_empty[s]);
                    tc::umma_commit(&B.t_full[tb]);
                    ++ci;
                    ++ti;
                }
                tc::umma_commit(&B.q_empty[qsd]);
                ++qi;
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
            }
            tc::umma_commit(&B.done);
            if (!tc::mbar_wait(&B.done, 0, WAIT_LIMIT)) *abort_flag = 1;
            if (tracing) {
                a.trace[IVF_T_MMA_WAIT_C] = (unsigned long long)c_wait_c;
                a.trace[IVF_T_MMA_WAIT_T] = (unsigned long long)c_wait_t;
                a.trace[IVF_T_TILES] = ti;
            }
        }
        __syncwarp();
    } else {
        // ── epilogue: row half h, column half g, TMEM lane quarter w % 4 ──
        const int h = w >> 3, g = (w >> 2) & 1;
        const int row = h * 128 + (w & 3) * 32 + lane;
        const uint32_t lane_base = uint32_t((w & 3) * 32) << 16;
        const bool t0 = tracing && tid == 0;
        const bool buffered = a.buffered != 0;
        float* bd = bdall + size_t(g) * WBUF * WQ + row;
        uint32_t* bi = biall + size_t(g) * WBUF * WQ + row;
        float* srow = stash + size_t(tid) * WSTASH;
        // 16-byte groups of the stash row swizzled so that 8 lanes' stores
        // (64-byte rows) cover all 32 banks
        const int swz = ((lane >> 1) & 3) << 2;
        uint32_t ti = 0;
        uint32_t nb = 0, nqs = 0, nqe = 0, nts = 0;
        auto load_job = [&](uint32_t j) {
            if (j < a.njobs) {
                nb = a.job_bucket[j];
                nqs = a.job_qstart[j];
                nqe = a.job_qend[j];
                nts = a.job_tstart ? a.job_tstart[j] : 0u;
            }
        };
        load_job(blockIdx.x);
        for (uint32_t job = blockIdx.x; job < a.njobs && !*abort_flag; job += gridDim.x) {
            const uint32_t b = nb, qs = nqs, qe = nqe, ts = nts;
            load_job(job + gridDim.x);
            const uint32_t cs = a.c_off[b], ce = a.c_off[b + 1];
            const uint32_t nct = (ce - cs + WCN - 1) / WCN;
            const uint32_t tfirst = ts < nct ? ts : 0u;
            const uint32_t entry = qs + row;
            const bool valid = entry < qe;
            const float qn = valid ? a.qnorm[entry] : __int_as_float(0x7f800000);
            const uint32_t qself = valid ? a.qself[entry] : 0xFFFFFFFFu;
            const float thr0 = (valid && a.qthr) ? a.qthr[entry] : __int_as_float(0x7f800000);
            const uint32_t slot = (valid && a.out_slot) ? a.out_slot[entry] : entry;
            float thr = thr0;
            float ath = (qn - thr) * 0.5f;
            float sv[S];
            uint32_t sx[S];
#pragma unroll
            for (int j = 0; j < S; ++j) {
                sv[j] = __int_as_float(0x7f800000);
                sx[j] = 0xFFFFFFFFu;
            }
            int cnt = 0;
            auto flush = [&]() {
                for (int u = 0; u < cnt; ++u) {
                    const float d = bd[u * WQ];
                    if (d < thr) {
                        shortlist_push<S>(sv, sx, d, bi[u * WQ]);
                        thr = fminf(thr0, sv[S - 1]);
                    }
                }
                cnt = 0;
                ath = (qn - thr) * 0.5f;
            };
            bool ok = true;
            for (uint32_t t = 0; t < nct; ++t) {
                const int tb = int(ti & 1);
                long long c0 = t0 ? clock64() : 0;
                ok = tc::mbar_wait(&B.t_full[tb], (ti >> 1) & 1, WAIT_LIMIT);
                ok = __all_sync(FULL, ok);
                if (!ok) break;
                tc::tc_fence_after();
                const uint32_t tcol =
                    taddr + lane_base + uint32_t(tb * 2 * WCN + h * WCN + g * WCPG);
                const uint32_t tt = tfirst + t >= nct ? tfirst + t - nct : tfirst + t;
                const int lim = int(ce) - int(cs + tt * WCN + g * WCPG);
                const uint32_t cbase = cs + tt * WCN + g * WCPG;
                long long c1 = t0 ? clock64() : 0;
#pragma unroll 1
                for (int q = 0; q < WCPG / 16; ++q) {
                    uint32_t r[16];
                    tc::tmem_ld16(tcol + uint32_t(q * 16), r);
                    tc::tmem_ld_wait();
                    float v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
                    if (lim < (q + 1) * 16) {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (q * 16 + j >= lim) v[j] = __int_as_float(0xff800000);
                    }
                    if (!__any_sync(FULL, max16(v) > ath)) continue;
                    const long long cs0 = t0 ? clock64() : 0;
                    uint32_t lm = 0;
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (v[j] > ath) lm |= 1u << j;
#pragma unroll
                    for (int j = 0; j < 16; j += 4)
                        *reinterpret_cast<float4*>(srow + (j ^ swz)) =
                            make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    if (tracing) {
                        const uint32_t na = __reduce_add_sync(FULL, uint32_t(__popc(lm)));
                        const uint32_t wm = __reduce_or_sync(FULL, lm);
                        if (t0) {
                            et[ET_SLOW] += 1;
                            et[ET_ADMITS] += na;
                            et[ET_WMBITS] += __popc(wm);
                        }
                    }
                    if (buffered &&
                        __reduce_max_sync(FULL, uint32_t(cnt + __popc(lm))) > uint32_t(WBUF))
                        flush();
                    const uint32_t cb0 = cbase + q * 16;
                    while (__any_sync(FULL, lm != 0)) {
                        if (lm) {
                            const int j = __ffs(lm) - 1;
                            lm &= lm - 1;
                            const float dj = fmaf(-2.0f, srow[j ^ swz], qn);
                            if (dj < thr && cb0 + j != qself) {
                                if (buffered) {
                                    bd[cnt * WQ] = dj;
                                    bi[cnt * WQ] = cb0 + j;
                                    ++cnt;
                                } else {
                                    shortlist_push<S>(sv, sx, dj, cb0 + j);
                                    thr = fminf(thr0, sv[S - 1]);
                                    ath = (qn - thr) * 0.5f;
                                }
                            }
                        }
                    }
                    if (t0) et[ET_SLOW_CYC] += clock64() - cs0;
                }
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&B.t_empty[tb]);
                ++ti;
                if (t0) {
                    const long long c2 = clock64();
                    et[ET_WAIT] += c1 - c0;
                    et[ET_WORK] += c2 - c1;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                break;
            }
            long long c3 = t0 ? clock64() : 0;
            if (cnt > 0) flush();
            if (valid) {
                int live = S;
                if (a.out_n) {
                    live = 0;
#pragma unroll
                    for (int j = 0; j < S; ++j)
                        live += sv[j] < __int_as_float(0x7f800000) ? 1 : 0;
                    a.out_n[size_t(slot) * NG + g] = uint8_t(live);
                }
                float4* od = reinterpret_cast<float4*>(a.out_d + (size_t(entry) * NG + g) * S);
                uint4* oi = reinterpret_cast<uint4*>(a.out_i + (size_t(entry) * NG + g) * S);
#pragma unroll
                for (int j = 0; j < S / 4; ++j)
                    if (4 * j < live) {
                        od[j] = make_float4(sv[4 * j], sv[4 * j + 1], sv[4 * j + 2], sv[4 * j + 3]);
                        oi[j] = make_uint4(sx[4 * j], sx[4 * j + 1], sx[4 * j + 2], sx[4 * j + 3]);
                    }
            }
            if (t0) {
                et[ET_JOBS] += 1;
                et[ET_END] += clock64() - c3;
            }
        }
        if (t0) {
            a.trace[IVF_T_EPI_WAIT] = et[ET_WAIT];
            a.trace[IVF_T_EPI_WORK] = et[ET_WORK];
            a.trace[IVF_T_EPI_END] = et[ET_END];
            a.trace[IVF_T_JOBS] = et[ET_JOBS];
            a.trace[IVF_T_SLOW] = et[ET_SLOW];
            a.trace[IVF_T_ADMITS] = et[ET_ADMITS];
            a.trace[IVF_T_WMBITS] = et[ET_WMBITS];
            a.trace[IVF_T_SLOW_CYC] = et[ET_SLOW_CYC];
        }
    }
    __syncthreads();
    if (tracing && tid == 0) a.trace[IVF_T_TOTAL] = (unsigned long long)(clock64() - c_start);
    if (*abort_flag && tid == 0) atomicExch(a.err, 2);
    tc::tc_fence_after();
    if (w == 0) tc::tmem_dealloc(taddr, 512);
}

// ── host: tensor maps ────────────────────────────────────────────────────
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

template <int S, bool F8>
size_t tiles_smem() {
    return 1024 + size_t(QST) * TQ * ROWB + size_t(cand_stages(S, F8)) * TCN * ROWB +
           size_t(NG) * BUF * TQ * 8 + (F8 ? 2 * 2 * NG * CPG * 4 : size_t(NEPI) * STASH * 4);
}

template <int S, bool F8>
cudaError_t launch_s(const CUtensorMap& tmQ, const CUtensorMap& tmC, const IvfTileArgs& a,
                     int grid, cudaStream_t st) {
    const size_t sm = tiles_smem<S, F8>();
    cudaError_t e = cudaFuncSetAttribute(k_ivf_tiles<S, F8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return e;
    k_ivf_tiles<S, F8><<<grid, NT, sm, st>>>(tmQ, tmC, a); count_launch();
    return cudaGetLastError();
}

}  // namespace

// A [rows x 64] BF16 row-major matrix (128-byte rows) as 128-byte-swizzled
// boxes of box_rows x 64.
bool make_bf16_map(CUtensorMap* map, const void* base, uint64_t rows, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {64, rows};
    cuuint64_t strides[1] = {ROWB};
    cuuint32_t box[2] = {64, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool make_bf16_map_ld(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols,
                      uint64_t ld, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn || (ld * 2) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {ld * 2};
    cuuint32_t box[2] = {64, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool make_fp8_map(CUtensorMap* map, const void* base, uint64_t rows, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {128, rows};
    cuuint64_t strides[1] = {ROWB};
    cuuint32_t box[2] = {128, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

int ivf_groups() { return NG; }

int ivf_shortlist(int want) { return want <= 16 ? 16 : (want <= 32 ? 32 : 0); }

cudaError_t launch_ivf_tiles(const CUtensorMap& tmQ, const CUtensorMap& tmC,
                             const IvfTileArgs& a, int grid, cudaStream_t st) {
    if (a.njobs == 0) return cudaSuccess;
    if (a.wide) {
        if (a.fp8 || a.S != 16) return cudaErrorInvalidValue;
        const size_t sm = wide_smem();
        cudaError_t e = cudaFuncSetAttribute(k_ivf_wide, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(sm));
        if (e != cudaSuccess) return e;
        k_ivf_wide<<<grid, WNT, sm, st>>>(tmQ, tmC, a); count_launch();
        return cudaGetLastError();
    }
    if (a.fp8) {
        if (a.S == 16) return launch_s<16, true>(tmQ, tmC, a, grid, st);
        if (a.S == 32) return launch_s<32, true>(tmQ, tmC, a, grid, st);
        return cudaErrorInvalidValue;
    }
    if (a.S == 1) return launch_s<1, false>(tmQ, tmC, a, grid, st);
    if (a.S == 16) return launch_s<16, false>(tmQ, tmC, a, grid, st);
    if (a.S == 32) return launch_s<32, false>(tmQ, tmC, a, grid, st);
    return cudaErrorInvalidValue;
}

}  // namespace pq
