// ORACLE — test infrastructure only, never shipped and never on the product path.
//
// A step-for-step C++17 restatement of the reference's CPU NN-Descent
// (crates/polariseq-core/src/nndescent.rs:78-1003) and of its f32 distance
// kernels (crates/polariseq-core/src/simd.rs:14-81).  It is the bit-exactness
// oracle for the CUDA plain form and, threaded with OpenMP over the same block
// (4096 rows) / generation-chunk (512 rows) / 64 destination-bucket structure
// as the reference's rayon code, the timed CPU baseline.
//
// Parity status: the reference is Rust and cannot be compiled in this
// environment (no cargo/rustc, no vendored crates) and ships no NN-Descent
// golden vectors, so this restatement is pinned by the reference's own
// property tests restated in tests/ (structure, determinism, recall,
// gather-bound invariance, tiny inputs, simd known answers) — "parity
// unpinned" against reference-produced bytes.
//
// Build: compiled with -ffp-contract=off and without -ffast-math so that every
// f32 operation rounds exactly as Rust's (Rust never contracts a*b+c into FMA).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Mirrors NndescentOptions (nndescent.rs:42-76); zero means "auto" for the
// sized fields, exactly as there.
typedef struct oracle_opts {
    uint64_t k;
    uint64_t max_candidates;
    uint64_t max_iterations;
    double delta;
    uint64_t n_trees;
    uint64_t leaf_size;
    uint64_t gather_max;
    uint64_t seed;
} oracle_opts;

// Optional probe: snapshots of the internal state for parity bisection.
// stop_after: -2 = full run; -1 = stop after initialisation (forest + random
// fill); r >= 0 = stop after round r's apply (before the convergence test).
// All pointers may be null.
typedef struct oracle_probe {
    int32_t stop_after;
    int32_t rounds_run;           // out
    uint32_t* heap_idx;           // n*k, state at the stop point
    float* heap_dist;             // n*k
    uint8_t* heap_flag;           // n*k
    uint32_t* cand_new;           // n*m, candidate heaps of the last round run
    uint32_t* cand_old;           // n*m
    uint64_t* round_changed;      // [max_iterations] heap entries changed
    uint64_t* round_emitted;      // [max_iterations] updates that passed a threshold
    uint64_t* round_pairs;        // [max_iterations] join distances evaluated
    uint64_t resolved[6];         // out: k, max_cand, n_iters, n_trees, leaf, stop_at
} oracle_probe;

}  // extern "C"

namespace {

constexpr uint32_t EMPTY = 0xFFFFFFFFu;   // nndescent.rs:116
constexpr size_t N_BUCKETS = 64;          // nndescent.rs:275
constexpr size_t BLOCK = 4096;            // nndescent.rs:279
constexpr size_t GEN_CHUNK = 512;         // nndescent.rs:281
constexpr size_t GATHER_MAX = size_t(1) << 20;  // nndescent.rs:467

// ── deterministic hashing RNG (nndescent.rs:80-112) ─────────────────────
inline uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline float hash_unit(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t h = splitmix(seed ^ splitmix(a) ^ splitmix(b * 0x9E3779B97F4A7C15ull));
    return float(h >> 40) / float(uint64_t(1) << 24);
}

inline size_t hash_index(uint64_t seed, uint64_t a, uint64_t b, size_t n) {
    return size_t(splitmix(seed ^ splitmix(a) ^ splitmix(b + 0x12345678ull)) % uint64_t(n));
}

struct Rng {
    uint64_t s;
    uint64_t next_u64() { s = splitmix(s); return s; }
    size_t below(size_t n) { return size_t(next_u64() % uint64_t(n)); }
};

// ── simd.rs:14-81: 8 independent lane sums, fixed pairwise reduce, tail ──
inline float reduce8(const float* a) {
    return ((a[0] + a[4]) + (a[1] + a[5])) + ((a[2] + a[6]) + (a[3] + a[7]));
}

inline float sq_dist(const float* a, const float* b, size_t d) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t full = d / 8 * 8;
    for (size_t c = 0; c < full; c += 8)
        for (int l = 0; l < 8; ++l) {
            float t = a[c + l] - b[c + l];
            acc[l] = acc[l] + t * t;
        }
    float tail = 0.0f;
    for (size_t j = full; j < d; ++j) {
        float t = a[j] - b[j];
        tail = tail + t * t;
    }
    return reduce8(acc) + tail;
}

inline float dot(const float* a, const float* b, size_t d) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t full = d / 8 * 8;
    for (size_t c = 0; c < full; c += 8)
        for (int l = 0; l < 8; ++l) acc[l] = acc[l] + a[c + l] * b[c + l];
    float tail = 0.0f;
    for (size_t j = full; j < d; ++j) tail = tail + a[j] * b[j];
    return reduce8(acc) + tail;
}

// ── flagged neighbour heaps (nndescent.rs:118-206) ──────────────────────
struct NeighborHeap {
    size_t k;
    std::vector<uint32_t> idx;
    std::vector<float> dist;
    std::vector<uint8_t> flag;
    NeighborHeap(size_t n, size_t k_)
        : k(k_), idx(n * k_, EMPTY), dist(n * k_, INFINITY), flag(n * k_, 0) {}
};

// HeapRowsMut::push on one row (nndescent.rs:168-205).
inline bool heap_push(uint32_t* idx, float* dist, uint8_t* flg, size_t k, uint32_t j, float d,
                      uint8_t flag) {
    if (d >= dist[0]) return false;  // `d >= dist[0]` rejects (a NaN passes, as there)
    for (size_t s = 0; s < k; ++s)
        if (idx[s] == j) return false;
    idx[0] = j;
    dist[0] = d;
    flg[0] = flag;
    size_t p = 0;
    for (;;) {
        size_t l = 2 * p + 1, r = 2 * p + 2, sw = p;
        if (l < k && dist[l] > dist[sw]) sw = l;
        if (r < k && dist[r] > dist[sw]) sw = r;
        if (sw == p) break;
        std::swap(idx[p], idx[sw]);
        std::swap(dist[p], dist[sw]);
        std::swap(flg[p], flg[sw]);
        p = sw;
    }
    return true;
}

// CandidateHeap::push_row (nndescent.rs:244-269).
inline void cand_push(uint32_t* idx, float* prio, size_t m, uint32_t j, float p) {
    if (p >= prio[0]) return;
    for (size_t s = 0; s < m; ++s)
        if (idx[s] == j) return;
    idx[0] = j;
    prio[0] = p;
    size_t q = 0;
    for (;;) {
        size_t l = 2 * q + 1, r = 2 * q + 2, sw = q;
        if (l < m && prio[l] > prio[sw]) sw = l;
        if (r < m && prio[r] > prio[sw]) sw = r;
        if (sw == q) break;
        std::swap(idx[q], idx[sw]);
        std::swap(prio[q], prio[sw]);
        q = sw;
    }
}

struct Update { uint32_t dest, nbr; float dist; };                 // nndescent.rs:286-291
struct CandUpdate { uint32_t dest, nbr; float prio; bool is_new; };  // nndescent.rs:293-298

inline size_t rows_per_bucket(size_t n) {  // nndescent.rs:300-302
    size_t r = (n + N_BUCKETS - 1) / N_BUCKETS;
    return r > 0 ? r : 1;
}

using Buckets = std::vector<std::vector<Update>>;
using CandBuckets = std::vector<std::vector<CandUpdate>>;

// apply_updates (nndescent.rs:307-324): each bucket owns a row range and
// consumes the generation chunks in order.
size_t apply_updates(NeighborHeap& h, const std::vector<Buckets>& gen, size_t n) {
    size_t rpb = rows_per_bucket(n);
    size_t nb = (n + rpb - 1) / rpb;
    size_t k = h.k;
    size_t changed = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : changed)
    for (size_t b = 0; b < nb; ++b) {
        for (const Buckets& chunk : gen)
            for (const Update& u : chunk[b]) {
                size_t base = size_t(u.dest) * k;
                if (heap_push(&h.idx[base], &h.dist[base], &h.flag[base], k, u.nbr, u.dist, 1))
                    ++changed;
            }
    }
    return changed;
}

// apply_candidates (nndescent.rs:326-354).
void apply_candidates(std::vector<uint32_t>& idx, std::vector<float>& prio, size_t m,
                      const std::vector<CandBuckets>& gen, size_t n, bool want_new) {
    size_t rpb = rows_per_bucket(n);
    size_t nb = (n + rpb - 1) / rpb;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t b = 0; b < nb; ++b) {
        for (const CandBuckets& chunk : gen)
            for (const CandUpdate& u : chunk[b])
                if (u.is_new == want_new) {
                    size_t base = size_t(u.dest) * m;
                    cand_push(&idx[base], &prio[base], m, u.nbr, u.prio);
                }
    }
}

// ── random projection trees (nndescent.rs:356-641) ──────────────────────
struct Tree {
    std::vector<uint32_t> ids;
    std::vector<std::pair<uint32_t, uint32_t>> leaves;
};

// random_hyperplane (nndescent.rs:367-385).
float random_hyperplane(const float* data, size_t d, const uint32_t* ids, size_t n, Rng& rng,
                        float* normal) {
    size_t a = ids[rng.below(n)];
    size_t b = ids[rng.below(n)];
    int tries = 0;
    while (b == a && tries < 8) {
        b = ids[rng.below(n)];
        ++tries;
    }
    const float* xa = data + a * d;
    const float* xb = data + b * d;
    for (size_t j = 0; j < d; ++j) normal[j] = xa[j] - xb[j];
    // Rust's f32 `sum` folds left from -0.0; the sign of a zero offset is
    // never observable (|margin| < 1e-8 is a tie either way).
    float s = -0.0f;
    for (size_t j = 0; j < d; ++j) s = s + (normal[j] * 0.5f) * (xa[j] + xb[j]);
    return -s;
}

// partition_in_place (nndescent.rs:389-405): two-pointer swap partition,
// `sides` indexed by original position.
size_t partition_in_place(uint32_t* ids, size_t n, const uint8_t* sides) {
    size_t lo = 0, hi = n;
    std::vector<uint32_t> pos(n);
    for (size_t i = 0; i < n; ++i) pos[i] = uint32_t(i);
    while (lo < hi) {
        if (sides[pos[lo]]) {
            ++lo;
        } else {
            --hi;
            std::swap(ids[lo], ids[hi]);
            std::swap(pos[lo], pos[hi]);
        }
    }
    return lo;
}

// random_split (nndescent.rs:408-415): Fisher-Yates, then cut in half.
size_t random_split(uint32_t* ids, size_t n, Rng& rng) {
    for (size_t i = n; i-- > 1;) {
        size_t j = rng.below(i + 1);
        std::swap(ids[i], ids[j]);
    }
    return n / 2;
}

// rp_tree_leaves (nndescent.rs:419-457): sequential recursion drawing every
// random choice from one `rng` in depth-first order.
void rp_tree_leaves(const float* data, size_t d, uint32_t* ids, size_t n, size_t base,
                    size_t leaf_size, Rng& rng, size_t depth,
                    std::vector<std::pair<uint32_t, uint32_t>>& out, std::vector<float>& normal,
                    std::vector<uint8_t>& sides) {
    if (n <= leaf_size || depth > 100) {
        out.emplace_back(uint32_t(base), uint32_t(base + n));
        return;
    }
    float offset = random_hyperplane(data, d, ids, n, rng, normal.data());
    sides.resize(n);
    for (size_t i = 0; i < n; ++i) {
        float margin = dot(normal.data(), data + size_t(ids[i]) * d, d) + offset;
        if (std::fabs(margin) < 1e-8f)
            sides[i] = (rng.next_u64() & 1) == 0;
        else
            sides[i] = margin > 0.0f;
    }
    size_t split = partition_in_place(ids, n, sides.data());
    if (split == 0 || split == n) {
        split = random_split(ids, n, rng);
        if (split == 0 || split == n) {
            out.emplace_back(uint32_t(base), uint32_t(base + n));
            return;
        }
    }
    rp_tree_leaves(data, d, ids, split, base, leaf_size, rng, depth + 1, out, normal, sides);
    rp_tree_leaves(data, d, ids + split, n - split, base + split, leaf_size, rng, depth + 1, out,
                   normal, sides);
}

// rp_tree_sequential (nndescent.rs:474-581): identical to rp_tree_leaves, on
// the input rows while a subtree exceeds gather_max and on a gathered copy
// of its rows below that.
void rp_tree_sequential(const float* data, size_t d, uint32_t* ids, size_t n, size_t base,
                        size_t leaf_size, Rng& rng, size_t depth, size_t gather_max,
                        std::vector<std::pair<uint32_t, uint32_t>>& out,
                        std::vector<float>& normal, std::vector<uint8_t>& sides) {
    if (n <= gather_max) {
        std::vector<float> local(n * d);
        for (size_t i = 0; i < n; ++i)
            std::memcpy(&local[i * d], data + size_t(ids[i]) * d, d * sizeof(float));
        std::vector<uint32_t> local_ids(n);
        for (size_t i = 0; i < n; ++i) local_ids[i] = uint32_t(i);
        rp_tree_leaves(local.data(), d, local_ids.data(), n, base, leaf_size, rng, depth, out,
                       normal, sides);
        std::vector<uint32_t> snap(ids, ids + n);
        for (size_t i = 0; i < n; ++i) ids[i] = snap[local_ids[i]];
        return;
    }
    if (n <= leaf_size || depth > 100) {
        out.emplace_back(uint32_t(base), uint32_t(base + n));
        return;
    }
    float offset = random_hyperplane(data, d, ids, n, rng, normal.data());
    std::vector<uint8_t> sd(n);
    for (size_t i = 0; i < n; ++i) {
        float margin = dot(normal.data(), data + size_t(ids[i]) * d, d) + offset;
        if (std::fabs(margin) < 1e-8f)
            sd[i] = (rng.next_u64() & 1) == 0;
        else
            sd[i] = margin > 0.0f;
    }
    size_t split = partition_in_place(ids, n, sd.data());
    sd.clear();
    sd.shrink_to_fit();
    if (split == 0 || split == n) {
        split = random_split(ids, n, rng);
        if (split == 0 || split == n) {
            out.emplace_back(uint32_t(base), uint32_t(base + n));
            return;
        }
    }
    rp_tree_sequential(data, d, ids, split, base, leaf_size, rng, depth + 1, gather_max, out,
                       normal, sides);
    rp_tree_sequential(data, d, ids + split, n - split, base + split, leaf_size, rng, depth + 1,
                       gather_max, out, normal, sides);
}

// rp_tree_parallel (nndescent.rs:587-641): the top levels (n >= 8192 and
// depth < 6) split with ties decided by splitmix(seed ^ id) and hand each
// child a fresh seed; the leaves come back in depth-first order.
void rp_tree_parallel(const float* data, size_t d, uint32_t* ids, size_t n, size_t base,
                      size_t leaf_size, uint64_t seed, size_t depth, size_t gather_max,
                      std::vector<std::pair<uint32_t, uint32_t>>& out) {
    std::vector<float> normal(d);
    if (n < 8192 || depth >= 6) {
        Rng rng{seed};
        std::vector<uint8_t> sides;
        rp_tree_sequential(data, d, ids, n, base, leaf_size, rng, depth, gather_max, out, normal,
                           sides);
        return;
    }
    Rng rng{seed};
    float offset = random_hyperplane(data, d, ids, n, rng, normal.data());
    std::vector<uint8_t> sides(n);
    for (size_t i = 0; i < n; ++i) {
        uint32_t id = ids[i];
        float margin = dot(normal.data(), data + size_t(id) * d, d) + offset;
        if (std::fabs(margin) < 1e-8f)
            sides[i] = (splitmix(seed ^ uint64_t(id)) & 1) == 0;
        else
            sides[i] = margin > 0.0f;
    }
    size_t split = partition_in_place(ids, n, sides.data());
    if (split == 0 || split == n) split = random_split(ids, n, rng);
    std::vector<uint8_t>().swap(sides);
    rp_tree_parallel(data, d, ids, split, base, leaf_size, splitmix(seed ^ 1), depth + 1,
                     gather_max, out);
    rp_tree_parallel(data, d, ids + split, n - split, base + split, leaf_size,
                     splitmix(seed ^ 2), depth + 1, gather_max, out);
}

Tree build_tree(const float* data, size_t d, size_t n, size_t leaf_size, uint64_t seed,
                size_t gather_max) {  // nndescent.rs:643-646
    Tree t;
    t.ids.resize(n);
    for (size_t i = 0; i < n; ++i) t.ids[i] = uint32_t(i);
    rp_tree_parallel(data, d, t.ids.data(), n, 0, leaf_size, seed, 0, gather_max, t.leaves);
    return t;
}

struct Resolved {
    size_t k, max_cand, n_iters, n_trees, leaf_size, gather_max, stop_at;
};

// Auto defaults (nndescent.rs:722-752) and the stop threshold (:850).
Resolved resolve(size_t n, const oracle_opts& o) {
    Resolved r;
    size_t k = o.k < n - 1 ? o.k : n - 1;
    r.k = k > 0 ? k : 1;
    size_t mc = o.max_candidates > 0 ? o.max_candidates : std::min<size_t>(2 * r.k, 60);
    r.max_cand = mc > 0 ? mc : 1;
    if (o.max_iterations > 0) {
        r.n_iters = o.max_iterations;
    } else {
        double lg = std::round(std::log2(double(n)));
        size_t it = lg > 0 ? size_t(lg) : 0;
        r.n_iters = it > 5 ? it : 5;
    }
    if (o.n_trees > 0) {
        r.n_trees = o.n_trees;
    } else {
        double t = std::round(std::sqrt(double(n)) / 10.0);
        r.n_trees = std::min<size_t>(8 + size_t(t), 48);
    }
    r.leaf_size = o.leaf_size > 0 ? o.leaf_size : std::max<size_t>(r.k, 10);
    r.gather_max = o.gather_max > 0 ? o.gather_max : GATHER_MAX;
    double sa = o.delta * double(n) * double(r.k);
    r.stop_at = (sa > 0 && sa == sa) ? (sa >= 1.8e19 ? SIZE_MAX : size_t(sa)) : 0;
    return r;
}

}  // namespace

extern "C" {

uint64_t oracle_effective_k(uint64_t n_obs, uint64_t k) {  // nndescent.rs:648-650
    uint64_t m = n_obs > 0 ? n_obs - 1 : 0;
    uint64_t e = k < m ? k : m;
    return e > 0 ? e : 1;
}

// One tree, for forest parity checks: ids (n) and leaves (2 * n_leaves).
// Returns the number of leaves (or the required count if cap is too small).
uint64_t oracle_build_tree(const float* data, uint64_t n, uint64_t d, uint64_t leaf_size,
                           uint64_t seed, uint64_t gather_max, uint32_t* ids_out,
                           uint32_t* leaves_out, uint64_t leaves_cap) {
    Tree t = build_tree(data, d, n, leaf_size, seed, gather_max ? gather_max : GATHER_MAX);
    std::memcpy(ids_out, t.ids.data(), n * sizeof(uint32_t));
    if (t.leaves.size() <= leaves_cap)
        for (size_t i = 0; i < t.leaves.size(); ++i) {
            leaves_out[2 * i] = t.leaves[i].first;
            leaves_out[2 * i + 1] = t.leaves[i].second;
        }
    return t.leaves.size();
}

uint64_t oracle_splitmix(uint64_t x) { return splitmix(x); }
float oracle_hash_unit(uint64_t s, uint64_t a, uint64_t b) { return hash_unit(s, a, b); }
uint64_t oracle_hash_index(uint64_t s, uint64_t a, uint64_t b, uint64_t n) {
    return hash_index(s, a, b, n);
}
float oracle_sq_dist(const float* a, const float* b, uint64_t d) { return sq_dist(a, b, d); }
float oracle_dot(const float* a, const float* b, uint64_t d) { return dot(a, b, d); }

// The reference's two-pointer partition, exposed for the permutation tests.
uint64_t oracle_partition(uint32_t* ids, uint64_t n, const uint8_t* sides) {
    return partition_in_place(ids, n, sides);
}

void oracle_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

int oracle_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// nndescent_into (nndescent.rs:699-1003).  Returns 0 and writes *nnz_out, or
// a negative code for the inputs on which the reference panics.
int oracle_nndescent_into(const float* data, uint64_t n_obs, uint64_t n_dim,
                          const oracle_opts* opts, uint32_t* indptr_out, uint64_t indptr_len,
                          uint32_t* indices_out, uint64_t indices_len, float* dists_out,
                          uint64_t dists_len, uint64_t* nnz_out, oracle_probe* probe) {
    if (n_obs == 0 || n_dim == 0) return -1;           // "empty data"
    if (opts->k == 0) return -2;                         // "k must be >= 1"
    if (indptr_len != n_obs + 1) return -3;              // indptr length
    uint64_t cap = n_obs * oracle_effective_k(n_obs, opts->k);
    if (indices_len < cap || dists_len < cap) return -4;  // "graph arrays are too short"

    const size_t n = n_obs, d = n_dim;
    Resolved R = resolve(n, *opts);
    const size_t k = R.k, max_cand = R.max_cand;
    const uint64_t seed = opts->seed;
    const size_t rpb = rows_per_bucket(n);
    auto row = [&](size_t i) { return data + i * d; };
    if (probe) {
        probe->rounds_run = 0;
        uint64_t res[6] = {R.k, R.max_cand, R.n_iters, R.n_trees, R.leaf_size, R.stop_at};
        std::memcpy(probe->resolved, res, sizeof(res));
    }

    NeighborHeap heap(n, k);

    // ── 1. RP-tree forest (nndescent.rs:768-780) ──
    std::vector<Tree> forest(R.n_trees);
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t t = 0; t < R.n_trees; ++t)
        forest[t] = build_tree(data, d, n, R.leaf_size, splitmix(seed ^ (uint64_t(t) + 1)),
                               R.gather_max);

    // Leaf all-pairs, one tree at a time (nndescent.rs:785-815).
    for (const Tree& tree : forest) {
        size_t nl = tree.leaves.size();
        size_t nchunks = (nl + 63) / 64;
        std::vector<Buckets> gen(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t c = 0; c < nchunks; ++c) {
            Buckets b(N_BUCKETS);
            size_t lend = std::min(nl, (c + 1) * 64);
            for (size_t li = c * 64; li < lend; ++li) {
                const uint32_t* leaf = tree.ids.data() + tree.leaves[li].first;
                size_t len = tree.leaves[li].second - tree.leaves[li].first;
                for (size_t i = 0; i < len; ++i)
                    for (size_t j = i + 1; j < len; ++j) {
                        uint32_t p = leaf[i], q = leaf[j];
                        float dist = sq_dist(row(p), row(q), d);
                        b[p / rpb].push_back({p, q, dist});
                        b[q / rpb].push_back({q, p, dist});
                    }
            }
            gen[c] = std::move(b);
        }
        apply_updates(heap, gen, n);
    }
    std::vector<Tree>().swap(forest);

    // Random fill of empty slots, own row only (nndescent.rs:820-845).
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) {
        uint32_t* idx = &heap.idx[i * k];
        float* dist = &heap.dist[i * k];
        uint8_t* flg = &heap.flag[i * k];
        uint64_t attempt = 0;
        auto has_empty = [&] {
            for (size_t s = 0; s < k; ++s)
                if (idx[s] == EMPTY) return true;
            return false;
        };
        while (has_empty() && attempt < 64) {
            size_t j = hash_index(seed, uint64_t(i), attempt, n);
            if (j == i) j = (j + 1) % n;
            heap_push(idx, dist, flg, k, uint32_t(j), sq_dist(row(i), row(j), d), 1);
            ++attempt;
        }
    }

    auto snapshot_heap = [&] {
        if (!probe) return;
        if (probe->heap_idx) std::memcpy(probe->heap_idx, heap.idx.data(), n * k * 4);
        if (probe->heap_dist) std::memcpy(probe->heap_dist, heap.dist.data(), n * k * 4);
        if (probe->heap_flag) std::memcpy(probe->heap_flag, heap.flag.data(), n * k);
    };
    if (probe && probe->stop_after == -1) {
        snapshot_heap();
        return 0;
    }

    // ── 2. NN-Descent iterations (nndescent.rs:848-975) ──
    std::vector<uint32_t> new_idx(n * max_cand), old_idx(n * max_cand);
    std::vector<float> new_prio(n * max_cand), old_prio(n * max_cand);
    std::vector<float> thresholds(n);
    for (size_t iter = 0; iter < R.n_iters; ++iter) {
        // 2a. candidate sampling (nndescent.rs:855-892)
        std::fill(new_idx.begin(), new_idx.end(), EMPTY);
        std::fill(old_idx.begin(), old_idx.end(), EMPTY);
        std::fill(new_prio.begin(), new_prio.end(), INFINITY);
        std::fill(old_prio.begin(), old_prio.end(), INFINITY);
        for (size_t bs = 0; bs < n; bs += BLOCK) {
            size_t be = std::min(n, bs + BLOCK);
            size_t nch = (be - bs + GEN_CHUNK - 1) / GEN_CHUNK;
            std::vector<CandBuckets> gen(nch);
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t c = 0; c < nch; ++c) {
                CandBuckets b(N_BUCKETS);
                size_t c0 = bs + c * GEN_CHUNK, c1 = std::min(be, c0 + GEN_CHUNK);
                for (size_t i = c0; i < c1; ++i)
                    for (size_t s = 0; s < k; ++s) {
                        uint32_t j = heap.idx[i * k + s];
                        if (j == EMPTY) continue;
                        bool is_new = heap.flag[i * k + s] != 0;
                        float prio = hash_unit(seed, uint64_t(iter), uint64_t(i * k + s));
                        b[i / rpb].push_back({uint32_t(i), j, prio, is_new});
                        b[j / rpb].push_back({j, uint32_t(i), prio, is_new});
                    }
                gen[c] = std::move(b);
            }
            apply_candidates(new_idx, new_prio, max_cand, gen, n, true);
            apply_candidates(old_idx, old_prio, max_cand, gen, n, false);
        }

        // 2b. neighbours that made it into the new list become old (:895-909)
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i) {
            const uint32_t* cands = &new_idx[i * max_cand];
            for (size_t s = 0; s < k; ++s) {
                uint32_t j = heap.idx[i * k + s];
                if (heap.flag[i * k + s] && j != EMPTY) {
                    for (size_t c = 0; c < max_cand; ++c)
                        if (cands[c] == j) {
                            heap.flag[i * k + s] = 0;
                            break;
                        }
                }
            }
        }

        // 2c. local join, thresholds frozen for the round (:914-969)
        for (size_t i = 0; i < n; ++i) thresholds[i] = heap.dist[i * k];
        size_t changed = 0;
        uint64_t emitted = 0, pairs = 0;
        for (size_t bs = 0; bs < n; bs += BLOCK) {
            size_t be = std::min(n, bs + BLOCK);
            size_t nch = (be - bs + GEN_CHUNK - 1) / GEN_CHUNK;
            std::vector<Buckets> gen(nch);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : emitted, pairs)
            for (size_t c = 0; c < nch; ++c) {
                Buckets b(N_BUCKETS);
                size_t c0 = bs + c * GEN_CHUNK, c1 = std::min(be, c0 + GEN_CHUNK);
                auto emit = [&](uint32_t p, uint32_t q, float dist) {
                    if (dist < thresholds[p]) {
                        b[p / rpb].push_back({p, q, dist});
                        ++emitted;
                    }
                    if (dist < thresholds[q]) {
                        b[q / rpb].push_back({q, p, dist});
                        ++emitted;
                    }
                };
                for (size_t i = c0; i < c1; ++i) {
                    const uint32_t* news = &new_idx[i * max_cand];
                    const uint32_t* olds = &old_idx[i * max_cand];
                    for (size_t a = 0; a < max_cand; ++a) {
                        uint32_t p = news[a];
                        if (p == EMPTY) continue;
                        const float* xp = row(p);
                        for (size_t bq = a + 1; bq < max_cand; ++bq) {
                            uint32_t q = news[bq];
                            if (q == EMPTY || q == p) continue;
                            ++pairs;
                            emit(p, q, sq_dist(xp, row(q), d));
                        }
                        for (size_t bq = 0; bq < max_cand; ++bq) {
                            uint32_t q = olds[bq];
                            if (q == EMPTY || q == p) continue;
                            ++pairs;
                            emit(p, q, sq_dist(xp, row(q), d));
                        }
                    }
                }
                gen[c] = std::move(b);
            }
            changed += apply_updates(heap, gen, n);
        }
        if (probe) {
            probe->rounds_run = int32_t(iter + 1);
            if (probe->round_changed) probe->round_changed[iter] = changed;
            if (probe->round_emitted) probe->round_emitted[iter] = emitted;
            if (probe->round_pairs) probe->round_pairs[iter] = pairs;
            if (probe->stop_after == int32_t(iter)) {
                snapshot_heap();
                if (probe->cand_new) std::memcpy(probe->cand_new, new_idx.data(), n * max_cand * 4);
                if (probe->cand_old) std::memcpy(probe->cand_old, old_idx.data(), n * max_cand * 4);
                return 0;
            }
        }
        if (changed <= R.stop_at) break;
    }

    // ── 3. extract: stable sort by distance, sqrt, CSR (nndescent.rs:978-996) ──
    indptr_out[0] = 0;
    size_t pos = 0;
    std::vector<std::pair<uint32_t, float>> rowbuf;
    rowbuf.reserve(k);
    for (size_t i = 0; i < n; ++i) {
        rowbuf.clear();
        for (size_t s = 0; s < k; ++s) {
            uint32_t j = heap.idx[i * k + s];
            if (j != EMPTY) rowbuf.emplace_back(j, heap.dist[i * k + s]);
        }
        std::stable_sort(rowbuf.begin(), rowbuf.end(),
                         [](const std::pair<uint32_t, float>& a,
                            const std::pair<uint32_t, float>& b) { return a.second < b.second; });
        for (auto& e : rowbuf) {
            indices_out[pos] = e.first;
            dists_out[pos] = std::sqrt(e.second);
            ++pos;
        }
        indptr_out[i + 1] = uint32_t(pos);
    }
    if (probe) snapshot_heap();
    *nnz_out = pos;
    return 0;
}

}  // extern "C"
