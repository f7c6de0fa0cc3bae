"""ORACLE — test infrastructure only, never shipped and never on the product path.

A second, independent restatement of the reference's NN-Descent
(crates/polariseq-core/src/nndescent.rs:78-1003, simd.rs:14-81), written
literally and sequentially in Python so that it can be read against the Rust
line by line: the same recursion for the RP trees (rp_tree_parallel,
rp_tree_sequential, rp_tree_leaves), the same two-pointer partition with its
position array, Fisher-Yates random splits, the same 64 destination buckets
filled chunk by chunk and applied chunk by chunk, the same 4096-row blocks and
512-row generation chunks in the rounds, the same heap push (replace the root,
sift down by swaps) and the same stable extract.  Every f32 operation is a
NumPy float32 operation (IEEE single rounding, no fused multiply-add), in the
reference's order: eight lane accumulators, the fixed pairwise reduce, the
sequential tail.

It shares no code with the C++ restatement (nndescent_ref.cpp) nor with the
CUDA kernels; the tests compare the three byte for byte.  It is slow (pure
Python), so it runs on small inputs (a few hundred to a few thousand cells)
and, for the forest's parallel levels, on single trees of larger inputs.

It also restates, from their published algorithms, the random inputs of the
reference's own unit tests (make_clustered_data, nndescent.rs:1012-1022):
ChaCha with 8 rounds (rand_chacha 0.10.0 ChaCha8Rng: 64-bit block counter and
64-bit stream, both starting at zero), seeded by rand_core 0.10.1's
SeedableRng::seed_from_u64 (a PCG32 stream expanding the u64 into the 32-byte
key), and rand 0.10.2's StandardUniform f32 ((next_u32 >> 8) * 2^-24).
"""

from __future__ import annotations

import numpy as np

F32 = np.float32
EMPTY = 0xFFFFFFFF
M64 = (1 << 64) - 1
N_BUCKETS = 64
BLOCK = 4096
GEN_CHUNK = 512
GATHER_MAX = 1 << 20
LANES = 8


# ── hashing RNG (nndescent.rs:80-112) ───────────────────────────────────────

def splitmix(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def hash_unit(seed: int, a: int, b: int) -> F32:
    h = splitmix(seed ^ splitmix(a) ^ splitmix((b * 0x9E3779B97F4A7C15) & M64))
    return F32(F32(h >> 40) / F32(1 << 24))


def hash_index(seed: int, a: int, b: int, n: int) -> int:
    return splitmix(seed ^ splitmix(a) ^ splitmix((b + 0x12345678) & M64)) % n


class Rng:
    def __init__(self, s: int):
        self.s = s

    def next_u64(self) -> int:
        self.s = splitmix(self.s)
        return self.s

    def below(self, n: int) -> int:
        return self.next_u64() % n


# ── f32 kernels (simd.rs:14-81): scalar and vectorised over rows ────────────

def _reduce(acc):
    return F32(F32(F32(acc[0] + acc[4]) + F32(acc[1] + acc[5]))
               + F32(F32(acc[2] + acc[6]) + F32(acc[3] + acc[7])))


def sq_dist(a: np.ndarray, b: np.ndarray) -> F32:
    acc = [F32(0.0)] * LANES
    d = len(a)
    full = d // LANES
    for c in range(full):
        for lane in range(LANES):
            t = F32(a[c * LANES + lane] - b[c * LANES + lane])
            acc[lane] = F32(acc[lane] + F32(t * t))
    tail = F32(0.0)
    for j in range(full * LANES, d):
        t = F32(a[j] - b[j])
        tail = F32(tail + F32(t * t))
    return F32(_reduce(acc) + tail)


def dot_rows(v: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """simd::dot(v, row) for every row of `rows` (m x d float32), each with
    the scalar order: lane accumulators over the rows at once."""
    d = len(v)
    full = d // LANES
    acc = [np.zeros(len(rows), F32) for _ in range(LANES)]
    for c in range(full):
        for lane in range(LANES):
            j = c * LANES + lane
            acc[lane] = (acc[lane] + (rows[:, j] * v[j]).astype(F32)).astype(F32)
    tail = np.zeros(len(rows), F32)
    for j in range(full * LANES, d):
        tail = (tail + (v[j] * rows[:, j]).astype(F32)).astype(F32)
    r = ((acc[0] + acc[4]).astype(F32) + (acc[1] + acc[5]).astype(F32)).astype(F32)
    r2 = ((acc[2] + acc[6]).astype(F32) + (acc[3] + acc[7]).astype(F32)).astype(F32)
    return ((r + r2).astype(F32) + tail).astype(F32)


# ── heaps (nndescent.rs:114-270) ────────────────────────────────────────────

def heap_push(idx, dist, flag, base, k, j, dd, fl) -> bool:
    if dd >= dist[base]:
        return False
    for s in range(k):
        if idx[base + s] == j:
            return False
    idx[base], dist[base], flag[base] = j, dd, fl
    p = 0
    while True:
        lft, rgt = 2 * p + 1, 2 * p + 2
        swap = p
        if lft < k and dist[base + lft] > dist[base + swap]:
            swap = lft
        if rgt < k and dist[base + rgt] > dist[base + swap]:
            swap = rgt
        if swap == p:
            break
        a, b = base + p, base + swap
        idx[a], idx[b] = idx[b], idx[a]
        dist[a], dist[b] = dist[b], dist[a]
        flag[a], flag[b] = flag[b], flag[a]
        p = swap
    return True


def cand_push(idx, prio, base, m, j, p) -> None:
    if p >= prio[base]:
        return
    for s in range(m):
        if idx[base + s] == j:
            return
    idx[base], prio[base] = j, p
    q = 0
    while True:
        lft, rgt = 2 * q + 1, 2 * q + 2
        swap = q
        if lft < m and prio[base + lft] > prio[base + swap]:
            swap = lft
        if rgt < m and prio[base + rgt] > prio[base + swap]:
            swap = rgt
        if swap == q:
            break
        a, b = base + q, base + swap
        idx[a], idx[b] = idx[b], idx[a]
        prio[a], prio[b] = prio[b], prio[a]
        q = swap


def rows_per_bucket(n: int) -> int:
    return max(-(-n // N_BUCKETS), 1)


# ── random projection trees (nndescent.rs:356-646) ──────────────────────────

def random_hyperplane(data, ids, rng):
    n = len(ids)
    a = ids[rng.below(n)]
    b = ids[rng.below(n)]
    tries = 0
    while b == a and tries < 8:
        b = ids[rng.below(n)]
        tries += 1
    xa, xb = data[a], data[b]
    normal = (xa - xb).astype(F32)
    s = F32(-0.0)
    for p, q, nv in zip(xa, xb, normal):
        s = F32(s + F32(F32(nv * F32(0.5)) * F32(p + q)))
    return normal, F32(-s)


def partition_in_place(ids, sides) -> int:
    lo, hi = 0, len(ids)
    pos = list(range(len(ids)))
    while lo < hi:
        if sides[pos[lo]]:
            lo += 1
        else:
            hi -= 1
            ids[lo], ids[hi] = ids[hi], ids[lo]
            pos[lo], pos[hi] = pos[hi], pos[lo]
    return lo


def random_split(ids, rng) -> int:
    for i in range(len(ids) - 1, 0, -1):
        j = rng.below(i + 1)
        ids[i], ids[j] = ids[j], ids[i]
    return len(ids) // 2


def _sides_seq(data, ids, normal, offset, rng):
    margins = (dot_rows(normal, data[np.asarray(ids, np.int64)]) + offset).astype(F32)
    sides = []
    for m in margins:
        if abs(m) < F32(1e-8):
            sides.append(rng.next_u64() & 1 == 0)
        else:
            sides.append(bool(m > 0.0))
    return sides


def rp_tree_leaves(data, ids, lo, hi, base, leaf_size, rng, depth, out):
    """ids[lo:hi] is the slice (a list, recursed in place)."""
    n = hi - lo
    if n <= leaf_size or depth > 100:
        out.append((base, base + n))
        return
    sl = ids[lo:hi]
    normal, offset = random_hyperplane(data, sl, rng)
    sides = _sides_seq(data, sl, normal, offset, rng)
    split = partition_in_place(sl, sides)
    if split == 0 or split == n:
        split = random_split(sl, rng)
        if split == 0 or split == n:
            ids[lo:hi] = sl
            out.append((base, base + n))
            return
    ids[lo:hi] = sl
    rp_tree_leaves(data, ids, lo, lo + split, base, leaf_size, rng, depth + 1, out)
    rp_tree_leaves(data, ids, lo + split, hi, base + split, leaf_size, rng, depth + 1, out)


def rp_tree_sequential(data, ids, lo, hi, base, leaf_size, rng, depth, gather_max, out):
    n = hi - lo
    if n <= gather_max:
        local = data[np.asarray(ids[lo:hi], np.int64)]
        local_ids = list(range(n))
        rp_tree_leaves(local, local_ids, 0, n, base, leaf_size, rng, depth, out)
        snapshot = ids[lo:hi]
        ids[lo:hi] = [snapshot[li] for li in local_ids]
        return
    if n <= leaf_size or depth > 100:
        out.append((base, base + n))
        return
    sl = ids[lo:hi]
    normal, offset = random_hyperplane(data, sl, rng)
    sides = _sides_seq(data, sl, normal, offset, rng)
    split = partition_in_place(sl, sides)
    if split == 0 or split == n:
        split = random_split(sl, rng)
        if split == 0 or split == n:
            ids[lo:hi] = sl
            out.append((base, base + n))
            return
    ids[lo:hi] = sl
    rp_tree_sequential(data, ids, lo, lo + split, base, leaf_size, rng, depth + 1, gather_max,
                       out)
    rp_tree_sequential(data, ids, lo + split, hi, base + split, leaf_size, rng, depth + 1,
                       gather_max, out)


def rp_tree_parallel(data, ids, lo, hi, base, leaf_size, seed, depth, gather_max):
    n = hi - lo
    if n < 8192 or depth >= 6:
        out = []
        rp_tree_sequential(data, ids, lo, hi, base, leaf_size, Rng(seed), depth, gather_max, out)
        return out
    rng = Rng(seed)
    sl = ids[lo:hi]
    normal, offset = random_hyperplane(data, sl, rng)
    margins = (dot_rows(normal, data[np.asarray(sl, np.int64)]) + offset).astype(F32)
    sides = [(splitmix(seed ^ i) & 1 == 0) if abs(m) < F32(1e-8) else bool(m > 0.0)
             for i, m in zip(sl, margins)]
    split = partition_in_place(sl, sides)
    if split == 0 or split == n:
        split = random_split(sl, rng)
    ids[lo:hi] = sl
    left = rp_tree_parallel(data, ids, lo, lo + split, base, leaf_size, splitmix(seed ^ 1),
                            depth + 1, gather_max)
    right = rp_tree_parallel(data, ids, lo + split, hi, base + split, leaf_size,
                             splitmix(seed ^ 2), depth + 1, gather_max)
    return left + right


def build_tree(data, leaf_size, seed, gather_max=GATHER_MAX):
    """(ids, leaves) of one tree (nndescent.rs:643-646)."""
    data = np.ascontiguousarray(data, F32)
    n = data.shape[0]
    ids = list(range(n))
    leaves = rp_tree_parallel(data, ids, 0, n, 0, leaf_size, seed, 0, gather_max)
    return np.asarray(ids, np.uint32), np.asarray(leaves, np.uint32).reshape(-1, 2)


# ── the algorithm (nndescent.rs:699-1003) ───────────────────────────────────

def effective_k(n_obs, k):
    return max(min(k, max(n_obs - 1, 0)), 1)


def resolve(n, k, max_candidates=0, max_iterations=0, n_trees=0, leaf_size=0):
    k = max(min(k, n - 1), 1)
    max_cand = max(max_candidates if max_candidates > 0 else min(2 * k, 60), 1)
    n_iters = max_iterations if max_iterations > 0 else max(int(_round(np.log2(n))), 5)
    trees = n_trees if n_trees > 0 else min(8 + int(_round(np.sqrt(n) / 10.0)), 48)
    leaf = leaf_size if leaf_size > 0 else max(k, 10)
    return k, max_cand, n_iters, trees, leaf


def _round(x: float) -> float:
    """Rust's f64::round: half away from zero."""
    return float(np.floor(x + 0.5)) if x >= 0 else -float(np.floor(-x + 0.5))


def _apply(idx, dist, flag, k, gen, changed_out=None):
    """apply_updates (nndescent.rs:307-324): per bucket, chunk by chunk."""
    changed = 0
    for b in range(N_BUCKETS):
        for chunk in gen:
            for dest, nbr, dd in chunk[b]:
                if heap_push(idx, dist, flag, dest * k, k, nbr, dd, True):
                    changed += 1
    return changed


def nndescent(data, k=15, *, max_iterations=0, seed=0, max_candidates=0, n_trees=0, delta=0.001,
              leaf_size=0, gather_max=0):
    """The CSR graph {indptr, indices, data} and the per-round changed counts."""
    data = np.ascontiguousarray(data, F32)
    n, d = data.shape
    assert n > 0 and d > 0 and k > 0
    k, max_cand, n_iters, trees, leaf = resolve(n, k, max_candidates, max_iterations, n_trees,
                                                leaf_size)
    gmax = gather_max if gather_max > 0 else GATHER_MAX
    rpb = rows_per_bucket(n)
    idx = [EMPTY] * (n * k)
    dist = [F32(np.inf)] * (n * k)
    flag = [False] * (n * k)

    # 1. forest and leaf pairs, one tree after another
    forest = [build_tree(data, leaf, splitmix(seed ^ (t + 1)), gmax) for t in range(trees)]
    for ids, leaves in forest:
        gen = []
        for c0 in range(0, len(leaves), 64):
            buckets = [[] for _ in range(N_BUCKETS)]
            for a, b in leaves[c0:c0 + 64]:
                leaf_ids = [int(v) for v in ids[a:b]]
                for i, p in enumerate(leaf_ids):
                    for q in leaf_ids[i + 1:]:
                        dd = sq_dist(data[p], data[q])
                        buckets[p // rpb].append((p, q, dd))
                        buckets[q // rpb].append((q, p, dd))
            gen.append(buckets)
        _apply(idx, dist, flag, k, gen)

    # random fill of empty slots
    for i in range(n):
        attempt = 0
        while EMPTY in idx[i * k:(i + 1) * k] and attempt < 64:
            j = hash_index(seed, i, attempt, n)
            if j == i:
                j = (j + 1) % n
            heap_push(idx, dist, flag, i * k, k, j, sq_dist(data[i], data[j]), True)
            attempt += 1

    # 2. rounds
    stop_at = int(delta * n * k)
    changed_per_round = []
    for it in range(n_iters):
        new_i, new_p = [EMPTY] * (n * max_cand), [F32(np.inf)] * (n * max_cand)
        old_i, old_p = [EMPTY] * (n * max_cand), [F32(np.inf)] * (n * max_cand)
        for b0 in range(0, n, BLOCK):
            b1 = min(b0 + BLOCK, n)
            gen = []
            for c0 in range(b0, b1, GEN_CHUNK):
                buckets = [[] for _ in range(N_BUCKETS)]
                for i in range(c0, min(c0 + GEN_CHUNK, b1)):
                    for s in range(k):
                        j = idx[i * k + s]
                        if j == EMPTY:
                            continue
                        is_new = flag[i * k + s]
                        pr = hash_unit(seed, it, i * k + s)
                        buckets[i // rpb].append((i, j, pr, is_new))
                        buckets[j // rpb].append((j, i, pr, is_new))
                gen.append(buckets)
            for want_new, ci, cp in ((True, new_i, new_p), (False, old_i, old_p)):
                for b in range(N_BUCKETS):
                    for chunk in gen:
                        for dest, nbr, pr, is_new in chunk[b]:
                            if is_new == want_new:
                                cand_push(ci, cp, dest * max_cand, max_cand, nbr, pr)
        for i in range(n):
            row = new_i[i * max_cand:(i + 1) * max_cand]
            for s in range(k):
                if flag[i * k + s] and idx[i * k + s] != EMPTY and idx[i * k + s] in row:
                    flag[i * k + s] = False
        thr = [dist[i * k] for i in range(n)]
        changed = 0
        for b0 in range(0, n, BLOCK):
            b1 = min(b0 + BLOCK, n)
            gen = []
            for c0 in range(b0, b1, GEN_CHUNK):
                buckets = [[] for _ in range(N_BUCKETS)]
                for i in range(c0, min(c0 + GEN_CHUNK, b1)):
                    news = new_i[i * max_cand:(i + 1) * max_cand]
                    olds = old_i[i * max_cand:(i + 1) * max_cand]
                    for a, p in enumerate(news):
                        if p == EMPTY:
                            continue
                        for q in list(news[a + 1:]) + list(olds):
                            if q == EMPTY or q == p:
                                continue
                            dd = sq_dist(data[p], data[q])
                            if dd < thr[p]:
                                buckets[p // rpb].append((p, q, dd))
                            if dd < thr[q]:
                                buckets[q // rpb].append((q, p, dd))
                gen.append(buckets)
            changed += _apply(idx, dist, flag, k, gen)
        changed_per_round.append(changed)
        if changed <= stop_at:
            break

    # 3. extract: stable sort by distance, sqrt
    indptr = [0]
    indices, dists = [], []
    for i in range(n):
        row = [(idx[i * k + s], dist[i * k + s]) for s in range(k) if idx[i * k + s] != EMPTY]
        row.sort(key=lambda e: e[1])  # stable, as Rust's sort_by
        for j, dd in row:
            indices.append(j)
            dists.append(np.sqrt(F32(dd)).astype(F32))
        indptr.append(len(indices))
    return {"indptr": np.asarray(indptr, np.uint32), "indices": np.asarray(indices, np.uint32),
            "data": np.asarray(dists, F32), "round_changed": changed_per_round}


# ── the reference tests' random inputs (nndescent.rs:1012-1022) ─────────────

_MASK32 = 0xFFFFFFFF


def _rotl(v, c):
    return ((v << c) & _MASK32) | (v >> (32 - c))


def chacha_block(key_words, counter: int, stream: int, rounds: int):
    """One ChaCha block (16 little-endian u32 words): constants, 8 key words,
    64-bit block counter, 64-bit stream id; `rounds` of column / diagonal
    quarter rounds, then the input added word by word."""
    st = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574, *key_words,
          counter & _MASK32, (counter >> 32) & _MASK32, stream & _MASK32, (stream >> 32) & _MASK32]
    x = list(st)

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & _MASK32
        x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & _MASK32
        x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & _MASK32
        x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & _MASK32
        x[b] = _rotl(x[b] ^ x[c], 7)

    for _ in range(rounds // 2):
        qr(0, 4, 8, 12)
        qr(1, 5, 9, 13)
        qr(2, 6, 10, 14)
        qr(3, 7, 11, 15)
        qr(0, 5, 10, 15)
        qr(1, 6, 11, 12)
        qr(2, 7, 8, 13)
        qr(3, 4, 9, 14)
    return [(a + b) & _MASK32 for a, b in zip(x, st)]


def seed_from_u64(state: int) -> bytes:
    """rand_core's SeedableRng::seed_from_u64 for a 32-byte seed: each 4-byte
    chunk is the output of one PCG32 step (advance, then XSH RR)."""
    mul, inc = 6364136223846793005, 11634580027462260723
    out = b""
    for _ in range(8):
        state = (state * mul + inc) & M64
        xorshifted = (((state >> 18) ^ state) >> 27) & _MASK32
        rot = state >> 59
        x = ((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & _MASK32
        out += x.to_bytes(4, "little")
    return out


class ChaCha8Rng:
    """rand_chacha's ChaCha8Rng from a 32-byte seed: the keystream's u32 words
    in order, block counter from 0, stream 0."""

    def __init__(self, seed: bytes, rounds: int = 8):
        self.key = [int.from_bytes(seed[4 * i:4 * i + 4], "little") for i in range(8)]
        self.rounds = rounds
        self.counter = 0
        self.buf = []

    @classmethod
    def seed_from_u64(cls, state: int) -> "ChaCha8Rng":
        return cls(seed_from_u64(state))

    def next_u32(self) -> int:
        if not self.buf:
            self.buf = chacha_block(self.key, self.counter, 0, self.rounds)
            self.counter += 1
        return self.buf.pop(0)

    def random_f32(self) -> F32:
        """rand's StandardUniform f32: 24 high bits of a u32 times 2^-24."""
        return F32(F32(self.next_u32() >> 8) * F32(1.0 / (1 << 24)))


def make_clustered_data(n: int, d: int, n_clusters: int, seed: int) -> np.ndarray:
    """The reference tests' input: row i = (i % n_clusters) * 10 + U[0, 1)
    per coordinate, drawn in row-major order from ChaCha8Rng::seed_from_u64."""
    rng = ChaCha8Rng.seed_from_u64(seed)
    out = np.empty(n * d, F32)
    for i in range(n):
        c = F32(i % n_clusters)
        for j in range(d):
            out[i * d + j] = F32(F32(c * F32(10.0)) + rng.random_f32())
    return out.reshape(n, d)


def make_blob_data(n: int = 6000, d: int = 20, seed: int = 9) -> np.ndarray:
    """The input of the reference's recall test (nndescent.rs:1109-1133):
    row i, coordinate j = (i % 12) * 3 * (j % 3) + 4 U[0, 1)."""
    rng = ChaCha8Rng.seed_from_u64(seed)
    out = np.empty(n * d, F32)
    for i in range(n):
        c = F32(i % 12)
        for j in range(d):
            out[i * d + j] = F32(F32(F32(c * F32(3.0)) * F32(j % 3))
                                 + F32(rng.random_f32() * F32(4.0)))
    return out.reshape(n, d)
