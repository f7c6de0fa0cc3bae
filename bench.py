"""Benchmark: kNN-graph build throughput (cells/s) on one B200 per rank.

Workload (one "step" = one complete kNN-graph build): 4,000,000 cells x 50 PCs
f32, k = 15, a 60-component Gaussian mixture with log-normal cluster sizes, a
j^-0.5 per-dimension spectrum and 5% doublet-like midpoints (seeded synthetic
data standing in for a PCA embedding; no dataset is needed or available).

  value  cells/s with the embedding already resident in HBM (device entry point)
  e2e    cells/s through the C ABI with pinned HOST buffers: the embedding's
         host->device copy and the graph's device->host copy are inside the
         timed region
  roofline  the dominant kernel's algorithmic work per launch (flops for the
         tensor-core tiles, bytes for the plain form's subtrees) over its
         CUDA-event duration, against the measured peak (sustained BF16 GEMM,
         HBM copy)
  cpu_baseline  the C++ restatement of the reference's CPU NN-Descent (oracle/)
         on the whole workload, all host threads; the same build checks the
         plain form's graph byte for byte (plain_bit_exact)
  forms  the plain form at the reference defaults and with the best reference
         options found (plain_tuned; recall@15 >= 0.99 is out of the reference
         algorithm's reach on this workload), the BF16 and E4M3 shortlist
         forms, and the learned-init NN-Descent; forms_k30 the same at k = 30
  configs  1.3M x 50 (plain, plain_tuned, BF16) and the batched doublet-scoring
         workload (one persistent launch vs 64 launches, CPU knn_exact)

Multi-GPU (torchrun): each rank builds the graph of its own embedding (replicas
of the workload with different seeds); per-step time is the max over ranks.

`--impl reference` times the reference algorithm's CPU implementation (the
oracle port; the Rust reference cannot be built here) on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "kNN build cells/s, 4M×50, k=15: plain vs chosen form at recall@15≥0.99"
UNIT = "cells/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4_000_000)
    ap.add_argument("--d", type=int, default=50)
    ap.add_argument("--k", type=int, default=15)
    ap.add_argument("--comps", type=int, default=60)
    ap.add_argument("--queries", type=int, default=20_000)
    ap.add_argument("--cpu-sample", type=int, default=262_144)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--form", default="bf16",
                    choices=["plain", "plain_tuned", "bf16", "fp8", "learned"],
                    help="the headline form (the others are measured too unless --skip-other)")
    ap.add_argument("--others", default="plain,plain_tuned,bf16,fp8,learned",
                    help="comma-separated forms measured besides the headline")
    ap.add_argument("--skip-other", action="store_true")
    ap.add_argument("--skip-k30", action="store_true")
    ap.add_argument("--skip-configs", action="store_true")
    ap.add_argument("--profile-only", action="store_true",
                    help="run W warm-up and K device-resident builds, print nothing else "
                         "(for ncu launch lists)")
    return ap.parse_args()


def max_over_ranks(torch, value: float, device, world: int) -> float:
    """The largest of every rank's value (per-step times are reported as the
    slowest rank's); a no-op on one rank."""
    if world <= 1:
        return value
    import torch.distributed as dist

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(args, rank):
    from polariseq_b200 import synth

    return synth.mixture_lognormal(args.n, args.d, args.comps, seed=1000 + rank)


def config(args):
    return {"workload": f"kNN graph build, {args.n} cells x {args.d} PCs f32, k={args.k}, "
                        f"{args.comps}-component log-normal Gaussian mixture, 5% doublets",
            "n_cells": args.n, "n_pcs": args.d, "k": args.k,
            "form": {"plain": "plain (bit-exact)",
                     "plain_tuned": "plain (bit-exact) with the best reference options found",
                     "learned": "learned-init NN-Descent (router's top buckets seed the lists)",
                     "bf16": "chosen: bf16 tensor-core shortlist + FP32 re-rank + FP64 boundary",
                     "fp8": "e4m3 tensor-core shortlist + FP32 re-rank + FP64 boundary"}[args.form],
            "l2": "inputs larger than L2 (embedding 800 MB, graph 480 MB)"}


# ── clocks sampled during the timed region ─────────────────────────────────
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ── recall vs FP64 exact on sampled queries ────────────────────────────────
def recall_fp64(torch, x_dev, indices, dists, k, nq, seed=7):
    """recall@k and max relative distance error against an FP64 brute force
    (self excluded, (distance, index) order) on nq seeded query rows."""
    n = x_dev.shape[0]
    g = np.random.default_rng(seed)
    q = np.sort(g.choice(n, size=min(nq, n), replace=False))
    xd = x_dev.double()
    x2 = (xd * xd).sum(1)
    hits = 0
    max_rel = 0.0
    ind = indices.reshape(n, k)
    dst = dists.reshape(n, k)
    qt = torch.from_numpy(q).to(x_dev.device)
    # query chunks whose FP64 distance rows stay near 2 GB
    qc = int(max(8, min(256, (2 << 30) // (8 * n))))
    for s in range(0, len(q), qc):
        qi = qt[s:s + qc]
        xq = xd[qi]
        d2 = x2[qi][:, None] + x2[None, :] - 2.0 * (xq @ xd.T)
        d2[torch.arange(len(qi), device=d2.device), qi] = float("inf")
        # (distance, index) order: the k+8 nearest, ties at equal FP64
        # distance ordered by index, then the first k
        vals, idx = torch.topk(d2, k + 8, dim=1, largest=False, sorted=True)
        vals, idx = vals.cpu().numpy(), idx.cpu().numpy()
        order = np.lexsort((idx, vals), axis=1)
        exact = np.take_along_axis(idx, order, axis=1)[:, :k]
        a = ind[q[s:s + qc]]
        for r in range(len(qi)):
            hits += len(set(exact[r].tolist()) & set(a[r].tolist()))
        # max relative error of returned distances vs the FP64 distance of each pair
        aj = torch.from_numpy(a.astype(np.int64)).to(x_dev.device)
        true = torch.sqrt(((xq[:, None, :] - xd[aj]) ** 2).sum(-1))
        got = torch.from_numpy(dst[q[s:s + qc]].astype(np.float64)).to(x_dev.device)
        rel = ((got - true).abs() / true.clamp_min(1e-30)).max().item()
        max_rel = max(max_rel, rel)
    del xd, x2
    # hand the cached blocks back: the library allocates its own workspace
    torch.cuda.empty_cache()
    return hits / (len(q) * k), max_rel


def cpu_baseline(args, x, threads=None):
    """The oracle (C++ restatement of the reference CPU algorithm) on the
    first `cpu_sample` cells of the workload, all host threads."""
    import oracle

    oracle.lib()
    if threads:
        oracle.set_threads(threads)
    s = min(args.cpu_sample, x.shape[0])
    sample = np.ascontiguousarray(x[:s])
    t0 = time.perf_counter()
    oracle.nndescent(sample, args.k, seed=0)
    dt = time.perf_counter() - t0
    return {"value": s / dt, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port",
            "sample": f"first {s} of the workload's {x.shape[0]} cells, one full build "
                      f"({dt:.2f} s); per-cell cost grows with n, so the sample flatters the CPU"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    x = workload(args, 0)
    for _ in range(args.warmup):
        cpu_baseline(args, x)
    vals = [cpu_baseline(args, x) for _ in range(args.steps)]
    v = statistics.median([r["value"] for r in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    s = min(args.cpu_sample, args.n)
    cfg = config(args)
    cfg["reference_sample_cells"] = s
    cfg["reference_sample"] = (f"each step builds the graph of the first {s} cells of the "
                               f"{args.n}-cell workload (a full build of all cells takes "
                               "about a minute on the host, too long for K steps)")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * s / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) per tile pair (128 x 256 or 256 x 128 contractions)
# of the shortlist tile kernels, from ncu captures (--set full) of their two
# passes at 1M x 50: the wide kernel (BF16, 16-entry shortlists) read and wrote
# 0.528 GB over 170,761 pairs (primary pass) and 1.379 GB over 721,611 (other
# probes), 2,137 bytes per pair over both; the standard kernel 0.537 GB over
# 184,331 and 1.443 GB over 806,044, 1,999 bytes per pair.  A launch's traffic
# is taken to scale with the tile pairs it processes.
TILE_DRAM_BYTES_PER_PAIR = {"k_ivf_wide": 2137.0, "k_ivf_tiles": 1999.0}


def tiles_roofline(per, st, args, peaks):
    """The shortlist tile kernel against the tensor pipe: algorithmic flops are
    2 * (query entry, candidate) pairs * d (unpadded), per launch, over the
    launch's CUDA-event time."""
    g = per.get("tiles")
    if not g or g["launches_per_build"] == 0:
        return None
    cells = st["shortlist"][3]
    tile_pairs = st["shortlist"][0]
    L = g["launches_per_build"]
    sec = g["ms_per_build"] / L / 1000.0
    flops = 2.0 * cells * args.d / L
    achieved = flops / sec / 1e12
    peak = peaks.get("bf16_tflops_sustained") or 1400.0
    padded = 2.0 * tile_pairs * 128 * 256 * 64 / L / sec / 1e12
    # BF16 tiles with 16-entry shortlists (k <= 15) run the wide kernel
    kernel = ("k_ivf_wide" if args.form in ("bf16", "learned") and args.k <= 15
              else "k_ivf_tiles")
    traffic = TILE_DRAM_BYTES_PER_PAIR[kernel] * tile_pairs / L
    return {"bound": "tensor", "kernel": kernel, "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "padded_tflops": padded, "launches_per_build": L,
            "peak_source": ("measured sustained bf16" if "bf16_tflops_sustained" in peaks
                            else "fallback")}


def seqtree_roofline(per, st, n, d, peaks):
    """The plain form's dominant kernel group, the depth-first RP subtrees,
    against HBM: each tree's rows read once below its parallel top levels
    (trees x n x 4d bytes) over the group's CUDA-event time.  The kernel is
    bound by its depth-first chain of dependent nodes, not by bandwidth, so
    the fraction is small by nature."""
    g = per.get("seqtree")
    if not g or g["launches_per_build"] == 0:
        return None
    ab = float(st["n_trees"]) * n * 4 * d
    sec = g["ms_per_build"] / 1000.0
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = ab / sec / 1e9
    return {"bound": "hbm", "kernel": "k_seqtree", "achieved": achieved, "peak": hbm,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
            "ms_per_build": g["ms_per_build"],
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}


# The best of the reference's own NndescentOptions (nndescent.rs:42-76) found
# for recall@15 on the 4M x 50 workload: the bit-exact plain form, graph for
# graph.  A sweep (max_candidates 30-120, delta down to 1e-4 with 40
# iterations, leaf_size 15-40, 48-96 trees) tops out at 0.955 with these
# (defaults 0.888, 120 candidates 0.924): recall@15 >= 0.99 is out of the
# reference algorithm's reach on this workload at k = 15.
PLAIN_TUNED = {"max_candidates": 60, "n_trees": 96, "leaf_size": 40}

FORMS = {"plain": {"mode": "plain"}, "plain_tuned": dict(mode="plain", **PLAIN_TUNED),
         "bf16": {"mode": "bf16"}, "fp8": {"mode": "fp8"},
         # learned-init NN-Descent: the router's top-4 buckets seed the lists,
         # the reference's rounds (default options) run to convergence
         "learned": {"mode": "plain", "init": "learned"}}


def form_opts(pq, name, k):
    f = FORMS[name]
    return pq._opts(k, f.get("max_iterations", 0), 0, f.get("max_candidates", 0),
                    f.get("n_trees", 0), f.get("delta", 0.001), f.get("leaf_size", 0),
                    mode=pq.MODES[f["mode"]],
                    init=pq.INITS[f.get("init", "rp")])


def measure_form(torch, pq, _lib, ctx, name, xd, dev, stream, steps, warmup, barrier, world, k,
                 queries, keep=False):
    """`warmup` untimed then `steps` device-resident builds of one form, timed
    with CUDA events on the launching stream (max over ranks), with
    per-group events; recall@k against FP64 on `queries` cells and a check
    that every row is ascending."""
    n = xd.shape[0]
    cap = n * pq.effective_k(n, k)
    opts = form_opts(pq, name, k)
    ip = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ix = torch.empty(cap, dtype=torch.int32, device=dev)
    dx = torch.empty(cap, dtype=torch.float32, device=dev)

    def step():
        return ctx.nndescent_device(xd, opts, ip, ix, dx, stream=stream.cuda_stream)

    for _ in range(max(3, warmup)):
        step()
    torch.cuda.synchronize(dev)
    _lib.load().pq_ctx_set_profiling(ctx._h, 1)
    kg_ms = np.zeros(16)
    kg_l = np.zeros(16, np.int64)
    launches = 0
    stats = []
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        nnz = step()
        stats.append(ctx.stats())
        s = _lib.NndStats()
        _lib.load().pq_ctx_stats(ctx._h, s)
        kg_ms += np.array(s.kg_ms[:16])
        kg_l += np.array(s.kg_launches[:16], np.int64)
        launches += s.launches
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    _lib.load().pq_ctx_set_profiling(ctx._h, 0)
    ms = max_over_ranks(torch, e0.elapsed_time(e1) / steps, dev, world)
    names = _lib.KERNEL_GROUPS
    per = {names[g]: {"ms_per_build": float(kg_ms[g] / steps),
                      "launches_per_build": int(kg_l[g] // steps)}
           for g in range(len(names)) if kg_l[g] > 0}
    kk = pq.effective_k(n, k)
    full = nnz == n * kk
    d2 = dx[:nnz].view(n, kk) if full else None
    ascending = bool((d2[:, 1:] >= d2[:, :-1]).all()) if full else None
    if full:
        rec, max_rel = recall_fp64(torch, xd, ix[:nnz].cpu().numpy().view(np.uint32),
                                   dx[:nnz].cpu().numpy(), kk, queries)
    else:
        rec, max_rel = None, None
    st = stats[-1]
    out = {"ms": ms, "value": world * n / (ms / 1000.0), "launches": launches // steps,
           "launches_timed": int(launches), "groups": per, "stats": st, "steps": steps,
           "recall_at_k": rec, "max_rel_dist_err": max_rel, "rounds_run": st["rounds_run"],
           "rows_ascending": ascending}
    if keep:
        out["graph"] = {"indptr": ip.cpu().numpy().view(np.uint32),
                        "indices": ix[:nnz].cpu().numpy().view(np.uint32),
                        "data": dx[:nnz].cpu().numpy()}
    return out


def summary(f):
    st = f["stats"]
    return {"cells_per_s": f["value"], "ms_per_build": f["ms"], "steps": f["steps"],
            "recall_at_k": f["recall_at_k"], "max_rel_dist_err": f["max_rel_dist_err"],
            "rows_ascending": f["rows_ascending"], "rounds_run": f["rounds_run"],
            "launches_per_build": f["launches"],
            "phases_ms": {"init": st["ms_forest"], "layout_or_leaves": st["ms_leaves"],
                          "search_or_rounds": st["ms_rounds"], "finish": st["ms_extract"]},
            "kernel_groups": f["groups"],
            **({"learned": {k: st[k] for k in ("est_recall", "est_recall_learned",
                                               "est_recall_rp", "fell_back", "learned_rounds",
                                               "ms_learn_train", "ms_learn_route",
                                               "learn_loss_first", "learn_loss_last")}}
               if st.get("ms_learn_train") else {})}


def plain_bit_exact(x, k, graph):
    """The oracle's graph of the same workload (reference defaults, seed 0),
    timed on all host threads, compared byte for byte with the plain form's."""
    import oracle

    oracle.lib()
    t0 = time.perf_counter()
    r = oracle.nndescent(x, k, seed=0)
    dt = time.perf_counter() - t0
    same = (np.array_equal(r["indptr"], graph["indptr"])
            and np.array_equal(r["indices"], graph["indices"])
            and r["data"].tobytes() == graph["data"].tobytes())
    return same, dt


def bench_batched(torch, pq, ctx, dev, args, steps, warmup):
    """The doublet-scoring workload: 64 samples, cell counts log-uniform in
    [2,000, 60,000] plus 2x simulated doublets (30 PCs), k = round(0.5 sqrt(n))
    per sample, exact kNN of every point within its sample.  One persistent,
    work-queued, graph-captured launch for all samples against 64 launches of
    one sample each; recall against FP64 on sampled points of the largest
    sample; the reference's tiled knn_exact restated in C++ (all host
    threads) on a bounded subset of the samples."""
    from polariseq_b200 import synth

    samples = synth.doublet_samples(64, 2000, 60000, seed=0, device=f"cuda:{dev.index}")
    cells = [len(a) // 3 for a in samples]
    ks = np.array([max(1, int(round(0.5 * np.sqrt(c)))) for c in cells], np.uint32)
    sizes = np.array([len(a) for a in samples], np.uint64)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    pts = int(sizes.sum())
    total = int(np.sum(sizes * ks.astype(np.uint64)))
    x = torch.from_numpy(np.concatenate(samples)).to(dev)
    oi = torch.empty(total, dtype=torch.int32, device=dev)
    od = torch.empty(total, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    shape = ctx.knn_batched_device(x, offs, ks, oi, od, autotune=True, graph=True,
                                   stream=stream.cuda_stream)
    for _ in range(max(3, warmup)):
        ctx.knn_batched_device(x, offs, ks, oi, od, graph=True, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.knn_batched_device(x, offs, ks, oi, od, graph=True, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    one = e0.elapsed_time(e1) / steps
    # 64 separate launches, one sample each (the same kernel)
    out_off = np.concatenate([[0], np.cumsum(sizes * ks.astype(np.uint64))]).astype(np.int64)
    e0.record(stream)
    for s in range(len(samples)):
        a, b = int(offs[s]), int(offs[s + 1])
        o0, o1 = int(out_off[s]), int(out_off[s + 1])
        ctx.knn_batched_device(x[a:b], np.array([0, b - a], np.uint64), ks[s:s + 1],
                               oi[o0:o1], od[o0:o1], graph=False, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    sep = e0.elapsed_time(e1)
    # recall of the largest sample against FP64
    big = int(np.argmax(sizes))
    a, b = int(offs[big]), int(offs[big + 1])
    o0, o1 = int(out_off[big]), int(out_off[big + 1])
    kb = int(ks[big])
    rec, max_rel = recall_fp64(torch, x[a:b], oi[o0:o1].cpu().numpy().view(np.uint32),
                               od[o0:o1].cpu().numpy(), kb, 2000)
    pairs = float(np.sum(sizes.astype(np.float64) ** 2))
    out = {"workload": "64 samples, cells log-uniform in [2000, 60000] + 2x simulated doublets, "
                       "30 PCs, k = round(0.5 sqrt(cells)) per sample",
           "points": pts, "samples": len(samples), "k_range": [int(ks.min()), int(ks.max())],
           "tile_shape": shape, "steps": steps,
           "one_launch_ms": one, "points_per_s": pts / (one / 1000.0),
           "separate_launches_ms": sep, "distance_pairs": pairs,
           "pair_rate_tflops_fp32": 2.0 * pairs * 30 / (one / 1000.0) / 1e12,
           "recall_at_k_largest_sample": rec, "max_rel_dist_err": max_rel}
    if not args.no_cpu:
        import oracle

        oracle.lib()
        # a bounded subset: the samples in order until ~5e10 point pairs
        sub, acc = [], 0.0
        for s in range(len(samples)):
            if sub and acc + float(sizes[s]) ** 2 > 5e10:
                break
            sub.append(s)
            acc += float(sizes[s]) ** 2
        t0 = time.perf_counter()
        oracle.knn_exact_batched([samples[s] for s in sub], [int(ks[s]) for s in sub])
        dt = time.perf_counter() - t0
        sp = int(sum(int(sizes[s]) for s in sub))
        out["cpu_baseline"] = {"value": sp / dt, "unit": "points/s",
                               "cores": oracle.max_threads(), "kind": "port",
                               "sample": f"the first {len(sub)} samples ({sp} points), one "
                                         f"call ({dt:.2f} s)"}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    import polariseq_b200 as pq
    from polariseq_b200 import _lib, synth

    x = workload(args, rank)
    n, d, k = x.shape[0], x.shape[1], args.k
    cap = n * pq.effective_k(n, k)
    ctx = pq.Context(local)
    stream = torch.cuda.current_stream(dev)
    xd = torch.from_numpy(x).to(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    if args.profile_only:
        opts = form_opts(pq, args.form, k)
        ip = torch.empty(n + 1, dtype=torch.int32, device=dev)
        ix = torch.empty(cap, dtype=torch.int32, device=dev)
        dx = torch.empty(cap, dtype=torch.float32, device=dev)
        for _ in range(args.warmup + args.steps):
            ctx.nndescent_device(xd, opts, ip, ix, dx, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        st = ctx.stats()
        print(json.dumps({"profile_only": True, "n": n, "form": args.form,
                          "ms_total": st["ms_total"], "shortlist": st.get("shortlist")}),
              flush=True)
        return

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    # secondary forms and configurations: fewer timed builds, one GPU only
    sec = min(args.steps, 5)
    others = world == 1 and not args.skip_other

    # ── device-resident timed region of the headline form (clocks sampled) ──
    clocks = Clocks(local)
    clocks.start()
    head = measure_form(torch, pq, _lib, ctx, args.form, xd, dev, stream, args.steps,
                        args.warmup, barrier, world, k, args.queries)
    ck = clocks.stop()
    forms = {args.form: head}
    forms_k30 = {}
    if others:
        for other in [f for f in args.others.split(",") if f]:
            if other != args.form:
                forms[other] = measure_form(torch, pq, _lib, ctx, other, xd, dev, stream, sec, 3,
                                            barrier, world, k, args.queries,
                                            keep=other == "plain")
        for other in ([] if args.skip_k30 else ["bf16", "fp8", "plain"]):
            try:
                forms_k30[other] = measure_form(torch, pq, _lib, ctx, other, xd, dev, stream,
                                                sec, 3, barrier, world, 30, args.queries)
            except NotImplementedError as e:
                forms_k30[other] = {"unsupported": str(e)}

    # ── end to end through the public API with pinned host buffers ──
    hx = torch.from_numpy(x).pin_memory()
    hip = torch.empty(n + 1, dtype=torch.int32).pin_memory()
    hix = torch.empty(cap, dtype=torch.int32).pin_memory()
    hdx = torch.empty(cap, dtype=torch.float32).pin_memory()
    hxn, hipn = hx.numpy(), hip.numpy().view(np.uint32)
    hixn, hdxn = hix.numpy().view(np.uint32), hdx.numpy()
    hopts = form_opts(pq, args.form, k)

    def e2e_build():
        # the host-buffer entry point (nndescent_into with caller arrays)
        return ctx.nndescent_into(hxn, hopts, hipn, hixn, hdxn)

    nnz = e2e_build()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        nnz = e2e_build()
    e2e_ms = max_over_ranks(torch, (time.perf_counter() - t0) * 1000.0 / args.steps, dev, world)
    e2e = {"value": world * n / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": int(x.nbytes),
           "d2h_bytes_per_step": int(4 * (n + 1) + 8 * nnz), "steps": args.steps}

    roof = (tiles_roofline(head["groups"], head["stats"], args, peaks) if args.form != "plain"
            else seqtree_roofline(head["groups"], head["stats"], n, d, peaks))

    # ── the CPU baseline: the oracle on the whole workload (which also checks
    #    the plain form's graph byte for byte), else on a bounded sample ──
    cpu = None
    bit_exact = None
    if rank == 0 and not args.no_cpu:
        try:
            if "plain" in forms and "graph" in forms["plain"]:
                bit_exact, dt = plain_bit_exact(x, k, forms["plain"].pop("graph"))
                import oracle

                cpu = {"value": n / dt, "unit": UNIT, "cores": oracle.max_threads(),
                       "kind": "port", "sample": f"the whole workload ({n} cells), one build "
                                                 f"({dt:.1f} s), also the bit-exact check"}
            else:
                cpu = cpu_baseline(args, x)
        except Exception as e:  # pragma: no cover
            cpu = {"error": str(e)}

    # ── the other configurations ──
    configs = {}
    if others and not args.skip_configs:
        del xd
        x2 = synth.mixture_lognormal(1_300_000, d, 40, seed=2000)
        xd2 = torch.from_numpy(x2).to(dev)
        c2 = {}
        for f in ("plain", "plain_tuned", "bf16"):
            c2[f] = summary(measure_form(torch, pq, _lib, ctx, f, xd2, dev, stream, sec, 3,
                                         barrier, world, k, args.queries))
        configs["c2_1.3M"] = {"workload": "1,300,000 cells x 50 PCs f32, k=15, 40-component "
                                          "log-normal Gaussian mixture, 5% doublets",
                              "forms": c2}
        del xd2
        configs["c4_batched"] = bench_batched(torch, pq, ctx, dev, args, sec, 3)

    forms_out = {f: summary(v) for f, v in forms.items()}
    forms_k30_out = {f: (summary(v) if "stats" in v else v) for f, v in forms_k30.items()}
    if "plain" in forms:
        forms_out["plain"]["roofline"] = seqtree_roofline(forms["plain"]["groups"],
                                                          forms["plain"]["stats"], n, d, peaks)
        forms_out["plain"]["bit_exact_vs_oracle"] = bit_exact
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": head["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16" if args.form != "plain" else "f32", "data": "synthetic",
            "config": config(args), "e2e": e2e, "gpu_launches": head["launches_timed"],
            "roofline": roof, "cpu_baseline": cpu, "clocks": ck,
            "quality": {"recall_at_k": head["recall_at_k"],
                        "max_rel_dist_err": head["max_rel_dist_err"],
                        "rows_ascending": head["rows_ascending"],
                        "queries": min(args.queries, n), "oracle": "FP64 brute force"},
            "plain_bit_exact": bit_exact, "plain_tuned_options": PLAIN_TUNED,
            "forms": forms_out, "forms_k30": forms_k30_out, "configs": configs}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
