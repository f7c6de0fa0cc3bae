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
         tensor-core tiles, bytes for the plain form's join) over its CUDA-event
         duration, against the measured peak (sustained BF16 GEMM, HBM copy)
  cpu_baseline  the C++ restatement of the reference's CPU NN-Descent (oracle/)
         on a bounded sample of the same workload, all host threads

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
    ap.add_argument("--form", default="bf16", choices=["plain", "bf16", "fp8"],
                    help="the headline form (the other is measured too unless --skip-other)")
    ap.add_argument("--skip-other", action="store_true")
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
    for s in range(0, len(q), 256):
        qi = qt[s:s + 256]
        xq = xd[qi]
        d2 = x2[qi][:, None] + x2[None, :] - 2.0 * (xq @ xd.T)
        d2[torch.arange(len(qi), device=d2.device), qi] = float("inf")
        # (distance, index) order: stable sort of the k+8 best by distance
        vals, idx = torch.topk(d2, k + 8, dim=1, largest=False, sorted=True)
        exact = idx[:, :k].cpu().numpy()
        a = ind[q[s:s + 256]]
        for r in range(len(qi)):
            hits += len(set(exact[r].tolist()) & set(a[r].tolist()))
        # max relative error of returned distances vs the FP64 distance of each pair
        aj = torch.from_numpy(a.astype(np.int64)).to(x_dev.device)
        true = torch.sqrt(((xq[:, None, :] - xd[aj]) ** 2).sum(-1))
        got = torch.from_numpy(dst[q[s:s + 256]].astype(np.float64)).to(x_dev.device)
        rel = ((got - true).abs() / true.clamp_min(1e-30)).max().item()
        max_rel = max(max_rel, rel)
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
            "sample": f"first {s} cells of the workload, one full build ({dt:.2f} s)"}


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
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * s / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config(args), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) per 128 x 256 tile pair of the shortlist tile kernel:
# an ncu capture (--set full) of its two passes at 1M x 50 read
# and wrote 0.537 GB over 184,331 tile pairs (primary pass) and 1.443 GB over
# 806,044 (other probes), 1,999 bytes per pair over both; a launch's traffic
# is taken to scale with the tile pairs it processes.
TILE_DRAM_BYTES_PER_PAIR = 1999.0


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
    traffic = (TILE_DRAM_BYTES_PER_PAIR * tile_pairs / L
               if TILE_DRAM_BYTES_PER_PAIR is not None else None)
    return {"bound": "tensor", "kernel": "k_ivf_tiles", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "padded_tflops": padded, "launches_per_build": L,
            "peak_source": ("measured sustained bf16" if "bf16_tflops_sustained" in peaks
                            else "fallback")}


def join_roofline(per, st, args, peaks):
    """The plain form's join pass 1 against HBM: every non-empty candidate row
    of every source row read once, the candidate ids and thresholds, and the
    emit bits written, per launch over the launch's CUDA-event time."""
    g = per.get("join_count")
    if not g or g["launches_per_build"] == 0:
        return None
    n, d = args.n, args.d
    m = st["max_candidates"]
    ab = n * (2 * m * 4 * d + 2 * m * 8 + (4 * m * m) // 8 + 4) * g["launches_per_build"]
    L = g["launches_per_build"]
    sec = g["ms_per_build"] / L / 1000.0
    achieved = ab / L / sec / 1e9
    hbm = peaks.get("hbm_gbs", 6650.0)
    return {"bound": "hbm", "kernel": "k_join_count", "achieved": achieved, "peak": hbm,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}


def measure_form(torch, pq, _lib, ctx, form, xd, dev, stream, args, barrier, world, k=None):
    """W warm-up then K device-resident builds of one form, timed with CUDA
    events on the launching stream (max over ranks), with per-group events."""
    n, k = xd.shape[0], (k or args.k)
    cap = n * pq.effective_k(n, k)
    opts = pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES[form])
    ip = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ix = torch.empty(cap, dtype=torch.int32, device=dev)
    dx = torch.empty(cap, dtype=torch.float32, device=dev)

    def step():
        return ctx.nndescent_device(xd, opts, ip, ix, dx, stream=stream.cuda_stream)

    for _ in range(max(3, args.warmup)):
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
    for _ in range(args.steps):
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
    ms = max_over_ranks(torch, e0.elapsed_time(e1) / args.steps, dev, world)
    names = _lib.KERNEL_GROUPS
    per = {names[g]: {"ms_per_build": float(kg_ms[g] / args.steps),
                      "launches_per_build": int(kg_l[g] // args.steps)}
           for g in range(len(names)) if kg_l[g] > 0}
    rec, max_rel = recall_fp64(torch, xd, ix[:nnz].cpu().numpy().view(np.uint32),
                               dx[:nnz].cpu().numpy(), k, args.queries)
    st = stats[-1]
    return {"ms": ms, "value": world * n / (ms / 1000.0), "launches": launches // args.steps,
            "launches_timed": int(launches), "groups": per, "stats": st,
            "recall_at_k": rec, "max_rel_dist_err": max_rel, "rounds_run": st["rounds_run"]}


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
    from polariseq_b200 import _lib

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
        opts = pq._opts(k, 0, 0, 0, 0, 0.001, mode=pq.MODES[args.form])
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

    # ── device-resident timed region of the headline form (clocks sampled) ──
    clocks = Clocks(local)
    clocks.start()
    head = measure_form(torch, pq, _lib, ctx, args.form, xd, dev, stream, args, barrier, world)
    ck = clocks.stop()
    forms = {args.form: head}
    forms_k30 = {}
    if not args.skip_other:
        for other in ("plain", "bf16", "fp8"):
            if other != args.form:
                forms[other] = measure_form(torch, pq, _lib, ctx, other, xd, dev, stream, args,
                                            barrier, world)
        # k = 30 (the E4M3 form supports k <= 15)
        for other in ("bf16", "plain"):
            forms_k30[other] = measure_form(torch, pq, _lib, ctx, other, xd, dev, stream, args,
                                            barrier, world, k=30)

    # ── end to end through the public API with pinned host buffers ──
    hx = torch.from_numpy(x).pin_memory()
    hip = torch.empty(n + 1, dtype=torch.int32).pin_memory()
    hix = torch.empty(cap, dtype=torch.int32).pin_memory()
    hdx = torch.empty(cap, dtype=torch.float32).pin_memory()
    hxn, hipn = hx.numpy(), hip.numpy().view(np.uint32)
    hixn, hdxn = hix.numpy().view(np.uint32), hdx.numpy()
    r = pq.nndescent_dense(hxn, k, out=(hipn, hixn, hdxn), device=local, mode=args.form)
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        r = pq.nndescent_dense(hxn, k, out=(hipn, hixn, hdxn), device=local, mode=args.form)
    e2e_ms = max_over_ranks(torch, (time.perf_counter() - t0) * 1000.0 / e2e_steps, dev, world)
    e2e = {"value": world * n / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": int(x.nbytes),
           "d2h_bytes_per_step": int(4 * (n + 1) + 8 * r["nnz"]), "steps": e2e_steps}

    roof = (tiles_roofline(head["groups"], head["stats"], args, peaks) if args.form != "plain"
            else join_roofline(head["groups"], head["stats"], args, peaks))

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            cpu = cpu_baseline(args, x)
        except Exception as e:  # pragma: no cover
            cpu = {"error": str(e)}

    def summary(f):
        st = f["stats"]
        out = {"cells_per_s": f["value"], "ms_per_build": f["ms"],
               "recall_at_k": f["recall_at_k"], "max_rel_dist_err": f["max_rel_dist_err"],
               "rounds_run": f["rounds_run"], "launches_per_build": f["launches"],
               "phases_ms": {"init": st["ms_forest"], "layout_or_leaves": st["ms_leaves"],
                             "search_or_rounds": st["ms_rounds"], "finish": st["ms_extract"]},
               "kernel_groups": f["groups"]}
        return out

    forms_out = {f: summary(v) for f, v in forms.items()}
    forms_k30_out = {f: summary(v) for f, v in forms_k30.items()}
    if "plain" in forms:
        forms_out["plain"]["roofline"] = join_roofline(forms["plain"]["groups"],
                                                       forms["plain"]["stats"], args, peaks)
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": head["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16" if args.form != "plain" else "f32", "data": "synthetic",
            "config": config(args), "e2e": e2e, "gpu_launches": head["launches_timed"],
            "roofline": roof, "cpu_baseline": cpu, "clocks": ck,
            "quality": {"recall_at_k": head["recall_at_k"],
                        "max_rel_dist_err": head["max_rel_dist_err"],
                        "queries": min(args.queries, n), "oracle": "FP64 brute force"},
            "forms": forms_out, "forms_k30": forms_k30_out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
