#!/usr/bin/env python
"""Benchmark of the Galerkin triple product C = R*A*P on one or more B200s.

Workload: the 128^3 7-point Poisson operator with 2x2x2 aggregation and one
damped-Jacobi smoothing step (A: 2,097,152 rows, 14.6M nonzeros; P:
2,097,152 x 262,144; R = P^T), FP64, seeded synthetic data.  A step is one
complete R*A*P product on the device (default: direct variant, upper-bound
flavour), inputs resident in HBM, output allocated and freed each step.

Metric: compulsory-byte throughput in GB/s -- R, A and P read once plus C
written once, counted in the device format (int32 indices, FP64 values).  The
inputs (~390 MB) exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs (torchrun, one rank per GPU) are replicas: every rank runs
its own product (weak scaling, no data-path collective); the time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sp3mm4amg_b200 import problems as pb  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "roofline_traffic.json")
FALLBACK_HBM_GBS = 6650.0

VARIANTS = {"pair": 0, "direct": 1, "pair_right": 2}
FLAVOURS = {"ub": 0, "symbnum": 1}

# nvidia-smi clocks_event_reasons bits.
REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
           0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
           0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
           0x100: "display_clock_setting"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="direct", choices=list(VARIANTS))
    ap.add_argument("--flavour", default="ub", choices=list(FLAVOURS))
    ap.add_argument("--side", type=int, default=128, help="grid side of the 3D problem")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=2.5,
                    help="seconds of reference work per step of --impl reference")
    ap.add_argument("--no-ref-full", action="store_true",
                    help="--impl reference: skip the one unsampled full product")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the cpu_baseline sample")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched workload")
    ap.add_argument("--no-served", action="store_true", help="skip the served workload")
    ap.add_argument("--no-irregular", action="store_true", help="skip the irregular workload")
    ap.add_argument("--no-hierarchy", action="store_true",
                    help="skip the hierarchy build of the main grid")
    ap.add_argument("--no-library", action="store_true",
                    help="skip the cuSPARSE context measurement")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--serve-count", type=int, default=200)
    ap.add_argument("--serve-rate", type=float, default=100.0, help="requests per second")
    return ap.parse_args()


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_name(side):
    return f"poisson3d_{side}^3_7pt_agg2x2x2_jacobi"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.cmd = ["nvidia-smi", f"--id={index}",
                    "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                    "--format=csv,noheader,nounits", "-lms", "50"]
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        for line in out.splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 3:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
                bits = int(parts[2], 16)
            except ValueError:
                continue
            for b, name in REASONS.items():
                if bits & b and name != "gpu_idle":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def smi_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own OpenMP code (oracle/_ref) on a bounded
# row sample of the same product, extrapolated to the full product.

def cpu_reference_runner(prob, threads, variant="direct"):
    """Returns (kind, fn(rows) -> seconds, description) for the reference's
    own code (oracle/_ref) on the first `rows` rows of R: the direct
    upper-bound product sp3mmRowByRowMerged_0 -- the variant the main line
    runs -- or (variant "pair") sp3mmRowByRowPair_0 with spmmRowByRow_0."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle
    try:
        ref = oracle.Reference(threads=threads)
        ref.adapt_grid(0)
        if variant == "direct":
            def run(rows):
                Rs = prob.R.rows(0, rows)
                t0 = time.perf_counter()
                ref.sp3mm_direct(Rs, prob.A, prob.P, 0)
                return time.perf_counter() - t0
            return ("reference", run,
                    "reference sp3mmRowByRowMerged_0 (direct, upper-bound: the main line's "
                    "variant)")

        def run(rows):
            Rs = prob.R.rows(0, rows)
            t0 = time.perf_counter()
            ref.sp3mm_pair("spmmRowByRow_", Rs, prob.A, prob.P, 0)
            return time.perf_counter() - t0
        return ("reference", run,
                "reference sp3mmRowByRowPair_0 with spmmRowByRow_0 (pair-wise, upper-bound 1D)")
    except (FileNotFoundError, OSError):
        orc = oracle.Oracle()
        orc.set_threads(threads)

        def run(rows):
            Rs = prob.R.rows(0, rows)
            t0 = time.perf_counter()
            if variant == "direct":
                orc.sp3mm_direct(Rs, prob.A, prob.P)
            else:
                orc.sp3mm_pair(Rs, prob.A, prob.P)
            return time.perf_counter() - t0
        return "port", run, f"oracle restatement ({variant}), reference library not built"


def calibrated_sample(run, M, seconds):
    rows = 64
    t = run(rows)
    while t < 0.5 and rows < M:
        rows = min(M, rows * 4)
        t = run(rows)
    want = int(rows * seconds / max(t, 1e-6))
    return max(1, min(M, want))


def run_reference_arm(args, prob, nnz_c):
    """The reference's own CPU code on the main line's product (direct,
    upper-bound) with all host threads: each step a row sample of R, its
    time scaled to the whole product (the reference's cost is linear in the
    rows of R: every row resets its dense accumulators); once per run the
    whole product unsampled (`full_product`, unless --no-ref-full), which
    checks that scaling; and a sample of the pair-wise upper-bound product
    (`pair_ub`) beside it."""
    threads = os.cpu_count() or 1
    total_bytes = prob.compulsory_bytes(nnz_c=nnz_c, idx_bytes=4)
    ref_variant = "direct" if args.variant == "direct" else "pair"
    kind, run, desc = cpu_reference_runner(prob, threads, ref_variant)
    M = prob.R.M
    rows = calibrated_sample(run, M, args.ref_seconds)
    vals, times = [], []
    for i in range(args.warmup + args.steps):
        t = run(rows)
        if i >= args.warmup:
            times.append(t)
            vals.append(total_bytes / (t * M / rows) / 1e9)
    value = statistics.median(vals)
    scaled_s = statistics.median(times) * M / rows
    sample = f"rows 0..{rows} of {M} of R per step ({desc}), time scaled by {M}/{rows}"
    full = None
    if not args.no_ref_full:
        t_full = run(M) if rows < M else statistics.median(times)
        full = {"seconds": t_full, "value": total_bytes / t_full / 1e9, "unit": "GB/s",
                "scaled_estimate_s": scaled_s, "scaled_over_full": scaled_s / t_full}
    pkind, prun, pdesc = cpu_reference_runner(prob, threads, "pair")
    prows = calibrated_sample(prun, M, args.ref_seconds)
    ptimes = [prun(prows) for _ in range(3)]
    pair = {"value": total_bytes / (statistics.median(ptimes) * M / prows) / 1e9, "unit": "GB/s",
            "seconds_per_product": statistics.median(ptimes) * M / prows,
            "sample": f"rows 0..{prows} of {M} of R, median of 3 ({pdesc})"}
    line = {
        "impl": "reference", "metric": "rap_compulsory_GBps", "value": value, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_bytes / (value * 1e9) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.side), "variant": args.variant,
                   "flavour": args.flavour, "rows_R": M, "nnz_A": prob.A.nnz,
                   "nnz_P": prob.P.nnz, "nnz_C": nnz_c, "bytes_per_product": total_bytes,
                   "byte_basis": "int32 idx + f64 val"},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "full_product": full,
        "pair_ub": pair,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Batched and served workloads.

def _events_time(torch, stream, fn):
    """Seconds of fn() between events on the context stream (host waits
    inside fn are part of it)."""
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) * 1e-3


def run_batched(S, torch, ctx, stream, count, seed=3, min_coarse=1000):
    """Many uneven products: the R*A*P products of `count` device-built
    smoothed-aggregation hierarchies (2D 5-point / 3D 7-point, n log-uniform
    in [1e3, 2e5], each repeated until n < 1000), computed one product per
    call versus as one batch (plan + execute) and as graph replays."""
    specs = pb.config3_specs(seed, count)
    ops = [pb.stencil_operator(d) for d in specs]
    dA = [ctx.upload(o) for o in ops]
    # Warm-up at full size: the memory pool grows to the workload's needs.
    for h in ctx.hierarchies(dA, specs, min_coarse=min_coarse, max_levels=20):
        h.free()
    # Median of three builds each way: some builds stall on the host for
    # 0.3-1 s (seen in the batched build's planning; cause not known), which
    # a single sample would report as the build time.
    hb_runs, hs = [], []
    for rep in range(3):
        got = []
        hb_runs.append(_events_time(torch, stream, lambda: got.extend(
            ctx.hierarchies(dA, specs, min_coarse=min_coarse, max_levels=20))))
        if rep < 2:
            for h in got:
                h.free()
        else:
            hs = got
    t_hb = float(np.median(hb_runs))

    def singles():
        for a, d in zip(dA, specs):
            ctx.hierarchy(a, d, min_coarse=min_coarse, max_levels=20).free()
    hs_runs = [_events_time(torch, stream, singles) for _ in range(3)]
    t_hs = float(np.median(hs_runs))
    prods = []
    for h in hs:
        for lvl in range(len(h) - 1):
            A, P, R = h.level(lvl)
            prods.append((R, A, P))
    rows = sum(p[0].shape[0] for p in prods)

    def plain():
        for R, A, P in prods:
            ctx.rap(R, A, P, S.DIRECT, S.UB).free()
    plain()   # warm-up
    t_plain = min(_events_time(torch, stream, plain) for _ in range(2))
    t_full, reps = [], 10
    launches0 = ctx.launches()
    for i in range(3):
        box = {}
        t = _events_time(torch, stream, lambda: box.update(b=ctx.batch(prods)) or box["b"].run())
        b = box["b"]
        if i > 0:
            t_full.append(t)
        if i < 2:
            b.free()
    full_launches = (ctx.launches() - launches0) // 3
    tune = b.autotune(3)
    t_rep = _events_time(torch, stream, lambda: [b.execute() for _ in range(reps)]) / reps
    info = b.info()
    b.free()
    for h in hs:
        h.free()
    for a in dA:
        a.free()
    n = len(prods)
    tf = min(t_full)
    return {
        "workload": f"{count} hierarchies (2D 5-pt / 3D 7-pt, n log-uniform 1e3..2e5, "
                    f"seed {seed}), every R*A*P level product until n < {min_coarse}",
        "products": n, "rows_C": rows, "nnz_C": info["nnz"],
        "plain_products_per_s": n / t_plain,
        "batch_products_per_s": n / tf, "speedup": t_plain / tf,
        "replay_products_per_s": n / t_rep, "replay_speedup": t_plain / t_rep,
        "plain_s": t_plain, "batch_s": tf, "replay_s": t_rep,
        "batch_launches": full_launches, "tiers": info["tiers"],
        "autotune": tune.strip().splitlines()[:3],
        "hierarchy_build_batched_s": t_hb, "hierarchy_build_single_s": t_hs,
        "hierarchy_build_batched_s_each": hb_runs, "hierarchy_build_single_s_each": hs_runs,
        "hierarchy_build_speedup": t_hs / t_hb,
        "timing": "CUDA events on the context stream around each whole pass",
    }


def run_irregular(S, torch, ctx, stream, npoints=1_000_000, steps=10):
    """The irregular product: kNN graph Laplacian of `npoints` seeded points
    (16 neighbours, symmetrised), greedy aggregation, one Jacobi step;
    direct upper-bound R*A*P timed on the device, inputs resident."""
    prob = pb.knn_problem(npoints, seed=2)
    d = [ctx.upload(m) for m in (prob.R, prob.A, prob.P)]
    nnz_c = 0
    for _ in range(3):
        C = ctx.rap(*d, S.DIRECT, S.UB)
        nnz_c = C.nnz
        C.free()
    t = _events_time(torch, stream, lambda: [ctx.rap(*d, S.DIRECT, S.UB).free()
                                             for _ in range(steps)]) / steps
    ctx.set_profiling(True)
    ctx.rap(*d, S.DIRECT, S.UB).free()
    prof = ctx.profile()
    ctx.set_profiling(False)
    for m in d:
        m.free()
    total = prob.compulsory_bytes(nnz_c=nnz_c, idx_bytes=4)
    deg = np.diff(prob.A.indptr) - 1
    return {"workload": f"knn16 Laplacian, {npoints} points (seed 2), greedy aggregation "
                        f"(mean {prob.A.M / prob.P.N:.2f} per aggregate), Jacobi-smoothed P",
            "rows_R": prob.R.M, "nnz_A": prob.A.nnz, "nnz_P": prob.P.nnz, "nnz_C": nnz_c,
            "degree_min_max": [int(deg.min()), int(deg.max())],
            "ms_per_product": t * 1e3, "GBps": total / t / 1e9, "bytes_per_product": total,
            "kernels_ms": {k: v[1] for k, v in prof.items()}}


def run_hierarchy(S, torch, ctx, stream, side=128, steps=3):
    """The AMG caller of the path: a device hierarchy over the 3D 7-point
    operator on a side^3 grid (2x2x2 aggregation, one Jacobi step, R = P^T,
    A_{l+1} = R_l A_l P_l direct, until fewer than 1000 rows), its build time,
    and every level's R*A*P product timed alone with its kernels."""
    dims = (side, side, side)
    dA = ctx.upload(pb.stencil_operator(dims))
    for _ in range(2):
        ctx.hierarchy(dA, dims, min_coarse=1000).free()
    t_build = _events_time(torch, stream, lambda: [ctx.hierarchy(dA, dims, min_coarse=1000).free()
                                                   for _ in range(steps)]) / steps
    h = ctx.hierarchy(dA, dims, min_coarse=1000)
    levels = []
    for l in range(len(h)):
        A, P, R = h.level(l)
        if P is None:
            levels.append({"level": l, "rows": A.d.M, "nnz": A.d.nnz})
            continue
        for _ in range(2):
            ctx.rap(R, A, P, S.DIRECT, S.UB).free()
        t = _events_time(torch, stream, lambda: [ctx.rap(R, A, P, S.DIRECT, S.UB).free()
                                                 for _ in range(steps)]) / steps
        ctx.set_profiling(True)
        ctx.rap(R, A, P, S.DIRECT, S.UB).free()
        prof = ctx.profile()
        ctx.set_profiling(False)
        levels.append({"level": l, "rows_R": R.d.M, "nnz_A": A.d.nnz, "nnz_P": P.d.nnz,
                       "ms_per_product": t * 1e3,
                       "kernels_ms": {k: round(v[1], 4) for k, v in prof.items()}})
    h.free()
    dA.free()
    return {"workload": f"3D 7-point {side}^3, block 2 aggregation, one Jacobi step, direct UB "
                        "products until n < 1000",
            "build_ms": t_build * 1e3, "levels": levels}


def run_library(torch, prob, steps=5):
    """Context only, not the product: the same product as (R*A)*P through
    torch's sparse CSR matrix product on the device (cuSPARSE SpGEMM), FP64,
    inputs resident."""
    try:
        dev = torch.device("cuda")

        def t(m):
            return torch.sparse_csr_tensor(
                torch.as_tensor(m.indptr, dtype=torch.int64, device=dev),
                torch.as_tensor(m.indices, dtype=torch.int64, device=dev),
                torch.as_tensor(m.data, dtype=torch.float64, device=dev), size=m.shape)
        R, A, P = t(prob.R), t(prob.A), t(prob.P)
        C = (R @ A) @ P
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            C = (R @ A) @ P
        b.record()
        b.synchronize()
        nnz = int(C._nnz())
        del R, A, P, C
        torch.cuda.empty_cache()
        return {"library": "cuSPARSE SpGEMM via torch sparse CSR, (R*A)*P, FP64, int64 indices",
                "ms_per_product": a.elapsed_time(b) / steps, "nnz_C": nnz}
    except Exception as e:  # noqa: BLE001 - report, do not fail the bench
        return {"library": "cuSPARSE SpGEMM via torch sparse CSR", "unavailable": repr(e)[:200]}


def run_served(S, ctx, count, rate, seed=4, reps=3):
    """A Poisson stream of hierarchy-setup requests (90% of config-3 sizes,
    10% 3D 64^3..128^3) served by continuous batching versus one request at
    a time, at `rate` requests/s and saturated (all arriving at once)."""
    from sp3mm4amg_b200 import serving
    specs = pb.config4_specs(seed, count)
    ops = [pb.stencil_operator(d) for d in specs]
    arrivals = pb.poisson_arrivals(rate, count, seed + 1)
    # Warm-up at full size in both value types (the memory pool grows to the
    # workload's needs; every kernel instantiation is loaded).
    for cvt in (S.F64, S.F32):
        serving.serve_batched(ctx, specs, np.zeros(count), coarse_val_type=cvt, operators=ops)
    serving.serve_plain(ctx, specs[:8], np.zeros(8), operators=ops[:8])
    res = {"workload": f"{count} requests (seed {seed}): 90% 2D/3D n log-uniform 1e3..2e5, "
                       f"10% 3D side 64..128; hierarchy to n < 1000",
           "rate_per_s": rate, "repeats": reps}
    runs = {"fp64": [], "fp32_coarse": [], "plain_fp64": []}
    for _ in range(reps):
        for name, cvt in (("fp64", S.F64), ("fp32_coarse", S.F32)):
            st, _ = serving.serve_batched(ctx, specs, arrivals, coarse_val_type=cvt,
                                          operators=ops)
            sat, _ = serving.serve_batched(ctx, specs, np.zeros(count), coarse_val_type=cvt,
                                           operators=ops)
            runs[name].append((st, sat))
        plain = serving.serve_plain(ctx, specs, arrivals, operators=ops)
        plain_sat = serving.serve_plain(ctx, specs, np.zeros(count), operators=ops)
        runs["plain_fp64"].append((plain, plain_sat))

    def med(xs):
        return float(np.median(xs))
    for name, rr in runs.items():
        res[name] = {"p50_s": med([st["p50_s"] for st, _ in rr]),
                     "p99_s": med([st["p99_s"] for st, _ in rr]),
                     "p99_s_each": [st["p99_s"] for st, _ in rr],
                     "products_per_s": med([st["products_per_s"] for st, _ in rr]),
                     "products": rr[0][0]["products"],
                     "saturated_products_per_s": med([sat["products_per_s"] for _, sat in rr]),
                     "saturated_products_per_s_each": [sat["products_per_s"] for _, sat in rr],
                     "saturated_p99_s": med([sat["p99_s"] for _, sat in rr])}
        if name != "plain_fp64":
            res[name]["peak_active"] = max(st["peak_active"] for st, _ in rr)
            res[name]["failed"] = sum(st["failed"] + sat["failed"] for st, sat in rr)
    kept = {}
    for name, cvt in (("fp64", S.F64), ("fp32_coarse", S.F32)):
        _, kept[name] = serving.serve_batched(ctx, specs, np.zeros(count), coarse_val_type=cvt,
                                              operators=ops, keep=True)
    # FP32 coarse storage: every request's every level against its FP64
    # hierarchy (which equals the oracle chain bit for bit), on the device.
    per_level = {}
    for a, b in zip(kept["fp32_coarse"], kept["fp64"]):
        for lvl, e in enumerate(serving.level_errors(a, b)):
            per_level.setdefault(lvl, []).append(e)
        a.free()
        b.free()
    lv = sorted(per_level.items())
    res["fp32_level_max_rel_err"] = {str(l): max(e[0] for e in v) for l, v in lv}
    res["fp32_level_median_rel_err"] = {str(l): float(np.median([e[0] for e in v]))
                                        for l, v in lv}
    res["fp32_level_max_err_over_max"] = {str(l): max(e[1] for e in v) for l, v in lv}
    # How many entries the large relative errors are (cancellation near zero).
    res["fp32_level_entries_rel_err_over_1e-3"] = {str(l): sum(e[2] for e in v) for l, v in lv}
    res["fp32_level_entries"] = {str(l): sum(e[3] for e in v) for l, v in lv}
    res["fp32_error_coverage"] = f"all {count} requests, every level (device comparison)"
    res["saturated_speedup_fp64"] = (res["fp64"]["saturated_products_per_s"] /
                                     res["plain_fp64"]["saturated_products_per_s"])
    return res


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The slowest rank's time: every rank contributes, all receive the max."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(units_per_rank: float, world: int, elapsed_s: float) -> float:
    """Whole-job throughput: the units all ranks processed over the max time."""
    return world * units_per_rank / elapsed_s


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        prob = pb.stencil_problem(3, args.side)
        nnz_c = 8_382_712 if args.side == 128 else None
        if nnz_c is None:
            import oracle
            nnz_c = oracle.Oracle().sp3mm_pair(prob.R, prob.A, prob.P).nnz
        run_reference_arm(args, prob, nnz_c)
        return

    import torch
    import sp3mm4amg_b200 as S
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    def barrier():
        if dist is not None:
            dist.barrier()

    prob = pb.stencil_problem(3, args.side)
    variant, flavour = VARIANTS[args.variant], FLAVOURS[args.flavour]
    ctx = S.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))
    dR, dA, dP = ctx.upload(prob.R), ctx.upload(prob.A), ctx.upload(prob.P)

    # Warm-up (also fixes the output size).
    nnz_c = 0
    for _ in range(max(args.warmup, 3)):
        C = ctx.rap(dR, dA, dP, variant, flavour)
        nnz_c = C.nnz
        C.free()
    ctx.sync()
    total_bytes = prob.compulsory_bytes(nnz_c=nnz_c, idx_bytes=4)

    clocks = ClockSampler(smi_index(local_rank))
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        C = ctx.rap(dR, dA, dP, variant, flavour)
        C.free()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launches() - launches0
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    elapsed_ms = max_over_ranks(elapsed_ms, dist, "cuda")
    ms_per_step = elapsed_ms / args.steps
    value = job_value(args.steps * total_bytes, world, elapsed_ms * 1e-3) / 1e9

    # Per-kernel device times (separate pass with per-launch events).
    ctx.set_profiling(True)
    nprof = 10
    for _ in range(nprof):
        C = ctx.rap(dR, dA, dP, variant, flavour)
        C.free()
    prof = ctx.profile()
    ctx.set_profiling(False)
    dom_label, (dom_n, dom_total, _) = max(prof.items(), key=lambda kv: kv[1][1])
    all_ms = sum(v[1] for v in prof.values())
    peak, peak_kind = peaks()
    # The dominant row kernel reads R, A and P and writes C: its algorithmic
    # bytes per launch are the product's compulsory bytes.
    dom_avg_ms = dom_total / nprof
    achieved = total_bytes / (dom_avg_ms * 1e-3) / 1e9
    traffic = None
    try:
        with open(TRAFFIC_PATH) as f:
            tj = json.load(f)
        if tj.get("kernel_label") == dom_label and tj.get("variant") == args.variant:
            traffic = tj.get("dram_bytes_per_launch")
    except Exception:
        pass

    # End to end through the drop-in C entry point: pinned host spmat in,
    # malloc'd host spmat out, host<->device copies inside the timed region.
    import ctypes
    from sp3mm4amg_b200 import capi
    from sp3mm4amg_b200.spmat import CONFIG, HostSpMat
    lib = capi.load()
    hR, hA, hP = (HostSpMat(m, 0, pinned=True) for m in (prob.R, prob.A, prob.P))
    fname = {(1, 0): "sp3mmRowByRowMerged_0", (1, 1): "sp3mmRowByRowMerged_SymbNum_0",
             (0, 0): "sp3mmRowByRowPair_0", (0, 1): "sp3mmRowByRowPair_SymbNum_0",
             (2, 0): "sp3mmRowByRowPairRight_0", (2, 1): "sp3mmRowByRowPairRight_0"}[
        (variant, flavour)]
    fn = getattr(lib, fname)
    cfg = CONFIG(gridRows=1, gridCols=1, symbMMRowImplID=0, threadNum=1, chunkDistrbFunc=None)
    spmm_arg = None
    if variant == 2 and flavour == 1:
        spmm_arg = ctypes.cast(lib.spmmRowByRow_SymbNum_0, ctypes.c_void_p).value
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    from sp3mm4amg_b200.spmat import SPMAT_P
    e2e_times = []
    nz = nnz_c
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p = fn(hR.ptr, hA.ptr, hP.ptr, ctypes.byref(cfg), spmm_arg)
        t1 = time.perf_counter()
        if not p:
            raise RuntimeError("e2e call returned NULL")
        m = ctypes.cast(p, SPMAT_P).contents
        nz = int(m.NZ)
        for arr in (m.AS, m.JA, m.IRP):
            libc.free(ctypes.cast(arr, ctypes.c_void_p))
        libc.free(p)
        if i > 0:
            e2e_times.append(t1 - t0)
    e2e_t = statistics.median(e2e_times) if e2e_times else None
    h2d = sum((mm.M + 1) * 8 + mm.nnz * 16 for mm in (prob.R, prob.A, prob.P))
    d2h = (prob.R.M + 1) * 8 + nz * 16

    line = {
        "metric": "rap_compulsory_GBps", "value": value, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": workload_name(args.side), "variant": args.variant,
                   "flavour": args.flavour, "rows_R": prob.R.M, "nnz_A": prob.A.nnz,
                   "nnz_P": prob.P.nnz, "nnz_C": nnz_c,
                   "bytes_per_product": total_bytes, "byte_basis": "int32 idx + f64 val",
                   "products_per_s": world * args.steps / (elapsed_ms * 1e-3),
                   "l2": "inputs exceed L2 (126 MB); no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": dom_label, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel_share": dom_total / all_ms if all_ms else None,
                     "kernels_ms_per_product": {k: v[1] / nprof for k, v in prof.items()}},
        "e2e": None if e2e_t is None else {
            "value": total_bytes / e2e_t / 1e9, "unit": "GB/s", "seconds_per_product": e2e_t,
            "entry_point": fname, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and not args.no_library:
        line["library_context"] = run_library(torch, prob)
    if rank == 0 and not args.no_batched:
        line["batched"] = run_batched(S, torch, ctx, stream, args.batch_count)
    if rank == 0 and not args.no_served:
        line["served"] = run_served(S, ctx, args.serve_count, args.serve_rate)
    if rank == 0 and not args.no_irregular:
        line["irregular"] = run_irregular(S, torch, ctx, stream)
    if rank == 0 and not args.no_hierarchy:
        line["hierarchy"] = run_hierarchy(S, torch, ctx, stream, side=args.side)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        kind, run, desc = cpu_reference_runner(
            prob, threads, "direct" if args.variant == "direct" else "pair")
        rows = calibrated_sample(run, prob.R.M, args.cpu_seconds)
        t = run(rows)
        full = t * prob.R.M / rows
        line["cpu_baseline"] = {
            "value": total_bytes / full / 1e9, "unit": "GB/s", "cores": threads, "kind": kind,
            "sample": f"rows 0..{rows} of {prob.R.M} of R ({desc}); {t:.2f} s, scaled to the "
                      f"full product ({full:.1f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
