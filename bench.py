"""Benchmark of the lane-packing subinterval search on B200.

One step = the box refinement of all six families from a uniform lattice seed
(64 subdivisions per axis over lambda in [0.5, 0.99], the reference's dependent
radius ranges), not-proved boxes bisected on every axis (16 children for the
3-disk families, 8 for the 2-disk ones) down to a bounded depth.  `value` is the
box throughput of the best form (FP32 enclosure pre-pass + FP64); the plain
FP64 form runs on the same boxes and both must give identical verdict counts.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--depth L]
    python bench.py --impl reference     # the CPU restatement on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "full-domain proof wall time & boxes/s: batched+learned vs plain FP64, same verdicts"
UNIT = "boxes/s"
FAMILIES = range(6)
DIMS = (4, 3, 4, 4, 3, 4)
SEED_RES = 64
LEVEL_CAP = 1 << 25


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--depth", type=int, default=2, help="bisection levels below the 64^dims seed")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--families", default="0,1,2,3,4,5", help="comma list (profiling runs)")
    ap.add_argument("--seed-res", type=int, default=64, help="lattice subdivisions per axis of the seed")
    ap.add_argument("--level-capacity", type=int, default=1 << 25, help="boxes per worklist level buffer")
    ap.add_argument("--no-autotune", action="store_true", help="default kernel variants, FP64 (profiling runs)")
    return ap.parse_args()


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        backend = "nccl"
        import torch

        torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=__import__("datetime").timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for k, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- workload
def seed_opts(family, precision, depth):
    import circlepacking_b200 as cp

    return dict(precision=precision, policy=cp.SPLIT_UNIFORM, max_depth=depth,
                seed_sizes=[SEED_RES] * DIMS[family], seed_lambda=(cp.LAMBDA_MIN, cp.LAMBDA_MAX),
                level_capacity=LEVEL_CAP)


def run_step(prover, precision, depth):
    """One step over all families; precision: a cp precision or a per-family dict."""
    reps = []
    for f in FAMILIES:
        prec = precision[f] if isinstance(precision, dict) else precision
        reps.append(prover.refine(f, **seed_opts(f, prec, depth)))
    return reps


def autotune(prover, cp):
    """Per family: the fastest level-kernel variant for each precision on a
    calibration refinement (32^dims seed, one level), then the faster precision.
    Both precisions give identical verdicts, so the choice is speed only."""
    chosen, table = {}, {}
    for f in FAMILIES:
        calib = dict(policy=cp.SPLIT_UNIFORM, max_depth=1, seed_sizes=[32] * DIMS[f])
        t = {}
        for prec in (cp.FP64, cp.FP32_PREFILTER):
            v, ms = prover.autotune(f, precision=prec, **calib)
            t[prec] = (min(ms), v, ms)
        best = min(t, key=lambda k: t[k][0])
        chosen[f] = best
        table[cp.FAMILIES[f]] = {"precision": "fp64" if best == cp.FP64 else "fp32-prefilter",
                                 "variant": t[best][1],
                                 "calib_ms": {"fp64": t[cp.FP64][2], "fp32-prefilter": t[cp.FP32_PREFILTER][2]}}
    return chosen, table


def seed_boxes_host(family):
    """The 64^dims lattice seed of a family in pinned host memory (numpy view)."""
    import torch

    import circlepacking_b200 as cp

    total = SEED_RES ** DIMS[family]
    idx = torch.arange(total, device="cuda", dtype=torch.int64)
    lo, hi, vis = cp.lattice_boxes(family, (cp.LAMBDA_MIN, cp.LAMBDA_MAX), [SEED_RES] * DIMS[family], idx,
                                   visited=True)
    hlo = torch.empty(lo.shape, dtype=torch.float64, pin_memory=True)
    hhi = torch.empty(hi.shape, dtype=torch.float64, pin_memory=True)
    hdp = torch.empty(vis.shape, dtype=torch.uint8, pin_memory=True)
    hlo.copy_(lo)
    hhi.copy_(hi)
    hdp.copy_(torch.where(vis != 0, 0, 255).to(torch.uint8))  # 255: boxes the lattice never visits
    return hlo, hhi, hdp


def roofline_work():
    """Primitive-op counts per box (CPU oracle, the reference's evaluation path)
    on a sample of each family's seed lattice."""
    from oracle import oracle as O

    counts = {}
    rng = np.random.default_rng(0)
    for f in FAMILIES:
        dims = DIMS[f]
        total = SEED_RES ** dims
        idx = np.sort(rng.choice(total, size=min(4000, total), replace=False))
        lo, hi = O.lattice_boxes(f, (0.5, 0.9900000000000001), [SEED_RES] * dims, idx)
        counts[f] = O.count_ops(f, lo, hi)
    return counts


def roofline_of(cp, device, reps_plain) -> dict:
    """Roofline of the FP64 level kernel: DFMA-equivalent work per box (each
    primitive weighted by the measured DFMA rate over its own measured rate)
    against the measured DFMA peak."""
    rates = cp.measure_primitives(device)
    counts = roofline_work()
    work = 0.0
    for f, r in zip(FAMILIES, reps_plain):
        c = counts[f]
        per_box = (c["add"] * rates["dfma"] / rates["dadd_rd"] + c["mul"] * rates["dfma"] / rates["dmul_rd"]
                   + c["div"] * rates["dfma"] / rates["ddiv_rd"] + c["asin"] * rates["dfma"] / rates["asin"]) / c["boxes"]
        work += r["evaluated"] * per_box
    kernel_ms = sum(r["device_ms"] for r in reps_plain)
    achieved = 2.0 * work / (kernel_ms / 1e3) / 1e12
    peak = 2.0 * rates["dfma"] / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": None, "kernel": "k_level<family, fp64> (per-box FP64 criteria + split)",
            "work_model": "per box: CPU-oracle-counted add/mul/div/asin of the reference's evaluation path on the "
                          "seed lattices, each weighted by measured DFMA rate / primitive rate; peak = measured DFMA",
            "peaks_measured_tops": {k: v / 1e12 for k, v in rates.items()}, "peak_source": "measured in-process",
            "ops_per_box": {cp.FAMILIES[f]: {k: counts[f][k] / counts[f]["boxes"] for k in ("add", "mul", "div", "asin")}
                            for f in FAMILIES}}


def cpu_baseline(seconds: float) -> dict:
    """The CPU oracle (all host threads) on a bounded sample of the workload:
    boxes drawn uniformly from the seed lattices of the families, in rounds of
    growing size until about `seconds` of CPU time have been spent."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    rng = np.random.default_rng(1)
    total_boxes, t_total, per_family, rounds = 0, 0.0, 4000, 0
    while t_total < seconds:
        for f in FAMILIES:
            dims = DIMS[f]
            total = SEED_RES ** dims
            idx = np.sort(rng.choice(total, size=min(per_family, total), replace=False))
            lo, hi = O.lattice_boxes(f, (0.5, 0.9900000000000001), [SEED_RES] * dims, idx)
            t0 = time.perf_counter()
            O.eval_boxes(f, lo, hi, threads=threads)
            t_total += time.perf_counter() - t0
            total_boxes += idx.size
        rounds += 1
        if t_total < seconds / 3:
            per_family = min(per_family * 4, 4_000_000)
    return {"value": total_boxes / t_total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{total_boxes} boxes drawn from the 64^dims seed lattices of the families "
                      f"({', '.join(str(f) for f in FAMILIES)}) in {rounds} rounds, CPU restatement "
                      f"(oracle/cpu_oracle.cpp), {threads} threads, {t_total:.1f} s of evaluation"}


def main_reference(args, world, rank):
    if rank != 0:
        return
    res = []
    for _ in range(args.warmup):
        cpu_baseline(min(2.0, args.cpu_seconds))
    for _ in range(args.steps):
        res.append(cpu_baseline(args.cpu_seconds / max(args.steps, 1)))
    v = float(np.mean([r["value"] for r in res]))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "64^dims lattice seed boxes of the six lane-packing families (sampled)",
                       "parallelism": "host threads"},
            "cpu_baseline": {**res[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    global FAMILIES, SEED_RES, LEVEL_CAP
    FAMILIES = [int(x) for x in args.families.split(",")]
    SEED_RES, LEVEL_CAP = args.seed_res, args.level_capacity
    world, rank, local = dist_init()
    if args.impl == "reference":
        main_reference(args, world, rank)
        return
    import torch

    import circlepacking_b200 as cp

    torch.cuda.set_device(local)
    prover = cp.Prover(local)
    stream = prover.stream
    FP64, PRE = cp.FP64, cp.FP32_PREFILTER

    # ---- autotune (outside the timed region): kernel variant and precision per family
    if args.no_autotune:
        chosen = {f: FP64 for f in FAMILIES}
        tuning = {cp.FAMILIES[f]: {"precision": "fp64", "variant": 0} for f in FAMILIES}
    else:
        chosen, tuning = autotune(prover, cp)

    def use_plain(on):
        # the plain arm: FP64 with the untuned default kernel variant
        for f in FAMILIES:
            if on:
                prover.set_level_variant(f, FP64, 0)
            elif tuning[cp.FAMILIES[f]]["precision"] == "fp64":
                prover.set_level_variant(f, FP64, tuning[cp.FAMILIES[f]]["variant"])

    # ---- warm-up (also the verdict-identity check between the two forms)
    for _ in range(max(args.warmup, 3)):
        best = run_step(prover, chosen, args.depth)
    use_plain(True)
    plain = run_step(prover, FP64, args.depth)
    use_plain(False)
    identical = all(b["verdicts"] == p["verdicts"] and b["unresolved"] == p["unresolved"] for b, p in zip(best, plain))

    # ---- timed: best form, K steps on the prover's stream
    def timed(precision):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = []
        for _ in range(args.steps):
            reps = run_step(prover, precision, args.depth)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1) / args.steps
        return max_over_ranks(world, ms), reps

    with ClockSampler(local) as clk:
        ms_best, reps_best = timed(chosen)
    use_plain(True)
    ms_plain, reps_plain = timed(FP64)
    use_plain(False)
    boxes_step = sum(r["evaluated"] for r in reps_best)
    value = sum_over_ranks(world, boxes_step) / (ms_best / 1e3)
    plain_value = sum_over_ranks(world, sum(r["evaluated"] for r in reps_plain)) / (ms_plain / 1e3)
    launches_step = sum(r["launches"] + 2 for r in reps_best)  # level kernels + slab-bound + seed kernels

    # ---- e2e: the host-buffer C-ABI call (seed boxes from pinned host memory)
    e2e = None
    if not args.no_e2e:
        seeds = {f: seed_boxes_host(f) for f in FAMILIES}
        h2d = sum(int(seeds[f][0].numel() * 8 * 2 + seeds[f][2].numel()) for f in FAMILIES)
        d2h = len(FAMILIES) * __import__("ctypes").sizeof(cp.RefineReport)

        def e2e_step():
            tot = 0
            for f in FAMILIES:
                lo, hi, dp = seeds[f]
                r = prover.refine_boxes(f, lo.numpy(), hi.numpy(), depth=dp.numpy(),
                                        **{k: v for k, v in seed_opts(f, chosen[f], args.depth).items()
                                           if k not in ("seed_sizes", "seed_lambda")})
                tot += r["evaluated"]
            return tot

        e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        tot = 0
        for _ in range(args.steps):
            tot += e2e_step()
        torch.cuda.synchronize()
        dt = max_over_ranks(world, (time.perf_counter() - t0) / args.steps)
        e2e = {"value": sum_over_ranks(world, tot / args.steps) / dt, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3,
               "call": "cp_refine_boxes_host per family (host seed boxes, report back)"}

    # ---- roofline of the FP64 criterion kernel (plain run)
    roofline = None if args.no_roofline else roofline_of(cp, local, reps_plain)
    cpu = cpu_baseline(args.cpu_seconds) if (rank == 0 and not args.no_cpu) else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_best, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"config-2 box set: 64^dims lattice seed per family over lambda [0.5,0.99], "
                               f"not-proved boxes bisected on all axes, {args.depth} levels, six families",
                   "precision": "per family, autotuned: fp64 or fp32 enclosure pre-pass + fp64 (identical verdicts)",
                   "autotune": tuning, "boxes_per_step": boxes_step,
                   "l2": "worklists of several GB per level (inputs > L2)", "parallelism": f"replicas x{world}"},
        "plain_fp64": {"value": plain_value, "ms_per_step": ms_plain},
        "verdicts_identical": identical,
        "fp32_decided_fraction": sum(r["fp32_decided"] for r in reps_best) / max(1, boxes_step),
        "per_family": [{"family": cp.FAMILIES[f], "evaluated": r["evaluated"], "verdicts": r["verdicts"],
                        "unresolved": r["unresolved"], "fp32_decided": r["fp32_decided"]}
                       for f, r in zip(FAMILIES, reps_best)],
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
        "gpu_launches": launches_step * args.steps,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    prover.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
