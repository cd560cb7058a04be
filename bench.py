"""Benchmark of the lane-packing subinterval search on B200.

One step = the box refinement of all six families from a uniform lattice seed
(64 subdivisions per axis over lambda in [0.5, 0.99], the reference's dependent
radius ranges), not-proved boxes bisected on every axis (16 children for the
3-disk families, 8 for the 2-disk ones) down to a bounded depth.  `value` is the
box throughput of the best form, picked per family outside the timed region
(graph engine or host-driven level loop, kernel shape, FP64 or FP32 pre-pass,
learned criterion order when faster); the plain FP64 form runs on the same
boxes, and both must give the same per-box verdict digest (every evaluated box
and its verdict, hashed on the device).

Beside the headline the line carries: the uneven-depth worklist (64^4 lattice
plus 10M seeded random boxes at depths 0-8), the FP32 pre-pass form of the
whole step, the learned criterion order and learned split on the uneven-depth
worklist, the full-domain proofs of the families lambda-only refinement closes
(one or two of them also by the reference's own lambda loop), the roofline of
the level kernel on the reference kernel's own operation counts, and the CPU
restatement on the host cores.

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
SHARD = (0.5, 0.9900000000000001)  # lambda range of the seeds (the whole domain)
PART, PARTS = 0, 1  # this rank's interleaved piece of every lattice seed (strong scaling over ranks)


_T0 = time.perf_counter()


def log(msg: str):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}\n")
    sys.stderr.flush()


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
    ap.add_argument("--no-autotune", action="store_true", help="default kernel shapes, FP64 (profiling runs)")
    ap.add_argument("--no-learned", action="store_true", help="no proposal networks (reference criterion order)")
    ap.add_argument("--no-proof", action="store_true", help="skip the full-domain proof leg")
    ap.add_argument("--reference-proof", default="3,5",
                    help="families (comma list, '' = none) whose full-domain proof also runs by the reference's own "
                         "method: its lambda loop over its lattice sizes, on this library's FP64 lattice kernel")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-depth worklist legs")
    ap.add_argument("--uneven-family", type=int, default=3, help="family of the uneven-depth worklist legs")
    ap.add_argument("--uneven-random", type=int, default=10_000_000, help="random boxes added to the lattice seed")
    ap.add_argument("--no-fp32-leg", action="store_true", help="skip the FP32 pre-pass form of the whole step")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="with --no-autotune: the precision of the graph-engine form (profiling runs)")
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
def seed_opts(family, form, depth, digest=False):
    """Refinement options of one family in a form: {"precision", "engine", "learned_order"}."""
    import circlepacking_b200 as cp

    return dict(precision=form["precision"], policy=cp.SPLIT_UNIFORM, max_depth=depth,
                seed_sizes=[SEED_RES] * DIMS[family], seed_lambda=SHARD,
                level_capacity=LEVEL_CAP, engine=form["engine"], learned_order=form.get("learned_order", False),
                digest=digest, seed_part=PART, seed_parts=PARTS)


def run_step(prover, forms, depth, digest=False):
    """One step: the refinement of every family in its form."""
    return [prover.refine(f, **seed_opts(f, forms[f], depth, digest)) for f in FAMILIES]


def same_boxes_and_verdicts(a, b):
    """Two reports of refinements that must have evaluated the same boxes with
    the same verdicts: equal per-box digests (and counts)."""
    return (a["digest"] == b["digest"] and a["digest"] != (0, 0) and a["verdicts"] == b["verdicts"]
            and a["unresolved"] == b["unresolved"] and a["per_depth"] == b["per_depth"])


def autotune(prover, cp, learned: bool):
    """Per family, outside the timed region: the fastest form on a calibration
    refinement (32^dims seed, one level) among the device-driven graph engine
    (block size x boxes per thread) and the host-driven level loop (register
    variants), each in FP64 and with the FP32 pre-pass, then (with `learned`)
    whether the trained network's criterion order is faster still.  Every
    candidate gives identical verdicts, so the choice is speed only."""
    forms, table = {}, {}
    for f in FAMILIES:
        calib = dict(policy=cp.SPLIT_UNIFORM, max_depth=1, seed_sizes=[32] * DIMS[f])
        cands = []
        for prec in (cp.FP64, cp.FP32_PREFILTER):
            blk, bpt, ms = prover.autotune_graph(f, precision=prec, **calib)
            cands.append((min(min(r) for r in ms), prec, cp.ENGINE_GRAPH, {"block": blk, "boxes_per_thread": bpt}))
            v, ms = prover.autotune(f, precision=prec, **calib)
            cands.append((min(ms), prec, cp.ENGINE_LEVELS, {"variant": v}))
            prover.set_level_variant(f, prec, v)
        ms, prec, eng, shape = min(cands, key=lambda c: c[0])
        form = {"precision": prec, "engine": eng, "learned_order": False}
        entry = {"precision": "fp64" if prec == cp.FP64 else "fp32-prefilter",
                 "engine": "graph" if eng == cp.ENGINE_GRAPH else "levels", **shape, "calib_ms": ms,
                 "candidates_ms": {f"{'fp64' if c[1] == cp.FP64 else 'fp32'}-{'graph' if c[2] else 'levels'}": c[0]
                                   for c in cands}}
        if learned and cp.N_CRITERIA[f] > 1:
            kw = dict(calib, precision=prec, engine=eng)
            base = min(prover.refine(f, **kw)["device_ms"] for _ in range(3))
            lrn = min(prover.refine(f, learned_order=True, **kw)["device_ms"] for _ in range(3))
            entry["calib_ms_learned_order"] = lrn
            entry["calib_ms_reference_order"] = base
            if lrn < base:
                form["learned_order"] = True
        entry["learned_order"] = form["learned_order"]
        forms[f], table[cp.FAMILIES[f]] = form, entry
    return forms, table


def train_models(prover, cp, depth):
    """The proposal network of every family with more than one criterion, trained
    on the GPU on records of its own refinement (outside the timed region)."""
    out = {}
    for f in FAMILIES:
        if cp.N_CRITERIA[f] < 2:
            continue
        t0 = time.perf_counter()
        n = prover.model_collect(f, 1 << 21, sample_stride=8, policy=cp.SPLIT_UNIFORM, max_depth=depth,
                                 seed_sizes=[32] * DIMS[f], level_capacity=LEVEL_CAP)
        losses = prover.model_train(f, epochs=20, batch=4096, lr=1e-3, seed=1)
        out[cp.FAMILIES[f]] = {"records": n, "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                               "seconds": time.perf_counter() - t0}
    return out


# DRAM traffic of the graph refinement per evaluated box, from one ncu capture
# (middle family, 32^4 seed, one level: 11.95M boxes evaluated, 10.9M children
# written, 1.118 GB read + 1.208 GB written); algorithmic: 65 B read per 4-D box
# and 65 B written per child.  FP64 pipe activity of the same capture.
TRAFFIC_PER_BOX, ALGORITHMIC_BYTES_PER_BOX = 2.326e9 / 11.95e6, 124.0
FP64_PIPE_ACTIVE_NCU = 0.239

PROOF_FAMILIES = (0, 1, 2, 3, 4, 5)


def proof_leg(prover, cp, forms, families, world=1):
    """Full-domain proofs by the library's proof driver (cp_prove_family with
    cp_proof_defaults): each family's whole domain (lambda in [0.5, 0.99], the
    dependent radius ranges) from lattice seeds with the radius resolution the
    family needs -- for start, lambda slabs narrowing geometrically toward 0.99,
    each seeded with the reference's own radius lattice -- not-proved boxes
    bisected in lambda only (the reference's own refinement rule,
    run_kernel.cuh:110-127).  A family is proved when no box is left
    unresolved.  The best form runs every slab as one graph launch, the plain
    form as the FP64 host-driven level loop; both evaluate the same tree, which
    the per-box verdict digests confirm."""
    out = []
    for f in families:
        prover.set_level_variant(f, cp.FP64, 0)
        # each rank refines its interleaved piece of every slab's lattice
        best_kw = dict(engine=cp.ENGINE_GRAPH, precision=forms[f]["precision"], digest=1, seed_parts=PARTS,
                       seed_part=PART)
        plain_kw = dict(best_kw, engine=cp.ENGINE_LEVELS, precision=cp.FP64, reuse=0)
        # warm-up (graph build): one slab of a 4^dims seed as given, no per-slab scaling
        prover.prove_family(f, **dict(best_kw, slabs=1, seed_sizes=[4, 4, 4, 4], slab_radii=[]))
        b = prover.prove_family(f, **best_kw)
        p = prover.prove_family(f, **plain_kw)
        same = (b["digest"] == p["digest"] and b["verdicts"] == p["verdicts"] and b["per_depth"] == p["per_depth"]
                and b["unresolved"] == p["unresolved"])
        unresolved = sum_over_ranks(world, b["unresolved"] + p["unresolved"])
        d = prover.proof_defaults(f)
        out.append({"family": cp.FAMILIES[f], "proved": unresolved == 0,
                    "seeds": {"slabs": d["slabs"], "geometric": bool(d["geometric"]),
                              "lattice_per_slab": d["seed_sizes"][:DIMS[f]], "max_depth": d["max_depth"]},
                    "boxes": int(sum_over_ranks(world, b["evaluated"])), "max_depth": b["max_depth_seen"],
                    "best_wall_ms": max_over_ranks(world, b["wall_ms"]),
                    "best_device_ms": max_over_ranks(world, b["device_ms"]),
                    "plain_wall_ms": max_over_ranks(world, p["wall_ms"]),
                    "plain_device_ms": max_over_ranks(world, p["device_ms"]),
                    "verdicts_identical": sum_over_ranks(world, 0 if same else 1) == 0})
    return out


def seed_boxes_host(family):
    """The 64^dims lattice seed of a family in pinned host memory (numpy view)."""
    import torch

    import circlepacking_b200 as cp

    total = SEED_RES ** DIMS[family]
    idx = torch.from_numpy(cp.seed_partition(total, PART, PARTS)).cuda()  # this rank's piece of the seed
    lo, hi, vis = cp.lattice_boxes(family, SHARD, [SEED_RES] * DIMS[family], idx, visited=True)
    hlo = torch.empty(lo.shape, dtype=torch.float64, pin_memory=True)
    hhi = torch.empty(hi.shape, dtype=torch.float64, pin_memory=True)
    hdp = torch.empty(vis.shape, dtype=torch.uint8, pin_memory=True)
    hlo.copy_(lo)
    hhi.copy_(hi)
    hdp.copy_(torch.where(vis != 0, 0, 255).to(torch.uint8))  # 255: boxes the lattice never visits
    return hlo, hhi, hdp


def roofline_of(cp, device, reps, counts) -> dict:
    """Roofline of the FP64 criterion evaluation (the level kernel): the
    reference kernel's own primitive operations per evaluated box (add/sub,
    mul, div, asin, each counting one), weighted by the step's boxes per depth,
    per second of the step's device time, against the measured FP64 instruction
    peak (one DFMA per lane and cycle).  Two weighted readings stand beside it:
    each primitive weighted by DFMA rate / its own measured rate, once with the
    reference's __ddiv_rd and once with this library's division."""
    rates = cp.measure_primitives(device)
    ops = {"add": 0.0, "mul": 0.0, "div": 0.0, "asin": 0.0}
    boxes = 0
    for f, r in zip(FAMILIES, reps):
        per = counts[f]
        depths = sorted(per)
        for d, n in enumerate(r["per_depth"]):
            if not n:
                continue
            use = per[d] if d in per else per[min(depths, key=lambda x: abs(x - d))]
            for k in ops:
                ops[k] += n * use[k]
            boxes += n
    kernel_s = sum(r["device_ms"] for r in reps) / 1e3
    unweighted = sum(ops.values())
    peak = rates["dfma"]

    def weighted(div_rate):
        return (ops["add"] * peak / rates["dadd_rd"] + ops["mul"] * peak / rates["dmul_rd"]
                + ops["div"] * peak / div_rate + ops["asin"] * peak / rates["asin"])

    achieved = unweighted / kernel_s
    return {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": TRAFFIC_PER_BOX * boxes,
            "traffic_note": f"DRAM bytes per step: {TRAFFIC_PER_BOX:.0f} B per evaluated box from one ncu capture of "
                            f"the graph refinement (algorithmic {ALGORITHMIC_BYTES_PER_BOX:.0f} B), scaled by the "
                            f"step's {boxes} evaluated boxes",
            "kernel": "k_level_persist<family, precision, block> (per-box criteria + split), graph engine",
            "work_model": "per evaluated box: the reference kernel's own add/sub, mul, div and asin count (it stops "
                          "at the first failing sub-check and handle), counted by the CPU restatement while it refines "
                          "sampled seeds of the same workload, per family and depth, weighted by the step's boxes per "
                          "depth; each primitive counts 1 against the FP64 instruction peak (DFMA per lane per cycle)",
            "ops_per_second": {k: v / kernel_s / 1e12 for k, v in ops.items()} | {"unit": "T/s"},
            "frac_weighted_ddiv_rd": weighted(rates["ddiv_rd"]) / kernel_s / peak,
            "frac_weighted_library_div": weighted(rates["div_rd_lib"]) / kernel_s / peak,
            "fp64_pipe_active_ncu": FP64_PIPE_ACTIVE_NCU,
            "peaks_measured_tops": {k: v / 1e12 for k, v in rates.items()},
            "peak_source": "measured in-process (MEASURED_PEAKS.json has no FP64 figure): DFMA instruction rate",
            "ops_per_box": {cp.FAMILIES[f]: {str(d): v for d, v in counts[f].items()} for f in FAMILIES}}


def cpu_baseline(seconds: float, depth: int):
    """The CPU restatement (oracle/cpu_oracle.cpp, all host threads) on a bounded
    sample of the same workload: the uniform refinement below randomly drawn
    boxes of each family's 64^dims seed lattice down to `depth` levels, every
    box on the reference kernel's own evaluation path, in rounds of growing size
    until about `seconds` of CPU time have been spent.  Returns the baseline and
    the primitive operations per evaluated box, per family and depth (the
    roofline's work model)."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    rng = np.random.default_rng(1)
    boxes, t_total, rounds, seeds = 0, 0.0, 0, 16
    ops = {f: np.zeros((16, 4), np.float64) for f in FAMILIES}
    per_depth = {f: np.zeros(16, np.float64) for f in FAMILIES}
    n_seeds = 0
    while t_total < seconds:
        for f in FAMILIES:
            total = SEED_RES ** DIMS[f]
            idx = np.sort(rng.choice(total, size=min(seeds, total), replace=False))
            t0 = time.perf_counter()
            r = O.refine_sample(f, [SEED_RES] * DIMS[f], idx, depth, outer=SHARD, threads=threads)
            t_total += time.perf_counter() - t0
            boxes += r["evaluated"]
            n_seeds += idx.size
            ops[f] += r["ops"]
            per_depth[f] += np.asarray(r["per_depth"], np.float64)
        rounds += 1
        if t_total < seconds / 3:
            seeds = min(seeds * 4, 1 << 16)
    counts = {}
    for f in FAMILIES:
        counts[f] = {d: dict(zip(("add", "mul", "div", "asin"), (ops[f][d] / per_depth[f][d]).tolist()),
                             boxes=int(per_depth[f][d])) for d in range(16) if per_depth[f][d] > 0}
    base = {"value": boxes / t_total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n_seeds} seed boxes drawn from the 64^dims lattices of the families "
                      f"({', '.join(str(f) for f in FAMILIES)}), each refined with the uniform split to depth "
                      f"{depth} ({boxes} boxes evaluated on the reference kernel's path), CPU restatement "
                      f"(oracle/cpu_oracle.cpp), {threads} threads, {t_total:.1f} s, {rounds} rounds"}
    return base, counts


def uneven_seeds(prover, cp, family, n_random):
    """The uneven-depth worklist: the family's 64^dims lattice seed (depth 0)
    followed by n_random seeded random boxes (seed 0xC1C1E5, log-uniform widths
    2^-20..2^-4, depth labels 0..8), as device tensors."""
    import torch

    dims = DIMS[family]
    total = SEED_RES ** dims
    lo, hi, vis = cp.lattice_boxes(family, SHARD, [SEED_RES] * dims, torch.arange(total, device="cuda"),
                                   visited=True)
    rlo, rhi, rdp = prover.random_boxes(family, n_random, seed=0xC1C1E5, max_label=8)
    dp = torch.where(vis != 0, 0, 255).to(torch.uint8)
    return (torch.cat([lo, rlo], 1).contiguous(), torch.cat([hi, rhi], 1).contiguous(),
            torch.cat([dp, rdp]).contiguous())


def uneven_legs(prover, cp, forms, args, models_ready):
    """Uneven-depth worklist of one family, seeded with its 64^dims lattice plus
    10M random boxes at depths 0..8, refined with the uniform split down to the
    step's depth: every box is evaluated once; boxes above the depth limit that
    are not proved get their children evaluated too.  Forms: the best form
    (graph engine: one persistent kernel over the whole worklist, autotuned
    shape, the family's precision), the plain FP64 level loop, the best form with
    the learned criterion order, and the learned split axis (another tree).
    Each form's verdicts are compared box by box with the plain form's digest."""
    import torch

    f = args.uneven_family
    lo, hi, dp = uneven_seeds(prover, cp, f, args.uneven_random)
    cap = max(LEVEL_CAP, lo.shape[1])
    base = dict(policy=cp.SPLIT_UNIFORM, max_depth=args.depth, level_capacity=cap)
    best_kw = dict(base, precision=forms[f]["precision"], engine=cp.ENGINE_GRAPH)
    plain_kw = dict(base, precision=cp.FP64, engine=cp.ENGINE_LEVELS)

    def timed(kw, reps=2):
        prover.refine_boxes(f, lo, hi, depth=dp, **kw)  # warm-up (graph build)
        best = None
        for _ in range(reps):
            r = prover.refine_boxes(f, lo, hi, depth=dp, **kw)
            best = r if best is None or r["device_ms"] < best["device_ms"] else best
        return best

    def entry(r, ref=None):
        e = {"evaluated": r["evaluated"], "boxes_per_s": r["evaluated"] / (r["device_ms"] / 1e3),
             "device_ms": r["device_ms"], "unresolved": r["unresolved"], "per_depth": r["per_depth"],
             "criteria_per_box": r["handles_evaluated"] / max(1, r["evaluated"]),
             "fp32_decided_fraction": r["fp32_decided"] / max(1, r["evaluated"])}
        if ref is not None:
            e["verdicts_identical"] = same_boxes_and_verdicts(r, ref)
        return e

    prover.set_level_variant(f, cp.FP64, 0)
    plain = timed(plain_kw)
    plain_dig = prover.refine_boxes(f, lo, hi, depth=dp, digest=True, **plain_kw)
    best = timed(best_kw)
    best_dig = prover.refine_boxes(f, lo, hi, depth=dp, digest=True, **best_kw)
    out = {"family": cp.FAMILIES[f], "seeds": int(lo.shape[1]),
           "seed_depths": np.bincount(dp.cpu().numpy(), minlength=256)[:9].tolist(),
           "dropped_random_boxes": int((dp == 255).sum().item()),
           "workload": f"64^dims lattice seed + {args.uneven_random} random boxes (seed 0xC1C1E5, widths 2^-20..2^-4 "
                       f"log-uniform, depth labels 0..8), uniform split to depth {args.depth}",
           "plain_fp64": entry(plain), "best": dict(entry(best, plain_dig), form=
                                                      {"engine": "graph", "precision": "fp64" if
                                                       forms[f]["precision"] == cp.FP64 else "fp32-prefilter"})}
    out["best"]["verdicts_identical"] = same_boxes_and_verdicts(best_dig, plain_dig)
    out["best"]["speedup_vs_plain"] = plain["device_ms"] / best["device_ms"]
    if models_ready and cp.N_CRITERIA[f] > 1:
        lrn = timed(dict(best_kw, learned_order=True))
        lrn_dig = prover.refine_boxes(f, lo, hi, depth=dp, digest=True, learned_order=True, **best_kw)
        e = entry(lrn)
        e["verdicts_identical"] = same_boxes_and_verdicts(lrn_dig, plain_dig)
        e["time_vs_best"] = lrn["device_ms"] / best["device_ms"]
        e["time_vs_plain"] = lrn["device_ms"] / plain["device_ms"]
        out["learned_order"] = e
        split = timed(dict(best_kw, policy=cp.SPLIT_LEARNED), reps=1)
        e = entry(split)
        e["note"] = "learned split axis: another tree of boxes (per-box verdicts are the FP64 kernel's own)"
        out["learned_split"] = e
    prover.set_level_variant(f, cp.FP64, forms[f].get("variant", 1))
    del lo, hi, dp
    torch.cuda.empty_cache()
    return out


def fp32_leg(prover, cp, args, plain_digests):
    """The FP32 pre-pass form of the whole step (every family, graph engine):
    time, the fraction of boxes the FP32 pass decides, and per-box verdict
    identity with the plain FP64 form."""
    forms = {f: {"precision": cp.FP32_PREFILTER, "engine": cp.ENGINE_GRAPH} for f in FAMILIES}
    run_step(prover, forms, args.depth)  # warm-up
    reps = run_step(prover, forms, args.depth)
    digs = run_step(prover, forms, args.depth, digest=True)
    boxes = sum(r["evaluated"] for r in reps)
    ms = sum(r["device_ms"] for r in reps)
    return {"boxes_per_s": boxes / (ms / 1e3), "device_ms": ms,
            "fp32_decided_fraction": sum(r["fp32_decided"] for r in reps) / max(1, boxes),
            "per_family_fp32_decided": {cp.FAMILIES[f]: r["fp32_decided"] / max(1, r["evaluated"])
                                        for f, r in zip(FAMILIES, reps)},
            "per_family_device_ms": {cp.FAMILIES[f]: r["device_ms"] for f, r in zip(FAMILIES, reps)},
            "verdicts_identical": all(same_boxes_and_verdicts(d, p) for d, p in zip(digs, plain_digests))}


def main_reference(args, world, rank):
    if rank != 0:
        return
    res = []
    for _ in range(args.warmup):
        cpu_baseline(min(2.0, args.cpu_seconds), args.depth)
    for _ in range(args.steps):
        res.append(cpu_baseline(args.cpu_seconds / max(args.steps, 1), args.depth)[0])
    v = float(np.mean([r["value"] for r in res]))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"uniform-bisection box set: 64^dims lattice seed per family over lambda "
                                   f"[0.5,0.99], not-proved boxes bisected on all axes, {args.depth} levels, six "
                                   f"families (sampled seeds, CPU)",
                       "parallelism": "host threads"},
            "cpu_baseline": {**res[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    global FAMILIES, SEED_RES, LEVEL_CAP, PART, PARTS
    FAMILIES = [int(x) for x in args.families.split(",")]
    SEED_RES, LEVEL_CAP = args.seed_res, args.level_capacity
    world, rank, local = dist_init()
    if args.impl == "reference":
        main_reference(args, world, rank)
        return
    import torch

    import circlepacking_b200 as cp

    # strong scaling: every rank refines an interleaved piece of the same seeds
    # (lattice boxes rank, rank + world, ...); boxes are independent, so the
    # pieces need no data exchange and their counts and digests add up
    PART, PARTS = rank, world

    torch.cuda.set_device(local)
    prover = cp.Prover(local)
    stream = prover.stream
    FP64 = cp.FP64
    plain_forms = {f: {"precision": FP64, "engine": cp.ENGINE_LEVELS} for f in FAMILIES}

    # ---- outside the timed region: proposal networks, kernel shapes, precisions
    models = None
    if args.no_autotune:
        prec = FP64 if args.precision == "fp64" else cp.FP32_PREFILTER
        forms = {f: {"precision": prec, "engine": cp.ENGINE_GRAPH} for f in FAMILIES}
        tuning = {cp.FAMILIES[f]: {"precision": args.precision, "engine": "graph"} for f in FAMILIES}
    else:
        if not args.no_learned:
            models = train_models(prover, cp, args.depth)
        forms, tuning = autotune(prover, cp, learned=not args.no_learned)

    tuned_variant = {f: tuning[cp.FAMILIES[f]].get("variant", 1) for f in FAMILIES}

    def use_plain(on):
        # the plain arm: FP64, host-driven level loop, untuned kernel variant 0
        for f in FAMILIES:
            prover.set_level_variant(f, FP64, 0 if on else tuned_variant[f])

    log("autotuned: " + json.dumps({cp.FAMILIES[f]: {k: v for k, v in tuning[cp.FAMILIES[f]].items() if k != "candidates_ms"} for f in FAMILIES}))
    # ---- warm-up, then the per-box verdict identity of the two forms (one
    # step each with the device digest of every evaluated box and its verdict)
    for _ in range(max(args.warmup, 3)):
        run_step(prover, forms, args.depth)
    best_dig = run_step(prover, forms, args.depth, digest=True)
    use_plain(True)
    plain_dig = run_step(prover, plain_forms, args.depth, digest=True)
    use_plain(False)
    identical = all(same_boxes_and_verdicts(b, p) for b, p in zip(best_dig, plain_dig))

    log(f"warm-up done; verdicts identical: {identical}")
    # ---- timed: K steps on the prover's stream
    def timed(fm):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = []
        for _ in range(args.steps):
            reps = run_step(prover, fm, args.depth)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1) / args.steps
        return max_over_ranks(world, ms), reps

    with ClockSampler(local) as clk:
        ms_best, reps_best = timed(forms)
    use_plain(True)
    ms_plain, reps_plain = timed(plain_forms)
    use_plain(False)
    boxes_step = sum(r["evaluated"] for r in reps_best)
    value = sum_over_ranks(world, boxes_step) / (ms_best / 1e3)
    plain_value = sum_over_ranks(world, sum(r["evaluated"] for r in reps_plain)) / (ms_plain / 1e3)
    # kernels per step: the graph engine's chunk launches (+ scheduler, + inference
    # with a learned order), the seed and slab-bound kernels
    launches_step = sum(r["launches"] * ((3 if forms[f].get("learned_order") else 2)
                                         if forms[f]["engine"] == cp.ENGINE_GRAPH else
                                         (2 if forms[f].get("learned_order") else 1)) + 2
                        for f, r in zip(FAMILIES, reps_best))

    log(f"timed: best {ms_best:.1f} ms/step, plain {ms_plain:.1f} ms/step")
    # ---- e2e: the host-buffer C-ABI call (seed boxes from pinned host memory)
    e2e = None
    if not args.no_e2e:
        seeds = {f: seed_boxes_host(f) for f in FAMILIES}
        h2d = sum(int(seeds[f][0].numel() * 8 * 2 + seeds[f][2].numel()) for f in FAMILIES)
        d2h = len(FAMILIES) * __import__("ctypes").sizeof(cp.RefineReport)

        def stage(k, f):
            lo, hi, dp = seeds[f]
            prover.stage_boxes(k % 2, lo.numpy(), hi.numpy(), dp.numpy())

        def e2e_steps(steps):
            """`steps` steps of the host-buffer path: every family's seeds are copied
            from pinned host memory into a staging slot while the previous family
            refines (cp_stage_boxes_host / cp_refine_staged, two slots); each report
            comes back to the host."""
            jobs = [f for _ in range(steps) for f in FAMILIES]
            tot = 0
            stage(0, jobs[0])
            for k, f in enumerate(jobs):
                if k + 1 < len(jobs):
                    stage(k + 1, jobs[k + 1])
                r = prover.refine_staged(f, k % 2, **{kk: v for kk, v in seed_opts(f, forms[f], args.depth).items()
                                                      if kk not in ("seed_sizes", "seed_lambda")})
                tot += r["evaluated"]
            return tot

        e2e_steps(1)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        tot = e2e_steps(args.steps)
        torch.cuda.synchronize()
        dt = max_over_ranks(world, (time.perf_counter() - t0) / args.steps)
        e2e = {"value": sum_over_ranks(world, tot / args.steps) / dt, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": dt * 1e3,
               "call": "cp_stage_boxes_host + cp_refine_staged per family (host seed boxes copied while the "
                       "previous family refines, report back), best form"}

    log("e2e done")
    # ---- the FP32 pre-pass form of the whole step, and the uneven-depth worklist
    fp32 = None if args.no_fp32_leg else fp32_leg(prover, cp, args, plain_dig)
    uneven = None
    if not args.no_uneven and args.uneven_family in FAMILIES and world == 1:
        uneven = uneven_legs(prover, cp, forms, args, models_ready=models is not None)

    log("fp32 / uneven legs done")
    # ---- full-domain proofs of the families that lambda-only refinement closes
    proofs = None if args.no_proof else proof_leg(prover, cp, forms, [f for f in PROOF_FAMILIES if f in FAMILIES], world)
    if proofs is not None and args.reference_proof:
        # the same proofs by the reference's own method (run_kernel.cuh:61-132 with
        # the lattice sizes of its family kernels), timed on this GPU
        for f in [int(x) for x in args.reference_proof.split(",")]:
            if f not in FAMILIES or PARTS != 1:
                continue
            prover.set_level_variant(f, FP64, 0)
            t0 = time.perf_counter()
            ref = prover.prove_family_reference(f)
            t_ref = time.perf_counter() - t0
            for e in proofs:
                if e["family"] == cp.FAMILIES[f]:
                    e["reference_method_library_kernel"] = {
                        "method": "the reference's lambda loop (run_kernel.cuh:61-132) over its lattice sizes, each "
                                  "launch on this library's slab-ordered FP64 lattice kernel (not the reference's "
                                  "own kernels)",
                        "proved": ref["proved"], "wall_ms": t_ref * 1e3, "device_ms": ref["device_ms"],
                        "launches": ref["launches"], "boxes": ref["boxes_evaluated"],
                        "lattice": list(cp.REFERENCE_SIZES[f][:DIMS[f]])}
                    e["speedup_vs_reference_method_library_kernel"] = t_ref * 1e3 / e["best_wall_ms"]
    use_plain(False)

    log("proofs done")
    # ---- CPU leg (rank 0): the CPU restatement timed on the host cores, and its
    # op count of the reference kernel's path on device-recorded samples of the
    # step's boxes; then the roofline of the level kernel (best form)
    cpu, counts = None, None
    if rank == 0 and not args.no_cpu:
        cpu, counts = cpu_baseline(args.cpu_seconds, args.depth)
    roofline = roofline_of(cp, local, reps_best, counts) if (counts and not args.no_roofline) else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_best, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"uniform-bisection box set: 64^dims lattice seed per family over lambda [0.5,0.99], "
                               f"not-proved boxes bisected on all axes, {args.depth} levels, six families",
                   "form": "per family, autotuned: graph engine (block size x boxes per thread) or host-driven "
                           "level loop (register variant), fp64 or fp32 pre-pass + fp64, learned criterion order "
                           "when faster (identical verdicts)",
                   "autotune": tuning, "models": models, "boxes_per_step": boxes_step,
                   "l2": "worklists of several GB per level (inputs > L2)",
                   "parallelism": f"seed pieces x{world} (rank r refines lattice boxes r, r+{world}, ... of every "
                                  f"seed; counts and digests summed over ranks)"},
        "plain_fp64": {"value": plain_value, "ms_per_step": ms_plain,
                       "form": "fp64, host-driven level loop, kernel variant 0, reference criterion order"},
        "verdicts_identical": identical,
        "verdicts_identical_by": "device digest (sum and xor of a 64-bit hash of every evaluated box's bounds and "
                                 "verdict) equal between the best and plain forms, per family",
        "fp32_decided_fraction": sum(r["fp32_decided"] for r in reps_best) / max(1, boxes_step),
        "fp32_prepass_step": fp32,
        "uneven_depth_worklist": uneven,
        "criteria_per_box": {"best": sum(r["handles_evaluated"] for r in reps_best) / max(1, boxes_step),
                             "plain": sum(r["handles_evaluated"] for r in reps_plain) /
                             max(1, sum(r["evaluated"] for r in reps_plain))},
        "per_family": [{"family": cp.FAMILIES[f], "evaluated": r["evaluated"], "verdicts": r["verdicts"],
                        "unresolved": r["unresolved"], "fp32_decided": r["fp32_decided"], "device_ms": r["device_ms"],
                        "plain_device_ms": p["device_ms"], "digest": ["%016x" % x for x in d["digest"]]}
                       for f, r, p, d in zip(FAMILIES, reps_best, reps_plain, best_dig)],
        "full_domain_proofs": proofs,
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
