"""TEST INFRASTRUCTURE ONLY -- times the reference's own family kernels.

The reference's lambda loop (run_kernel.cuh:61-132) driven over the unmodified
reference kernels (lane_packing/*_configuration.cu, compiled from the reference
sources into oracle/_ref/libcp_refcheck.so by `make -C oracle ref`), one
launch per step through refc_kernel_once (the launch run_kernel.cuh:81-84
issues: same grid, block and Atomic_ordered_double protocol), under a wall-time
budget.  The same number of steps is then run by this library's
cp_prove_family_reference (same loop, this library's lattice kernel), and the
two traces of (lambda interval, first failing lambda) are compared step by step.

    python oracle/time_reference_kernels.py [--families 3,5] [--budget 300]

Prints one JSON object per family.  Not part of the product: the product never
imports or runs anything under oracle/.
"""
from __future__ import annotations

import argparse
import heapq
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# run as a script, this file's own directory comes first on the path, where
# `oracle` would name oracle/oracle.py instead of the package
sys.path[:] = [ROOT] + [p for p in sys.path if os.path.abspath(p or ".") != os.path.dirname(os.path.abspath(__file__))]

LAMBDA = (0.5, 0.9900000000000001)  # values.hpp:31-32
DBL_MAX = np.finfo(np.float64).max


def reference_loop(refcheck, family: int, budget_s: float):
    """run_kernel_until_no_criticals (run_kernel.cuh:61-132) over the reference
    kernel of `family`, stopped after `budget_s` seconds of wall time."""
    q = [LAMBDA]
    trace, dev_ms = [], 0.0
    t0 = time.perf_counter()
    finished = False
    while True:
        if not q:
            finished = True
            break
        if time.perf_counter() - t0 > budget_s:
            break
        lb, ub = heapq.heappop(q)
        first, ms = refcheck.kernel_once(family, lb, ub)
        dev_ms += ms
        trace.append((lb, ub, first))
        if first != DBL_MAX:
            width_before = ub - lb
            width_after = ub - first
            if width_before >= 2 * width_after:
                heapq.heappush(q, (first, ub))
            else:
                mid = 0.5 * (first + ub)
                if first < mid:
                    heapq.heappush(q, (first, mid))
                if mid <= ub:
                    heapq.heappush(q, (mid, ub))
    return dict(finished=finished, launches=len(trace), device_ms=dev_ms, wall_s=time.perf_counter() - t0,
                trace=trace, remaining=(q[0] if q else None))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--families", default="3,5")
    ap.add_argument("--budget", type=float, default=300.0, help="wall seconds per family for the reference kernels")
    args = ap.parse_args()

    import circlepacking_b200 as cp
    from oracle import refcheck

    prover = cp.Prover(0)
    for f in [int(x) for x in args.families.split(",")]:
        ref = reference_loop(refcheck, f, args.budget)
        n = ref["launches"]
        t0 = time.perf_counter()
        ours = prover.prove_family_reference(f, max_launches=n, trace_cap=n)
        wall_ours = time.perf_counter() - t0
        tr_ref = np.array(ref["trace"], dtype=np.float64).reshape(-1, 3)
        tr_ours = np.asarray(ours["trace"], dtype=np.float64).reshape(-1, 3)
        # the reference returns DBL_MAX where no box fails; this library +inf
        tr_ours_cmp = np.where(np.isinf(tr_ours), DBL_MAX, tr_ours)
        same = tr_ref.shape == tr_ours_cmp.shape and bool((tr_ref == tr_ours_cmp).all())
        top = float(tr_ref[:, 2][tr_ref[:, 2] != DBL_MAX].max()) if n and (tr_ref[:, 2] != DBL_MAX).any() else None
        out = {
            "family": cp.FAMILIES[f], "lattice": list(cp.REFERENCE_SIZES[f][:cp.DIMS[f]]),
            "budget_s": args.budget,
            "reference_kernels": {"finished": ref["finished"], "launches": n, "device_ms": ref["device_ms"],
                                  "wall_s": ref["wall_s"], "ms_per_launch": ref["device_ms"] / max(n, 1),
                                  "remaining_first_interval": ref["remaining"], "highest_first_lambda": top},
            "library_kernel_same_launches": {"status": ours["status"], "launches": ours["launches"],
                                             "device_ms": ours["device_ms"], "wall_s": wall_ours,
                                             "ms_per_launch": ours["device_ms"] / max(ours["launches"], 1)},
            "traces_identical": same,
            "device_time_ratio": ref["device_ms"] / max(ours["device_ms"], 1e-9),
        }
        print(json.dumps(out), flush=True)
    prover.close()


if __name__ == "__main__":
    main()
