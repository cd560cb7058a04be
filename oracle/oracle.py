"""TEST INFRASTRUCTURE ONLY -- Python bindings of the CPU oracle.

``oracle/cpu_oracle.cpp`` restates the reference's lane-packing criteria on the
CPU (see its header).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU baseline / reference arm may import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libcp_oracle.so")

FAMILIES = ("start", "start_end_2d", "start_end_3d", "middle", "end_2d", "end_3d")
DIMS = (4, 3, 4, 4, 3, 4)
# sub-criteria per family (bits 0..K-1 of the mask)
N_CRITERIA = (2, 1, 1, 4, 2, 2)
PROVED, CRITICAL, NOFIT, EMPTY, ERROR = 0, 1, 2, 3, 4
M_FIT, M_TRAP = 0x40, 0x80

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle library (make -C oracle)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
        os.path.join(_HERE, "cpu_oracle.cpp")
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "_build/libcp_oracle.so"], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        P, I64, I32, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
        L.orc_eval_boxes.argtypes = [I32, P, P, I64, I64, P, P, P, I32]
        L.orc_count_ops.argtypes = [I32, P, P, I64, I64, P]
        L.orc_count_ops_mode.argtypes = [I32, P, P, I64, I64, I32, P]
        L.orc_refine_sample.argtypes = [I32, D, D, P, P, I64, I32, P, P, P, I32]
        L.orc_single_placement.argtypes = [D]
        L.orc_single_placement.restype = D
        L.orc_asin_pad.argtypes = [P, I64, P, P]
        L.orc_round_op.argtypes = [I32, I32, P, P, I64, P]
        L.orc_round_op_fenv.argtypes = [I32, I32, P, P, I64, P]
        L.orc_primitive.argtypes = [I32, P, I64, P, P]
        L.orc_lattice_boxes.argtypes = [I32, D, D, P, I32, P, I64, P, P, I64, I32]
        L.orc_eval_lattice.argtypes = [I32, D, D, P, I32, P, P, I32]
        L.orc_reference_loop.argtypes = [I32, P, I32, I64, P, P, I32]
        L.orc_reference_loop.restype = I64
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def eval_boxes(family: int, lo: np.ndarray, hi: np.ndarray, trace: bool = False, threads: int = 0):
    """Per-box verdict / fail mask (and optional (lhs, rhs) trace) of raw boxes.

    lo, hi: float64 arrays of shape (dims, n)."""
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    n = lo.shape[1]
    v = np.empty(n, np.uint8)
    m = np.empty(n, np.uint8)
    t = np.empty((n, 8, 2), np.float64) if trace else None
    rc = lib().orc_eval_boxes(family, _p(lo), _p(hi), n, n, _p(v), _p(m), _p(t) if trace else None, threads)
    if rc:
        raise ValueError("orc_eval_boxes failed")
    return (v, m, t) if trace else (v, m)


def count_ops(family: int, lo: np.ndarray, hi: np.ndarray, decide: bool = False) -> dict:
    """Primitive operations (add/sub, mul, div, asin) of evaluating boxes lo/hi:
    every sub-criterion (decide=False), or the reference kernel's own path, which
    stops at the first failing sub-check and handle (decide=True)."""
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    c = np.zeros(4, np.uint64)
    lib().orc_count_ops_mode(family, _p(lo), _p(hi), lo.shape[1], lo.shape[1], int(decide), _p(c))
    return dict(add=int(c[0]), mul=int(c[1]), div=int(c[2]), asin=int(c[3]), boxes=int(lo.shape[1]))


def refine_sample(family: int, sizes, idx, max_depth: int, outer=(0.5, 0.9900000000000001), threads: int = 0) -> dict:
    """The device engine's uniform refinement below the lattice seed boxes `idx`
    of the lattice `sizes` over `outer`, restated on the CPU on the reference
    kernel's own evaluation path: verdict counts, unresolved, clipped, boxes
    evaluated per depth and primitive operations (add, mul, div, asin) per depth."""
    s = np.zeros(4, np.int32)
    s[: len(sizes)] = sizes
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.zeros(7, np.int64)
    per_depth = np.zeros(16, np.int64)
    ops = np.zeros((16, 4), np.uint64)
    rc = lib().orc_refine_sample(family, float(outer[0]), float(outer[1]), _p(s), _p(idx), idx.size, max_depth,
                                 _p(out), _p(per_depth), _p(ops), threads)
    if rc:
        raise ValueError("orc_refine_sample: bad arguments")
    return dict(verdicts=out[:5].tolist(), unresolved=int(out[5]), clipped=int(out[6]),
                evaluated=int(out[:5].sum()), per_depth=per_depth.tolist(), ops=ops.astype(np.int64))


def single_placement(lb_lambda: float) -> float:
    return lib().orc_single_placement(float(lb_lambda))


def asin_pad(x: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float64)
    rd = np.empty_like(x)
    ru = np.empty_like(x)
    lib().orc_asin_pad(_p(x), x.size, _p(rd), _p(ru))
    return rd, ru


def round_op(op: int, up: bool, a: np.ndarray, b: np.ndarray, fenv: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty_like(a)
    f = lib().orc_round_op_fenv if fenv else lib().orc_round_op
    f(op, int(up), _p(a), _p(b), a.size, _p(out))
    return out


PRIM_INNER_INNER, PRIM_OUTER_INNER, PRIM_INNER_OUTER, PRIM_OUTER_OUTER, PRIM_SEMI_OUTER, PRIM_SEMI_INNER = range(6)
PRIM_NARGS = (3, 3, 3, 2, 1, 2)


def primitive(kind: int, args: np.ndarray):
    """args: float64 (2*nargs, n) rows = lb0, ub0, lb1, ub1, ...  Returns (lb, ub, trap)."""
    args = np.ascontiguousarray(args, dtype=np.float64)
    n = args.shape[1]
    full = np.zeros((6, n), np.float64)
    full[: args.shape[0]] = args
    out = np.empty((2, n), np.float64)
    trap = np.empty(n, np.uint8)
    lib().orc_primitive(kind, _p(full), n, _p(out), _p(trap))
    return out[0], out[1], trap


def lattice_boxes(family: int, outer, sizes, idx: np.ndarray, fused: bool = True, threads: int = 0):
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    dims = DIMS[family]
    s = np.zeros(4, np.int32)
    s[: len(sizes)] = sizes
    lo = np.empty((dims, idx.size), np.float64)
    hi = np.empty((dims, idx.size), np.float64)
    lib().orc_lattice_boxes(family, float(outer[0]), float(outer[1]), _p(s), int(fused), _p(idx), idx.size,
                            _p(lo), _p(hi), idx.size, threads)
    return lo, hi


def eval_lattice(family: int, outer, sizes, fused: bool = True, threads: int = 0):
    s = np.zeros(4, np.int32)
    s[: len(sizes)] = sizes
    hist = np.zeros(5, np.int64)
    fc = np.zeros(1, np.float64)
    lib().orc_eval_lattice(family, float(outer[0]), float(outer[1]), _p(s), int(fused), _p(hist), _p(fc), threads)
    return hist, float(fc[0])


def reference_loop(family: int, sizes, max_steps: int = 1000, fused: bool = True, threads: int = 0):
    s = np.zeros(4, np.int32)
    s[: len(sizes)] = sizes
    steps = np.zeros((max_steps, 3), np.float64)
    proved = np.zeros(1, np.int32)
    k = lib().orc_reference_loop(family, _p(s), int(fused), max_steps, _p(steps), _p(proved), threads)
    return steps[:k].copy(), bool(proved[0])
