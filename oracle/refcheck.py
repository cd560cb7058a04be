"""TEST INFRASTRUCTURE ONLY -- bindings of the reference-derived GPU checker.

``oracle/_ref/libcp_refcheck.so`` is the reference's own lane_packing device code
(compiled unchanged from the reference sources by ``make -C oracle ref``, with
an include shim that turns its device trap into a recorded flag).  It runs on a
GPU and is the bit-exact oracle for the FP64 path.  Only tests/ and
``__graft_entry__.smoke()`` use it, as the checker.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "_ref", "libcp_refcheck.so")
RC_EMPTY, RC_FIT, RC_TRAP = 0x20, 0x40, 0x80
_lib = None


def available() -> bool:
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(SO)
        P, I, D, L64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
        L.refc_eval_boxes.argtypes = [I, P, P, L64, P]
        L.refc_lattice_boxes.argtypes = [I, D, D, P, P, L64, P, P]
        L.refc_kernel_once.argtypes = [I, D, D, P, P]
        L.refc_primitive.argtypes = [I, P, L64, P, P]
        L.refc_single_placement.argtypes = [P, L64, P]
        L.refc_asin_pad.argtypes = [P, L64, P, P]
        L.refc_trap_count_reset.restype = ctypes.c_uint
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def eval_boxes(family: int, lo, hi) -> np.ndarray:
    """Per-box bits of the reference's own criteria: bit k = handle k failed,
    0x20 empty, 0x40 fit check fired, 0x80 trap site reached."""
    lo, hi = _c(lo, np.float64), _c(hi, np.float64)
    n = lo.shape[1]
    bits = np.empty(n, np.uint8)
    rc = lib().refc_eval_boxes(family, lo.ctypes.data, hi.ctypes.data, n, bits.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_eval_boxes failed ({rc})")
    return bits


def lattice_boxes(family: int, outer, sizes, idx):
    idx = _c(idx, np.int64)
    dims = 3 if family in (1, 4) else 4
    s = _c(list(sizes) + [1] * (4 - len(sizes)), np.int32)
    lo = np.empty((dims, idx.size), np.float64)
    hi = np.empty((dims, idx.size), np.float64)
    rc = lib().refc_lattice_boxes(family, float(outer[0]), float(outer[1]), s.ctypes.data, idx.ctypes.data, idx.size,
                                  lo.ctypes.data, hi.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_lattice_boxes failed ({rc})")
    return lo, hi


def kernel_once(family: int, la_lb: float, la_ub: float):
    first = np.zeros(1, np.float64)
    ms = np.zeros(1, np.float32)
    rc = lib().refc_kernel_once(family, la_lb, la_ub, first.ctypes.data, ms.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_kernel_once failed ({rc})")
    return float(first[0]), float(ms[0])


def primitive(kind: int, args):
    args = _c(args, np.float64)
    n = args.shape[1]
    full = np.zeros((6, n), np.float64)
    full[: args.shape[0]] = args
    out = np.empty((2, n), np.float64)
    trap = np.empty(n, np.uint8)
    rc = lib().refc_primitive(kind, full.ctypes.data, n, out.ctypes.data, trap.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_primitive failed ({rc})")
    return out[0], out[1], trap


def single_placement(lam):
    lam = _c(lam, np.float64)
    out = np.empty_like(lam)
    rc = lib().refc_single_placement(lam.ctypes.data, lam.size, out.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_single_placement failed ({rc})")
    return out


def asin_pad(x):
    x = _c(x, np.float64)
    rd = np.empty_like(x)
    ru = np.empty_like(x)
    rc = lib().refc_asin_pad(x.ctypes.data, x.size, rd.ctypes.data, ru.ctypes.data)
    if rc:
        raise RuntimeError(f"refc_asin_pad failed ({rc})")
    return rd, ru


def trap_count_reset() -> int:
    return int(lib().refc_trap_count_reset())
