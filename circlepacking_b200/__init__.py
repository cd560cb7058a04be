"""B200-native lane-packing prover (host-side mirror of the C ABI in include/cp_prover.h).

The compute path is the CUDA library ``circlepacking_b200/_lib/libcp_b200.so``
(built by ``python -m circlepacking_b200.build``).  This module only binds it with
ctypes and moves data with torch; there is no CPU fallback: every entry point
raises when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libcp_b200.so")

FAMILIES = ("start", "start_end_2d", "start_end_3d", "middle", "end_2d", "end_3d")
START, START_END_2D, START_END_3D, MIDDLE, END_2D, END_3D = range(6)
DIMS = (4, 3, 4, 4, 3, 4)
N_CRITERIA = (2, 1, 1, 4, 2, 2)
PROVED, CRITICAL, NOFIT, EMPTY, ERROR = range(5)
VERDICT_NAMES = ("proved", "critical", "nofit", "empty", "error")
MASK_FIT, MASK_TRAP = 0x40, 0x80
FP64, FP32_PREFILTER = 0, 1
EVAL_FULL, EVAL_DECIDE = 0, 1
LAMBDA_MIN, LAMBDA_MAX = 0.5, 0.9900000000000001

STATUS = {
    0: "CP_OK", 1: "CP_ERR_INVALID", 2: "CP_ERR_CUDA", 3: "CP_ERR_NOMEM", 4: "CP_ERR_CAPACITY",
    5: "CP_ERR_DEVICE", 6: "CP_ERR_TRAP_SITE", 7: "CP_ERR_NOFIT", 8: "CP_ERR_INTERRUPTED",
    9: "CP_ERR_NOT_PROVED", 10: "CP_ERR_NO_DEVICE",
}


class ProverError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        detail = ""
        if _lib is not None:
            detail = _lib.cp_last_error_string().decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(status, status)} {detail}".strip())


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m circlepacking_b200.build` "
                "(the prover has no CPU fallback)"
            )
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    P, I, D, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    L.cp_family_dims.argtypes = [I]
    L.cp_family_criteria.argtypes = [I]
    L.cp_status_string.argtypes = [I]
    L.cp_status_string.restype = ctypes.c_char_p
    L.cp_last_error_string.restype = ctypes.c_char_p
    L.cp_version.restype = ctypes.c_char_p
    L.cp_eval_boxes.argtypes = [I, I, I, P, P, SZ, SZ, P, P, P, P, P]
    L.cp_eval_boxes_host.argtypes = [I, I, I, P, P, SZ, P, P]
    L.cp_lattice_boxes.argtypes = [I, D, D, P, P, SZ, P, P, SZ, P]
    L.cp_single_placement.argtypes = [P, SZ, P, P]
    L.cp_eval_primitive.argtypes = [I, P, SZ, P, P, P]
    L.cp_asin_pad.argtypes = [P, SZ, P, P, P]


def _check(status: int, where: str):
    if status != 0:
        raise ProverError(status, where)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("circlepacking_b200 needs a CUDA device (no CPU fallback)")
    return torch


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(x, dtype):
    """A contiguous CUDA tensor of the given torch dtype."""
    torch = _torch()
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x))
    return x.to(device="cuda", dtype=dtype).contiguous()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def eval_boxes(family: int, lo, hi, precision: int = FP64, mode: int = EVAL_FULL, order=None, trace: bool = False):
    """Per-box verdicts of raw boxes lo/hi of shape (dims, n) (numpy or torch).

    Returns CUDA tensors (verdict uint8[n], mask uint8[n][, trace float64[n, 8, 2]])."""
    torch = _torch()
    lo = _dev(lo, torch.float64)
    hi = _dev(hi, torch.float64)
    n = lo.shape[1]
    v = torch.empty(n, dtype=torch.uint8, device="cuda")
    m = torch.empty(n, dtype=torch.uint8, device="cuda")
    o = _dev(order, torch.uint8) if order is not None else None
    tr = torch.full((n, 8, 2), float("nan"), dtype=torch.float64, device="cuda") if trace else None
    _check(lib().cp_eval_boxes(family, precision, mode, _ptr(lo), _ptr(hi), n, n, _ptr(v), _ptr(m), _ptr(o),
                               _ptr(tr), _stream()), "cp_eval_boxes")
    return (v, m, tr) if trace else (v, m)


def eval_boxes_host(family: int, lo: np.ndarray, hi: np.ndarray, precision: int = FP64, mode: int = EVAL_FULL):
    """As eval_boxes with host (numpy) buffers through cp_eval_boxes_host."""
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    n = lo.shape[1]
    v = np.empty(n, np.uint8)
    m = np.empty(n, np.uint8)
    _check(lib().cp_eval_boxes_host(family, precision, mode, lo.ctypes.data, hi.ctypes.data, n, v.ctypes.data,
                                    m.ctypes.data), "cp_eval_boxes_host")
    return v, m


def lattice_boxes(family: int, outer, sizes, index):
    """Raw boxes of a family lattice at the given linear indices (CUDA tensors (dims, n))."""
    torch = _torch()
    idx = _dev(index, torch.int64)
    n = idx.numel()
    dims = DIMS[family]
    s = (ctypes.c_int32 * 4)(*(list(sizes) + [1] * (4 - len(sizes))))
    lo = torch.empty((dims, n), dtype=torch.float64, device="cuda")
    hi = torch.empty((dims, n), dtype=torch.float64, device="cuda")
    _check(lib().cp_lattice_boxes(family, float(outer[0]), float(outer[1]), s, _ptr(idx), n, _ptr(lo), _ptr(hi), n,
                                  _stream()), "cp_lattice_boxes")
    return lo, hi


def single_placement(lb_lambda):
    torch = _torch()
    x = _dev(lb_lambda, torch.float64)
    out = torch.empty_like(x)
    _check(lib().cp_single_placement(_ptr(x), x.numel(), _ptr(out), _stream()), "cp_single_placement")
    return out


def eval_primitive(kind: int, args):
    """args: (2*nargs, n) lb/ub rows.  Returns (lb, ub, trap) CUDA tensors."""
    torch = _torch()
    a = _dev(args, torch.float64)
    n = a.shape[1]
    full = torch.zeros((6, n), dtype=torch.float64, device="cuda")
    full[: a.shape[0]] = a
    out = torch.empty((2, n), dtype=torch.float64, device="cuda")
    trap = torch.empty(n, dtype=torch.uint8, device="cuda")
    _check(lib().cp_eval_primitive(kind, _ptr(full), n, _ptr(out), _ptr(trap), _stream()), "cp_eval_primitive")
    return out[0], out[1], trap


def asin_pad(x):
    torch = _torch()
    x = _dev(x, torch.float64)
    rd = torch.empty_like(x)
    ru = torch.empty_like(x)
    _check(lib().cp_asin_pad(_ptr(x), x.numel(), _ptr(rd), _ptr(ru), _stream()), "cp_asin_pad")
    return rd, ru
