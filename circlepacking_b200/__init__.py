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
    L.cp_lattice_boxes.argtypes = [I, D, D, P, P, SZ, P, P, SZ, P, P]
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


def lattice_boxes(family: int, outer, sizes, index, visited: bool = False):
    """Raw boxes of a family lattice at the given linear indices (CUDA tensors
    (dims, n)); with visited=True also the byte mask of boxes the kernel visits."""
    torch = _torch()
    idx = _dev(index, torch.int64)
    n = idx.numel()
    dims = DIMS[family]
    s = (ctypes.c_int32 * 4)(*(list(sizes) + [1] * (4 - len(sizes))))
    lo = torch.empty((dims, n), dtype=torch.float64, device="cuda")
    hi = torch.empty((dims, n), dtype=torch.float64, device="cuda")
    vis = torch.empty(n, dtype=torch.uint8, device="cuda") if visited else None
    _check(lib().cp_lattice_boxes(family, float(outer[0]), float(outer[1]), s, _ptr(idx), n, _ptr(lo), _ptr(hi), n,
                                  _ptr(vis), _stream()), "cp_lattice_boxes")
    return (lo, hi, vis) if visited else (lo, hi)


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


# ---------------------------------------------------------------- prover handle
SPLIT_UNIFORM, SPLIT_LAMBDA, SPLIT_WIDEST, SPLIT_LEARNED, SPLIT_HYBRID = range(5)
ENGINE_LEVELS, ENGINE_GRAPH = 0, 1
GRAPH_BLOCKS, GRAPH_BPT = (64, 128, 256, 512, 1024), (1, 2, 4, 8)
REFERENCE_SIZES = ((256, 256, 256, 64), (4096, 4096, 4096), (256, 256, 256, 64), (512, 256, 256, 64),
                   (4096, 1024, 1024), (1024, 256, 128, 128))


class RefineOpts(ctypes.Structure):
    _fields_ = [("family", ctypes.c_int32), ("precision", ctypes.c_int32), ("policy", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("seed_sizes", ctypes.c_int32 * 4), ("seed_lambda", ctypes.c_double * 2),
                ("level_capacity", ctypes.c_int64), ("block", ctypes.c_int32), ("learned_order", ctypes.c_int32),
                ("engine", ctypes.c_int32), ("boxes_per_thread", ctypes.c_int32), ("lambda_scale", ctypes.c_double),
                ("digest", ctypes.c_int32), ("seed_parts", ctypes.c_int32), ("seed_part", ctypes.c_int32),
                ("reuse", ctypes.c_int32)]


class RefineReport(ctypes.Structure):
    _fields_ = [("evaluated", ctypes.c_int64), ("verdicts", ctypes.c_int64 * 5), ("unresolved", ctypes.c_int64),
                ("clipped", ctypes.c_int64), ("fp32_decided", ctypes.c_int64), ("per_depth", ctypes.c_int64 * 64),
                ("max_depth_seen", ctypes.c_int32), ("launches", ctypes.c_int32), ("device_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double), ("handles_evaluated", ctypes.c_int64), ("digest", ctypes.c_uint64 * 2)]

    def as_dict(self) -> dict:
        return dict(evaluated=self.evaluated, verdicts=list(self.verdicts), unresolved=self.unresolved,
                    clipped=self.clipped, fp32_decided=self.fp32_decided,
                    per_depth=list(self.per_depth)[: self.max_depth_seen + 1], max_depth_seen=self.max_depth_seen,
                    launches=self.launches, device_ms=self.device_ms, wall_ms=self.wall_ms,
                    handles_evaluated=self.handles_evaluated, digest=(int(self.digest[0]), int(self.digest[1])))


class ReferenceReport(ctypes.Structure):
    _fields_ = [("proved", ctypes.c_int32), ("interrupted", ctypes.c_int32), ("launches", ctypes.c_int64),
                ("boxes_evaluated", ctypes.c_int64), ("remaining", ctypes.c_double * 2), ("device_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return dict(proved=bool(self.proved), interrupted=bool(self.interrupted), launches=self.launches,
                    boxes_evaluated=self.boxes_evaluated, remaining=list(self.remaining), device_ms=self.device_ms,
                    wall_ms=self.wall_ms)


class ProofOpts(ctypes.Structure):
    _fields_ = [("family", ctypes.c_int32), ("precision", ctypes.c_int32), ("engine", ctypes.c_int32),
                ("policy", ctypes.c_int32), ("max_depth", ctypes.c_int32), ("slabs", ctypes.c_int32),
                ("geometric", ctypes.c_int32), ("seed_sizes", ctypes.c_int32 * 4), ("level_capacity", ctypes.c_int64),
                ("digest", ctypes.c_int32), ("seed_parts", ctypes.c_int32), ("seed_part", ctypes.c_int32),
                ("reuse", ctypes.c_int32), ("slab_radii", (ctypes.c_int32 * 3) * 32)]

    def as_dict(self) -> dict:
        d = {k: (list(getattr(self, k)) if k == "seed_sizes" else getattr(self, k)) for k, _ in self._fields_}
        d["slab_radii"] = [list(r) for r in self.slab_radii]
        return d


class ProofReport(ctypes.Structure):
    _fields_ = [("proved", ctypes.c_int32), ("slabs_done", ctypes.c_int32), ("evaluated", ctypes.c_int64),
                ("verdicts", ctypes.c_int64 * 5), ("unresolved", ctypes.c_int64), ("clipped", ctypes.c_int64),
                ("per_depth", ctypes.c_int64 * 64), ("max_depth_seen", ctypes.c_int32),
                ("first_unresolved_slab", ctypes.c_int32), ("device_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
                ("digest", ctypes.c_uint64 * 2)]

    def as_dict(self) -> dict:
        return dict(proved=bool(self.proved), slabs_done=self.slabs_done, evaluated=self.evaluated,
                    verdicts=list(self.verdicts), unresolved=self.unresolved, clipped=self.clipped,
                    per_depth=list(self.per_depth)[: self.max_depth_seen + 1], max_depth_seen=self.max_depth_seen,
                    first_unresolved_slab=self.first_unresolved_slab, device_ms=self.device_ms, wall_ms=self.wall_ms,
                    digest=(int(self.digest[0]), int(self.digest[1])))


def _declare_handle(L):
    P, I, D, SZ, I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_int64
    L.cp_create.argtypes = [I, ctypes.POINTER(P)]
    L.cp_destroy.argtypes = [P]
    L.cp_destroy.restype = None
    L.cp_request_interrupt.argtypes = [P]
    L.cp_request_interrupt.restype = None
    L.cp_refine.argtypes = [P, ctypes.POINTER(RefineOpts), ctypes.POINTER(RefineReport)]
    L.cp_refine_boxes.argtypes = [P, ctypes.POINTER(RefineOpts), P, P, P, SZ, ctypes.POINTER(RefineReport)]
    L.cp_refine_boxes_host.argtypes = [P, ctypes.POINTER(RefineOpts), P, P, P, SZ, ctypes.POINTER(RefineReport)]
    L.cp_stage_boxes_host.argtypes = [P, I, P, P, P, SZ, I]
    L.cp_refine_staged.argtypes = [P, ctypes.POINTER(RefineOpts), I, ctypes.POINTER(RefineReport)]
    L.cp_reference_step.argtypes = [P, I, D, D, P, P, P]
    L.cp_prove_family_reference.argtypes = [P, I, D, D, P, I64, P, ctypes.POINTER(ReferenceReport)]
    L.cp_reference_criticals.argtypes = [P, I, D, D, P, SZ, P, P, ctypes.POINTER(SZ)]
    L.cp_measure_primitives.argtypes = [I, P]
    L.cp_get_stream.argtypes = [P]
    L.cp_get_stream.restype = P
    L.cp_autotune.argtypes = [P, ctypes.POINTER(RefineOpts), ctypes.POINTER(ctypes.c_int), P]
    L.cp_refine_boxes_static.argtypes = [I, I, I, I, P, P, P, SZ, ctypes.POINTER(RefineReport), P]
    L.cp_set_level_variant.argtypes = [P, I, I, I]
    L.cp_refine_resume.argtypes = [P, ctypes.POINTER(RefineReport)]
    L.cp_checkpoint_save.argtypes = [P, ctypes.c_char_p]
    L.cp_checkpoint_load.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(RefineOpts)]
    L.cp_autotune_graph.argtypes = [P, ctypes.POINTER(RefineOpts), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int), P]
    L.cp_random_boxes.argtypes = [P, I, ctypes.c_uint64, I, SZ, P, P, P]
    L.cp_proof_defaults.argtypes = [I, ctypes.POINTER(ProofOpts)]
    L.cp_prove_family.argtypes = [P, ctypes.POINTER(ProofOpts), ctypes.POINTER(ProofReport)]
    L.cp_prove_all.argtypes = [P, I, I, ctypes.POINTER(ProofReport)]
    L.cp_set_chunk_callback.argtypes = [P, P, P]
    L.cp_set_chunk_callback.restype = None


def measure_primitives(device: int = 0) -> dict:
    L = lib()
    _declare_handle(L)
    rates = np.zeros(9, np.float64)
    _check(L.cp_measure_primitives(device, rates.ctypes.data), "cp_measure_primitives")
    return dict(zip(("dfma", "dadd_rd", "dmul_rd", "ddiv_rd", "asin", "ffma", "div_rd_lib", "div_rd_f32seed_inline",
                     "div_rd_inline"), rates.tolist()))


def div_check(a, b):
    """(library RD, library RU, __ddiv_rd, __ddiv_ru) of a/b on the device, as numpy arrays."""
    torch = _torch()
    L = lib()
    L.cp_div_check.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    a = _dev(a, torch.float64)
    b = _dev(b, torch.float64)
    out = torch.empty((a.numel(), 4), dtype=torch.float64, device="cuda")
    _check(L.cp_div_check(_ptr(a), _ptr(b), a.numel(), _ptr(out), _stream()), "cp_div_check")
    return out.cpu().numpy().T


def fdiv_check(a, b):
    """(library RD, library RU, __fdiv_rd, __fdiv_ru) of float32 a/b on the device, as numpy arrays."""
    torch = _torch()
    L = lib()
    L.cp_fdiv_check.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    a = _dev(np.asarray(a, np.float32), torch.float32)
    b = _dev(np.asarray(b, np.float32), torch.float32)
    out = torch.empty((a.numel(), 4), dtype=torch.float32, device="cuda")
    _check(L.cp_fdiv_check(_ptr(a), _ptr(b), a.numel(), _ptr(out), _stream()), "cp_fdiv_check")
    return out.cpu().numpy().T


def _sizes4(sizes):
    if sizes is None:
        return None
    return (ctypes.c_int32 * 4)(*(list(sizes) + [1] * (4 - len(sizes))))


class Prover:
    """A prover handle (device scratch, stream and counters) over the C ABI."""

    def __init__(self, device: int = 0):
        L = lib()
        _declare_handle(L)
        self._L = L
        h = ctypes.c_void_p()
        _check(L.cp_create(device, ctypes.byref(h)), "cp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.cp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        """The handle's CUDA stream as a torch ExternalStream."""
        torch = _torch()
        return torch.cuda.ExternalStream(self._L.cp_get_stream(self._h))

    def interrupt(self):
        self._L.cp_request_interrupt(self._h)

    _CHUNK_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64)

    def set_chunk_callback(self, fn):
        """fn(evaluated, waiting) after every chunk of a host-driven refinement
        (cp_set_chunk_callback); fn may call interrupt().  None removes it."""
        if fn is None:
            self._chunk_cb = None
            self._L.cp_set_chunk_callback(self._h, None, None)
            return
        self._chunk_cb = self._CHUNK_CB(lambda _u, e, w: fn(int(e), int(w)))
        self._L.cp_set_chunk_callback(self._h, ctypes.cast(self._chunk_cb, ctypes.c_void_p), None)

    @staticmethod
    def opts(family, precision=FP64, policy=SPLIT_UNIFORM, max_depth=2, seed_sizes=None, seed_lambda=None,
             level_capacity=0, learned_order=False, engine=ENGINE_LEVELS, block=0, boxes_per_thread=0,
             lambda_scale=0.0, digest=False, seed_part=0, seed_parts=1, reuse=True) -> RefineOpts:
        o = RefineOpts()
        o.family, o.precision, o.policy, o.max_depth = family, precision, policy, max_depth
        ss = list(seed_sizes or [64] * DIMS[family]) + [1] * 4
        for d in range(4):
            o.seed_sizes[d] = ss[d]
        sl = seed_lambda or (LAMBDA_MIN, LAMBDA_MAX)
        o.seed_lambda[0], o.seed_lambda[1] = sl
        o.level_capacity = level_capacity
        o.block = block
        o.learned_order = int(bool(learned_order))
        o.engine = engine
        o.boxes_per_thread = boxes_per_thread
        o.lambda_scale = lambda_scale
        o.digest = int(bool(digest))
        o.seed_parts, o.seed_part = seed_parts, seed_part
        o.reuse = int(bool(reuse))
        return o

    def autotune(self, family, **kw):
        """Times every level-kernel variant on this refinement and keeps the fastest."""
        o = self.opts(family, **kw)
        best = ctypes.c_int()
        ms = np.zeros(4, np.float64)
        _check(self._L.cp_autotune(self._h, ctypes.byref(o), ctypes.byref(best), ms.ctypes.data), "cp_autotune")
        return best.value, ms.tolist()

    def autotune_graph(self, family, **kw):
        """Times every graph-engine kernel shape (block size x boxes per thread) on
        this refinement and keeps the fastest; returns (block, bpt, ms[5][4])."""
        o = self.opts(family, **kw)
        blk, bpt = ctypes.c_int(), ctypes.c_int()
        ms = np.zeros(20, np.float64)
        _check(self._L.cp_autotune_graph(self._h, ctypes.byref(o), ctypes.byref(blk), ctypes.byref(bpt),
                                         ms.ctypes.data), "cp_autotune_graph")
        return blk.value, bpt.value, ms.reshape(5, 4).tolist()

    def set_level_variant(self, family, precision, variant):
        _check(self._L.cp_set_level_variant(self._h, family, precision, variant), "cp_set_level_variant")

    def refine(self, family, **kw) -> dict:
        o = self.opts(family, **kw)
        r = RefineReport()
        _check(self._L.cp_refine(self._h, ctypes.byref(o), ctypes.byref(r)), "cp_refine")
        return r.as_dict()

    def stage_boxes(self, slot, lo, hi, depth=None):
        """Starts the host-to-device copy of seed boxes (numpy [dims][n]; page-locked
        memory, e.g. a pinned torch tensor's numpy view, for the copy to overlap)
        into staging slot 0 or 1 (cp_stage_boxes_host) and returns at once.  The
        arrays are kept alive until refine_staged(slot) returns."""
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        dp = np.ascontiguousarray(depth, np.uint8) if depth is not None else None
        staged = self.__dict__.setdefault("_staged", [None, None])
        staged[slot] = (lo, hi, dp)
        _check(self._L.cp_stage_boxes_host(self._h, slot, lo.ctypes.data, hi.ctypes.data,
                                           dp.ctypes.data if dp is not None else None, lo.shape[1], lo.shape[0]),
               "cp_stage_boxes_host")

    def refine_staged(self, family, slot, **kw) -> dict:
        """Refines the boxes staged in a slot (cp_refine_staged); same report as refine_boxes."""
        o = self.opts(family, **kw)
        r = RefineReport()
        try:
            _check(self._L.cp_refine_staged(self._h, ctypes.byref(o), slot, ctypes.byref(r)), "cp_refine_staged")
        finally:
            self.__dict__.setdefault("_staged", [None, None])[slot] = None
        return r.as_dict()

    def refine_boxes(self, family, lo, hi, depth=None, **kw) -> dict:
        """Refine explicit seed boxes: torch CUDA tensors (device) or numpy (host entry)."""
        o = self.opts(family, **kw)
        r = RefineReport()
        if isinstance(lo, np.ndarray):
            lo = np.ascontiguousarray(lo, np.float64)
            hi = np.ascontiguousarray(hi, np.float64)
            dp = np.ascontiguousarray(depth, np.uint8).ctypes.data if depth is not None else None
            _check(self._L.cp_refine_boxes_host(self._h, ctypes.byref(o), lo.ctypes.data, hi.ctypes.data, dp,
                                               lo.shape[1], ctypes.byref(r)), "cp_refine_boxes_host")
        else:
            torch = _torch()
            lo = _dev(lo, torch.float64)
            hi = _dev(hi, torch.float64)
            dp = _dev(depth, torch.uint8) if depth is not None else None
            torch.cuda.synchronize()
            _check(self._L.cp_refine_boxes(self._h, ctypes.byref(o), _ptr(lo), _ptr(hi), _ptr(dp), lo.shape[1],
                                          ctypes.byref(r)), "cp_refine_boxes")
        return r.as_dict()

    def random_boxes(self, family, n, seed=0xC1C1E5, max_label=8):
        """n seeded random boxes on the family's domain (cp_random_boxes):
        CUDA tensors lo, hi of shape (dims, n) and depth labels uint8[n] (255 = dropped)."""
        torch = _torch()
        lo = torch.empty((DIMS[family], n), dtype=torch.float64, device="cuda")
        hi = torch.empty_like(lo)
        dp = torch.empty(n, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        _check(self._L.cp_random_boxes(self._h, family, seed, max_label, n, _ptr(lo), _ptr(hi), _ptr(dp)),
               "cp_random_boxes")
        return lo, hi, dp

    def proof_defaults(self, family) -> dict:
        """The library's settings for a family's full-domain proof (cp_proof_defaults)."""
        o = ProofOpts()
        _check(self._L.cp_proof_defaults(family, ctypes.byref(o)), "cp_proof_defaults")
        return o.as_dict()

    def prove_family(self, family, **overrides) -> dict:
        """The full-domain proof of a family (cp_prove_family): the library's
        defaults for the family, with any field of cp_proof_opts overridden.
        An interrupted proof (interrupt()) returns with interrupted=True."""
        o = ProofOpts()
        _check(self._L.cp_proof_defaults(family, ctypes.byref(o)), "cp_proof_defaults")
        for k, v in overrides.items():
            if k == "seed_sizes":
                ss = list(v) + [1] * 4
                for d in range(4):
                    o.seed_sizes[d] = ss[d]
            elif k == "slab_radii":
                rows = [list(r) for r in v] + [[0, 0, 0]] * 32
                for i in range(32):
                    for d in range(3):
                        o.slab_radii[i][d] = rows[i][d]
            else:
                setattr(o, k, int(v))
        r = ProofReport()
        st = self._L.cp_prove_family(self._h, ctypes.byref(o), ctypes.byref(r))
        if st not in (0, 8):
            raise ProverError(st, "cp_prove_family")
        d = r.as_dict()
        d["interrupted"] = st == 8
        return d

    def prove_all(self, precision=FP64, engine=ENGINE_GRAPH) -> list:
        """The full-domain proofs of the six families in the reference's order (cp_prove_all)."""
        reps = (ProofReport * 6)()
        _check(self._L.cp_prove_all(self._h, precision, engine, reps), "cp_prove_all")
        return [r.as_dict() for r in reps]

    def refine_resume(self) -> dict:
        """Continues the refinement interrupted by interrupt() (or loaded from a checkpoint)."""
        r = RefineReport()
        _check(self._L.cp_refine_resume(self._h, ctypes.byref(r)), "cp_refine_resume")
        return r.as_dict()

    def checkpoint_save(self, path):
        _check(self._L.cp_checkpoint_save(self._h, os.fsencode(path)), "cp_checkpoint_save")

    def checkpoint_load(self, path) -> RefineOpts:
        o = RefineOpts()
        _check(self._L.cp_checkpoint_load(self._h, os.fsencode(path), ctypes.byref(o)), "cp_checkpoint_load")
        return o

    def reference_step(self, family, la_lb, la_ub, sizes=None):
        """One reference-semantics lattice launch: smallest failing lambda.lb (inf if none)."""
        first = ctypes.c_double()
        err = (ctypes.c_double * 8)()
        st = self._L.cp_reference_step(self._h, family, la_lb, la_ub, _sizes4(sizes), ctypes.byref(first), err)
        if st != 0:
            raise ProverError(st, f"cp_reference_step (box {list(err)})")
        return first.value

    def prove_family_reference(self, family, la_lb=LAMBDA_MIN, la_ub=LAMBDA_MAX, sizes=None, max_launches=0,
                               trace_cap=0):
        r = ReferenceReport()
        trace = np.zeros((max(trace_cap, 1), 3), np.float64)
        st = self._L.cp_prove_family_reference(self._h, family, la_lb, la_ub, _sizes4(sizes), max_launches,
                                               trace.ctypes.data if trace_cap else None, ctypes.byref(r))
        d = r.as_dict()
        d["status"] = STATUS.get(st, st)
        if trace_cap:
            d["trace"] = trace[: min(r.launches, trace_cap)]
        return d

    def reference_criticals(self, family, la_lb, la_ub, sizes=None, max_boxes=1000):
        boxes = np.zeros((max(max_boxes, 1), 8), np.float64)
        handles = np.zeros(max(max_boxes, 1), np.uint8)
        count = ctypes.c_size_t()
        _check(self._L.cp_reference_criticals(self._h, family, la_lb, la_ub, _sizes4(sizes), max_boxes,
                                             boxes.ctypes.data, handles.ctypes.data, ctypes.byref(count)),
               "cp_reference_criticals")
        m = min(count.value, max_boxes)
        return count.value, boxes[:m], handles[:m]


STATIC_MAX_SEEDS, STATIC_MAX_DEPTH = 65536, 6


def refine_boxes_static(family, lo, hi, depth=None, precision=FP64, policy=SPLIT_WIDEST, max_depth=6) -> dict:
    """cp_refine_boxes_static: the refinement of explicit device seed boxes for
    callers that cannot let the library allocate (all scratch lives in a fixed
    array inside the library; see include/cp_prover.h)."""
    torch = _torch()
    L = lib()
    _declare_handle(L)
    lo = _dev(lo, torch.float64)
    hi = _dev(hi, torch.float64)
    dp = _dev(depth, torch.uint8) if depth is not None else None
    r = RefineReport()
    _check(L.cp_refine_boxes_static(family, precision, policy, max_depth, _ptr(lo), _ptr(hi), _ptr(dp), lo.shape[1],
                                    ctypes.byref(r), _stream()), "cp_refine_boxes_static")
    return r.as_dict()


# ---------------------------------------------------------------- learned proposal model
def _declare_model(L):
    P, I, SZ, I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_int64
    L.cp_model_collect.argtypes = [P, ctypes.POINTER(RefineOpts), I64, ctypes.c_int32, ctypes.POINTER(I64)]
    L.cp_model_records.argtypes = [P, P, P, P, P, P, SZ, ctypes.POINTER(SZ)]
    L.cp_model_train.argtypes = [P, I, I, I, ctypes.c_float, ctypes.c_uint64, P]
    L.cp_model_get_params.argtypes = [P, I, P]
    L.cp_model_set_params.argtypes = [P, I, P]
    L.cp_model_loss_grad.argtypes = [I, P, P, P, P, SZ, P, P]
    L.cp_model_loss_grad_kind.argtypes = [I, I, P, P, P, P, SZ, P, P]
    L.cp_model_set_training.argtypes = [P, I]
    L.cp_model_predict.argtypes = [P, I, P, P, P, SZ, P, P, P]
    L.cp_model_set_inference.argtypes = [P, I]
    L.cp_model_set_wait_limit.argtypes = [P, ctypes.c_int32]


def model_param_count() -> int:
    return int(lib().cp_model_param_count())


def model_loss_grad(family, params, feats, crit, axis, kind=0):
    """One GPU forward+backward pass (no optimiser step): (loss, grad).
    kind 0: warp-level mma.sync kernel; 1: tcgen05 kernel (tensor memory)."""
    L = lib()
    _declare_model(L)
    params = np.ascontiguousarray(params, np.float32)
    feats = np.ascontiguousarray(feats, np.float32)
    crit = np.ascontiguousarray(crit, np.uint8)
    axis = np.ascontiguousarray(axis, np.int8)
    loss = np.zeros(1, np.float32)
    grad = np.zeros(params.size, np.float32)
    _check(L.cp_model_loss_grad_kind(kind, family, params.ctypes.data, feats.ctypes.data, crit.ctypes.data,
                                     axis.ctypes.data, feats.shape[0], loss.ctypes.data, grad.ctypes.data),
           "cp_model_loss_grad")
    return float(loss[0]), grad


class _ModelMixin:
    def model_collect(self, family, max_records, sample_stride=1, **kw) -> int:
        _declare_model(self._L)
        o = self.opts(family, **kw)
        n = ctypes.c_int64()
        _check(self._L.cp_model_collect(self._h, ctypes.byref(o), max_records, sample_stride, ctypes.byref(n)),
               "cp_model_collect")
        return n.value

    def model_records(self, cap=None) -> dict:
        _declare_model(self._L)
        n = ctypes.c_size_t()
        _check(self._L.cp_model_records(self._h, None, None, None, None, None, 0, ctypes.byref(n)), "cp_model_records")
        k = n.value if cap is None else min(cap, n.value)
        feats = np.zeros((max(k, 1), 16), np.float32)
        crit = np.zeros(max(k, 1), np.uint8)
        axis = np.zeros(max(k, 1), np.int8)
        boxes = np.zeros((max(k, 1), 8), np.float64)
        depth = np.zeros(max(k, 1), np.uint8)
        _check(self._L.cp_model_records(self._h, feats.ctypes.data, crit.ctypes.data, axis.ctypes.data,
                                        boxes.ctypes.data, depth.ctypes.data, k, ctypes.byref(n)), "cp_model_records")
        return dict(feats=feats[:k], crit=crit[:k], axis=axis[:k], boxes=boxes[:k], depth=depth[:k])

    def model_train(self, family, epochs=20, batch=4096, lr=1e-3, seed=1):
        _declare_model(self._L)
        losses = np.zeros(epochs, np.float32)
        _check(self._L.cp_model_train(self._h, family, epochs, batch, lr, seed, losses.ctypes.data), "cp_model_train")
        return losses

    def model_params(self, family):
        _declare_model(self._L)
        p = np.zeros(model_param_count(), np.float32)
        _check(self._L.cp_model_get_params(self._h, family, p.ctypes.data), "cp_model_get_params")
        return p

    def model_set_params(self, family, params):
        _declare_model(self._L)
        p = np.ascontiguousarray(params, np.float32)
        _check(self._L.cp_model_set_params(self._h, family, p.ctypes.data), "cp_model_set_params")

    def model_set_inference(self, kind):
        """0: warp-level mma.sync inference kernel; 1: tcgen05 + tensor memory."""
        _declare_model(self._L)
        _check(self._L.cp_model_set_inference(self._h, kind), "cp_model_set_inference")

    def model_set_training(self, kind):
        """The training kernel of model_train: 1 = tcgen05 (default), 0 = mma.sync."""
        _declare_model(self._L)
        _check(self._L.cp_model_set_training(self._h, kind), "cp_model_set_training")

    def model_set_wait_limit(self, polls):
        """Polls per bounded completion wait of the tcgen05 inference kernel (0: every wait times out)."""
        _declare_model(self._L)
        _check(self._L.cp_model_set_wait_limit(self._h, polls), "cp_model_set_wait_limit")

    def model_predict(self, family, lo, hi, depth=None):
        _declare_model(self._L)
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        n = lo.shape[1]
        dp = np.ascontiguousarray(depth, np.uint8).ctypes.data if depth is not None else None
        logits = np.zeros((n, 8), np.float32)
        axis = np.zeros(n, np.uint8)
        order = np.zeros(n, np.uint8)
        _check(self._L.cp_model_predict(self._h, family, lo.ctypes.data, hi.ctypes.data, dp, n, logits.ctypes.data,
                                        axis.ctypes.data, order.ctypes.data), "cp_model_predict")
        return logits, axis, order


for _name in ("model_collect", "model_records", "model_train", "model_params", "model_set_params", "model_predict",
              "model_set_inference", "model_set_wait_limit", "model_set_training"):
    setattr(Prover, _name, getattr(_ModelMixin, _name))


# ---------------------------------------------------------------- multi-GPU sharding
def lambda_shard(rank: int, world: int, lo: float = LAMBDA_MIN, hi: float = LAMBDA_MAX, balance: str = "work"):
    """The lambda sub-range of `rank` among `world` ranks.

    balance="work": the cut points equalise the integral of (1 - lambda)^-2 over
    the pieces -- the needed lambda width of the proofs shrinks about like
    (1 - lambda)^2 toward the top of the domain, so the boxes per unit of lambda
    grow like its inverse, and equal pieces of that integral carry about equal
    work.  balance="width": equal widths.  Neighbouring ranks compute their shared
    boundary by the same expression, so the pieces tile [lo, hi] exactly.  Boxes
    are independent: ranks refine their pieces with no data exchange and only
    the final counts are summed (reduce_report)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    if balance not in ("work", "width"):
        raise ValueError("balance must be 'work' or 'width'")

    def cut(k):
        if k == 0:
            return lo
        if k == world:
            return hi
        if balance == "width":
            return lo + (hi - lo) / world * k
        # W(x) = 1 / (1 - x) is an antiderivative of (1 - x)^-2
        a, b = 1.0 / (1.0 - lo), 1.0 / (1.0 - hi)
        return 1.0 - 1.0 / (a + (b - a) * k / world)

    return cut(rank), cut(rank + 1)


def seed_partition(total: int, rank: int, world: int) -> np.ndarray:
    """The lattice indices of `rank`'s piece of a seed of `total` boxes split
    among `world` ranks (cp_refine_opts.seed_part / seed_parts): rank, rank +
    world, rank + 2 world, ...  Interleaving spreads the lambda slabs, where the
    work concentrates, evenly over the ranks; the pieces are disjoint and their
    union is the whole seed, so the ranks' reports add up to the single-GPU one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    return np.arange(rank, total, world, dtype=np.int64)


def reduce_report(report: dict, group=None) -> dict:
    """Sums a refinement report's counts over the ranks of a torch.distributed
    group (any backend): the scalar counts, the verdict histogram, the launches
    and the per-depth histogram (padded to 64 depths, the report's bins);
    max_depth_seen is recomputed from the summed histogram and the times become
    the maximum over ranks; a per-box digest is combined as the device combines
    it (sum mod 2^64, xor), which is exact for disjoint pieces of a seed.  Every
    rank must call it (two all-reduces, and an all-gather when the report
    carries a digest)."""
    import torch
    import torch.distributed as dist

    import numpy as _np

    keys = ("evaluated", "unresolved", "clipped", "fp32_decided", "handles_evaluated", "launches")
    depth = list(report["per_depth"])[:64]
    depth += [0] * (64 - len(depth))
    v = torch.tensor([report[k] for k in keys] + list(report["verdicts"]) + depth, dtype=torch.float64)
    t = torch.tensor([report["device_ms"], report["wall_ms"]], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        v, t = v.cuda(), t.cuda()
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    v, t = v.cpu().tolist(), t.cpu().tolist()
    out = dict(report)
    for i, k in enumerate(keys):
        out[k] = int(v[i])
    nk = len(keys)
    out["verdicts"] = [int(x) for x in v[nk:nk + 5]]
    hist = [int(x) for x in v[nk + 5:nk + 5 + 64]]
    seen = max((d for d, c in enumerate(hist) if c), default=0)
    out["per_depth"] = hist[: seen + 1]
    out["max_depth_seen"] = seen
    out["device_ms"], out["wall_ms"] = t
    if "digest" in report:
        # digests add up over disjoint pieces: sum mod 2^64 and xor (gathered:
        # collectives have no xor for every backend)
        world = dist.get_world_size(group)
        mine = torch.tensor([int(x) - (1 << 64) if int(x) >= (1 << 63) else int(x) for x in report["digest"]],
                            dtype=torch.int64)
        if dist.get_backend(group) == "nccl":
            mine = mine.cuda()
        parts = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine, group=group)
        words = _np.array([p_.cpu().numpy().view(_np.uint64) for p_ in parts], dtype=_np.uint64)
        with _np.errstate(over="ignore"):
            total = int(words[:, 0].sum(dtype=_np.uint64))
        out["digest"] = (total, int(_np.bitwise_xor.reduce(words[:, 1])))
    return out
