"""Seeded box generators shared by the tests and the golden-fixture script.

All boxes live on the reference's domain: lambda in [0.5, 0.99] and radii in
the dependent ranges of the family lattices."""
from __future__ import annotations

import numpy as np

LAMBDA = (0.5, 0.9900000000000001)
DIMS = (4, 3, 4, 4, 3, 4)
FAMILY_NAMES = ("start", "start_end_2d", "start_end_3d", "middle", "end_2d", "end_3d")


def lattice_indices(family: int, sizes, n: int, seed: int) -> np.ndarray:
    total = int(np.prod(sizes[: DIMS[family]]))
    rng = np.random.default_rng(seed)
    if total <= n:
        return np.arange(total, dtype=np.int64)
    return np.sort(rng.choice(total, size=n, replace=False)).astype(np.int64)


def sub_boxes(lo: np.ndarray, hi: np.ndarray, seed: int, min_frac: float = 1e-6) -> tuple[np.ndarray, np.ndarray]:
    """A random sub-box of every box: per axis a log-uniform fraction of the
    width at a uniform position."""
    rng = np.random.default_rng(seed)
    w = hi - lo
    frac = np.exp(rng.uniform(np.log(min_frac), 0.0, size=lo.shape))
    sw = w * frac
    start = lo + rng.uniform(0.0, 1.0, size=lo.shape) * (w - sw)
    nlo = np.minimum(start, hi)
    nhi = np.minimum(np.maximum(start + sw, nlo), hi)
    return nlo, nhi


def point_boxes(lo: np.ndarray, hi: np.ndarray, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Degenerate boxes (lb == ub on every axis) at random points."""
    rng = np.random.default_rng(seed)
    p = lo + rng.uniform(0.0, 1.0, size=lo.shape) * (hi - lo)
    return p.copy(), p.copy()


def handle_bits(family: int, mask: np.ndarray) -> np.ndarray:
    """Map the sub-criterion mask to the reference's per-handle failures
    (middle: bits 0|1 = handle_case_1_1, bits 2|3 = handle_case_2_1)."""
    m = mask.astype(np.uint8)
    if family == 3:
        h0 = ((m & 0x3) != 0).astype(np.uint8)
        h1 = ((m & 0xC) != 0).astype(np.uint8)
        return h0 | (h1 << 1)
    return m & 0x3


def product_to_ref_bits(family: int, verdict: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Product (verdict, mask) in the reference checker's bit layout."""
    bits = handle_bits(family, mask) | (mask & 0xC0)
    bits = np.where(verdict == 3, np.uint8(0x20), bits).astype(np.uint8)
    return bits


# ---------------------------------------------------------------- verdict digests
M64 = (1 << 64) - 1


def _mix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def host_digest(lo, hi, verdict):
    """The library's per-box verdict digest (cp_refine_report.digest) of boxes
    lo/hi (dims, n) with the given verdicts: sum mod 2^64 and xor of a splitmix64
    hash of the bounds' bit patterns and the verdict, restated in numpy."""
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    with np.errstate(over="ignore"):
        h = np.uint64(0x9E3779B97F4A7C15) * (np.asarray(verdict).astype(np.uint64) + np.uint64(1))
        for d in range(lo.shape[0]):
            h = _mix64(h ^ np.ascontiguousarray(lo[d]).view(np.uint64))
            h = _mix64(h + np.ascontiguousarray(hi[d]).view(np.uint64))
        x = _mix64(h ^ np.uint64(0x5851F42D4C957F2D))
    return int(h.sum(dtype=np.uint64)) & M64, int(np.bitwise_xor.reduce(x)) if x.size else 0
