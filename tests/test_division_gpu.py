"""The library's directed division (Newton reciprocal + exact FMA remainders,
used for every interval division) is bit-identical to CUDA's __ddiv_rd /
__ddiv_ru, which the reference calls (interval.cuh:261-310)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(seed):
    rng = np.random.default_rng(seed)
    n = 400_000
    parts = []
    # magnitudes across and beyond the fast path's range [2^-500, 2^500]
    ea = rng.integers(-540, 540, n)
    eb = rng.integers(-540, 540, n)
    a = rng.uniform(1, 2, n) * np.exp2(ea.astype(float)) * rng.choice([-1, 1], n)
    b = rng.uniform(1, 2, n) * np.exp2(eb.astype(float)) * rng.choice([-1, 1], n)
    parts.append((a, b))
    # the prover's operand ranges: angles, radii, lane widths
    a = rng.uniform(-1.0, 4.0, n)
    b = rng.uniform(1e-6, 2.0, n) * rng.choice([-1, 1], n)
    parts.append((a, b))
    # exact quotients, and quotients next to a representable value
    k = rng.integers(1, 1 << 20, n).astype(float)
    b = rng.uniform(0.5, 1, n)
    a = b * k
    parts.append((a, b))
    parts.append((np.nextafter(a, np.inf), b))
    parts.append((np.nextafter(a, -np.inf), b))
    # same-significand operands (quotient a power of two) and zeros / subnormals / infinities
    m = rng.uniform(1, 2, n)
    parts.append((m * 8.0, m))
    special = np.array([0.0, -0.0, 5e-324, -5e-324, 1e-310, np.inf, -np.inf, 1.0, -1.0, 3.0])
    sa, sb = np.meshgrid(special, special)
    parts.append((sa.ravel(), sb.ravel()))
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    return a, b


@pytest.mark.parametrize("seed", [1, 2])
def test_directed_division_bit_identical(cp, seed):
    a, b = _cases(seed)
    rd, ru, want_rd, want_ru = cp.div_check(a, b)
    same_rd = (rd.view(np.int64) == want_rd.view(np.int64)) | (np.isnan(rd) & np.isnan(want_rd))
    same_ru = (ru.view(np.int64) == want_ru.view(np.int64)) | (np.isnan(ru) & np.isnan(want_ru))
    bad = np.nonzero(~(same_rd & same_ru))[0]
    assert bad.size == 0, [(a[i], b[i], rd[i], want_rd[i], ru[i], want_ru[i]) for i in bad[:5]]



def _fcases(seed):
    rng = np.random.default_rng(seed)
    n = 400_000
    parts = []
    # magnitudes across and beyond the fast path's range [2^-60, 2^61)
    ea = rng.integers(-140, 128, n)
    eb = rng.integers(-140, 128, n)
    a = rng.uniform(1, 2, n) * np.exp2(ea.astype(float)) * rng.choice([-1, 1], n)
    b = rng.uniform(1, 2, n) * np.exp2(eb.astype(float)) * rng.choice([-1, 1], n)
    parts.append((a, b))
    # the pre-pass's operand ranges
    parts.append((rng.uniform(-1.0, 4.0, n), rng.uniform(1e-6, 2.0, n) * rng.choice([-1, 1], n)))
    # exact quotients and their float neighbours
    k = rng.integers(1, 1 << 12, n).astype(np.float32)
    bf = rng.uniform(0.5, 1, n).astype(np.float32)
    af = (bf * k).astype(np.float32)
    parts.append((af, bf))
    parts.append((np.nextafter(af, np.float32(np.inf)), bf))
    parts.append((np.nextafter(af, np.float32(-np.inf)), bf))
    special = np.array([0.0, -0.0, 1e-45, -1e-45, 1e-40, np.inf, -np.inf, 1.0, -1.0, 3.0], np.float32)
    sa, sb = np.meshgrid(special, special)
    parts.append((sa.ravel(), sb.ravel()))
    a = np.concatenate([np.asarray(p[0], np.float32) for p in parts])
    b = np.concatenate([np.asarray(p[1], np.float32) for p in parts])
    return a, b


@pytest.mark.parametrize("seed", [3, 4])
def test_fp32_directed_division_bit_identical(cp, seed):
    """The FP32 pre-pass's directed division equals __fdiv_rd / __fdiv_ru bit for bit."""
    a, b = _fcases(seed)
    rd, ru, want_rd, want_ru = cp.fdiv_check(a, b)
    same_rd = (rd.view(np.int32) == want_rd.view(np.int32)) | (np.isnan(rd) & np.isnan(want_rd))
    same_ru = (ru.view(np.int32) == want_ru.view(np.int32)) | (np.isnan(ru) & np.isnan(want_ru))
    bad = np.nonzero(~(same_rd & same_ru))[0]
    assert bad.size == 0, [(a[i], b[i], rd[i], want_rd[i], ru[i], want_ru[i]) for i in bad[:5]]
