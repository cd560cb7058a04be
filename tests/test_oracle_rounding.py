"""The oracle's directed rounding (error-free transformations) against <cfenv>."""
import numpy as np
import pytest


def _inputs(seed: int, n: int = 20000):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-2, 2, n) * 10.0 ** rng.integers(-8, 3, n)
    b = rng.uniform(-2, 2, n) * 10.0 ** rng.integers(-8, 3, n)
    # exact cancellations, signed zeros, equal magnitudes, tiny and huge values
    edge = np.array([0.0, -0.0, 1.0, -1.0, 0.5, 3.0, 1e-300, -1e-300, 5e-324, -5e-324, 1e300, -1e300,
                     0.1, 0.2, 0.3, 1 / 3, 2.0 ** -1022, 1.7976931348623157e308])
    ea, eb = np.meshgrid(edge, edge)
    a = np.concatenate([a, ea.ravel(), a[:500]])
    b = np.concatenate([b, eb.ravel(), -a[:500]])
    return a, b


@pytest.mark.parametrize("op", [0, 1, 2])
@pytest.mark.parametrize("up", [False, True])
def test_directed_ops_match_fenv(oracle, op, up):
    a, b = _inputs(op * 2 + int(up))
    got = oracle.round_op(op, up, a, b)
    want = oracle.round_op(op, up, a, b, fenv=True)
    same = (got.view(np.uint64) == want.view(np.uint64)) | (np.isnan(got) & np.isnan(want))
    assert same.all(), (a[~same][:5], b[~same][:5], got[~same][:5], want[~same][:5])


def test_directed_ops_bracket_nearest(oracle):
    a, b = _inputs(7)
    for op, f in ((0, np.add), (1, np.multiply), (2, np.divide)):
        with np.errstate(all="ignore"):
            rn = f(a, b)
        lo = oracle.round_op(op, False, a, b)
        hi = oracle.round_op(op, True, a, b)
        ok = np.isnan(rn) | ((lo <= rn) & (rn <= hi))
        assert ok.all()
