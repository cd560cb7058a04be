"""Properties of the CPU oracle that hold independently of the reference's bits."""
import numpy as np
import pytest

from tests import boxgen


def test_asin_padding_encloses_extended_precision(oracle):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-1, 1, 20000), rng.uniform(0.99, 1.0, 2000), [0.0, -0.0, 1.0, -1.0, 1e-300]])
    rd, ru = oracle.asin_pad(x)
    ref = np.arcsin(x.astype(np.longdouble))
    assert (rd.astype(np.longdouble) <= ref).all()
    assert (ru.astype(np.longdouble) >= ref).all()
    assert (rd <= ru).all()


@pytest.mark.parametrize("family", range(6))
def test_lattice_covers_ranges(oracle, family):
    """Neighbouring subintervals of every axis share their endpoint bits, so the
    lattice covers the dependent ranges completely (subintervals.hpp:31-42)."""
    dims = boxgen.DIMS[family]
    sizes = [8, 6, 5, 4][:dims]
    total = int(np.prod(sizes))
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, np.arange(total))
    shape = tuple(sizes)
    L = lo.reshape((dims,) + shape)
    H = hi.reshape((dims,) + shape)
    for d in range(dims):
        a = np.moveaxis(L[d], d, 0)
        b = np.moveaxis(H[d], d, 0)
        assert (a[1:] == b[:-1]).all(), f"axis {d} has gaps"
    assert L[0].min() == 0.5 and H[0].max() == boxgen.LAMBDA[1]


@pytest.mark.parametrize("family", range(6))
def test_trace_consistent_with_mask(oracle, family):
    dims = boxgen.DIMS[family]
    sizes = [64, 16, 16, 8][:dims]
    idx = boxgen.lattice_indices(family, sizes, 3000, seed=family)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, idx)
    v, m, t = oracle.eval_boxes(family, lo, hi, trace=True)
    live = (v != oracle.EMPTY) & ((m & oracle.M_TRAP) == 0)
    for k in range(oracle.N_CRITERIA[family]):
        ev = ~np.isnan(t[:, k, 0])
        if family == 3:
            fail = t[:, k, 0] < t[:, k, 1]
        else:
            fail = ~(t[:, k, 0] >= t[:, k, 1])
        bit = ((m >> k) & 1).astype(bool)
        assert (bit[live & ev] == fail[live & ev]).all()
        assert not bit[live & ~ev].any()


@pytest.mark.parametrize("family", range(6))
def test_sub_boxes_monotone(oracle, family):
    """Interval evaluation is inclusion-monotone in spirit: a sub-box of a PROVED
    box is never CRITICAL unless a guard or trap path differs -- checked here
    for the fraction of violations staying tiny."""
    dims = boxgen.DIMS[family]
    sizes = [512, 32, 32, 8][:dims]
    idx = boxgen.lattice_indices(family, sizes, 4000, seed=10 + family)
    lo, hi = oracle.lattice_boxes(family, (0.6, 0.62), sizes, idx)
    v, _ = oracle.eval_boxes(family, lo, hi)
    slo, shi = boxgen.sub_boxes(lo, hi, seed=family)
    sv, _ = oracle.eval_boxes(family, slo, shi)
    proved = v == oracle.PROVED
    bad = proved & (sv == oracle.CRITICAL)
    assert bad.sum() <= max(2, proved.sum() // 1000)


def test_single_placement_monotone(oracle):
    lam = np.linspace(0.5, 0.99, 200)
    s = np.array([oracle.single_placement(x) for x in lam])
    assert (np.diff(s) <= 0).all()
    assert (s < 0.5 * (1 - lam) + 1e-12).all()


def test_reference_loop_small(oracle):
    """The reference's lambda loop restated on a tiny lattice terminates or
    records monotone progress."""
    steps, proved = oracle.reference_loop(3, [16, 4, 4, 2], max_steps=40)
    assert len(steps) > 0
    assert (steps[:, 0] <= steps[:, 1]).all()


@pytest.mark.parametrize("family", range(6))
def test_decide_path_op_counts(oracle, family):
    """The reference kernel's own path (stop at the first failing sub-check and
    handle) costs no more than evaluating every sub-criterion, and exactly as
    much on proved boxes, where nothing stops early."""
    dims = boxgen.DIMS[family]
    sizes = [64, 16, 16, 8][:dims]
    idx = boxgen.lattice_indices(family, sizes, 2000, seed=10 + family)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, idx)
    v, _ = oracle.eval_boxes(family, lo, hi)
    full = oracle.count_ops(family, lo, hi)
    dec = oracle.count_ops(family, lo, hi, decide=True)
    for k in ("add", "mul", "div", "asin"):
        assert dec[k] <= full[k]
    proved = v == 0
    if proved.any():
        pf = oracle.count_ops(family, lo[:, proved], hi[:, proved])
        pd = oracle.count_ops(family, lo[:, proved], hi[:, proved], decide=True)
        assert pf == pd
    crit = v == 1
    if crit.any() and family in (0, 3, 4, 5):
        cf = oracle.count_ops(family, lo[:, crit], hi[:, crit])
        cd = oracle.count_ops(family, lo[:, crit], hi[:, crit], decide=True)
        assert cd["asin"] < cf["asin"]
