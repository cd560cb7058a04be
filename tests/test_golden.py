"""The CPU oracle pinned against golden outputs of the reference's own device
code (tests/golden/*.npz, made by tests/golden/gen_golden.py on a GPU)."""
import os

import numpy as np
import pytest

from tests import boxgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("family", range(6))
def test_oracle_box_verdicts_match_reference(oracle, family):
    d = _load(f"ref_{boxgen.FAMILY_NAMES[family]}.npz")
    v, m = oracle.eval_boxes(family, d["box_lo"], d["box_hi"])
    got = boxgen.product_to_ref_bits(family, v, m)
    want = d["box_bits"]
    trap = (want & 0x80) != 0
    same = np.where(trap, (got & 0xE0) == (want & 0xE0), got == want)
    assert same.all(), f"{(~same).sum()} of {same.size} boxes differ"
    # the fixture exercises proved, critical and trap-site boxes
    assert (want == 0).any() and ((want & 0x3) != 0).any()


@pytest.mark.parametrize("family", range(6))
def test_oracle_lattice_matches_reference(oracle, family):
    d = _load(f"ref_{boxgen.FAMILY_NAMES[family]}.npz")
    dims = boxgen.DIMS[family]
    specs = [("coarse", boxgen.LAMBDA, [64, 16, 16, 8])]
    specs += [(f"fine{j}", w, [512, 256, 256, 64]) for j, w in enumerate([(0.62, 0.6201), (0.9, 0.9001), (0.985, 0.98501)])]
    for key, outer, sizes in specs:
        lo, hi = oracle.lattice_boxes(family, outer, sizes[:dims], d[f"{key}_idx"])
        rlo, rhi = d[f"{key}_lo"], d[f"{key}_hi"]
        # the lambda axis involves no asin: bit-exact (fused multiply-add form)
        assert (lo[0] == rlo[0]).all() and (hi[0] == rhi[0]).all()
        # radius ranges inherit the single-placement bound (host asin): a few ulps
        assert np.allclose(lo, rlo, rtol=2e-14, atol=0) and np.allclose(hi, rhi, rtol=2e-14, atol=0)


@pytest.mark.parametrize("kind", range(6))
def test_oracle_primitives_match_reference(oracle, kind):
    d = _load("ref_primitives.npz")
    lo, hi, trap = oracle.primitive(kind, d[f"k{kind}_args"])
    assert (trap == d[f"k{kind}_trap"]).all()
    ok = trap == 0
    # angles are differences of asin values near 1: compare with an absolute
    # tolerance of a few ulps of pi/2 (host and CUDA asin differ in the last bits)
    assert np.allclose(lo[ok], d[f"k{kind}_lo"][ok], rtol=1e-12, atol=4e-15)
    assert np.allclose(hi[ok], d[f"k{kind}_hi"][ok], rtol=1e-12, atol=4e-15)


def test_oracle_asin_padding_overlaps_reference(oracle):
    d = _load("ref_primitives.npz")
    rd, ru = oracle.asin_pad(d["asin_x"])
    grd, gru = d["asin_rd"], d["asin_ru"]
    assert (rd <= gru).all() and (grd <= ru).all()
    ulp = np.spacing(np.abs(grd)) + 5e-324
    assert (np.abs(rd - grd) <= 8 * ulp).all() and (np.abs(ru - gru) <= 8 * ulp).all()


def test_oracle_single_placement_matches_reference(oracle):
    d = _load("ref_primitives.npz")
    got = np.array([oracle.single_placement(x) for x in d["single_lambda"]])
    assert np.allclose(got, d["single_out"], rtol=1e-13, atol=0)
