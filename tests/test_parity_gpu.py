"""Parity of the CUDA path with the reference's own device code (bit-exact) and
with the CPU oracle (verdicts; bounds within 1e-12 relative, since the host
libm asin differs from CUDA's in the last bits)."""
import numpy as np
import pytest

from tests import boxgen

pytestmark = pytest.mark.gpu

SIZES_COARSE = [64, 16, 16, 8]
SIZES_FINE = [512, 256, 256, 64]


def _mixed_boxes(oracle, family, seed, n=3000):
    """Lattice boxes (coarse, full lambda range; fine, narrow lambda ranges), random
    sub-boxes and point boxes, as (dims, N) arrays."""
    dims = boxgen.DIMS[family]
    parts = []
    idx = boxgen.lattice_indices(family, SIZES_COARSE[:dims], n, seed)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, SIZES_COARSE[:dims], idx)
    parts.append((lo, hi))
    parts.append(boxgen.sub_boxes(lo, hi, seed + 1))
    parts.append(boxgen.point_boxes(lo, hi, seed + 2))
    for j, outer in enumerate([(0.62, 0.6201), (0.9, 0.9001), (0.985, 0.98501)]):
        idx = boxgen.lattice_indices(family, SIZES_FINE[:dims], n // 3, seed + 10 + j)
        parts.append(oracle.lattice_boxes(family, outer, SIZES_FINE[:dims], idx))
    lo = np.concatenate([p[0] for p in parts], axis=1)
    hi = np.concatenate([p[1] for p in parts], axis=1)
    return lo, hi


@pytest.mark.parametrize("family", range(6))
def test_full_mode_matches_reference_device_code(cp, ref, oracle, family):
    lo, hi = _mixed_boxes(oracle, family, seed=100 + family)
    v, m = cp.eval_boxes(family, lo, hi, mode=cp.EVAL_FULL)
    got = boxgen.product_to_ref_bits(family, v.cpu().numpy(), m.cpu().numpy())
    want = ref.eval_boxes(family, lo, hi)
    trap = (want & 0x80) != 0
    # boxes that reached a trap site: compare the trap / empty / fit flags only
    same = np.where(trap, (got & 0xE0) == (want & 0xE0), got == want)
    bad = np.nonzero(~same)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first: box {bad[0]} got {got[bad[0]]:#x} want {want[bad[0]]:#x}"


@pytest.mark.parametrize("family", range(6))
def test_decide_mode_agrees_with_full(cp, oracle, family):
    lo, hi = _mixed_boxes(oracle, family, seed=200 + family)
    vf, _ = cp.eval_boxes(family, lo, hi, mode=cp.EVAL_FULL)
    for order in (0, 1):
        o = np.full(lo.shape[1], order, np.uint8)
        vd, _ = cp.eval_boxes(family, lo, hi, mode=cp.EVAL_DECIDE, order=o)
        vf_, vd_ = vf.cpu().numpy(), vd.cpu().numpy()
        settled = (vf_ == cp.PROVED) | (vf_ == cp.EMPTY)
        assert (vd_[settled] == vf_[settled]).all()
        assert ((vd_ == cp.PROVED) | (vd_ == cp.EMPTY))[~settled].sum() == 0


@pytest.mark.parametrize("family", range(6))
def test_verdicts_match_cpu_oracle(cp, oracle, family):
    lo, hi = _mixed_boxes(oracle, family, seed=300 + family, n=2000)
    v, m, t = cp.eval_boxes(family, lo, hi, mode=cp.EVAL_FULL, trace=True)
    v, m, t = v.cpu().numpy(), m.cpu().numpy(), t.cpu().numpy()
    ov, om, ot = oracle.eval_boxes(family, lo, hi, trace=True)
    # near-ties: any evaluated criterion within 1e-12 relative of its threshold
    with np.errstate(invalid="ignore"):
        rel = np.abs(ot[:, :, 0] - ot[:, :, 1]) / np.maximum(np.abs(ot[:, :, 1]), 1e-300)
    tie = np.nanmin(np.where(np.isnan(rel), np.inf, rel), axis=1) < 1e-12
    ok = tie | ((v == ov) & (m == om))
    assert ok.all(), f"{(~ok).sum()} verdict mismatches beyond near-ties"
    both = ~np.isnan(t[:, :, 0]) & ~np.isnan(ot[:, :, 0]) & (v != cp.ERROR)[:, None]
    for c in (0, 1):
        a, b = t[:, :, c][both], ot[:, :, c][both]
        assert np.allclose(a, b, rtol=1e-12, atol=1e-300)


def _prim_args(kind, seed, n=4000):
    rng = np.random.default_rng(seed)
    la_lo = rng.uniform(0.5, 0.99, n)
    la_w = np.exp(rng.uniform(np.log(1e-9), np.log(1e-2), n))
    lane = 1.0 - la_lo
    ra_lo = lane * rng.uniform(0.0, 0.5, n)
    ra_w = np.exp(rng.uniform(np.log(1e-12), np.log(1e-2), n)) * lane
    rb_lo = ra_lo * rng.uniform(0.0, 1.0, n)
    rb_w = np.exp(rng.uniform(np.log(1e-12), np.log(1e-2), n)) * lane
    la = (la_lo, la_lo + la_w)
    ra = (ra_lo, ra_lo + ra_w)
    rb = (rb_lo, np.minimum(rb_lo + rb_w, ra_lo + ra_w))
    if kind <= 2:
        rows = [*la, *ra, *rb]
    elif kind == 3:
        rows = [*ra, *rb]
    elif kind == 4:
        rows = [*ra]
    else:
        rows = [*la, *ra]
    return np.array(rows)


@pytest.mark.parametrize("kind", range(6))
def test_primitives_bit_exact(cp, ref, kind):
    args = _prim_args(kind, seed=kind)
    lo, hi, trap = cp.eval_primitive(kind, args)
    rlo, rhi, rtrap = ref.primitive(kind, args)
    lo, hi, trap = lo.cpu().numpy(), hi.cpu().numpy(), trap.cpu().numpy()
    ok = ((lo.view(np.uint64) == rlo.view(np.uint64)) & (hi.view(np.uint64) == rhi.view(np.uint64))) | (rtrap != 0)
    assert ok.all(), f"{(~ok).sum()} primitive mismatches"
    assert (trap == rtrap).all()


def test_asin_padding_bit_exact(cp, ref):
    rng = np.random.default_rng(5)
    tiny = np.array([5e-324, 1e-323, 2.5e-323, 3e-323, 4e-323, 1e-320, 2.2250738585072014e-308])
    x = np.concatenate([rng.uniform(-1, 1, 50000), rng.uniform(0.999, 1.0, 5000), tiny, -tiny,
                        [0.0, -0.0, 1.0, -1.0, 0.5, -0.5]])
    rd, ru = cp.asin_pad(x)
    want_rd, want_ru = ref.asin_pad(x)
    assert (rd.cpu().numpy().view(np.uint64) == want_rd.view(np.uint64)).all()
    assert (ru.cpu().numpy().view(np.uint64) == want_ru.view(np.uint64)).all()


def test_single_placement_bit_exact(cp, ref):
    lam = np.concatenate([np.linspace(0.5, 0.9900000000000001, 3000), np.random.default_rng(3).uniform(0.5, 0.99, 2000)])
    got = cp.single_placement(lam).cpu().numpy()
    want = ref.single_placement(lam)
    assert (got.view(np.uint64) == want.view(np.uint64)).all()


@pytest.mark.parametrize("family", range(6))
def test_lattice_bit_exact(cp, ref, oracle, family):
    dims = boxgen.DIMS[family]
    for sizes, outer in ((SIZES_COARSE, boxgen.LAMBDA), (SIZES_FINE, (0.9, 0.9001)), ([4096, 1024, 1024, 128], boxgen.LAMBDA)):
        idx = boxgen.lattice_indices(family, sizes[:dims], 5000, seed=family)
        lo, hi = cp.lattice_boxes(family, outer, sizes[:dims], idx)
        rlo, rhi = ref.lattice_boxes(family, outer, sizes[:dims], idx)
        assert (lo.cpu().numpy().view(np.uint64) == rlo.view(np.uint64)).all()
        assert (hi.cpu().numpy().view(np.uint64) == rhi.view(np.uint64)).all()


@pytest.mark.parametrize("family", [0, 3, 4])
def test_lattice_fma_form_pinned(ref, oracle, family):
    """The reference's device get_subinterval computes lb + diff*i as one fused
    multiply-add; the CPU oracle's fused form reproduces its la/r bits where no
    asin enters (lambda axis; r ranges bounded by the lane width)."""
    dims = boxgen.DIMS[family]
    sizes = [4096, 1024, 1024, 128][:dims]
    idx = boxgen.lattice_indices(family, sizes, 5000, seed=family)
    rlo, rhi = ref.lattice_boxes(family, boxgen.LAMBDA, sizes, idx)
    flo, fhi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, idx, fused=True)
    ulo, uhi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, idx, fused=False)
    fused_same = (flo[0] == rlo[0]).all() and (fhi[0] == rhi[0]).all()
    assert fused_same
    # the unfused form differs somewhere on this lattice, so the test discriminates
    assert not ((ulo[0] == rlo[0]).all() and (uhi[0] == rhi[0]).all())


@pytest.mark.parametrize("family", [1, 3])
def test_host_entry_matches_device_entry(cp, oracle, family):
    lo, hi = _mixed_boxes(oracle, family, seed=400 + family, n=500)
    v, m = cp.eval_boxes(family, lo, hi)
    hv, hm = cp.eval_boxes_host(family, lo, hi)
    assert (v.cpu().numpy() == hv).all() and (m.cpu().numpy() == hm).all()


@pytest.mark.parametrize("family", range(6))
def test_fp32_prepass_reproduces_fp64(cp, oracle, family):
    """The FP32 certified shadow issues a verdict only when it equals the FP64
    one: DECIDE verdict and mask per box, and the FULL-mode result."""
    lo, hi = _mixed_boxes(oracle, family, seed=500 + family)
    for mode in (cp.EVAL_DECIDE, cp.EVAL_FULL):
        for order in (0, 1):
            o = np.full(lo.shape[1], order, np.uint8)
            v64, m64 = cp.eval_boxes(family, lo, hi, precision=cp.FP64, mode=mode, order=o)
            v32, m32 = cp.eval_boxes(family, lo, hi, precision=cp.FP32_PREFILTER, mode=mode, order=o)
            assert (v64.cpu().numpy() == v32.cpu().numpy()).all()
            assert (m64.cpu().numpy() == m32.cpu().numpy()).all()


@pytest.mark.parametrize("family", [0, 3, 5])
def test_fp32_prepass_decides_most_fine_boxes(cp, oracle, family):
    """On fine lattice boxes (mostly proved) the pre-pass settles most of them;
    measured through the refinement report."""
    dims = boxgen.DIMS[family]
    p = cp.Prover(0)
    r = p.refine(family, precision=cp.FP32_PREFILTER, max_depth=0, seed_sizes=[64, 32, 32, 8][:dims],
                 seed_lambda=(0.6, 0.6005))
    p.close()
    assert r["fp32_decided"] >= 0.5 * r["evaluated"]
