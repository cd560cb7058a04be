"""Per-box verdict digests and the seeded random-box workload on the GPU.

The digest (cp_refine_opts.digest) folds every evaluated (box, verdict) pair
into an order-independent sum and xor of 64-bit hashes; two forms of a
refinement that evaluate the same boxes with the same verdicts must report the
same digest.  The hash is restated here in numpy, so the device digest of a
refinement without children is checked box by box against the verdicts
cp_eval_boxes returns."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from tests.boxgen import M64, host_digest


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


@pytest.mark.parametrize("family", [0, 1, 3, 5])
def test_digest_of_seed_matches_host_hash(cp, prover, family):
    """max_depth 0: the refinement evaluates the seed lattice only; its digest is
    the host hash of those boxes with cp_eval_boxes' DECIDE verdicts."""
    dims = cp.DIMS[family]
    sizes = [16, 8, 8, 4][:dims]
    r = prover.refine(family, max_depth=0, seed_sizes=sizes, digest=True)
    import torch

    total = int(np.prod(sizes))
    lo, hi, vis = cp.lattice_boxes(family, (cp.LAMBDA_MIN, cp.LAMBDA_MAX), sizes, np.arange(total), visited=True)
    keep = vis.bool()
    lo, hi = lo[:, keep].contiguous(), hi[:, keep].contiguous()
    v, _ = cp.eval_boxes(family, lo, hi, mode=cp.EVAL_DECIDE)
    torch.cuda.synchronize()
    v = v.cpu().numpy()
    assert r["evaluated"] == v.size
    assert r["digest"] == host_digest(lo.cpu().numpy(), hi.cpu().numpy(), v)


@pytest.mark.parametrize("family", [2, 3, 4])
def test_digest_identical_across_forms(cp, prover, family):
    """Graph engine and level loop, FP64 and the FP32 pre-pass: same boxes, same
    verdicts, same digest; another split policy gives another digest."""
    dims = cp.DIMS[family]
    kw = dict(policy=cp.SPLIT_UNIFORM, max_depth=2, seed_sizes=[8, 8, 8, 4][:dims], digest=True)
    base = prover.refine(family, **kw)
    assert base["digest"] != (0, 0)
    for extra in (dict(engine=cp.ENGINE_GRAPH), dict(precision=cp.FP32_PREFILTER),
                  dict(engine=cp.ENGINE_GRAPH, precision=cp.FP32_PREFILTER)):
        r = prover.refine(family, **kw, **extra)
        assert r["digest"] == base["digest"], extra
        assert r["verdicts"] == base["verdicts"]
    other = prover.refine(family, **dict(kw, policy=cp.SPLIT_LAMBDA))
    assert other["digest"] != base["digest"]
    off = prover.refine(family, **dict(kw, digest=False))
    assert off["digest"] == (0, 0) and off["verdicts"] == base["verdicts"]


def test_digest_is_additive_over_seed_sets(cp, prover):
    """The digest of a refinement from seeds A and B together is the sum (mod
    2^64) and xor of the digests from A and from B alone."""
    family = cp.MIDDLE
    lo, hi, dp = prover.random_boxes(family, 6000, seed=11, max_label=3)
    kw = dict(policy=cp.SPLIT_WIDEST, max_depth=4, digest=True)
    both = prover.refine_boxes(family, lo, hi, depth=dp, **kw)
    a = prover.refine_boxes(family, lo[:, :2500].contiguous(), hi[:, :2500].contiguous(), depth=dp[:2500], **kw)
    b = prover.refine_boxes(family, lo[:, 2500:].contiguous(), hi[:, 2500:].contiguous(), depth=dp[2500:], **kw)
    assert both["evaluated"] == a["evaluated"] + b["evaluated"]
    assert both["digest"][0] == (a["digest"][0] + b["digest"][0]) & M64
    assert both["digest"][1] == a["digest"][1] ^ b["digest"][1]


@pytest.mark.parametrize("family", [1, 3, 5])
def test_random_boxes_deterministic_and_in_domain(cp, prover, family):
    import torch

    n = 200000
    lo, hi, dp = prover.random_boxes(family, n, seed=0xC1C1E5, max_label=8)
    lo2, hi2, dp2 = prover.random_boxes(family, n, seed=0xC1C1E5, max_label=8)
    lo3, _, _ = prover.random_boxes(family, n, seed=0xC1C1E6, max_label=8)
    assert torch.equal(lo, lo2) and torch.equal(hi, hi2) and torch.equal(dp, dp2)
    assert not torch.equal(lo, lo3)
    lo, hi, dp = lo.cpu().numpy(), hi.cpu().numpy(), dp.cpu().numpy()
    alive = dp != 255
    assert alive.mean() > 0.5
    assert set(np.unique(dp[alive]).tolist()) == set(range(9))
    assert (lo[:, alive] <= hi[:, alive]).all()
    assert (lo[0, alive] >= cp.LAMBDA_MIN).all() and (hi[0, alive] <= cp.LAMBDA_MAX).all()
    # radii: within the family's dependent ranges (whose lower ends may be negative
    # for the start+end ranges, start_configuration.cu:74-77), never above 0.25
    assert (hi[1:, alive] <= 0.25).all() and (lo[1:, alive] > -0.25).all()
    w = hi[:, alive] - lo[:, alive]
    assert (w <= 2.0 ** -4 * (1 + 1e-12)).all()
    # radii never exceed the radius before them (the dependent ranges)
    assert (lo[2, alive] <= hi[1, alive]).all()
