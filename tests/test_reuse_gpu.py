"""Reuse of the start family's lambda-independent criterion terms
(cp_refine_opts.reuse): a child whose radii equal its parent's -- every child
of a lambda-only split that clipping to the dependent ranges leaves alone --
takes its parent's collision angle of disks 1 and 3 and semicircle angle of r1
(start_configuration.cu:126-162) instead of recomputing them.  The values are
functions of the radii alone, so the refinement must evaluate the same boxes
with the same verdicts as one that recomputes every term: equal per-box
digests, verdict counts and per-depth histograms, in every engine and
precision."""
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("evaluated", "verdicts", "unresolved", "clipped", "per_depth", "digest")


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("policy", [1, 4, 2])  # lambda only, hybrid, widest
def test_reuse_matches_recompute(cp, prover, policy, engine, precision):
    kw = dict(policy=policy, max_depth=10, seed_sizes=[8, 16, 16, 8], digest=True, engine=engine,
              precision=precision, level_capacity=1 << 22)
    a = prover.refine(cp.START, reuse=True, **kw)
    b = prover.refine(cp.START, reuse=False, **kw)
    for k in KEYS:
        assert a[k] == b[k], k
    assert a["evaluated"] > 4 * 8 * 16 * 16 * 8 // 2  # children were evaluated, not only the seed


def test_reuse_on_a_proof_slab(cp, prover):
    """The last lambda slab of the start proof (1 - lambda in its narrowest
    band) seeded with a coarse radius lattice, so that most boxes stay
    unresolved down to the depth limit: twelve levels of lambda-only children
    (at most 65536 * 2^12 boxes)."""
    lo, hi = 1.0 - 0.5 * (0.01 / 0.5) ** (17 / 18), cp.LAMBDA_MAX
    kw = dict(policy=cp.SPLIT_LAMBDA, max_depth=12, seed_sizes=[1, 64, 64, 16], seed_lambda=(lo, hi),
              digest=True, engine=cp.ENGINE_GRAPH, level_capacity=1 << 22)
    a = prover.refine(cp.START, reuse=True, **kw)
    b = prover.refine(cp.START, reuse=False, **kw)
    for k in KEYS:
        assert a[k] == b[k], k
    assert a["max_depth_seen"] >= 8


def test_reuse_switch_between_refinements(cp, prover):
    """Levels that hold terms from a refinement with reuse do not leak into a
    later refinement without it, nor into another family's."""
    kw = dict(policy=cp.SPLIT_LAMBDA, max_depth=8, seed_sizes=[8, 8, 8, 4], digest=True, level_capacity=1 << 20)
    ref = prover.refine(cp.START, reuse=False, **kw)
    prover.refine(cp.START, reuse=True, **kw)
    again = prover.refine(cp.START, reuse=False, **kw)
    mid_a = prover.refine(cp.MIDDLE, reuse=True, **kw)
    prover.refine(cp.START, reuse=True, **kw)
    mid_b = prover.refine(cp.MIDDLE, reuse=False, **kw)
    for k in KEYS:
        assert again[k] == ref[k], k
        assert mid_a[k] == mid_b[k], k
