"""Full-domain proofs on the GPU: five of the six families (all but start) are
proved over their whole domain (lambda in [0.5, 0.99] and the dependent radius
ranges) by lambda-only bisection -- the reference's own refinement rule, applied
per box -- from a lattice seed with 64 lambda slabs and the radius resolution
each family needs.  Both engines evaluate the same tree of boxes."""
import pytest

pytestmark = pytest.mark.gpu

SEEDS = {1: (64, 32, 32), 2: (64, 64, 64, 16), 3: (64, 32, 32, 8), 4: (64, 128, 128), 5: (64, 32, 32, 8)}


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


@pytest.mark.parametrize("family", [1, 2, 3, 4, 5])
def test_family_proved_over_full_domain(cp, prover, family):
    kw = dict(policy=cp.SPLIT_LAMBDA, max_depth=24, seed_sizes=list(SEEDS[family]),
              seed_lambda=(cp.LAMBDA_MIN, cp.LAMBDA_MAX), level_capacity=1 << 23)
    a = prover.refine(family, **kw)
    b = prover.refine(family, engine=cp.ENGINE_GRAPH, **kw)
    for k in ("evaluated", "verdicts", "unresolved", "clipped", "per_depth"):
        assert a[k] == b[k], k
    assert a["unresolved"] == 0, a
    assert a["verdicts"][cp.ERROR] == 0
    # every box was either proved, empty, or refined further (the leaves all proved)
    assert a["evaluated"] == sum(a["per_depth"]) and len(a["per_depth"]) - 1 <= 24
