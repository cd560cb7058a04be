"""Full-domain proofs on the GPU: the start+end (2 disks), middle and end (3
disks) families are proved over their whole domain (lambda in [0.5, 0.99] and
the dependent radius ranges) by lambda-only bisection -- the reference's own
refinement rule, applied per box -- from a 64 x 32 x 32 (x 8) lattice seed.  Both
engines evaluate the same tree of boxes."""
import pytest

pytestmark = pytest.mark.gpu

SEED = (64, 32, 32, 8)


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


@pytest.mark.parametrize("family", [1, 3, 5])
def test_family_proved_over_full_domain(cp, prover, family):
    kw = dict(policy=cp.SPLIT_LAMBDA, max_depth=24, seed_sizes=list(SEED[:cp.DIMS[family]]),
              seed_lambda=(cp.LAMBDA_MIN, cp.LAMBDA_MAX), level_capacity=1 << 23)
    a = prover.refine(family, **kw)
    b = prover.refine(family, engine=cp.ENGINE_GRAPH, **kw)
    for k in ("evaluated", "verdicts", "unresolved", "clipped", "per_depth"):
        assert a[k] == b[k], k
    assert a["unresolved"] == 0, a
    assert a["verdicts"][cp.ERROR] == 0
    # every box was either proved, empty, or refined further (the leaves all proved)
    assert a["evaluated"] == sum(a["per_depth"]) and len(a["per_depth"]) - 1 <= 24
