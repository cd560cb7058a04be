"""Full-domain proofs on the GPU: the families other than start are proved over
their whole domain (lambda in [0.5, 0.99] and the dependent radius ranges) by
lambda-only bisection -- the reference's own refinement rule, applied per box --
from one lattice seed over the whole lambda range with the resolution the
family needs (start, proved by lambda slabs, has its own test at the end).
Both engines evaluate the same tree of boxes."""
import pytest

pytestmark = pytest.mark.gpu

SEEDS = {1: (64, 32, 32), 2: (64, 64, 64, 16), 3: (51, 26, 21, 1), 4: (33, 66, 53), 5: (41, 17, 17, 4)}


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



@pytest.mark.parametrize("family", [1, 3, 5])
def test_prove_family_driver_matches_refinement(cp, prover, family):
    """cp_prove_family with the library's defaults for a family runs the same
    refinement as the explicit cp_refine call above (one slab, the family's
    seed lattice), box for box: same counts and the same per-box verdict digest
    in both engines."""
    d = prover.proof_defaults(family)
    assert d["slabs"] == 1 and d["policy"] == cp.SPLIT_LAMBDA
    assert tuple(d["seed_sizes"][:cp.DIMS[family]]) == SEEDS[family]
    kw = dict(policy=cp.SPLIT_LAMBDA, max_depth=d["max_depth"], seed_sizes=list(SEEDS[family]),
              seed_lambda=(cp.LAMBDA_MIN, cp.LAMBDA_MAX), level_capacity=d["level_capacity"], digest=True)
    want = prover.refine(family, **kw)
    for engine in (cp.ENGINE_GRAPH, cp.ENGINE_LEVELS):
        got = prover.prove_family(family, engine=engine, digest=1)
        assert got["proved"] and got["slabs_done"] == 1 and got["first_unresolved_slab"] == -1
        for k in ("evaluated", "verdicts", "unresolved", "clipped", "per_depth", "digest"):
            assert got[k] == want[k], (engine, k)


def test_prove_family_slabs_add_up(cp, prover):
    """Geometric lambda slabs: the slabs tile [0.5, 0.99], and a proof over k
    slabs reports the sums of the k slab refinements."""
    family = cp.END_3D
    got = prover.prove_family(family, slabs=4, geometric=1, seed_sizes=[16, 32, 32, 8], digest=1)
    assert got["slabs_done"] == 4
    lo = cp.LAMBDA_MIN
    tot_eval, tot_dig = 0, [0, 0]
    for k in range(4):
        # the library's cut: 1 - lambda from 0.5 to 0.01 by a constant factor (same expression, same libm pow)
        hi = cp.LAMBDA_MAX if k == 3 else 1.0 - (1.0 - cp.LAMBDA_MIN) * (
            ((1.0 - cp.LAMBDA_MAX) / (1.0 - cp.LAMBDA_MIN)) ** ((k + 1) / 4))
        r = prover.refine(family, policy=cp.SPLIT_LAMBDA, max_depth=24, seed_sizes=[16, 32, 32, 8],
                          seed_lambda=(lo, hi), level_capacity=1 << 23, engine=cp.ENGINE_GRAPH, digest=True)
        tot_eval += r["evaluated"]
        tot_dig = [(tot_dig[0] + r["digest"][0]) % (1 << 64), tot_dig[1] ^ r["digest"][1]]
        lo = hi
    assert got["evaluated"] == tot_eval and list(got["digest"]) == tot_dig


def test_slab_radii_set_each_slab_lattice(cp, prover):
    """cp_proof_opts.slab_radii: slab k seeds its own r1 x r2 x r3 subdivisions
    where given (here [16, 16, 4] in slab 0; slab 1 keeps seed_sizes); the proof
    reports the sums of the two slab refinements."""
    family = cp.END_3D
    got = prover.prove_family(family, slabs=2, geometric=1, seed_sizes=[16, 32, 32, 8], slab_radii=[[16, 16, 4]],
                              max_depth=16, digest=1)
    assert got["slabs_done"] == 2
    mid = 1.0 - (1.0 - cp.LAMBDA_MIN) * (((1.0 - cp.LAMBDA_MAX) / (1.0 - cp.LAMBDA_MIN)) ** 0.5)
    tot_eval, tot_dig = 0, [0, 0]
    for lam, sizes in (((cp.LAMBDA_MIN, mid), [16, 16, 16, 4]), ((mid, cp.LAMBDA_MAX), [16, 32, 32, 8])):
        r = prover.refine(family, policy=cp.SPLIT_LAMBDA, max_depth=16, seed_sizes=sizes, seed_lambda=lam,
                          level_capacity=1 << 23, engine=cp.ENGINE_GRAPH, digest=True)
        tot_eval += r["evaluated"]
        tot_dig = [(tot_dig[0] + r["digest"][0]) % (1 << 64), tot_dig[1] ^ r["digest"][1]]
    assert got["evaluated"] == tot_eval and list(got["digest"]) == tot_dig


def test_start_proved_over_full_domain(cp, prover):
    """The start family's proof with the library's defaults (18 geometric lambda
    slabs, a radius lattice per slab): every box proved, empty or clipped, in
    both engines, with and without reuse of the parents' lambda-independent
    terms, and the four runs evaluate the same boxes with the same verdicts."""
    runs = [prover.prove_family(cp.START, engine=e, reuse=u, digest=1)
            for e in (cp.ENGINE_GRAPH, cp.ENGINE_LEVELS) for u in (0, 1)]
    for r in runs:
        assert r["proved"] and r["unresolved"] == 0 and r["slabs_done"] == 18
        for k in ("evaluated", "verdicts", "clipped", "per_depth", "digest"):
            assert r[k] == runs[0][k], k
    assert runs[0]["verdicts"][1] > 0  # boxes were critical at coarser levels and got refined


def test_start_end_3d_proved_by_slabs(cp, prover):
    """start_end_3d's default proof (18 geometric lambda slabs, a radius
    lattice per slab): proved in both engines, with the same boxes and
    verdicts."""
    runs = [prover.prove_family(cp.START_END_3D, engine=e, digest=1) for e in (cp.ENGINE_GRAPH, cp.ENGINE_LEVELS)]
    for r in runs:
        assert r["proved"] and r["unresolved"] == 0 and r["slabs_done"] == 18
        for k in ("evaluated", "verdicts", "clipped", "per_depth", "digest"):
            assert r[k] == runs[0][k], k
