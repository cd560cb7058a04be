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



@pytest.mark.parametrize("family", [1, 3, 5])
def test_prove_family_driver_matches_refinement(cp, prover, family):
    """cp_prove_family with the library's defaults for a family runs the same
    refinement as the explicit cp_refine call above (one slab of 64 lambda
    cells), box for box: same counts and the same per-box verdict digest in
    both engines."""
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


def test_slab_scale_scales_each_slab_lattice(cp, prover):
    """cp_proof_opts.slab_scale: slab k scales the radius subdivisions of the
    seed by slab_scale[k] / 256 (here 128: [16, 16, 16, 4] in slab 0; 256: the
    given [16, 32, 32, 8] in slab 1); the proof reports the sums of the two slab
    refinements."""
    family = cp.END_3D
    got = prover.prove_family(family, slabs=2, geometric=1, seed_sizes=[16, 32, 32, 8], slab_scale=[128, 256],
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
