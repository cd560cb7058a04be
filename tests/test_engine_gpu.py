"""The refinement engine and the reference-semantics lambda loop on the GPU."""
import numpy as np
import pytest

from tests import boxgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


@pytest.mark.parametrize("family", range(6))
def test_refine_depth0_counts_match_oracle(cp, oracle, prover, family):
    dims = boxgen.DIMS[family]
    sizes = [32, 8, 8, 4][:dims]
    r = prover.refine(family, max_depth=0, seed_sizes=sizes)
    total = int(np.prod(sizes))
    # the device lattice (its radius ranges use CUDA's asin through the
    # single-placement bound, so the host lattice may differ in the last bit)
    lo, hi, vis = cp.lattice_boxes(family, boxgen.LAMBDA, sizes, np.arange(total), visited=True)
    vis = vis.cpu().numpy().astype(bool)
    v, _ = oracle.eval_boxes(family, lo.cpu().numpy()[:, vis], hi.cpu().numpy()[:, vis])
    assert r["evaluated"] == int(vis.sum()) and r["clipped"] == int((~vis).sum())
    assert r["verdicts"][cp.PROVED] == int((v == 0).sum())
    assert r["verdicts"][cp.EMPTY] == int((v == 3).sum())
    assert r["unresolved"] == int(((v != 0) & (v != 3)).sum())


@pytest.mark.parametrize("family", range(6))
@pytest.mark.parametrize("policy", [0, 1, 2])
def test_refine_prefilter_verdicts_identical(cp, prover, family, policy):
    dims = boxgen.DIMS[family]
    kw = dict(policy=policy, max_depth=3, seed_sizes=[16, 8, 8, 4][:dims])
    a = prover.refine(family, precision=cp.FP64, **kw)
    b = prover.refine(family, precision=cp.FP32_PREFILTER, **kw)
    assert a["verdicts"] == b["verdicts"] and a["unresolved"] == b["unresolved"] and a["clipped"] == b["clipped"]
    assert a["evaluated"] == sum(a["per_depth"])
    assert b["fp32_decided"] <= b["evaluated"]


@pytest.mark.parametrize("family", [0, 3, 5])
def test_refine_boxes_entries_agree(cp, prover, family):
    dims = boxgen.DIMS[family]
    sizes = [16, 8, 8, 4][:dims]
    total = int(np.prod(sizes))
    lo, hi, vis = cp.lattice_boxes(family, boxgen.LAMBDA, sizes, np.arange(total), visited=True)
    depth = np.where(vis.cpu().numpy() != 0, 0, 255).astype(np.uint8)  # 255: never visited (dropped)
    kw = dict(policy=cp.SPLIT_WIDEST, max_depth=4)
    a = prover.refine(family, seed_sizes=sizes, **kw)
    b = prover.refine_boxes(family, lo, hi, depth=depth, **kw)
    c = prover.refine_boxes(family, lo.cpu().numpy(), hi.cpu().numpy(), depth=depth, **kw)
    for k in ("evaluated", "verdicts", "unresolved", "clipped"):
        assert a[k] == b[k] == c[k]


def test_refine_capacity_chunking_is_transparent(cp, prover):
    """A small level capacity forces many chunks; the outcome does not change."""
    kw = dict(policy=cp.SPLIT_UNIFORM, max_depth=2, seed_sizes=[16, 8, 8, 4])
    a = prover.refine(3, **kw)
    b = prover.refine(3, level_capacity=4096, **kw)
    assert a["verdicts"] == b["verdicts"] and a["unresolved"] == b["unresolved"]
    assert b["launches"] > a["launches"]


@pytest.mark.parametrize("family", range(6))
def test_reference_step_matches_reference_kernel(cp, ref, prover, family):
    """One launch over [0.5, 0.99] with the reference's lattice: the same first
    failing lambda as the reference's own kernel (run_kernel.cuh:81-84)."""
    ref.trap_count_reset()
    want, _ = ref.kernel_once(family, cp.LAMBDA_MIN, cp.LAMBDA_MAX)
    ref_traps = ref.trap_count_reset()
    assert want != np.finfo(np.float64).max
    try:
        got = prover.reference_step(family, cp.LAMBDA_MIN, cp.LAMBDA_MAX)
    except cp.ProverError as e:
        # the engine reports a trap only where the reference kernel reaches one too
        assert ref_traps > 0 and e.status in (6, 7), (e, ref_traps)
        return
    assert got == want


def test_reference_step_proved_interval(cp, ref, prover):
    want, _ = ref.kernel_once(3, 0.6, 0.6005)
    got = prover.reference_step(3, 0.6, 0.6005)
    assert want == np.finfo(np.float64).max and got == np.inf


@pytest.mark.parametrize("family", [0, 3, 4])
def test_reference_loop_trace_matches_cpu_restatement(cp, oracle, prover, family):
    dims = boxgen.DIMS[family]
    sizes = [16, 4, 4, 2][:dims]
    steps, _ = oracle.reference_loop(family, sizes, max_steps=30)
    d = prover.prove_family_reference(family, sizes=sizes, max_launches=30, trace_cap=30)
    tr = d["trace"]
    n = min(len(tr), len(steps))
    assert n > 0
    assert np.array_equal(tr[:n, :2], steps[:n, :2])
    assert np.array_equal(tr[:n, 2], steps[:n, 2])


@pytest.mark.parametrize("family", [0, 3, 4])
def test_reference_criticals_consistent(cp, oracle, prover, family):
    dims = boxgen.DIMS[family]
    sizes = [16, 8, 8, 4][:dims]
    count, boxes, handles = prover.reference_criticals(family, 0.5, 0.6, sizes=sizes, max_boxes=100000)
    total = int(np.prod(sizes))
    lo, hi, vis = cp.lattice_boxes(family, (0.5, 0.6), sizes, np.arange(total), visited=True)
    vis = vis.cpu().numpy().astype(bool)
    v, m = oracle.eval_boxes(family, lo.cpu().numpy()[:, vis], hi.cpu().numpy()[:, vis])
    crit = (m & 0x3F) != 0
    assert count == int(crit.sum())
    assert len(boxes) == count and (handles != 0).all()


@pytest.mark.parametrize("family", [0, 3, 4])
def test_autotune_variants_keep_verdicts(cp, prover, family):
    dims = boxgen.DIMS[family]
    kw = dict(policy=cp.SPLIT_UNIFORM, max_depth=1, seed_sizes=[16, 8, 8, 4][:dims])
    best, ms = prover.autotune(family, **kw)
    assert 0 <= best < 4 and all(m > 0 for m in ms)
    outs = []
    for v in range(4):
        prover.set_level_variant(family, cp.FP64, v)
        outs.append(prover.refine(family, **kw))
    assert all(o["verdicts"] == outs[0]["verdicts"] and o["unresolved"] == outs[0]["unresolved"] for o in outs)


@pytest.mark.parametrize("family", range(6))
def test_cpu_restated_refinement_matches_device(cp, oracle, family):
    """The CPU restatement of the uniform refinement (the bench's CPU baseline
    workload) evaluates the same tree as the device engine below the same seed
    boxes: equal boxes per depth and verdict counts, up to the rare boxes whose
    criteria sit within the host-libm / CUDA asin difference of a threshold."""
    dims = cp.DIMS[family]
    sizes = [64] * dims
    idx = np.sort(np.random.default_rng(40 + family).choice(64 ** dims, 300, replace=False))
    want = oracle.refine_sample(family, sizes, idx, 2)
    lo, hi, vis = cp.lattice_boxes(family, (cp.LAMBDA_MIN, cp.LAMBDA_MAX), sizes, idx, visited=True)
    import torch

    dp = torch.where(vis != 0, 0, 255).to(torch.uint8)
    p = cp.Prover(0)
    try:
        got = p.refine_boxes(family, lo, hi, depth=dp, policy=cp.SPLIT_UNIFORM, max_depth=2)
    finally:
        p.close()
    for d in range(3):
        a, b = want["per_depth"][d], got["per_depth"][d] if d < len(got["per_depth"]) else 0
        assert abs(a - b) <= 1e-3 * max(a, b) + 2, (d, a, b)
    for v in range(5):
        a, b = want["verdicts"][v], got["verdicts"][v]
        assert abs(a - b) <= 1e-3 * max(a, b) + 2, (v, a, b)


def test_staged_host_seeds_match_host_entry(cp):
    """cp_stage_boxes_host + cp_refine_staged give the report of
    cp_refine_boxes_host, with the two slots alternating and the next slot's
    copy in flight while a refinement runs."""
    import torch

    p = cp.Prover(0)
    try:
        sets = []
        for f, sizes in ((cp.MIDDLE, [16, 8, 8, 4]), (cp.END_2D, [16, 16, 8]), (cp.START, [8, 8, 8, 4])):
            lo, hi, vis = cp.lattice_boxes(f, (cp.LAMBDA_MIN, cp.LAMBDA_MAX), sizes,
                                           np.arange(int(np.prod(sizes))), visited=True)
            hlo = torch.empty(lo.shape, dtype=torch.float64, pin_memory=True)
            hhi = torch.empty(hi.shape, dtype=torch.float64, pin_memory=True)
            hdp = torch.empty(vis.shape, dtype=torch.uint8, pin_memory=True)
            hlo.copy_(lo)
            hhi.copy_(hi)
            hdp.copy_(torch.where(vis != 0, 0, 255).to(torch.uint8))
            sets.append((f, hlo.numpy(), hhi.numpy(), hdp.numpy()))
        kw = dict(policy=cp.SPLIT_UNIFORM, max_depth=2, digest=True, engine=cp.ENGINE_GRAPH)
        want = [p.refine_boxes(f, lo, hi, depth=dp, **kw) for f, lo, hi, dp in sets]
        jobs = sets + sets
        p.stage_boxes(0, *jobs[0][1:])
        for k, (f, lo, hi, dp) in enumerate(jobs):
            if k + 1 < len(jobs):
                p.stage_boxes((k + 1) % 2, *jobs[k + 1][1:])
            got = p.refine_staged(f, k % 2, **kw)
            for key in ("evaluated", "verdicts", "unresolved", "clipped", "per_depth", "digest"):
                assert got[key] == want[k % len(sets)][key], (k, key)
        # a slot keeps its boxes on the device: refining it again gives the same report
        k = len(jobs) - 1
        again = p.refine_staged(jobs[k][0], k % 2, **kw)
        assert again["digest"] == want[k % len(sets)]["digest"]
        with pytest.raises(cp.ProverError):
            p.refine_staged(cp.END_2D, k % 2, **kw)  # 4-axis boxes staged, 3-axis family
    finally:
        p.close()
