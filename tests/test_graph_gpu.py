"""The device-driven refinement engine (one CUDA graph launch: scheduler kernel
+ persistent level kernel in a WHILE loop) against the host-driven level loop:
identical reports for every family, split policy, precision and kernel shape,
for lattice seeds and for explicit seeds at uneven depths."""
import numpy as np
import pytest

from tests import boxgen

pytestmark = pytest.mark.gpu

KEYS = ("evaluated", "verdicts", "unresolved", "clipped", "fp32_decided", "per_depth", "handles_evaluated")


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


def _same(a, b):
    for k in KEYS:
        assert a[k] == b[k], (k, a[k], b[k])


@pytest.mark.parametrize("family", range(6))
@pytest.mark.parametrize("policy,depth", [(0, 2), (1, 6), (2, 7), (4, 9)])
def test_graph_matches_level_loop(cp, prover, family, policy, depth):
    dims = boxgen.DIMS[family]
    kw = dict(policy=policy, max_depth=depth, seed_sizes=[16, 8, 8, 4][:dims], level_capacity=1 << 20)
    want = prover.refine(family, **kw)
    got = prover.refine(family, engine=cp.ENGINE_GRAPH, **kw)
    _same(want, got)
    assert got["launches"] >= 1


@pytest.mark.parametrize("block", [64, 128, 256, 512, 1024])
@pytest.mark.parametrize("bpt", [1, 3, 8])
def test_graph_kernel_shapes(cp, prover, block, bpt):
    kw = dict(policy=cp.SPLIT_WIDEST, max_depth=5, seed_sizes=[16, 8, 8, 4], level_capacity=1 << 19)
    want = prover.refine(cp.MIDDLE, **kw)
    got = prover.refine(cp.MIDDLE, engine=cp.ENGINE_GRAPH, block=block, boxes_per_thread=bpt, **kw)
    _same(want, got)


@pytest.mark.parametrize("family,precision", [(3, 0), (5, 1), (0, 1), (4, 0)])
def test_graph_uneven_depth_seeds(cp, oracle, prover, family, precision):
    """Explicit seeds at depths 0..8 (random sub-boxes of a lattice) in one worklist."""
    dims = boxgen.DIMS[family]
    idx = boxgen.lattice_indices(family, [64, 16, 16, 8][:dims], 4000, 21 + family)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, [64, 16, 16, 8][:dims], idx)
    lo, hi = boxgen.sub_boxes(lo, hi, 22 + family)
    depth = np.random.default_rng(23).integers(0, 9, lo.shape[1]).astype(np.uint8)
    kw = dict(policy=cp.SPLIT_WIDEST, max_depth=12, precision=precision, level_capacity=1 << 20)
    want = prover.refine_boxes(family, lo, hi, depth=depth, **kw)
    got = prover.refine_boxes(family, lo, hi, depth=depth, engine=cp.ENGINE_GRAPH, **kw)
    _same(want, got)


def test_graph_capacity_error(cp, prover):
    """The level stack sizes every chunk to the room left in the next level, so
    it only overflows when a level cannot hold one box's children (16 > 8)."""
    lo, hi, vis = cp.lattice_boxes(cp.MIDDLE, boxgen.LAMBDA, [2, 2, 2, 1], np.arange(8), visited=True)
    kw = dict(policy=cp.SPLIT_UNIFORM, max_depth=3, level_capacity=8)
    for engine in (cp.ENGINE_LEVELS, cp.ENGINE_GRAPH):
        with pytest.raises(cp.ProverError) as e:
            prover.refine_boxes(cp.MIDDLE, lo, hi, engine=engine, **kw)
        assert e.value.status == 4  # CP_ERR_CAPACITY
    # the handle stays usable
    r = prover.refine(cp.MIDDLE, engine=cp.ENGINE_GRAPH, policy=cp.SPLIT_WIDEST, max_depth=3,
                      seed_sizes=[8, 4, 4, 2], level_capacity=1 << 18)
    assert r["evaluated"] == sum(r["per_depth"])


def test_graph_learned_hints_match_level_loop(cp, prover):
    from oracle import mlp

    family = cp.END_3D
    prover.model_set_params(family, mlp.init_params(77))
    for kw in (dict(policy=cp.SPLIT_LEARNED), dict(policy=cp.SPLIT_WIDEST, learned_order=True)):
        kw.update(max_depth=7, seed_sizes=[16, 8, 8, 4], level_capacity=1 << 20)
        want = prover.refine(family, **kw)
        got = prover.refine(family, engine=cp.ENGINE_GRAPH, **kw)
        _same(want, got)


def test_graph_autotune(cp, prover):
    blk, bpt, ms = prover.autotune_graph(cp.MIDDLE, policy=cp.SPLIT_UNIFORM, max_depth=1, seed_sizes=[16, 8, 8, 8])
    assert blk in cp.GRAPH_BLOCKS and bpt in cp.GRAPH_BPT
    assert all(m > 0 for row in ms for m in row)
