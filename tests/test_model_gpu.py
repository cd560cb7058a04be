"""The learned proposal model on the GPU: BF16 tensor-core forward/backward
against the CPU restatement (oracle/mlp.py), trace labels against the CPU
oracle, training, and what the trained network gains over the plain method
(fewer guarded criteria evaluated per box, identical verdicts)."""
import numpy as np
import pytest

from oracle import mlp
from tests import boxgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prover(cp):
    p = cp.Prover(0)
    yield p
    p.close()


def _rows(seed, n):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 16), np.float32)
    x[:, :9] = rng.uniform(-1.2, 1.2, (n, 9))
    crit = rng.integers(0, 16, n).astype(np.uint8)
    axis = rng.integers(-1, 4, n).astype(np.int8)
    return x, crit, axis


@pytest.mark.parametrize("kind", [0, 1], ids=["mma_sync", "tcgen05"])
@pytest.mark.parametrize("family,n", [(3, 200), (5, 64), (4, 1000), (0, 130)])
def test_gradient_matches_oracle(cp, family, n, kind):
    """Loss and gradient of one forward + backward pass on the GPU against the
    CPU restatement, for both training kernels (warp-level mma.sync and tcgen05
    with tensor-memory accumulators)."""
    p = mlp.init_params(11 + family)
    x, crit, axis = _rows(family, n)
    axis = np.where(axis >= boxgen.DIMS[family], -1, axis).astype(np.int8)
    loss, grad = cp.model_loss_grad(family, p, x, crit, axis, kind=kind)
    want_loss, want_grad = mlp.loss_grad(family, p, x, crit, axis)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss) + 1e-6
    # BF16 operands: the GPU (FP32 accumulation) and the oracle (FP64) may round an
    # intermediate activation to neighbouring BF16 values; compare norm-wise
    err = np.linalg.norm(grad - want_grad) / np.linalg.norm(want_grad)
    assert err < 1e-2, err
    for name, (a, b) in zip([s[0] for s in mlp.SHAPES], zip(np.split(grad, np.cumsum(
            [int(np.prod(s[1])) for s in mlp.SHAPES])[:-1]), np.split(want_grad, np.cumsum(
            [int(np.prod(s[1])) for s in mlp.SHAPES])[:-1]))):
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, name


@pytest.mark.parametrize("family", [3, 4, 5])
def test_forward_matches_oracle(cp, oracle, prover, family):
    params = mlp.init_params(5 + family)
    prover.model_set_params(family, params)
    dims = boxgen.DIMS[family]
    idx = boxgen.lattice_indices(family, [64, 16, 16, 8][:dims], 3000, 7)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, [64, 16, 16, 8][:dims], idx)
    lo, hi = boxgen.sub_boxes(lo, hi, 8)
    depth = np.random.default_rng(9).integers(0, 30, lo.shape[1]).astype(np.uint8)
    logits, axis, order = prover.model_predict(family, lo, hi, depth)
    want = mlp.forward(params, mlp.features(family, lo, hi, depth))["z"]
    assert np.abs(logits - want).max() < 2e-2
    assert (axis == np.argmax(logits[:, 4:4 + dims], axis=1)).all()
    if family == 3:
        want_order = np.maximum(logits[:, 2], logits[:, 3]) > np.maximum(logits[:, 0], logits[:, 1])
    else:
        want_order = logits[:, 1] > logits[:, 0]
    assert (order == want_order).all()


@pytest.mark.parametrize("family", [3, 5])
def test_trace_labels_match_oracle(cp, oracle, prover, family):
    dims = boxgen.DIMS[family]
    n = prover.model_collect(family, 20000, sample_stride=3, policy=cp.SPLIT_WIDEST, max_depth=4,
                             seed_sizes=[16, 8, 8, 4][:dims])
    assert n > 1000
    r = prover.model_records()
    boxes = r["boxes"]
    lo, hi = boxes[:, 0:2 * dims:2].T.copy(), boxes[:, 1:2 * dims:2].T.copy()
    feats = mlp.features(family, lo, hi, r["depth"])
    assert np.abs(mlp.bf16(feats) - r["feats"]).max() <= 1e-2
    v, m, t = oracle.eval_boxes(family, lo, hi, trace=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        rel = np.abs(t[:, :, 0] - t[:, :, 1]) / np.maximum(np.abs(t[:, :, 1]), 1e-300)
    tie = np.nanmin(np.where(np.isnan(rel), np.inf, rel), axis=1) < 1e-12
    ok = tie | ((m & 0x0F) == r["crit"])
    assert ok.all()
    # split labels exist exactly for the critical boxes and name one of the family's axes
    crit_box = (v == cp.CRITICAL)
    assert ((r["axis"] >= 0) == crit_box)[~tie].all()
    assert (r["axis"] < dims).all()


def test_training_gains_over_plain_order(cp, prover):
    """Train the middle family's network on its own refinement traces; the
    learned criterion order must evaluate fewer guarded criteria per box than
    the reference order while every verdict count stays identical."""
    family = cp.MIDDLE
    kw = dict(policy=cp.SPLIT_WIDEST, max_depth=8, seed_sizes=[16, 8, 8, 4])
    n = prover.model_collect(family, 400000, sample_stride=2, **kw)
    assert n > 50000
    prover.model_set_training(1)  # tcgen05 training kernel (the default)
    losses = prover.model_train(family, epochs=8, batch=4096, lr=2e-3, seed=3)
    assert np.isfinite(losses).all() and losses[-1] < 0.8 * losses[0], losses
    plain = prover.refine(family, **kw)
    learned = prover.refine(family, learned_order=True, **kw)
    for k in ("evaluated", "verdicts", "unresolved", "clipped", "per_depth"):
        assert plain[k] == learned[k], k
    per_plain = plain["handles_evaluated"] / plain["evaluated"]
    per_learned = learned["handles_evaluated"] / learned["evaluated"]
    print(f"criteria evaluated per box: plain {per_plain:.4f}, learned {per_learned:.4f}; "
          f"device ms plain {plain['device_ms']:.2f}, learned {learned['device_ms']:.2f}")
    assert per_learned < per_plain
    # the learned split axis: a complete refinement with per-box proposals
    split = prover.refine(family, policy=cp.SPLIT_LEARNED, max_depth=8, seed_sizes=[16, 8, 8, 4])
    assert split["evaluated"] == sum(split["per_depth"])
    print(f"learned split: evaluated {split['evaluated']}, unresolved {split['unresolved']}; "
          f"widest: evaluated {plain['evaluated']}, unresolved {plain['unresolved']}")


@pytest.mark.parametrize("family", [3, 5, 1])
def test_tcgen05_inference_matches_mma_sync(cp, oracle, prover, family):
    """The tcgen05 (tensor-memory) inference kernel gives the warp-level mma.sync
    kernel's logits (same BF16 operands; FP32 sums in another order) and the
    same decisions away from ties."""
    params = mlp.init_params(31 + family)
    prover.model_set_params(family, params)
    dims = boxgen.DIMS[family]
    idx = boxgen.lattice_indices(family, [64, 16, 16, 8][:dims], 5000, 17)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, [64, 16, 16, 8][:dims], idx)
    lo, hi = boxgen.sub_boxes(lo, hi, 18)
    depth = np.random.default_rng(19).integers(0, 30, lo.shape[1]).astype(np.uint8)
    try:
        prover.model_set_inference(0)
        l0, a0, o0 = prover.model_predict(family, lo, hi, depth)
        prover.model_set_inference(1)
        l1, a1, o1 = prover.model_predict(family, lo, hi, depth)
        l1b, _, _ = prover.model_predict(family, lo, hi, depth)  # second call on the same handle
    finally:
        prover.model_set_inference(0)
    assert np.abs(l1 - l0).max() < 1e-3
    assert (l1b == l1).all()
    srt = np.sort(l0[:, 4:4 + dims], axis=1)
    clear = (srt[:, -1] - srt[:, -2]) > 1e-3
    assert (a1 == a0)[clear].all()
    want = np.abs(np.maximum(l0[:, 2], l0[:, 3]) - np.maximum(l0[:, 0], l0[:, 1])) > 1e-3 if family == 3 else \
        np.abs(l0[:, 1] - l0[:, 0]) > 1e-3
    assert (o1 == o0)[want].all()


@pytest.mark.parametrize("family", [3, 0])
def test_tcgen05_inference_matches_oracle(cp, oracle, prover, family):
    """The tcgen05 inference kernel against the CPU restatement of the network
    (oracle/mlp.py): logits within the BF16 tolerance of the mma.sync test."""
    params = mlp.init_params(41 + family)
    prover.model_set_params(family, params)
    dims = boxgen.DIMS[family]
    idx = boxgen.lattice_indices(family, [64, 16, 16, 8][:dims], 3000, 23)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, [64, 16, 16, 8][:dims], idx)
    lo, hi = boxgen.sub_boxes(lo, hi, 24)
    depth = np.random.default_rng(25).integers(0, 30, lo.shape[1]).astype(np.uint8)
    try:
        prover.model_set_inference(1)
        logits, axis, _ = prover.model_predict(family, lo, hi, depth)
    finally:
        prover.model_set_inference(0)
    want = mlp.forward(params, mlp.features(family, lo, hi, depth))["z"]
    assert np.abs(logits - want).max() < 2e-2
    assert (axis == np.argmax(logits[:, 4:4 + dims], axis=1)).all()


def test_tcgen05_wait_timeout_returns_error(cp, oracle, prover):
    """A completion wait of the tcgen05 kernel that runs out (limit 0: no poll)
    makes the kernel drain the MMA in flight, free its tensor memory and raise
    its error flag; the call returns CP_ERR_DEVICE and the handle keeps working
    once the time-out is cleared."""
    family = cp.MIDDLE
    params = mlp.init_params(51)
    prover.model_set_params(family, params)
    idx = boxgen.lattice_indices(family, [64, 16, 16, 8], 2000, 27)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, [64, 16, 16, 8], idx)
    try:
        prover.model_set_inference(1)
        good, _, _ = prover.model_predict(family, lo, hi)
        prover.model_set_wait_limit(0)
        with pytest.raises(cp.ProverError) as e:
            prover.model_predict(family, lo, hi)
        assert e.value.status == 5  # CP_ERR_DEVICE
        prover.model_set_wait_limit(1 << 22)
        prover.model_set_inference(1)  # clears the recorded time-out
        again, _, _ = prover.model_predict(family, lo, hi)
    finally:
        prover.model_set_wait_limit(1 << 22)
        prover.model_set_inference(0)
    assert (again == good).all()


def test_tcgen05_and_mma_sync_training_agree(cp, prover):
    """Both training kernels reach about the same loss from the same records,
    initialisation and shuffle (BF16 products summed in another order)."""
    family = cp.END_3D
    prover.model_collect(family, 100000, sample_stride=2, policy=cp.SPLIT_WIDEST, max_depth=6,
                         seed_sizes=[16, 8, 8, 4])
    try:
        prover.model_set_training(0)
        l0 = prover.model_train(family, epochs=4, batch=4096, lr=2e-3, seed=5)
        prover.model_set_training(1)
        l1 = prover.model_train(family, epochs=4, batch=4096, lr=2e-3, seed=5)
    finally:
        prover.model_set_training(1)
    assert np.isfinite(l1).all() and l1[-1] < l1[0]
    assert abs(l1[-1] - l0[-1]) <= 0.05 * abs(l0[-1]) + 1e-3, (l0, l1)
