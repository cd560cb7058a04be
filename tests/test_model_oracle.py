"""CPU checks of the proposal model's restatement (oracle/mlp.py): its analytic
gradient against central finite differences, and its BF16 rounding."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = mlp.init_params(3).astype(np.float64)
    n = 37
    x = rng.uniform(-1, 1, (n, 16))
    x[:, 9:] = 0
    crit = rng.integers(0, 16, n).astype(np.uint8)
    axis = rng.integers(-1, 4, n).astype(np.int8)
    for family in (3, 4):
        axis = np.where(axis >= mlp.DIMS[family], -1, axis).astype(np.int8)
        _, g = mlp.loss_grad(family, p, x, crit, axis, exact=True)
        idx = rng.choice(p.size, 60, replace=False)
        eps = 1e-6
        for i in idx:
            q = p.copy()
            q[i] += eps
            a, _ = mlp.loss_grad(family, q, x, crit, axis, exact=True)
            q[i] -= 2 * eps
            b, _ = mlp.loss_grad(family, q, x, crit, axis, exact=True)
            assert abs((a - b) / (2 * eps) - g[i]) < 1e-7


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
