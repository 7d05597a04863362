"""The CPU oracle of the code MLP: its analytic gradients against central
finite differences (float64, unrounded weights), and its BF16 rounding."""
import numpy as np

import mlp_oracle as mo
from nnm import mlp_init


def test_bf16_round():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0, 65504.0], np.float32)
    r = mo.bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie at 1 + 2^-8 rounds to even (1.0)
    assert r[2] == np.float32(1.0078125)  # above the tie rounds up
    assert abs(r[3] - a[3]) <= 2.0 ** -8 * 4
    assert (mo.bf16_round(r) == r).all()  # idempotent


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    d = 12
    m = mlp_init(d, seed=5, in_scale=1.0 / 64, in_shift=-1.0)
    x = rng.integers(0, 256, size=(40, d)).astype(np.float32)
    tr = rng.integers(0, 40, size=(16, 3))
    loss, g = mo.loss_and_grad(m, x, tr, margin=2.0, rounded=False)
    assert loss > 0
    eps = 1e-4
    for name, idxs in (("w1", [(0, 0), (17, 5), (255, 11)]), ("b1", [(3,), (200,)]),
                       ("w2", [(0, 0), (31, 255), (7, 100)]), ("b2", [(0,), (31,)])):
        for ix in idxs:
            mp = {k: (v.astype(np.float64).copy() if isinstance(v, np.ndarray) else v) for k, v in m.items()}
            mn = {k: (v.astype(np.float64).copy() if isinstance(v, np.ndarray) else v) for k, v in m.items()}
            mp[name][ix] += eps
            mn[name][ix] -= eps
            lp = mo.loss_and_grad(mp, x, tr, margin=2.0, rounded=False)[0]
            ln = mo.loss_and_grad(mn, x, tr, margin=2.0, rounded=False)[0]
            num = (lp - ln) / (2 * eps)
            assert abs(num - g[name][ix]) <= 1e-6 + 1e-4 * abs(num), (name, ix, num, g[name][ix])
