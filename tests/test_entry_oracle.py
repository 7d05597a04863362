"""The entry-network oracle itself (CPU): analytic gradients against finite
differences, labels against a direct search, probe order and ties."""
import numpy as np

import entry_oracle as eo
from nnm import entry_init


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    d, C, B = 6, 5, 7
    m = entry_init(d, C, seed=2, in_scale=0.5, in_shift=-0.1)
    m["b1"] = rng.standard_normal(256).astype(np.float32) * 0.1
    x = rng.standard_normal((B, d)).astype(np.float32)
    lab = rng.integers(0, C, B)
    loss, g = eo.loss_and_grad(m, x, lab, rounded=False)
    eps = 1e-6
    for k in ("w1", "b1", "w2", "b2"):
        flat = m[k].reshape(-1)
        for i in rng.choice(flat.size, min(6, flat.size), replace=False):
            keep = float(flat[i])
            mp = {**m, k: m[k].astype(np.float64).copy()}
            mp[k].reshape(-1)[i] = keep + eps
            lp = eo.loss_and_grad(mp, x, lab, rounded=False)[0]
            mp[k].reshape(-1)[i] = keep - eps
            lm = eo.loss_and_grad(mp, x, lab, rounded=False)[0]
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[k].reshape(-1)[i]) < 1e-5 * max(1.0, abs(num)), (k, i)
    assert np.isfinite(loss)


def test_nearest_class_matches_direct_search():
    rng = np.random.default_rng(3)
    x = rng.integers(0, 50, size=(300, 9)).astype(np.float32)
    rows = rng.integers(0, 300, 40)
    got = eo.nearest_class(x, rows, 64)
    for r, c in zip(rows, got):
        d = ((x[:64].astype(np.int64) - x[r].astype(np.int64)) ** 2).sum(1)
        assert c == int(np.flatnonzero(d == d.min())[0])


def test_probes_order_and_ties():
    s = np.array([[0.5, 2.0, 2.0, -1.0, 3.0], [1.0, 1.0, 1.0, 1.0, 1.0]])
    assert eo.probes(s, 3).tolist() == [[4, 1, 2], [0, 1, 2]]
