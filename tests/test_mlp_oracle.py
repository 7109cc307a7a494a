"""The MLP oracle's backward pass is the derivative of its forward pass
(checked with the bf16 roundings switched off, against central
differences)."""
import numpy as np

import oracle.mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(mo, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    rng = np.random.default_rng(0)
    n_params = 32 * 128 + 128 + 128 * 128 + 128 + 128 + 1
    p = rng.normal(0, 0.1, size=n_params)
    X = rng.normal(size=(16, 32))
    T = (rng.random(16) < 0.5).astype(float)
    g = mo.grad(p, X, T)
    for i in rng.choice(n_params, 40, replace=False):
        e = np.zeros(n_params)
        e[i] = 1e-6
        fd = (mo.loss(p + e, X, T) - mo.loss(p - e, X, T)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), i


def test_bf16_rounding_is_round_to_nearest_even():
    a = np.array([1.0, 1.00390625, 1.005859375, 3.0e38, -2.5], dtype=np.float32)
    r = mo.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert r[4] == -2.5
