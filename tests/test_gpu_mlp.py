"""The GPU scorer's BF16 / FP32-accumulate kernels against the float64
oracle: logits, the gradient of the mean loss (norm-wise relative error
below 1e-2 — bf16 operands, fp32 sums in a different order), and training
that actually fits a learnable rule."""
import numpy as np
import pytest

import oracle.mlp_oracle as mo
from coldcore_b200.mlp import GpuMlp

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 32)).astype(np.float32)
    T = ((X[:, 0] + 0.5 * X[:, 3] - X[:, 7] * X[:, 8]) > 0).astype(np.float32)
    return X, T


@pytest.mark.parametrize("n", [1, 64, 200, 1000])
def test_forward_and_gradient_match_oracle(n):
    X, T = _data(n, n)
    with GpuMlp(seed=3) as m:
        p = m.params()
        y = m.predict(X)
        yo = mo.forward(p, X)[3]
        assert np.allclose(y, yo, rtol=1e-3, atol=1e-3)
        g = m.grad(X, T)
        go = mo.grad(p, X, T)
        rel = np.linalg.norm(g - go) / max(np.linalg.norm(go), 1e-12)
        assert rel < 1e-2, rel
        for lo, hi in ((0, 4096), (4224, 20608), (20736, 20864)):
            part = np.linalg.norm(g[lo:hi] - go[lo:hi]) / max(
                np.linalg.norm(go[lo:hi]), 1e-12)
            assert part < 2e-2, (lo, part)


def test_training_fits_a_rule():
    X, T = _data(20000, 1)
    Xv, Tv = _data(4000, 2)
    with GpuMlp(seed=1) as m:
        l0 = mo.loss(m.params(), Xv, Tv)
        m.train(X, T, epochs=8, batch=256, lr=2e-3, seed=4)
        l1 = mo.loss(m.params(), Xv, Tv)
        acc = ((m.predict(Xv) > 0) == (Tv > 0.5)).mean()
    assert l1 < 0.5 * l0 and acc > 0.9, (l0, l1, acc)
