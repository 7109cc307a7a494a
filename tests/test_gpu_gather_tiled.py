"""The tiled gather (a block walks a tile of the support table for a group
of candidates), with and without the predicate bit plane, against the
oracle and against the per-word walk, for Hamming, Lee, torus and
mixed-radix cells, mu = 1 and 2, every role."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem,axes,R,mu", [
    ("hamming", [3] * 8, 3, 1), ("hamming", [3] * 12, 4, 1),
    ("hamming", [2, 3, 4, 5, 6, 7], 3, 2), ("lee", [7] * 6, 3, 1),
    ("torus_linf", [5, 6, 7], 1, 1), ("hamming", [2] * 16, 5, 2)])
def test_tiled_gather_matches(monkeypatch, problem, axes, R, mu):
    size = int(np.prod(axes))
    rng = np.random.default_rng(len(axes) * 7 + R)
    code = rng.choice(size, size=max(3, size // 40), replace=False)
    o = OracleBackend(axes, R, problem=problem, mu=mu)
    o.recount(code)
    cands = rng.integers(0, size, 333).astype(np.int64)
    with GpuBackend(axes, R, problem=problem, mu=mu) as b:
        b.recount(code)
        for role in (0, 1, 2):
            want = o.ball_gather(cands, role)
            monkeypatch.setenv("CC_GATHER_TILED", "1")
            monkeypatch.setenv("CC_GATHER_BITS", "1")
            bits = b.ball_gather(cands, role)
            monkeypatch.setenv("CC_GATHER_BITS", "0")
            tiled = b.ball_gather(cands, role)
            monkeypatch.setenv("CC_GATHER_TILED", "0")
            walk = b.ball_gather(cands, role)
            assert np.array_equal(bits, want), role
            assert np.array_equal(tiled, want), role
            assert np.array_equal(walk, want), role
