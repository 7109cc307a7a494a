"""The swap-neighbourhood polish on the B200 engine: every move is costed
by the engine's one-pass ``swap_eval`` and applied with ``ball_update``;
the incremental count must stay the exact count, and the polish must not
end worse than it started."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from coldcore_b200.search import Searcher

pytestmark = [pytest.mark.gpu, pytest.mark.late(1)]


@pytest.mark.parametrize("problem,axes,R,seed", [
    ("hamming", [3] * 6, 1, 3), ("hamming", [4] * 4, 1, 7),
    ("lee", [5, 5, 5], 1, 13)])
@pytest.mark.parametrize("nb", ["shell", "pool"])
def test_polish_keeps_exact_counts(problem, axes, R, seed, nb):
    with GpuBackend(axes, R, problem=problem) as b:
        s = Searcher(b, seed=seed)
        s.build_reserve_s = s.loop_reserve_s = 0.0
        s.load([])
        s.greedy_fill(10 ** 9)
        s.peel()
        M = len(s.code) - 1
        s.ruin(1, "low")
        start = s.uncov
        unc = s.anneal(M, 5.0, mode="lahc", neighbourhood=nb, log_every=0)
        assert unc <= start
        assert len(s.code) == M and len(np.unique(s.code)) == M
        assert s.verify_full() == unc
        assert s.stats["moves"] > 0
