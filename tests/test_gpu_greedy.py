"""Device-side exact greedy repair (``dct_b200_greedy_fill``) on the B200
against the brute-force exact greedy of the oracle: the same words in the
same order (largest exact gain, ties to the smallest index), the same
deficit, the same counters afterwards."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from oracle.dp_oracle import OracleBackend, exact_greedy

pytestmark = pytest.mark.gpu

CELLS = [("hamming", [3] * 7, 2, 1), ("hamming", [4, 3, 5, 2, 3], 2, 2),
         ("hamming", [2] * 11, 3, 1), ("lee", [5, 6, 7, 4], 2, 1),
         ("lee", [4] * 5, 3, 2), ("torus_linf", [7, 9, 11], 2, 1),
         ("torus_linf", [5, 5, 5], 1, 2), ("grid_linf", [4, 5, 6], 2, 1),
         ("grid_linf", [3, 3, 8], 1, 1), ("grid_linf", [6, 7], 3, 1)]


@pytest.mark.parametrize("cell", CELLS,
                         ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}-mu{c[3]}")
@pytest.mark.parametrize("max_add", [1, 7, 10 ** 6])
def test_device_greedy_matches_oracle(cell, max_add):
    prob, axes, R, mu = cell
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + 31 * R + mu)
    code = np.sort(rng.choice(size, size=max(1, size // 60), replace=False))
    if mu > 1:
        code = np.sort(np.concatenate([code, code[: len(code) // 2]]))
    ob = OracleBackend(axes, R, prob, mu=mu)
    ob.recount(code)
    want, wdef = exact_greedy(ob, code, max_add)
    with GpuBackend(axes, R, problem=prob, mu=mu) as b:
        b.recount(code)
        got, gdef = b.greedy_fill_device(max_add)
        assert got.tolist() == want.tolist()
        assert gdef == wdef == b.uncovered()
        assert np.array_equal(b.read_cnt(), ob.cnt.astype(np.uint16))
        # the placed words joined the active multiset: they can be removed
        if len(got):
            b.ball_update(got, -1)
            ob2 = OracleBackend(axes, R, prob, mu=mu)
            ob2.recount(code)
            assert np.array_equal(b.read_cnt(), ob2.cnt.astype(np.uint16))


def test_device_greedy_covers_from_empty():
    axes, R = [3] * 8, 2
    with GpuBackend(axes, R) as b:
        b.recount(np.zeros(0, dtype=np.int64))
        placed, deficit = b.greedy_fill_device(10 ** 5)
        assert deficit == 0 and b.uncovered() == 0
        assert len(np.unique(placed)) == len(placed)
        ob = OracleBackend(axes, R)
        ob.recount(placed)
        assert ob.uncovered() == 0


def test_searcher_device_repair_lns_is_exact():
    from coldcore_b200.search import Searcher
    with GpuBackend([3] * 9, 2) as b:
        s = Searcher(b, seed=5, repair="device")
        s.build_reserve_s = s.loop_reserve_s = 0.0
        s.load([])
        s.greedy_fill(10 ** 9)
        assert s.uncov == 0 and s.verify_full() == 0
        s.peel()
        M = len(s.code) - 3
        s.ruin(3, "low")
        s.lns(M, round_budget_s=3.0, kmin=4, kmax=20, select="adaptive",
              log_every=0)
        assert s.stats["rounds"] > 0
        inc = s.uncov
        assert s.verify_full() == inc
        assert len(np.unique(s.code)) == len(s.code) <= M
