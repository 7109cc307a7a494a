"""Set-side gathers on the B200: near a cover the engine lists the deficient
words once and counts each candidate's listed words by distance.  The
counts must equal the support walk's and the CPU oracle's, bit for bit, in
every problem family (coldcore dct_hc.cu:649-760 and the ``dct_stats``
counters 0, 1, 2, 3, 6)."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu

CELLS = [("hamming", [3] * 7, 2, 1), ("hamming", [4, 3, 5, 2, 3], 2, 2),
         ("hamming", [2] * 12, 3, 1), ("lee", [5, 6, 7, 4], 2, 1),
         ("lee", [4] * 5, 3, 2), ("torus_linf", [7, 9, 11], 2, 1),
         ("torus_linf", [5, 5, 5], 1, 2), ("grid_linf", [4, 5, 6], 3, 1),
         ("grid_linf", [3, 3, 8], 1, 1), ("grid_linf", [3, 3], 3, 1)]


def _near_cover(ob, rng, holes):
    """A greedy cover (best gain first, random ties) with a few codewords
    dropped, so the deficient set is small but not empty."""
    code = np.zeros(0, dtype=np.int64)
    ob.recount(code)
    while ob.uncovered() > 0:
        ob.gain_map()
        best = np.flatnonzero(ob.map == ob.map.max())
        code = np.append(code, int(rng.choice(best)))
        ob.recount(code)
    keep = rng.permutation(len(code))[holes:]
    return np.sort(code[keep])


@pytest.fixture
def set_env(monkeypatch):
    def setup(policy):
        monkeypatch.setenv("DCT_SET_GATHER", str(policy))
    return setup


@pytest.mark.parametrize("cell", CELLS,
                         ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}-mu{c[3]}")
def test_set_side_matches_walk_and_oracle(set_env, cell):
    prob, axes, R, mu = cell
    rng = np.random.default_rng(len(axes) * 100 + R)
    ob = OracleBackend(axes, R, prob, mu=mu)
    code = _near_cover(ob, rng, holes=2)
    if mu > 1:                               # a second copy of most words
        code = np.sort(np.concatenate([code, code[: len(code) * 3 // 4]]))
    ob.recount(code)
    cand = rng.integers(0, ob.space.size, 3000)
    want0 = ob.ball_gather(cand, 0)
    set_env(2)                                     # always try the list
    with GpuBackend(axes, R, problem=prob, mu=mu) as b:
        b.recount(code)
        got0 = b.ball_gather(cand, 0)
        st = b.gpu_stats()
        assert np.array_equal(got0, want0)
        if st["gather_set_side"] == 0:
            # the table is not the metric ball here: walks only
            assert st["set_scans"] == 0
        else:
            assert st["set_scans"] >= 1
        # the listed set follows incremental updates
        w = int(cand[0])
        b.ball_update(np.array([w]), +1)
        ob.ball_update(np.array([w]), +1)
        assert np.array_equal(b.ball_gather(cand, 0), ob.ball_gather(cand, 0))
        b.ball_update(np.array([w]), -1)
        ob.ball_update(np.array([w]), -1)
        assert np.array_equal(b.ball_gather(cand, 0), want0)
        if mu == 1:
            assert b.count_eq(0) == ob.count_eq(0)
    set_env(0)                                     # walks only
    with GpuBackend(axes, R, problem=prob, mu=mu) as b:
        b.recount(code)
        assert np.array_equal(b.ball_gather(cand, 0), want0)
        assert b.gpu_stats()["gather_set_side"] == 0


def test_hamming_table_is_ball_and_uses_list(set_env):
    set_env(2)
    axes, R = [3] * 8, 2
    rng = np.random.default_rng(3)
    ob = OracleBackend(axes, R, "hamming")
    code = _near_cover(ob, rng, holes=3)
    ob.recount(code)
    cand = rng.integers(0, 3 ** 8, 5000)
    with GpuBackend(axes, R) as b:
        b.recount(code)
        assert np.array_equal(b.ball_gather(cand, 0), ob.ball_gather(cand, 0))
        st = b.gpu_stats()
        assert st["gather_set_side"] >= 1 and st["set_scans"] == 1
        # same cnt state: the list is reused, and count_eq(0) reads it
        b.ball_gather(cand[:100], 0)
        assert b.gpu_stats()["set_scans"] == 1
        assert b.count_eq(0) == ob.count_eq(0)
        assert b.gpu_stats()["count_eq0_listed"] >= 1


def test_large_deficit_falls_back_to_walk(set_env):
    set_env(2)
    axes, R = [3] * 8, 2
    rng = np.random.default_rng(4)
    code = np.sort(rng.choice(3 ** 8, 5, replace=False))   # mostly uncovered
    ob = OracleBackend(axes, R, "hamming")
    ob.recount(code)
    cand = rng.integers(0, 3 ** 8, 2000)
    with GpuBackend(axes, R) as b:
        b.recount(code)
        assert np.array_equal(b.ball_gather(cand, 0), ob.ball_gather(cand, 0))
        st = b.gpu_stats()
        assert st["set_overflows"] >= 1 and st["gather_set_side"] == 0
        assert st["gather_walk"] >= 1


def test_auto_policy_needs_a_big_batch(set_env):
    set_env(1)
    axes, R = [3] * 8, 2
    rng = np.random.default_rng(5)
    ob = OracleBackend(axes, R, "hamming")
    code = _near_cover(ob, rng, holes=2)
    ob.recount(code)
    with GpuBackend(axes, R) as b:
        b.recount(code)
        small = rng.integers(0, 3 ** 8, 16)
        assert np.array_equal(b.ball_gather(small, 0),
                              ob.ball_gather(small, 0))
        assert b.gpu_stats()["gather_set_side"] == 0       # 16 x 129 words
        big = rng.integers(0, 3 ** 8, 20000)                # 2.6M >= 2^21
        assert np.array_equal(b.ball_gather(big, 0), ob.ball_gather(big, 0))
        assert b.gpu_stats()["gather_set_side"] >= 1


@pytest.mark.parametrize("cell", CELLS,
                         ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}-mu{c[3]}")
@pytest.mark.parametrize("policy", [1, 0])
def test_swap_eval_fast_path_matches_oracle(set_env, cell, policy):
    """With the metric-ball table the swap costs come from the drop lists
    in one pass (dct_stats[4]); with the set side off, from the
    drop / gather / undo sequence (dct_stats[5]).  Both equal the oracle's
    mutate-gather-undo values, and cnt is unchanged afterwards."""
    prob, axes, R, mu = cell
    rng = np.random.default_rng(len(axes) * 7 + R)
    ob = OracleBackend(axes, R, prob, mu=mu)
    code = _near_cover(ob, rng, holes=1)
    if mu > 1:
        code = np.sort(np.concatenate([code, code[: len(code) // 2]]))
    if len(code) == 0:
        code = np.array([0, ob.space.size - 1], dtype=np.int64)
    ob.recount(code)
    drops = np.unique(code)[: min(6, len(np.unique(code)))]
    parts = [rng.integers(0, ob.space.size, int(rng.integers(0, 40)))
             for _ in drops]
    ol, og = ob.swap_eval(drops, parts)
    set_env(policy)
    with GpuBackend(axes, R, problem=prob, mu=mu) as b:
        b.recount(code)
        before = b.read_cnt().copy()
        loss, gains = b.swap_eval(drops, parts)
        assert np.array_equal(loss, ol)
        for g, w in zip(gains, og):
            assert np.array_equal(g, w)
        shared = rng.integers(0, ob.space.size, 50)
        l2, g2 = b.swap_eval(drops, shared)
        ol2, og2 = ob.swap_eval(drops, shared)
        assert np.array_equal(l2, ol2) and np.array_equal(g2, og2)
        assert np.array_equal(b.read_cnt(), before)
        st = b.gpu_stats()
        if policy == 0:
            assert st["swap_eval_fast"] == 0 and st["swap_eval_fallback"] >= 2
        else:
            assert st["swap_eval_fast"] + st["swap_eval_fallback"] == 2
            if prob in ("hamming", "lee"):           # the table is the ball
                assert st["swap_eval_fast"] == 2
