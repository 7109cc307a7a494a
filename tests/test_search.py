"""The restated search core against the reference's own traces.

``tests/golden/search_traces.json`` holds what coldcore's ``Searcher`` did
over its CPU backend (``make_search_golden.py``).  The oracle backend has
the same fields and the same ascending ``map_extract`` order, so a seeded
run of :class:`coldcore_b200.search.Searcher` over it must make exactly the
same moves.
"""
import json
import os

import numpy as np
import pytest

from coldcore_b200.search import (FIXED_DRAW, RUIN_OPS, RUIN_OPS_EXT,
                                  RUIN_PRIOR_EXT, OperatorBandit, Searcher)
from oracle.dp_oracle import OracleBackend

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "search_traces.json")) as f:
    TRACES = json.load(f)


def _built(t):
    s = Searcher(OracleBackend(t["axes"], t["R"], t["problem"], mu=t["mu"]),
                 seed=t["seed"])
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    return s


def _id(t):
    return f"{t['problem']}-{'x'.join(map(str, t['axes']))}-R{t['R']}-mu{t['mu']}"


@pytest.mark.parametrize("t", TRACES, ids=_id)
def test_greedy_and_peel_match_reference(t):
    s = _built(t)
    assert s.code.tolist() == t["greedy"]
    assert s.uncov == 0
    s.peel()
    assert s.code.tolist() == t["peeled"]
    assert s.verify_full() == 0


@pytest.mark.parametrize("t", TRACES, ids=_id)
@pytest.mark.parametrize("mode", RUIN_OPS)
def test_ruin_operators_match_reference(t, mode):
    s = _built(t)
    s.peel()
    removed = s.ruin(3, mode)
    assert sorted(removed.tolist()) == t["ruin"][mode]["removed"]
    assert s.uncov == t["ruin"][mode]["uncov"]
    assert s.verify_full() == t["ruin"][mode]["uncov"]


@pytest.mark.parametrize("t", TRACES, ids=_id)
@pytest.mark.parametrize("select", ["fixed", "adaptive"])
def test_lns_matches_reference(t, select):
    g = t["lns"][select]
    if not g["solved"]:
        pytest.skip("the reference run hit its time budget (not replayable)")
    s = _built(t)
    s.peel()
    s.ruin(1, "low")
    unc = s.lns(g["M"], round_budget_s=120.0, kmin=2, kmax=4, select=select,
                log_every=0)
    assert unc == 0
    assert s.stats["rounds"] == g["rounds"]
    assert s.code.tolist() == g["code"]
    assert s.verify_full() == 0


def test_bandit_floor_and_prior():
    b = OperatorBandit(np.random.default_rng(0))
    p = b.probabilities()
    assert np.isclose(p.sum(), 1.0)
    assert p[RUIN_OPS.index("hole")] > p[RUIN_OPS.index("low")]
    for _ in range(200):
        b.update("random", 0.0)
    p = b.probabilities()
    assert p[RUIN_OPS.index("random")] >= 0.15 / len(RUIN_OPS) - 1e-12
    assert b.tier(True, 5, 5) == b.REWARD_BEST
    assert b.tier(False, 5, 4) == b.REWARD_BETTER
    assert b.tier(False, 5, 5) == b.REWARD_EQUAL
    assert b.tier(False, 5, 6) == b.REWARD_WORSE


def test_fixed_mix_is_the_record_mix():
    assert sorted(FIXED_DRAW) == sorted(["low", "hole", "hole", "cluster",
                                         "random"])


def test_descend_shrinks_and_stays_feasible():
    b = OracleBackend([3] * 5, 1, "hamming")
    sizes = []
    s = Searcher(b, seed=4, on_solved=lambda m, c: sizes.append((m, c.copy())))
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    M = s.descend(notch_budget_s=2.0, step0=2, reserve_s=0.0,
                  min_notch_s=0.5, fail_limit=1)
    assert sizes and sizes[-1][0] == M <= sizes[0][0]
    for m, code in sizes:
        b2 = OracleBackend([3] * 5, 1, "hamming")
        b2.recount(code)
        assert b2.uncovered() == 0 and len(code) == m


class _FixedProposer:
    """Proposes the first k positions; closes its gate every other round."""

    def __init__(self):
        self.calls = 0
        self.seen = []

    def propose(self, s, k):
        self.calls += 1
        return None if self.calls % 2 == 0 else np.arange(k)

    def observe(self, s, mode, pre, post, new_best):
        self.seen.append(mode)


def test_learned_selection_uses_proposer_and_falls_back():
    b = OracleBackend([3] * 5, 1, "hamming")
    prop = _FixedProposer()
    s = Searcher(b, seed=2, proposer=prop)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    s.peel()
    M = len(s.code) - 2
    s.ruin(2, "low")
    s.lns(M, round_budget_s=3.0, kmin=2, kmax=3, select="learned",
          log_every=0)
    assert s.stats["learned_rounds"] >= 1
    assert s.stats["fallback_rounds"] >= 1 or s.stats["rounds"] == 1
    assert "learned" in prop.seen
    assert s.verify_full() == s.uncov


def test_move_log_sees_every_round():
    b = OracleBackend([3] * 5, 1, "hamming")
    events = []

    def log(s, ev, **info):
        events.append((ev, info))

    s = Searcher(b, seed=6, move_log=log)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    s.peel()
    s.ruin(2, "low")
    s.lns(len(s.code), round_budget_s=2.0, kmin=2, kmax=3, log_every=0)
    kinds = [e for e, _ in events]
    assert kinds.count("pre") == kinds.count("ruin") == kinds.count("post")
    assert kinds.count("pre") == s.stats["rounds"]
    for ev, info in events:
        if ev == "ruin":
            assert len(info["pick"]) == len(set(info["pick"].tolist()))


with open(os.path.join(HERE, "golden", "search_deficit_traces.json")) as f:
    DEFICIT_TRACES = json.load(f)


@pytest.mark.parametrize("t", DEFICIT_TRACES, ids=_id)
def test_deficit_ruin_matches_reference(t):
    """The opt-in deficit-targeted ruin: the same uncovered words found by
    the rotating cnt scan, the same incumbents removed."""
    s = _built(t)
    s.peel()
    s.ruin(3, "low")
    assert s.uncovered_words().tolist() == t["ruin"]["targets"]
    removed = s.ruin(3, "deficit")
    assert sorted(removed.tolist()) == t["ruin"]["removed"]
    assert s.uncov == t["ruin"]["uncov"]
    assert s.stats.get("deficit_ruins", 0) == t["ruin"]["deficit_ruins"]


@pytest.mark.parametrize("t", DEFICIT_TRACES, ids=_id)
@pytest.mark.parametrize("select", ["fixed", "adaptive"])
def test_deficit_lns_matches_reference(t, select):
    g = t["lns"][select]
    if not g["solved"]:
        pytest.skip("the reference run hit its time budget (not replayable)")
    s = _built(t)
    s.peel()
    s.ruin(1, "low")
    unc = s.lns(g["M"], round_budget_s=120.0, kmin=2, kmax=4, select=select,
                log_every=0, deficit=True)
    assert unc == 0
    assert s.stats["rounds"] == g["rounds"]
    assert s.stats.get("deficit_ruins", 0) == g["deficit_ruins"]
    assert s.code.tolist() == g["code"]


def test_bandit_boost_hint():
    b = OperatorBandit(np.random.default_rng(0), ops=RUIN_OPS_EXT,
                       prior=RUIN_PRIOR_EXT)
    p0 = b.probabilities()
    p1 = b.probabilities({"deficit": 4.0})
    i = RUIN_OPS_EXT.index("deficit")
    assert np.isclose(p1.sum(), 1.0) and p1[i] > p0[i]
    for _ in range(300):
        b.update("deficit", 0.0)
    assert b.probabilities({"deficit": 4.0})[i] > b.probabilities()[i]
