"""The restated search core over explicit-incidence cells: covering designs
C(v,k,t) reach their known optima (the reference's own cases,
``tests/test_incidence.py:236-265``), on the oracle backend here and on
the B200 engine in ``test_gpu_incidence.py``."""
import time

import numpy as np
import pytest

from coldcore_b200.search import Searcher
from oracle.incidence_oracle import IncidenceOracle, design_incidence

KNOWN = [(7, 3, 2, 7), (9, 3, 2, 12), (8, 4, 3, 14)]


def design_cell(v, k, t, mu=1):
    from math import comb
    return IncidenceOracle(design_incidence(v, k, t), comb(v, t), mu=mu)


@pytest.mark.parametrize("v,k,t,opt", KNOWN)
def test_search_reaches_known_optimum(v, k, t, opt):
    b = design_cell(v, k, t)
    s = Searcher(b, seed=1, deadline=time.time() + 120)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(np.zeros(0, dtype=np.int64))
    assert s.greedy_fill(10 ** 6) == 0
    assert s.verify_full() == 0
    M = s.descend(floor=opt, notch_budget_s=20, step0=1, reserve_s=0.0,
                  min_notch_s=1.0)
    assert M <= opt and len(s.code) == M
    assert s.verify_full() == 0
    assert b.verify(s.code)
    assert len(np.unique(s.code)) == len(s.code)


def test_mu_fold_design_search():
    """Every pair twice with 3-subsets of a 7-set: 14 blocks suffice."""
    b = design_cell(7, 3, 2, mu=2)
    s = Searcher(b, seed=2, deadline=time.time() + 90)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(np.zeros(0, dtype=np.int64))
    assert s.greedy_fill(10 ** 6) == 0
    M = s.descend(floor=14, notch_budget_s=20, step0=1, reserve_s=0.0,
                  min_notch_s=1.0)
    assert M <= 14 and s.verify_full() == 0
    assert b.verify(s.code)


@pytest.mark.parametrize("v,k,t,opt", [(7, 3, 2, 7), (8, 4, 3, 14),
                                       (13, 4, 2, 13)])
def test_search_with_the_block_metric(v, k, t, opt):
    """Cluster / hole ruins and batched peel use the design's own metric
    when the backend has one (the protocol's locality hooks)."""
    from oracle.incidence_oracle import DesignOracle
    b = DesignOracle(v, k, t)
    s = Searcher(b, seed=3, deadline=time.time() + 120)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(np.zeros(0, dtype=np.int64))
    assert s.greedy_fill(10 ** 6) == 0
    s.peel()
    assert s.verify_full() == 0
    for mode in ("cluster", "hole"):
        removed = s.ruin(3, mode)
        assert len(removed) == 3
        s.greedy_fill(10 ** 6)
        assert s.verify_full() == 0
    M = s.descend(floor=opt, notch_budget_s=20, step0=1, reserve_s=0.0,
                  min_notch_s=1.0)
    assert M <= opt and s.verify_full() == 0 and b.verify(s.code)


def test_design_metric_helpers():
    from coldcore_b200.incidence import (block_distance, design_blocks,
                                         subset_ranks, universe_distance)
    from oracle.incidence_oracle import DesignOracle, colex_rank
    v, k, t = 9, 4, 2
    o = DesignOracle(v, k, t)
    every = np.arange(len(o.blocks))
    assert np.array_equal(design_blocks(v, k, every), o.blocks)
    assert np.array_equal(subset_ranks(o.blocks), every)
    rng = np.random.default_rng(9)
    idx = rng.choice(len(every), 40)
    D = block_distance(v, k, idx[:, None], idx[None, :])
    assert np.array_equal(D, o.distance(idx[:, None], idx[None, :]))
    assert (D == D.T).all() and (np.diag(D) == 0).all()
    u = rng.choice(o.n_univ, 6)
    ud = universe_distance(v, k, t, idx, u)
    for i in range(40):
        for j in range(6):
            assert (ud[i, j] == 0) == (u[j] in o.inc[idx[i]])
    # farther apart than k - t: no shared t-subset
    for i in range(40):
        for j in range(40):
            if D[i, j] > k - t:
                assert not set(o.inc[idx[i]]) & set(o.inc[idx[j]])
    assert colex_rank([0, 1, 2, 3]) == 0
    big = design_blocks(30, 8, [0, 5852924])
    assert big[0].tolist() == list(range(8))
    assert big[1].tolist() == list(range(22, 30))


def test_deficit_ruin_on_a_design():
    """The deficit ruin aims at the uncovered t-subsets through the
    design's own hooks (deficient_universe, universe_distance): C(10,4,3)
    reaches its optimum of 30 (the reference's locality case,
    tests/test_incidence.py:495-510)."""
    from oracle.incidence_oracle import DesignOracle
    b = DesignOracle(10, 4, 3)
    u = b.universe_distance([0, 1], np.arange(b.n_univ))
    assert ((u == 0).sum(axis=1) == 4).all()          # C(4,3) per block
    s = Searcher(b, seed=3, deadline=time.time() + 120)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(np.zeros(0, dtype=np.int64))
    assert s.greedy_fill(10 ** 6) == 0
    s.peel()
    M = s.descend(floor=30, notch_budget_s=30, step0=1, reserve_s=0.0,
                  min_notch_s=1.0, deficit=True)
    assert M <= 30 and s.verify_full() == 0 and b.verify(s.code)
    assert s.stats.get("deficit_ruins", 0) > 0


def test_block_neighbourhoods_and_coverers():
    """The remaining locality hooks of the design layer
    (covering_design.py:231-269), against the design oracle."""
    from math import comb

    from coldcore_b200.incidence import block_neighbours, candidates_covering
    from oracle.incidence_oracle import DesignOracle
    v, k, t = 9, 4, 2
    o = DesignOracle(v, k, t)
    rng = np.random.default_rng(9)
    c = int(rng.integers(len(o.blocks)))
    n1 = block_neighbours(v, k, c, 1)
    assert len(n1) == k * (v - k) == len(np.unique(n1))
    assert (o.distance(n1, c) == 1).all() and c not in n1
    assert len(block_neighbours(v, k, c, 1, m=7, rng=rng)) == 7
    n2 = block_neighbours(v, k, c, 2, m=50, rng=rng)
    assert 0 < len(n2) <= 50 and (o.distance(n2, c) == 2).all()
    assert len(block_neighbours(v, k, c, 99)) == 0
    for u in rng.choice(o.n_univ, 4):
        cc = candidates_covering(v, k, t, int(u))
        assert len(cc) == comb(v - t, k - t)
        assert np.array_equal(cc, np.flatnonzero((o.inc == u).any(axis=1)))
