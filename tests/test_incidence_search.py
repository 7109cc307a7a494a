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
