"""The explicit-incidence oracle (``oracle/incidence_oracle.py``) against the
reference's own backends (``tests/golden/incidence_golden.npz``, written by
``make_incidence_golden.py``) and against a dict-of-lists brute force.
Pins the oracle before the ABI-2 engine is checked against it."""
import numpy as np
import pytest

from golden_data import incidence_cells, incidence_golden
from oracle.incidence_oracle import (IncidenceOracle, WeightedIncidenceOracle,
                                     brute_cnt, brute_gather)


def make_oracle(g, key):
    meta = g[key + "/meta"]
    if key.startswith("weighted"):
        return WeightedIncidenceOracle(g[key + "/indptr"], g[key + "/indices"],
                                       g[key + "/w"], int(meta[0]),
                                       uw=g[key + "/uw"], mu=int(meta[1]))
    return IncidenceOracle(g[key + "/inc"], int(meta[0]), mu=int(meta[1]))


@pytest.mark.parametrize("key", incidence_cells())
def test_oracle_reproduces_the_reference(key):
    g = incidence_golden()
    o = make_oracle(g, key)
    for r in range(3):
        p = f"{key}/{r}/"
        o.recount(g[p + "sol"])
        assert np.array_equal(o.cnt, g[p + "cnt"])
        assert o.uncovered() == int(g[p + "uncovered"])
        assert [o.count_eq(t) for t in range(4)] == g[p + "count_eq"].tolist()
        o.gain_map()
        assert np.array_equal(o.map, g[p + "gain"])
        o.loss_map()
        assert np.array_equal(o.map, g[p + "loss"])
        for t in (0, 1, 2, 5):
            assert np.array_equal(o.ball_gather(g[p + "probe"], t),
                                  g[p + f"gather{t}"])
        o.ball_update(g[p + "add"], +1)
        o.ball_update(g[p + "add"][:3], -1)
        assert np.array_equal(o.cnt, g[p + "upd_cnt"])


@pytest.mark.parametrize("key", [k for k in incidence_cells()
                                 if not k.startswith("weighted")])
def test_oracle_matches_brute_force(key):
    g = incidence_golden()
    inc = g[key + "/inc"]
    n_univ, mu = (int(x) for x in g[key + "/meta"][:2])
    rows = [list(r) for r in inc]
    o = IncidenceOracle(inc, n_univ, mu=mu)
    sol = g[key + "/0/sol"]
    o.recount(sol)
    cnt = brute_cnt(rows, n_univ, sol)
    assert np.array_equal(o.cnt, cnt)
    every = np.arange(len(inc))
    for t in (0, 1, 2, 3):
        assert np.array_equal(o.ball_gather(every, t),
                              brute_gather(rows, cnt, mu, every, t))


def test_weighted_fields_reduce_to_roles_at_unit_weights():
    """With every weight 1 the weighted marginals are the role counts
    (the reference's own statement, incidence.py:386-392)."""
    rng = np.random.default_rng(5)
    inc = np.stack([np.sort(rng.choice(30, 5, replace=False))
                    for _ in range(40)])
    indptr = np.arange(0, 41 * 5, 5)
    for mu in (1, 2, 3):
        d = IncidenceOracle(inc, 30, mu=mu)
        w = WeightedIncidenceOracle(indptr, inc.ravel(), np.ones(200), 30,
                                    mu=mu)
        sol = rng.choice(40, 12, replace=False)
        d.recount(sol)
        w.recount(sol)
        assert np.array_equal(d.cnt, w.cnt)
        for t in (0, 1, 2):
            assert np.array_equal(d.ball_gather(np.arange(40), t),
                                  w.ball_gather(np.arange(40), t))
        assert d.uncovered() == w.uncovered()


def test_map_queries():
    o = IncidenceOracle(np.zeros((6, 1), dtype=np.int64), 1)
    o.map = np.array([0, 3, 7, 1, 0, 7])
    assert o.map_max() == 7
    assert o.map_hist(3, 7).tolist() == [2, 0, 2]
    assert o.map_hist(1, 7).tolist() == [4]
    idx, val, found = o.map_extract(3)
    assert idx.tolist() == [1, 2, 5] and val.tolist() == [3, 7, 7]
    assert found == 3
    o.map[:] = 0
    assert o.map_max() == 0 and o.map_hist(4, 1).tolist() == [0, 0, 0, 0]


def test_design_builder_matches_the_reference():
    """The restated C(v,k,t) builder gives the reference's
    build_incidence matrices (the golden design cells)."""
    from oracle.incidence_oracle import design_incidence
    g = incidence_golden()
    for key in [k for k in incidence_cells() if k.startswith("design")]:
        v, k, t = (int(x) for x in g[key + "/meta"][2:5])
        assert np.array_equal(design_incidence(v, k, t), g[key + "/inc"])
