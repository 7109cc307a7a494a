"""Group-invariant covering designs on the host: permutation groups, subset
orbits and the design quotient against the reference's own outputs
(``tests/golden/orbit_golden.npz``, written by ``make_orbit_golden.py``),
the quotient's defining identities against the full design, and orbit
searches reaching known optima over the oracle's weighted cell."""
import os
from math import comb

import numpy as np
import pytest

from coldcore_b200.design_orbits import (DesignOrbits, PermGroup,
                                         builtin_specs, orbit_search,
                                         parse_design_group, quotient_backend)
from oracle.incidence_oracle import DesignOracle, WeightedIncidenceOracle

HERE = os.path.dirname(os.path.abspath(__file__))
G = dict(np.load(os.path.join(HERE, "golden", "orbit_golden.npz")))


def _cases(prefix, nparts):
    keys = {"/".join(k.split("/")[1:1 + nparts]) for k in G
            if k.startswith(prefix + "/")}
    return sorted(keys)


@pytest.mark.parametrize("case", _cases("order", 2))
def test_group_orders_match_the_reference(case):
    v, spec = case.split("/", 1)
    g = parse_design_group(int(v), spec)
    assert g.order() == int(G[f"order/{case}"])
    keys = {e.tobytes() for e in g.elements()}
    assert len(keys) == g.order()
    for e in g.elements()[:20]:                  # closed under generators
        for gen in g.gens:
            assert gen[e].tobytes() in keys


def test_group_validation():
    with pytest.raises(ValueError):
        parse_design_group(8, "affine")          # not prime
    with pytest.raises(ValueError):
        parse_design_group(9, "prod:2x4")
    with pytest.raises(ValueError):
        parse_design_group(7, "nonsense")
    with pytest.raises(ValueError):
        PermGroup(5, [np.array([0, 0, 1, 2, 3])])
    big = PermGroup(9, [np.roll(np.arange(9), 1),
                        np.array([1, 0, 2, 3, 4, 5, 6, 7, 8])])
    with pytest.raises(ValueError):
        big.order(cap=5000)
    assert "cyclic" in builtin_specs(28) and "affine" in builtin_specs(31)


@pytest.mark.parametrize("case", _cases("subsets", 3))
def test_subset_orbits_match_the_reference(case):
    v, r, spec = case.split("/", 2)
    part = parse_design_group(int(v), spec).subset_orbits(int(r))
    assert np.array_equal(part.labels, G[f"subsets/{case}"])


@pytest.mark.parametrize("case", _cases("quotient", 4))
def test_quotients_match_the_reference(case):
    v, k, t, spec = case.split("/", 3)
    orb = DesignOrbits(int(v), int(k), int(t), spec)
    p = f"quotient/{case}/"
    assert np.array_equal(orb.block_part.sizes, G[p + "block_sizes"])
    assert np.array_equal(orb.block_part.reps, G[p + "block_reps"])
    assert np.array_equal(orb.univ_part.sizes, G[p + "univ_sizes"])
    assert np.array_equal(orb.univ_part.reps, G[p + "univ_reps"])
    for short in (False, True):
        q = p + ("short/" if short else "full/")
        for name, got in zip(("cand", "indptr", "indices", "w", "uw"),
                             orb.quotient_csr(short)):
            assert np.array_equal(got, G[q + name]), (short, name)


@pytest.mark.parametrize("v,k,t,spec", [(7, 3, 2, "cyclic"),
                                        (9, 3, 2, "prod:3x3"),
                                        (8, 4, 2, "dihedral"),
                                        (9, 4, 3, "cyclic-1")])
def test_quotient_identities_against_the_full_design(v, k, t, spec):
    """Quotient cnt = full cnt at the t-orbit representatives; weighted
    deficiency = full deficiency; an orbit's gain (loss) = the full
    deficiency drop (rise) of adding (removing) its blocks."""
    orb = DesignOrbits(v, k, t, spec)
    q = quotient_backend(orb, short_orbits=True,
                         backend=WeightedIncidenceOracle)
    f = DesignOracle(v, k, t)
    rng = np.random.default_rng(1)
    for _ in range(4):
        sel = rng.choice(q.n_cand, min(q.n_cand, 3), replace=False)
        q.recount(sel)
        f.recount(q.expand(sel))
        assert np.array_equal(q.cnt, f.cnt[orb.univ_part.reps])
        assert q.uncovered() == f.uncovered()
        assert q.block_count(sel) == len(q.expand(sel))
        q.gain_map()
        for c in range(q.n_cand):
            before = f.uncovered()
            f.ball_update(q.expand([c]), +1)
            assert q.map[c] == before - f.uncovered()
            assert q.ball_gather([c], 0)[0] == q.map[c]
            f.ball_update(q.expand([c]), -1)
        q.loss_map()
        for c in sel:
            before = f.uncovered()
            f.ball_update(q.expand([c]), -1)
            assert q.map[c] == f.uncovered() - before
            f.ball_update(q.expand([c]), +1)


QUOTIENT_OPTIMA = [(7, 3, 2, "cyclic", 7), (13, 4, 2, "cyclic", 13),
                   (21, 5, 2, "cyclic", 21)]


@pytest.mark.parametrize("v,k,t,spec,opt", QUOTIENT_OPTIMA)
def test_orbit_search_reaches_optimum(v, k, t, spec, opt):
    blocks, s, q = orbit_search(v, k, t, spec, budget_s=40, seed=1,
                                notch_budget_s=5, reserve_s=0.0,
                                backend=WeightedIncidenceOracle)
    assert len(blocks) == opt
    assert DesignOracle(v, k, t).verify(blocks)
    assert comb(v, k) >= len(blocks)


def test_release_keeps_feasibility_and_size():
    from coldcore_b200.design_orbits import release
    blocks, s, q = orbit_search(13, 4, 2, "cyclic", budget_s=5, seed=1,
                                notch_budget_s=2, reserve_s=0.0,
                                backend=WeightedIncidenceOracle)
    rel, s2 = release(13, 4, 2, blocks, 5, seed=1, notch_budget_s=2, step0=1,
                      reserve_s=0.0, backend=DesignOracle)
    assert len(rel) <= len(blocks) == 13
    assert DesignOracle(13, 4, 2).verify(rel)


def test_free_greedy_c24_8_5_is_759():
    """The exact greedy over all 735,471 blocks of C(24,8,5) finds the
    759-block Steiner system S(5,8,24) (the reference's case,
    tests/test_design_orbits.py:185-190)."""
    from coldcore_b200.design_orbits import design_rows
    from coldcore_b200.search import Searcher
    from oracle.incidence_oracle import IncidenceOracle
    b = IncidenceOracle(design_rows(24, 8, 5), comb(24, 5))
    s = Searcher(b, seed=1)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load(np.zeros(0, dtype=np.int64))
    assert s.greedy_fill(10 ** 9) == 0
    assert len(s.code) == 759
    cnt = np.zeros(comb(24, 5), dtype=np.int64)
    np.add.at(cnt, b.inc[s.code].ravel(), 1)
    assert (cnt == 1).all()                      # every 5-set exactly once
