"""The explicit-incidence engine (plugin ABI 2) on the B200 against the
reference's own backends (golden fixtures from ``make_incidence_golden.py``)
and the oracle: every field, gather, update and query, dense and weighted
CSR cells, both placements.  Integer work: bit-exact."""
import numpy as np
import pytest

from coldcore_b200.incidence import (GpuIncidenceBackend,
                                     GpuWeightedIncidenceBackend)
from golden_data import incidence_cells, incidence_golden
from oracle.incidence_oracle import IncidenceOracle, WeightedIncidenceOracle

pytestmark = [pytest.mark.gpu, pytest.mark.late(2)]


def open_cell(g, key, inc_mode, cap=16):
    meta = g[key + "/meta"]
    n_univ, mu = int(meta[0]), int(meta[1])
    if key.startswith("weighted"):
        args = (g[key + "/indptr"], g[key + "/indices"], g[key + "/w"], n_univ)
        return (GpuWeightedIncidenceBackend(*args, uw=g[key + "/uw"], mu=mu,
                                            extract_cap=cap,
                                            inc_mode=inc_mode),
                WeightedIncidenceOracle(*args, uw=g[key + "/uw"], mu=mu))
    return (GpuIncidenceBackend(g[key + "/inc"], n_univ, mu=mu,
                                extract_cap=cap, inc_mode=inc_mode),
            IncidenceOracle(g[key + "/inc"], n_univ, mu=mu))


@pytest.mark.parametrize("inc_mode", [0, 1])
@pytest.mark.parametrize("key", incidence_cells())
def test_engine_reproduces_the_reference(key, inc_mode):
    g = incidence_golden()
    cap = 16
    b, o = open_cell(g, key, inc_mode, cap)
    with b:
        assert b.inc_mode in (0, 2) and b.space.size == o.n_cand
        assert b.inc_mode == (0 if inc_mode == 0 else 2)
        for r in range(3):
            p = f"{key}/{r}/"
            sol = g[p + "sol"]
            b.recount(sol)
            o.recount(sol)
            assert np.array_equal(b.read_cnt(), g[p + "cnt"].astype(np.uint16))
            assert b.uncovered() == int(g[p + "uncovered"])
            assert [b.count_eq(t) for t in range(4)] == \
                g[p + "count_eq"].tolist()
            n_univ = o.n_univ
            assert np.array_equal(b.read_cnt(2, 6), o.cnt[2:8])
            assert np.array_equal(b.read_cnt(n_univ - 2, 9), o.cnt[n_univ - 2:])
            assert len(b.read_cnt(n_univ + 3, 2)) == 0
            every = np.arange(o.n_cand)
            for fld in ("gain", "loss"):
                getattr(b, fld + "_map")()
                getattr(o, fld + "_map")()
                assert np.array_equal(b.map_read_at(every), g[p + fld])
                assert np.array_equal(b.map_all(), o.map)
                assert b.map_max() == o.map_max()
                mx = max(1, o.map_max())
                for nbins in (1, 7, 1024):
                    assert np.array_equal(b.map_hist(nbins, mx),
                                          o.map_hist(nbins, mx))
                for thr in (0, 1, mx // 2, mx):
                    want, _, found = o.map_extract(thr)
                    gi, gv, gf = b.map_extract(thr)
                    assert gf == found and len(gi) == min(found, cap)
                    assert np.array_equal(o.map[gi], gv)
                    if found <= cap:
                        assert sorted(gi.tolist()) == want.tolist()
            for t in (0, 1, 2, 5):
                assert np.array_equal(b.ball_gather(g[p + "probe"], t),
                                      g[p + f"gather{t}"])
            assert b.ball_gather(g[p + "probe"][:0], 0).shape == (0,)
            b.ball_update(g[p + "add"], +1)
            b.ball_update(g[p + "add"][:3], -1)
            o.ball_update(g[p + "add"], +1)
            o.ball_update(g[p + "add"][:3], -1)
            assert np.array_equal(b.read_cnt(), g[p + "upd_cnt"].astype(
                np.uint16))
            o.recount(sol)
            assert b.verify(sol) == (o.uncovered() == 0)


def test_bad_candidates_are_rejected_before_any_change():
    g = incidence_golden()
    b, o = open_cell(g, "design1", 0)
    with b:
        sol = g["design1/0/sol"]
        b.recount(sol)
        before = b.read_cnt().copy()
        for bad in ([0, o.n_cand], [-1], [5, 2 ** 40]):
            with pytest.raises(RuntimeError):
                b.ball_update(bad, +1)
            with pytest.raises(RuntimeError):
                b.ball_gather(bad, 0)
            with pytest.raises(RuntimeError):
                b.map_read_at(bad)
            with pytest.raises(RuntimeError):
                b.recount(bad)
        assert np.array_equal(b.read_cnt(), before)
        b.recount([])
        assert b.uncovered() == o.n_univ * int(g["design1/meta"][1])


def test_row_lanes_follow_the_row_length():
    from coldcore_b200.incidence import load_sparse_plugin
    lib = load_sparse_plugin()
    for d, lanes in ((1, 1), (3, 4), (6, 8), (10, 16), (33, 32)):
        rng = np.random.default_rng(d)
        inc = np.stack([rng.choice(64, d, replace=False) for _ in range(50)])
        with GpuIncidenceBackend(inc, 64):
            assert lib.sparse_b200_row_lanes() == lanes


def test_covering_design_fields_against_the_oracle():
    """C(16,6,3): 8,008 blocks x 20 triples over 560 triples, mu = 2."""
    from itertools import combinations
    from math import comb
    v, k, t = 16, 6, 3
    blocks = list(combinations(range(v), k))
    # colex rank of a sorted t-subset: sum C(s_j, j + 1)
    inc = np.array([[sum(comb(s[j], j + 1) for j in range(t))
                     for s in combinations(b, t)] for b in blocks],
                   dtype=np.int32)
    n_univ = comb(v, t)
    rng = np.random.default_rng(16)
    o = IncidenceOracle(inc, n_univ, mu=2)
    with GpuIncidenceBackend(inc, n_univ, mu=2) as b:
        for M in (0, 40, 400):
            sol = rng.choice(len(blocks), M, replace=False)
            b.recount(sol)
            o.recount(sol)
            assert np.array_equal(b.read_cnt().astype(np.int64), o.cnt)
            assert b.uncovered() == o.uncovered()
            for fld in ("gain_map", "loss_map"):
                getattr(b, fld)()
                getattr(o, fld)()
                assert np.array_equal(b.map_all(), o.map)


@pytest.mark.parametrize("key", [k for k in incidence_cells()
                                 if k.startswith("design")])
def test_device_built_designs_match_the_reference(key):
    """Rows built on the device equal the reference's build_incidence, and
    the cell answers the golden sequence."""
    from coldcore_b200.incidence import GpuCoveringDesignBackend
    g = incidence_golden()
    meta = g[key + "/meta"]
    v, k, t = (int(x) for x in meta[2:5])
    with GpuCoveringDesignBackend(v, k, t, mu=int(meta[1])) as b:
        assert np.array_equal(b.rows(), g[key + "/inc"])
        assert np.array_equal(b.rows(3, 5), g[key + "/inc"][3:8])
        assert b.n_univ == int(meta[0])
        for r in range(3):
            p = f"{key}/{r}/"
            b.recount(g[p + "sol"])
            assert np.array_equal(b.read_cnt(), g[p + "cnt"].astype(np.uint16))
            b.gain_map()
            assert np.array_equal(b.map_all(), g[p + "gain"])
            b.loss_map()
            assert np.array_equal(b.map_all(), g[p + "loss"])


def test_device_built_larger_designs_against_the_oracle():
    from coldcore_b200.incidence import GpuCoveringDesignBackend
    from oracle.incidence_oracle import design_incidence
    for v, k, t in ((16, 6, 3), (20, 5, 2), (12, 12, 3), (9, 1, 1)):
        want = design_incidence(v, k, t)
        with GpuCoveringDesignBackend(v, k, t) as b:
            assert b.rows().shape == want.shape
            assert np.array_equal(b.rows(), want)


def test_engine_equals_the_reference_plugin():
    """The reference's own ABI-2 kernels (src/plugins/sparse/sparse.cu,
    built for sm_100a) and this engine on the same cells."""
    import os
    ref = os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "oracle", "_ref", "libref_sparse.so")
    if not os.path.exists(ref):
        pytest.skip("reference ABI-2 plugin not built")
    g = incidence_golden()
    for key in ("dense1", "design1", "weighted2"):
        meta = g[key + "/meta"]
        n_univ, mu = int(meta[0]), int(meta[1])
        sol, probe = g[key + "/1/sol"], g[key + "/1/probe"]
        res = []
        for path in (None, ref):
            if key.startswith("weighted"):
                b = GpuWeightedIncidenceBackend(
                    g[key + "/indptr"], g[key + "/indices"], g[key + "/w"],
                    n_univ, uw=g[key + "/uw"], mu=mu, plugin_path=path)
            else:
                b = GpuIncidenceBackend(g[key + "/inc"], n_univ, mu=mu,
                                        plugin_path=path)
            with b:
                b.recount(sol)
                out = [b.read_cnt(), b.uncovered()]
                for fld in ("gain_map", "loss_map"):
                    getattr(b, fld)()
                    out.append(b.map_all())
                for t in (0, 1, 3):
                    out.append(b.ball_gather(probe, t))
                res.append(out)
        for a, c in zip(*res):
            assert np.array_equal(a, c)


def test_design_search_on_the_engine():
    """The restated search core on the B200 engine: C(13,4,2) = 13 (the
    reference's own GPU case, tests/test_incidence.py:221-233)."""
    import time

    from coldcore_b200.incidence import GpuCoveringDesignBackend
    from coldcore_b200.search import Searcher
    with GpuCoveringDesignBackend(13, 4, 2) as b:
        s = Searcher(b, seed=1, deadline=time.time() + 90)
        s.build_reserve_s = s.loop_reserve_s = 0.0
        s.load(np.zeros(0, dtype=np.int64))
        assert s.greedy_fill(10 ** 6) == 0
        M = s.descend(floor=13, notch_budget_s=20, step0=1, reserve_s=0.0,
                      min_notch_s=1.0)
        assert M <= 13 and s.verify_full() == 0
        o = IncidenceOracle(b.rows(), b.n_univ)
        assert o.verify(s.code)


@pytest.mark.parametrize("d", [1, 2, 3, 5, 8, 9, 16, 17, 31, 32, 33, 64, 70])
def test_every_row_width_against_the_oracle(d):
    """Each lanes-per-row form (1..32 lanes, rows longer than a warp):
    fields, gathers and updates equal the oracle's."""
    rng = np.random.default_rng(d)
    n_univ, n_cand = 150, 301
    inc = np.stack([rng.choice(n_univ, d, replace=False)
                    for _ in range(n_cand)])
    o = IncidenceOracle(inc, n_univ, mu=2)
    with GpuIncidenceBackend(inc, n_univ, mu=2) as b:
        sol = rng.choice(n_cand, 40, replace=False)
        b.recount(sol)
        o.recount(sol)
        assert np.array_equal(b.read_cnt().astype(np.int64), o.cnt)
        for t in (0, 1, 3):
            o.field(t)
            assert b._lib.sparse_field(t) == 0
            assert np.array_equal(b.map_all(), o.map)
            probe = rng.choice(n_cand, 37)
            assert np.array_equal(b.ball_gather(probe, t),
                                  o.ball_gather(probe, t))
        add = rng.choice(n_cand, 9)
        b.ball_update(add, +1)
        o.ball_update(add, +1)
        assert np.array_equal(b.read_cnt().astype(np.int64), o.cnt)


@pytest.mark.parametrize("mean_len", [1, 3, 6, 12, 24, 40])
def test_every_csr_row_width_against_the_oracle(mean_len):
    rng = np.random.default_rng(100 + mean_len)
    n_univ, n_cand = 120, 257
    lens = rng.integers(0, 2 * mean_len + 1, n_cand)
    lens = np.minimum(lens, n_univ)
    indptr = np.concatenate(([0], np.cumsum(lens)))
    indices = np.concatenate([rng.choice(n_univ, int(k), replace=False)
                              for k in lens])
    w = rng.integers(1, 4, len(indices))
    uw = rng.integers(1, 5, n_univ)
    o = WeightedIncidenceOracle(indptr, indices, w, n_univ, uw=uw, mu=3)
    with GpuWeightedIncidenceBackend(indptr, indices, w, n_univ, uw=uw,
                                     mu=3) as b:
        sol = rng.choice(n_cand, 30, replace=False)
        b.recount(sol)
        o.recount(sol)
        assert np.array_equal(b.read_cnt().astype(np.int64), o.cnt)
        assert b.uncovered() == o.uncovered()
        for t in (0, 1, 2):
            probe = rng.choice(n_cand, 29)
            assert np.array_equal(b.ball_gather(probe, t),
                                  o.ball_gather(probe, t))
        b.gain_map()
        assert np.array_equal(b.map_all(), o.ball_gather(np.arange(n_cand), 0))
        b.loss_map()
        assert np.array_equal(b.map_all(), o.ball_gather(np.arange(n_cand), 1))


@pytest.mark.late(4)
@pytest.mark.parametrize("d,n_univ", [(1, 31), (3, 32), (6, 33), (17, 150),
                                      (33, 1000), (70, 27405)])
def test_role_bit_form_against_the_oracle(d, n_univ, monkeypatch):
    """CC_SPARSE_BITS=1: dense fields and gathers through the role bits in
    shared memory (universes of 31 to 27,405 elements, whole and partial
    bit words) equal the oracle's, before and after updates."""
    monkeypatch.setenv("CC_SPARSE_BITS", "1")
    rng = np.random.default_rng(d + n_univ)
    n_cand = 777
    inc = np.stack([rng.choice(n_univ, d, replace=False)
                    for _ in range(n_cand)])
    o = IncidenceOracle(inc, n_univ, mu=2)
    with GpuIncidenceBackend(inc, n_univ, mu=2) as b:
        for step in range(2):
            sol = rng.choice(n_cand, 60 + 40 * step, replace=False)
            b.recount(sol)
            o.recount(sol)
            for t in (0, 1, 2, 3):
                o.field(t)
                assert b._lib.sparse_field(t) == 0
                assert np.array_equal(b.map_all(), o.map), (step, t)
                probe = rng.choice(n_cand, 53)
                assert np.array_equal(b.ball_gather(probe, t),
                                      o.ball_gather(probe, t)), (step, t)
