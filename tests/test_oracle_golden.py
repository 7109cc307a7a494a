"""The CPU oracle against the reference's own outputs (golden fixtures) and
against the brute-force restatement.  Pins the oracle before any GPU result
is checked against it."""
import numpy as np
import pytest

from golden_data import (FAMILY_CELLS, TRANSFORM_CELLS, WIDE_CELLS, cell_id,
                         key, small)
from oracle.brute import BruteBackend
from oracle.dp_oracle import OracleBackend


def _fields(o, code):
    o.recount(code)
    cnt = o.read_cnt()
    o.gain_map()
    gain = o.map.astype(np.int32).copy()
    o.loss_map()
    loss = o.map.astype(np.int32).copy()
    o.recount(code)
    return cnt, gain, loss


@pytest.mark.parametrize("axes,R,mu", TRANSFORM_CELLS)
def test_transform_cells(axes, R, mu):
    g = small()
    cid = cell_id("hamming", axes, R, mu)
    o = OracleBackend(axes, R, mu=mu)
    for k in range(3):
        code = g[key(cid, k, "code")]
        cnt, gain, loss = _fields(o, code)
        assert np.array_equal(cnt, g[key(cid, k, "cnt")])
        assert np.array_equal(gain, g[key(cid, k, "gain")])
        assert np.array_equal(loss, g[key(cid, k, "loss")])


@pytest.mark.parametrize("problem,axes,R,mu", FAMILY_CELLS + WIDE_CELLS)
def test_family_cells(problem, axes, R, mu):
    g = small()
    cid = cell_id(problem, axes, R, mu)
    o = OracleBackend(axes, R, problem=problem, mu=mu)
    code = g[key(cid, "code")]
    cnt, gain, loss = _fields(o, code)
    assert np.array_equal(cnt, g[key(cid, "cnt")])
    assert np.array_equal(gain, g[key(cid, "gain")])
    assert np.array_equal(loss, g[key(cid, "loss")])
    probe = g[key(cid, "probe")]
    for t in (0, 1, 2):
        assert np.array_equal(o.ball_gather(probe, t),
                              g[key(cid, "gather", t)])
    for w, s in zip(g[key(cid, "upd_words")], g[key(cid, "upd_signs")]):
        o.ball_update([w], int(s))
    assert np.array_equal(o.read_cnt(), g[key(cid, "upd_cnt")])
    assert np.array_equal(o.ball_gather(probe, 0), g[key(cid, "upd_gather0")])
    assert np.array_equal(o.ball_gather(probe, 1), g[key(cid, "upd_gather1")])
    o.recount(code)
    o.gain_map()
    mx = o.map_max()
    assert mx == int(g[key(cid, "gain_max")])
    assert np.array_equal(o.map_hist(16, max(mx, 1)), g[key(cid, "gain_hist")])
    idx, _, found = o.map_extract(int(g[key(cid, "ext_thr")]))
    assert found == int(g[key(cid, "ext_found")])
    assert np.array_equal(idx, g[key(cid, "ext_idx")])     # ascending order
    assert o.uncovered() == int(g[key(cid, "deficit")])
    assert [o.count_eq(t) for t in range(4)] == list(g[key(cid, "count_eq")])


def test_k3_8_2_update_trace():
    """K_3(8,2), 30 codewords (seed 0), 100 seeded add/remove updates: the
    whole cnt field and count_eq(0..3) / deficit after every update."""
    g = small()
    o = OracleBackend([3] * 8, 2)
    code = g[key("K3_8_2", "code")]
    cnt, gain, loss = _fields(o, code)
    assert np.array_equal(cnt, g[key("K3_8_2", "cnt")])
    assert np.array_equal(gain, g[key("K3_8_2", "gain")])
    assert np.array_equal(loss, g[key("K3_8_2", "loss")])
    trace_cnt = g[key("K3_8_2", "trace_cnt")]
    trace_q = g[key("K3_8_2", "trace_q")]
    for i, (w, s) in enumerate(zip(g[key("K3_8_2", "upd_words")],
                                   g[key("K3_8_2", "upd_signs")])):
        o.ball_update([w], int(s))
        assert np.array_equal(o.read_cnt(), trace_cnt[i])
        q = [o.count_eq(t) for t in range(4)] + [o.uncovered()]
        assert q == list(trace_q[i])
    o.gain_map()
    assert np.array_equal(o.map.astype(np.int32), g[key("K3_8_2", "upd_gain")])
    o.loss_map()
    assert np.array_equal(o.map.astype(np.int32), g[key("K3_8_2", "upd_loss")])


@pytest.mark.parametrize("problem,axes,R,mu", [
    ("hamming", [3, 3, 3, 3], 2, 1), ("hamming", [2, 3, 4], 1, 2),
    ("lee", [6, 5], 2, 1), ("lee", [7, 7], 3, 2),
    ("torus_linf", [7, 5], 1, 1), ("torus_linf", [9, 11], 4, 2),
    ("grid_linf", [7, 5], 2, 1), ("grid_linf", [3, 4], 5, 1)])
def test_oracle_equals_brute_force(problem, axes, R, mu):
    o = OracleBackend(axes, R, problem=problem, mu=mu)
    b = BruteBackend(axes, R, problem=problem, mu=mu)
    rng = np.random.default_rng(3)
    code = rng.integers(0, o.space.size, size=max(3, o.space.size // 8))
    o.recount(code)
    b.recount(code)
    assert np.array_equal(o.cnt, b.cnt)
    for fn in ("gain_map", "loss_map"):
        getattr(o, fn)()
        getattr(b, fn)()
        assert np.array_equal(o.map, b.map)
    every = np.arange(o.space.size)
    for t in (0, 1, 2):
        assert np.array_equal(o.ball_gather(every, t), b.ball_gather(every, t))
    for w in rng.integers(0, o.space.size, size=5):
        assert np.array_equal(o.ball_indices(w), b.ball_indices(w))


def test_wide_axis_ball_is_the_metric_ball():
    """Axes above 255 (where the reference's uint8 digits wrap): the
    oracle's int64-digit ball equals the metric ball by direct distance."""
    axes, R = [300, 260], 1
    o = OracleBackend(axes, R, problem="torus_linf")
    for w in (0, 299, 300 * 259 + 299, 12345, 300 * 130):
        digs = o.space.digits(o.ball_indices(w))
        c = o.space.digits([w])[0]
        d = np.abs(digs - c)
        d = np.minimum(d, np.asarray(axes) - d)
        assert len(digs) == 9 and (d.max(axis=1) <= 1).all()
