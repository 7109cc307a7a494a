"""Host-side support tables against the reference's packed tables."""
import numpy as np
import pytest

from coldcore_b200.gpu import locality_order
from coldcore_b200.patterns import (ball_size, enumerate_ball, locality_key,
                                    v1_table, wide_table)
from golden_data import FAMILY_CELLS, cell_id, key, tables


def _multiset(a):
    return np.sort(np.asarray(a, dtype=np.uint64))


@pytest.mark.parametrize("problem,axes,R,mu", FAMILY_CELLS)
def test_v1_table_equals_reference(problem, axes, R, mu):
    t = tables()
    cid = cell_id(problem, axes, R, mu)
    ref = t[key(cid, "v1")]
    mine = v1_table(axes, R, problem)
    assert mine[0] == 0 and ref[0] == 0
    assert np.array_equal(_multiset(mine), _multiset(ref))
    assert len(np.unique(mine)) == len(mine)
    # the reference's locality order is a permutation sorted by the key
    loc = t[key(cid, "v1_local")]
    assert np.array_equal(_multiset(loc), _multiset(ref))
    mine_loc = locality_order(ref, axes)
    assert np.array_equal(_multiset(mine_loc), _multiset(ref))


@pytest.mark.parametrize("problem,axes,R", [
    ("hamming", [3, 4, 5], 2), ("lee", [7, 7, 7], 3),
    ("torus_linf", [2048, 2048], 1), ("grid_linf", [300, 17], 2),
    ("hamming", [2] * 26, 3), ("hamming", [3] * 16, 4)])
def test_wide_table_decodes_to_the_ball(problem, axes, R):
    tbl = wide_table(axes, R, problem)
    pos, dlt = enumerate_ball(axes, R, problem)
    assert tbl.shape == pos.shape
    assert (tbl[0] == 0).all()
    dec_p = np.where(tbl != 0, tbl >> 24, 0)
    dec_d = tbl & 0xFFFFFF
    key_a = locality_key(dec_p, dec_d, axes)
    assert (np.diff(key_a) >= 0).all()               # locality order
    assert np.array_equal(np.sort(key_a), np.sort(locality_key(pos, dlt,
                                                               axes)))


def test_ball_sizes():
    assert ball_size([2] * 26, 3, "hamming") == 2952
    assert ball_size([3] * 16, 4, "hamming") == 34113
    assert ball_size([7] * 8, 4, "lee") == 3633
    assert ball_size([2048, 2048], 1, "torus_linf") == 9
    assert ball_size([3] * 8, 2, "hamming") == 129


def test_ball_order_switch(monkeypatch):
    """COLDCORE_BALL_ORDER=native keeps the builder's order (coldcore
    gpu.py:119); either order holds the same patterns, centre first."""
    from coldcore_b200.gpu import ball_order, locality_order
    from coldcore_b200.patterns import v1_table
    axes, R = [3, 4, 5, 3], 2
    native = v1_table(axes, R, "hamming", order=False)
    assert ball_order()
    sorted_ = locality_order(native, axes)
    monkeypatch.setenv("COLDCORE_BALL_ORDER", "native")
    assert not ball_order()
    assert locality_order(native, axes) is native
    assert sorted_[0] == native[0] == 0
    assert sorted(sorted_.tolist()) == sorted(native.tolist())
