"""The C restatement of the reference's CPU DP (``oracle/cport``), which the
bench times as its CPU baseline, against the numpy oracle: the baseline
computes the same fields, so its rate is a rate for the same work."""
import numpy as np
import pytest

from oracle.cport import CPortCell, campaign_rate
from oracle.dp_oracle import OracleBackend

CELLS = [("hamming", [2] * 10, 3, 1), ("hamming", [3] * 7, 2, 1),
         ("hamming", [2, 3, 4, 5], 2, 2), ("hamming", [10, 9, 8], 4, 1),
         ("lee", [7] * 4, 3, 1), ("lee", [4, 6, 5], 2, 2),
         ("torus_linf", [7, 9, 11], 2, 1), ("torus_linf", [5] * 4, 1, 3),
         ("grid_linf", [4, 5, 6], 3, 1), ("grid_linf", [16, 4], 1, 2)]


@pytest.mark.parametrize("problem,axes,R,mu", CELLS,
                         ids=lambda v: str(v).replace(" ", ""))
def test_cport_fields_equal_the_oracle(problem, axes, R, mu):
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + R)
    code = np.sort(rng.choice(size, size=max(3, size // 20)))   # a multiset
    c = CPortCell(axes, R, problem, mu=mu)
    o = OracleBackend(axes, R, problem, mu=mu)
    c.recount(code)
    o.recount(code)
    assert np.array_equal(c.cnt.astype(np.int64), o.cnt.astype(np.int64))
    c.gain_map()
    o.gain_map()
    assert np.array_equal(c.map.astype(np.int64), o.map.astype(np.int64))
    c.loss_map()
    o.loss_map()
    assert np.array_equal(c.map.astype(np.int64), o.map.astype(np.int64))


def test_campaign_pool_runs_every_cell():
    rng = np.random.default_rng(1)
    cells = [("hamming", (3,) * 6, 2, rng.choice(729, 20, replace=False)),
             ("lee", (5,) * 4, 1, rng.choice(625, 30, replace=False)),
             ("hamming", (2,) * 12, 3, rng.choice(4096, 40, replace=False))]
    rate, wall, busy, workers = campaign_rate(cells, workers=2)
    assert workers == 2 and wall > 0 and busy > 0
    assert rate == pytest.approx(len(cells) / wall)


def test_incidence_field_port_equals_the_oracle():
    from oracle.cport import inc_field
    from oracle.incidence_oracle import IncidenceOracle
    rng = np.random.default_rng(3)
    for d in (1, 6, 33):
        inc = np.stack([rng.choice(90, d, replace=False) for _ in range(200)])
        o = IncidenceOracle(inc, 90, mu=2)
        o.recount(rng.choice(200, 30, replace=False))
        for t in (0, 1, 3):
            o.field(t)
            assert np.array_equal(inc_field(inc, o.cnt, t, mu=2), o.map)
