"""Full-size cells on the GPU against the reference's own checksums
(tests/golden/full_configs.json, written from the reference's numpy
backend): H2(26,3), H3(16,4), Lee Z_7^8 R4, king 2048^2 R1 and K_3(14,3),
fields plus 1,000 seeded updates; 10^5-candidate gathers."""
import hashlib

import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from coldcore_b200.workloads import CELLS, candidates, code_for, update_sequence
from golden_data import full
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu


def sha(a, dt):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dt).tobytes()
                          ).hexdigest()


@pytest.mark.parametrize("name", ["H3_14_3", "LEE_7_8_4", "KING_2048",
                                  "H3_16_4", "H2_26_3"])
def test_full_config_checksums(name):
    cell, ref = CELLS[name], full()[name]
    code = code_for(cell)
    assert sha(code, "<i8") == ref["code_sha"]
    with GpuBackend(list(cell.axes), cell.R, problem=cell.problem) as b:
        b.recount(code)
        assert sha(b.read_cnt(), "<u2") == ref["cnt_sha"]
        assert [b.count_eq(t) for t in range(4)] == ref["count_eq"]
        assert b.uncovered() == ref["deficit"]
        b.gain_map()
        assert sha(b.map_all(), "<i4") == ref["gain_sha"]
        assert b.map_max() == ref["gain_max"]
        hist = b.map_hist(1024, max(1, ref["gain_max"]))
        assert sha(hist, "<i4") == ref["gain_hist_sha"]
        b.loss_map()
        assert sha(b.map_all(), "<i4") == ref["loss_sha"]
        assert sha(b.map_read_at(code), "<i4") == ref["loss_at_code_sha"]
        if cell.problem == "hamming":
            words, signs = update_sequence(cell.size, code, 1000, 1000)
            for w, s in zip(words, signs):
                b.ball_update([w], int(s))
            assert sha(b.read_cnt(), "<u2") == ref["upd_cnt_sha"]
            assert b.uncovered() == ref["upd_deficit"]
            b.gain_map()
            assert sha(b.map_all(), "<i4") == ref["upd_gain_sha"]
        if cell.problem == "lee":
            b.recount(code)
            cand = candidates(cell.size, 100000, 2000)
            assert sha(cand, "<i8") == ref["cand_sha"]
            for t in (0, 1):
                assert sha(b.ball_gather(cand, t), "<i4") == ref[f"gather{t}_sha"]


def test_king_gathers_against_int64_oracle():
    """10^5 random candidates on the 2048x2048 torus (axes the reference's
    uint8 digits cannot walk): gathers roles 0/1 against the oracle."""
    cell = CELLS["KING_2048"]
    code = code_for(cell)
    o = OracleBackend(list(cell.axes), cell.R, problem=cell.problem,
                      dtype=np.int32)
    o.recount(code)
    cand = candidates(cell.size, 100000, 2001)
    with GpuBackend(list(cell.axes), cell.R, problem=cell.problem) as b:
        b.recount(code)
        for t in (0, 1):
            assert np.array_equal(b.ball_gather(cand, t), o.ball_gather(cand, t))
        w = cand[:50]
        b.ball_update(w, +1)
        o.ball_update(w, +1)
        assert np.array_equal(b.read_cnt(), o.read_cnt())


def test_lee_sparse_fields_against_oracle():
    """Lee Z_7^8 R4 at 0.05% density (the 3% cell is a complete cover, so
    its gain / loss maps are all zero): fields against the oracle."""
    axes, R = [7] * 8, 4
    o = OracleBackend(axes, R, problem="lee", dtype=np.int32)
    rng = np.random.default_rng(12)
    code = np.sort(rng.choice(o.space.size, 2900, replace=False))
    with GpuBackend(axes, R, problem="lee") as b:
        b.recount(code)
        o.recount(code)
        assert np.array_equal(b.read_cnt(), o.read_cnt())
        b.gain_map()
        o.gain_map()
        assert np.array_equal(b.map_all(), o.map)
        b.loss_map()
        o.loss_map()
        assert np.array_equal(b.map_all(), o.map)
