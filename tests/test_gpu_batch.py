"""Batched engine: every cell's fields and scalars against the oracle, in
the persistent graph launch and in the one-launch-per-pass form; the
bounded dependency wait ends a poisoned launch with an error status and
leaves the context usable."""
import numpy as np
import pytest

from coldcore_b200.batch import BatchEngine
from coldcore_b200.workloads import batch_cells
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu


def _mixed_cells():
    cells = batch_cells(count=20, seed=11, lo=2.0, hi=4.5)
    rng = np.random.default_rng(5)
    extra = [("torus_linf", (7, 9, 5), 1, 1), ("grid_linf", (6, 5, 4), 2, 1),
             ("hamming", (3, 4, 5, 6), 2, 2), ("lee", (7, 7, 7), 3, 1),
             # cells of >= 2^20 words: their own register-blocked launches
             ("hamming", (2,) * 20, 3, 1), ("lee", (5,) * 9, 2, 1)]
    out = [(p, a, R, c, 1) for p, a, R, c in cells]
    for p, a, R, mu in extra:
        size = int(np.prod(a))
        code = rng.integers(0, size, size=max(2, size // 30))
        out.append((p, a, R, code, mu))
    return out


@pytest.mark.parametrize("tile_kb", [0, 16, 96])
def test_batch_matches_oracle(tile_kb):
    cells = _mixed_cells()
    with BatchEngine() as b:
        for p, a, R, code, mu in cells:
            b.add(p, a, R, code, mu)
        b.build(tile_kb)
        for mode in (0, 1, 0):
            b.run(mode)
            sc = b.scalars()
            for i, (p, a, R, code, mu) in enumerate(cells):
                o = OracleBackend(list(a), R, problem=p, mu=mu)
                o.recount(code)
                assert np.array_equal(b.cnt(i), o.read_cnt()), (i, p, a, R)
                assert sc[i, 0] == o.uncovered()
                o.gain_map()
                assert np.array_equal(b.gain(i), o.map), (i, p, a, R)
                assert sc[i, 1] == o.map_max()
                o.loss_map()
                assert np.array_equal(b.loss(i), o.map), (i, p, a, R)
                assert sc[i, 2] == o.map_max()


def test_bounded_wait_reports_and_recovers():
    cells = _mixed_cells()[:6]
    with BatchEngine() as b:
        for p, a, R, code, mu in cells:
            b.add(p, a, R, code, mu)
        b.build(48)
        assert b.run_rc(2) == -7             # poisoned dependency: error
        b.run(0)                             # the next launch is correct
        p, a, R, code, mu = cells[0]
        o = OracleBackend(list(a), R, problem=p, mu=mu)
        o.recount(code)
        assert np.array_equal(b.cnt(0), o.read_cnt())


def test_campaign_of_256_cells_against_golden_digests():
    """The batched configuration the bench times (256 seeded cells, 292 M
    words): every cell's cnt, gain and loss maps and scalars, in the
    persistent graph launch and in one launch per pass, against the digests
    of tests/golden/batch256_golden.json."""
    import hashlib
    import json
    import os

    def digest(a):
        return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]

    with open(os.path.join(os.path.dirname(__file__), "golden",
                           "batch256_golden.json")) as f:
        golden = json.load(f)
    cells = batch_cells(256, seed=7)
    with BatchEngine() as b:
        for p, a, R, code in cells:
            b.add(p, a, R, code)
        b.build(0)
        for mode in (0, 1):
            b.run(mode)
            sc = b.scalars()
            for i, g in enumerate(golden):
                assert digest(b.cnt(i).astype("<u2")) == g["cnt"], (mode, i)
                assert digest(b.gain(i).astype("<i4")) == g["gain"], (mode, i)
                assert digest(b.loss(i).astype("<i4")) == g["loss"], (mode, i)
                assert tuple(sc[i]) == (g["deficit"], g["gain_max"],
                                        g["loss_max"]), (mode, i)
