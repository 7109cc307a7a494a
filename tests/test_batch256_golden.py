"""The 256-cell campaign digests (tests/golden/batch256_golden.json, made
by the C restatement) against the numpy oracle on the cells it finishes
in seconds, so the GPU test's reference values are pinned twice."""
import hashlib
import json
import os

import numpy as np
import pytest

from coldcore_b200.workloads import batch_cells
from oracle.dp_oracle import OracleBackend

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "batch256_golden.json")) as f:
    GOLDEN = json.load(f)
CELLS = batch_cells(256, seed=7)
SMALL = sorted(range(256), key=lambda i: int(np.prod(CELLS[i][1])))[:24]


def _d(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def test_golden_matches_the_workload():
    assert len(GOLDEN) == 256
    for g, (p, a, R, code) in zip(GOLDEN, CELLS):
        assert (g["problem"], g["axes"], g["R"], g["M"]) == \
            (p, list(a), R, len(code))


@pytest.mark.parametrize("i", SMALL)
def test_small_cells_against_the_oracle(i):
    p, a, R, code = CELLS[i]
    g = GOLDEN[i]
    o = OracleBackend(list(a), R, problem=p)
    o.recount(code)
    assert _d(o.read_cnt().astype("<u2")) == g["cnt"]
    assert o.uncovered() == g["deficit"]
    o.gain_map()
    assert _d(o.map.astype("<i4")) == g["gain"]
    assert o.map_max() == g["gain_max"]
    o.loss_map()
    assert _d(o.map.astype("<i4")) == g["loss"]
    assert o.map_max() == g["loss_max"]
