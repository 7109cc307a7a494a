"""coldcore's launch-size knob: with DCT_BLOCKS set at a cell's init, every
persistent transform launch runs that many CTAs (at least 256, at most one
per tile), striding its tiles by the grid; the fields stay equal to the
oracle's, bit for bit, whatever the grid."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("blocks", ["1", "300", "5000"])
@pytest.mark.parametrize("problem,axes,R", [
    ("hamming", [2] * 20, 3), ("hamming", [3] * 11, 4),
    ("lee", [7] * 6, 3), ("torus_linf", [96, 80], 1)])
def test_fields_under_dct_blocks(monkeypatch, blocks, problem, axes, R):
    monkeypatch.setenv("DCT_BLOCKS", blocks)
    monkeypatch.setenv("CC_TUNE", "0")
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + R + len(blocks))
    code = np.sort(rng.choice(size, size=max(8, size // 60), replace=False))
    o = OracleBackend(axes, R, problem)
    with GpuBackend(axes, R, problem=problem) as b:
        b.recount(code)
        o.recount(code)
        assert np.array_equal(b.read_cnt(), o.read_cnt())
        b.gain_map()
        o.gain_map()
        assert np.array_equal(b.map_all(), o.map)
        b.loss_map()
        o.loss_map()
        assert np.array_equal(b.map_all(), o.map)
