"""Lee distance on axes of size 2 or 3 is the Hamming distance (a nonzero
digit difference d has Lee weight min(d, q - d) = 1), which lets the engine
plan such cells as Hamming.  Checked on the oracle: every field of a Lee
cell with q <= 3 equals the Hamming cell's, and a Lee cell with a q = 4
axis differs."""
import numpy as np
import pytest

from oracle.dp_oracle import OracleBackend


def fields(problem, axes, R, code, mu=1):
    o = OracleBackend(axes, R, problem, mu=mu)
    o.recount(code)
    cnt = o.read_cnt().copy()
    o.gain_map()
    gain = o.map.copy()
    o.loss_map()
    return cnt, gain, o.map.copy()


@pytest.mark.parametrize("axes,R,mu", [
    ([2] * 9, 2, 1), ([3] * 7, 3, 2), ([2, 3, 3, 2, 3, 2], 2, 1)])
def test_lee_on_small_axes_is_hamming(axes, R, mu):
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + R)
    code = np.sort(rng.choice(size, size=max(3, size // 25), replace=False))
    for a, b in zip(fields("lee", axes, R, code, mu),
                    fields("hamming", axes, R, code, mu)):
        assert np.array_equal(a, b)


def test_lee_with_a_wider_axis_is_not_hamming():
    axes, R = [4, 3, 3, 3], 2
    code = np.array([0, 17, 50, 77])
    lee = fields("lee", axes, R, code)[0]
    ham = fields("hamming", axes, R, code)[0]
    assert not np.array_equal(lee, ham)
