"""The streamed form of the strided groups (tensor loads into shared-memory
stages, transform_tma.cu) against the oracle: with CC_TMA=1 every group it
serves takes it (the strided groups and the first group, read from cnt or
from the code); recount, gain and loss fields must equal the oracle's, bit
for bit, on binary Hamming cells of one to four groups, mu = 1 and 2."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu

TMA = 32                                 # GpuBackend.plan_forms bit


@pytest.mark.parametrize("axes,R,mu", [
    ([2] * 20, 3, 1), ([2] * 21, 3, 2), ([2] * 16, 3, 1),
    ([2] * 12, 3, 1), ([2] * 23, 3, 1), ([2] * 13 + [3], 3, 1)])
def test_streamed_groups_match_the_oracle(monkeypatch, axes, R, mu):
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_U8", "0")
    monkeypatch.setenv("CC_TUNE", "0")
    size = int(np.prod(axes))
    rng = np.random.default_rng(size % 1000 + R)
    code = np.sort(rng.choice(size, size=size // 200, replace=False))
    o = OracleBackend(axes, R, mu=mu)
    with GpuBackend(axes, R, mu=mu) as b:
        used = 0
        for step in range(2):
            if step:
                code = np.sort(rng.choice(size, size=size // 150,
                                          replace=False))
            b.recount(code)
            o.recount(code)
            assert np.array_equal(b.read_cnt(), o.read_cnt()), step
            b.gain_map()
            o.gain_map()
            assert np.array_equal(b.map_all(), o.map), step
            b.loss_map()
            o.loss_map()
            assert np.array_equal(b.map_all(), o.map), step
            for im, om in ((0, 2), (1, 1), (2, 1)):
                used += int(np.count_nonzero(b.plan_forms(im, om) & TMA))
        assert used > 0, "no launch took the streamed form"


@pytest.mark.parametrize("axes,R,mu", [
    ([3] * 11, 4, 1), ([3] * 13, 4, 1), ([3] * 12, 3, 2), ([3] * 14, 3, 1)])
def test_padded_ternary_plan_matches_the_oracle(monkeypatch, axes, R, mu):
    """Ternary cells: the first group (row pairs packed in 32-bit lanes)
    writes its 16-bit planes with rows padded to a multiple of 64 words, so
    the later groups stream them in packed pairs and the last one stores
    the canonical layout.  Every launch of every transform is streamed."""
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_TUNE", "0")
    size = int(np.prod(axes))
    rng = np.random.default_rng(size % 997 + R)
    o = OracleBackend(axes, R, mu=mu)
    with GpuBackend(axes, R, mu=mu) as b:
        for step in range(2):
            code = np.sort(rng.choice(size, size=size // (90 + 60 * step),
                                      replace=False))
            b.recount(code)
            o.recount(code)
            assert np.array_equal(b.read_cnt(), o.read_cnt()), step
            b.gain_map()
            o.gain_map()
            assert np.array_equal(b.map_all(), o.map), step
            b.loss_map()
            o.loss_map()
            assert np.array_equal(b.map_all(), o.map), step
            for im, om in ((0, 2), (1, 1), (2, 1)):
                forms = b.plan_forms(im, om)
                assert len(forms) >= 2 and (forms & TMA).all(), (im, forms)


def test_padded_ternary_plan_counts_a_multiset(monkeypatch):
    """A code with repeated words (the counts of the packed row pairs carry
    multiplicities) and mu = 3 (deficit and critical predicates)."""
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_TUNE", "0")
    axes, R, mu = [3] * 12, 3, 3
    size = 3 ** 12
    rng = np.random.default_rng(12)
    code = np.sort(rng.integers(0, size, size // 40))
    o = OracleBackend(axes, R, mu=mu)
    with GpuBackend(axes, R, mu=mu) as b:
        b.recount(code)
        o.recount(code)
        assert np.array_equal(b.read_cnt(), o.read_cnt())
        b.gain_map()
        o.gain_map()
        assert np.array_equal(b.map_all(), o.map)
        b.loss_map()
        o.loss_map()
        assert np.array_equal(b.map_all(), o.map)
        assert (b.plan_forms(0, 2) & TMA).all()


BYTE8 = 64                               # GpuBackend.plan_forms bit


@pytest.mark.parametrize("axes,R,mu", [
    ([2] * 20, 3, 1), ([2] * 21, 3, 2), ([2] * 23, 3, 1), ([2] * 26, 3, 1)])
def test_byte_planes_after_the_first_group(monkeypatch, axes, R, mu):
    """Gain and loss of binary R = 3 cells: the streamed first group (12
    axes at most, so every layer value is at most C(12, 3) = 220) writes
    8-bit planes past the 16-bit ones and the next launch stages them as
    bytes; fields equal the oracle's, and the recount keeps 16-bit planes.
    A 64 KB tile budget gives the 12-axis first group."""
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_TUNE", "0")
    monkeypatch.setenv("CC_SMEM_BUDGET_KB", "64")
    size = int(np.prod(axes))
    rng = np.random.default_rng(size % 991 + mu)
    o = OracleBackend(axes, R, mu=mu)
    with GpuBackend(axes, R, mu=mu) as b:
        for step in range(2):
            code = np.sort(rng.choice(size, size=size // (180 + 40 * step),
                                      replace=False))
            b.recount(code)
            o.recount(code)
            assert np.array_equal(b.read_cnt(), o.read_cnt()), step
            b.gain_map()
            o.gain_map()
            assert np.array_equal(b.map_all(), o.map), step
            b.loss_map()
            o.loss_map()
            assert np.array_equal(b.map_all(), o.map), step
        for im, om in ((1, 1), (2, 1)):
            forms = b.plan_forms(im, om)
            assert forms[0] & BYTE8 and forms[1] & BYTE8, (im, forms)
        assert not (b.plan_forms(0, 2) & BYTE8).any()


@pytest.mark.parametrize("axes,R,budget", [
    ([3] * 14, 3, "34"), ([3] * 13, 4, "42"), ([3] * 12, 3, "34")])
def test_six_axis_ternary_first_group(monkeypatch, axes, R, budget):
    """The padded plan with a six-axis first group (a 729-word row padded
    to 768, two rows a tile in the register kernel) and the later axes in
    two streamed groups: recount, gain and loss equal the oracle's over
    three codes, one a multiset."""
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_TUNE", "0")
    monkeypatch.setenv("CC_PIPE", "0")
    monkeypatch.setenv("CC_SMEM_BUDGET_KB", budget)
    size = int(np.prod(axes))
    rng = np.random.default_rng(size % 983 + R)
    o = OracleBackend(axes, R, mu=2)
    with GpuBackend(axes, R, mu=2) as b:
        for step in range(3):
            if step == 2:
                code = np.sort(rng.integers(0, size, size // 70))
            else:
                code = np.sort(rng.choice(size, size=size // (80 + 50 * step),
                                          replace=False))
            b.recount(code)
            o.recount(code)
            assert np.array_equal(b.read_cnt(), o.read_cnt()), step
            b.gain_map()
            o.gain_map()
            assert np.array_equal(b.map_all(), o.map), step
            b.loss_map()
            o.loss_map()
            assert np.array_equal(b.map_all(), o.map), step
        plan = b.plan(1, 1)
        assert int(plan[0][1]) == 6, plan
        assert (b.plan_forms(1, 1)[1:] & TMA).all()


@pytest.mark.parametrize("axes,R,mu,u8", [
    ([2] * 20, 3, 1, "1"), ([2] * 23, 3, 2, "1"), ([2] * 23, 3, 1, "0")])
def test_three_axis_rounds_in_the_eight_axis_group(monkeypatch, axes, R, mu,
                                                   u8):
    """The eight-axis streamed group with three-axis register rounds (8-word
    blocks, 512 threads), over 16-bit or 8-bit planes: fields equal the
    oracle's.  A 64 KB tile budget gives the 12 | 8 | ... grouping."""
    monkeypatch.setenv("CC_TMA", "1")
    monkeypatch.setenv("CC_TMA_BM", "3")
    monkeypatch.setenv("CC_U8", u8)
    monkeypatch.setenv("CC_TUNE", "0")
    monkeypatch.setenv("CC_SMEM_BUDGET_KB", "64")
    size = int(np.prod(axes))
    rng = np.random.default_rng(size % 977 + mu)
    o = OracleBackend(axes, R, mu=mu)
    with GpuBackend(axes, R, mu=mu) as b:
        for step in range(2):
            code = np.sort(rng.choice(size, size=size // (170 + 30 * step),
                                      replace=False))
            b.recount(code)
            o.recount(code)
            assert np.array_equal(b.read_cnt(), o.read_cnt()), step
            b.gain_map()
            o.gain_map()
            assert np.array_equal(b.map_all(), o.map), step
            b.loss_map()
            o.loss_map()
            assert np.array_equal(b.map_all(), o.map), step
        plan = b.plan(1, 1)
        assert [int(r[1]) for r in plan[:2]] == [12, 8], plan
