"""The streaming plan for cells larger than device memory, run on the host:
a numpy executor copies each planned piece into a small "device" array,
applies only that phase's axes there and copies it back.  The result must
be the oracle's whole-space transform, layer for layer, for every family
and for budgets that force many slabs and many narrow columns."""
from math import prod

import numpy as np
import pytest

from coldcore_b200.outofcore import columns, plan_stream, slabs
from oracle.dp_oracle import OracleBackend


def apply_axis(A, axes, j, problem, R):
    """One axis recurrence over a (layers, prod(axes)) array, in place
    (the oracle's per-axis passes on an arbitrary geometry)."""
    nl = A.shape[0]
    s = prod(axes[:j])
    q = axes[j]
    v = A.reshape(nl, A.shape[1] // (q * s), q, s)
    if problem == "hamming":
        tot = v.sum(axis=2)
        for d in range(nl - 1, 0, -1):
            v[d] += tot[d - 1][:, None, :] - v[d - 1]
    elif problem == "lee":
        half = q // 2
        for d in range(nl - 1, 0, -1):
            for w in range(1, min(d, half) + 1):
                v[d] += np.roll(v[d - w], w, axis=1)
                if not (q % 2 == 0 and w == half):
                    v[d] += np.roll(v[d - w], -w, axis=1)
    elif problem == "torus_linf":
        acc = np.zeros_like(v[0])
        for e in range(-R, R + 1):
            acc += np.roll(v[0], -e, axis=1)
        v[0] = acc
    else:
        h, _, inner = v.shape[1:]
        cs = np.zeros((h, q + 1, inner), dtype=A.dtype)
        np.cumsum(v[0], axis=1, out=cs[:, 1:, :])
        a = np.arange(q)
        lo, hi = np.maximum(a - R, 0), np.minimum(a + R, q - 1) + 1
        v[0] = cs[:, hi, :] - cs[:, lo, :]


def stream(A, axes, problem, R, plan):
    """Execute the plan on host layers A (layers, |X|), piece by piece."""
    s, p_low, p_high = plan["split"], plan["p_low"], plan["p_high"]
    nl = A.shape[0]
    for x, words in slabs(plan):                    # phase 1: low axes
        dev = A[:, x:x + words].copy()
        sub = list(axes[:s]) + [words // p_low]
        for j in range(s):
            apply_axis(dev, sub, j, problem, R)
        A[:, x:x + words] = dev
    grid = A.reshape(nl, p_high, p_low)
    for x0, w in columns(plan):                     # phase 2: high axes
        dev = np.ascontiguousarray(grid[:, :, x0:x0 + w]).reshape(nl, -1)
        sub = [w] + list(axes[s:])
        for j in range(1, len(sub)):
            apply_axis(dev, sub, j, problem, R)
        grid[:, :, x0:x0 + w] = dev.reshape(nl, p_high, w)


CELLS = [("hamming", [3] * 7, 2), ("hamming", [2] * 12, 3),
         ("hamming", [2, 3, 4, 5, 3], 3), ("lee", [5, 6, 7, 4], 3),
         ("torus_linf", [5, 7, 6, 5], 2), ("grid_linf", [4, 6, 5, 3], 2)]


@pytest.mark.parametrize("problem,axes,R", CELLS,
                         ids=lambda v: str(v).replace(" ", ""))
@pytest.mark.parametrize("budget_words", [64, 200, 1000])
def test_streamed_transform_equals_the_whole_space(problem, axes, R,
                                                   budget_words):
    layered = problem in ("hamming", "lee")
    nl = R + 1 if layered else 1
    o = OracleBackend(axes, R, problem)
    rng = np.random.default_rng(len(axes) * 10 + R)
    code = rng.choice(o.space.size, max(2, o.space.size // 30), replace=False)
    o.recount(code)                       # the oracle's whole-space layers
    want = o.layers().copy()
    A = np.zeros_like(want)
    np.add.at(A[0], code, 1)              # layer 0 of the code
    try:
        plan = plan_stream(axes, nl, 4, budget_words * nl * 4 * 2,
                           min_width=4)
    except ValueError:
        pytest.skip("no two-phase split at this budget")
    assert plan["n_slabs"] >= 1 and plan["n_cols"] >= 1
    stream(A, axes, problem, R, plan)
    assert np.array_equal(A, want)


def test_plan_geometry():
    plan = plan_stream([2] * 34, 4, 2, 64 << 30)    # 2^34 words, 64 GB
    assert plan["p_low"] * plan["p_high"] == 2 ** 34
    assert plan["slab_rows"] * plan["p_low"] * 4 * 2 * 2 <= 64 << 30
    assert plan["col_width"] * plan["p_high"] * 4 * 2 * 2 <= 64 << 30
    assert plan["col_width"] % 32 == 0
    covered = sum(w for _, w in slabs(plan))
    assert covered == 2 ** 34
    assert sum(w for _, w in columns(plan)) == plan["p_low"]
    with pytest.raises(ValueError):
        plan_stream([2] * 40, 8, 4, 1 << 20)         # far too small
