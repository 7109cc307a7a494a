"""The transform planner on the host, without a GPU (``plan_probe``): for
every geometry, transform, tile budget, prefetch mode and plane width, the
launches cover each axis once, their tiles fit, and the packed and
prefetching forms appear only where their alignment rules hold.  These are
the conditions the kernels index under, so a plan that broke one would read
or write out of place on the device."""
import math

import numpy as np
import pytest

from coldcore_b200.gpu import plan_probe

SRC_LAYERS, SRC_CNT, SRC_CODE = 0, 1, 2
DST_LAYERS, DST_MAP, DST_CNT = 0, 1, 2
MAX_SMEM = 227 * 1024

GEOMETRIES = [
    ("hamming", [2] * 26, 3), ("hamming", [2] * 22, 1),
    ("hamming", [2] * 12, 7), ("hamming", [2] * 5, 2),
    ("hamming", [3] * 16, 4), ("hamming", [3] * 14, 3),
    ("hamming", [4] * 11, 4), ("hamming", [5] * 10, 3),
    ("hamming", [6] * 9, 3), ("hamming", [2, 3, 4, 5, 6, 7], 3),
    ("hamming", [10, 9, 8, 7, 6], 5), ("hamming", [16, 3, 2], 2),
    ("hamming", [2, 2, 3, 3, 2, 2], 2),
    ("lee", [7] * 8, 4), ("lee", [2] * 23, 2), ("lee", [4] * 8, 3),
    ("lee", [5] * 10, 1), ("lee", [6] * 9, 3), ("lee", [16, 3, 2], 2),
    ("torus_linf", [7, 9, 11], 2), ("torus_linf", [5] * 8, 1),
    ("grid_linf", [4, 5, 6], 3), ("grid_linf", [16, 4], 1),
]
MODES = [(0, 2), (1, 1), (2, 1), (0, 3), (0, 1)]
KNOBS = [(16, 1), (24, 2), (64, 1), (100, 1), (100, 2), (100, 3), (160, 3),
         (200, 2)]


def smem_bytes(launch, R1):
    """Shared bytes of one launch: the tile's layers (skewed, one pad row),
    doubled for a prefetched layer source, plus two cnt windows for a
    prefetched cnt source."""
    tw = launch["Bo"] * launch["mid"]
    skw = tw + (tw >> launch["skew"]) if launch["skew"] else tw
    lanes = launch["W"] // 2 if launch["pack"] else launch["W"]
    lay = (skw + 1) * lanes * R1
    tile = (lay + 3) // 4 * 4 * 4
    if not launch["pipe"]:
        return tile
    if launch["src"] == SRC_CNT:
        return tile + 2 * ((tw + 16 + 7) // 8 * 8) * 2
    return 2 * tile


def live_layers(problem, axes, j, R):
    reach = sum(a // 2 if problem == "lee" else 1 for a in axes[:j])
    return min(reach, R) + 1


def check_plan(plan, problem, axes, R, mode, budget_kb, pipe, half):
    layered = problem in ("hamming", "lee")
    # Lee distance on axes of size 2 or 3 is the Hamming distance: such a
    # cell is planned as Hamming (transform_geometry)
    if problem == "lee" and max(axes) <= 3:
        problem = "hamming"
    R1 = R + 1 if layered else 1
    n = len(axes)
    space = math.prod(axes)
    init, out = mode
    final_dst = {1: DST_MAP, 2: DST_CNT, 3: DST_LAYERS}[out]
    half_on = half and R1 >= 2 and final_dst != DST_LAYERS
    assert plan, "no launch"
    j = 0
    for i, L in enumerate(plan):
        last = i == len(plan) - 1
        # ---- the launches cover axes 0..n-1 once, in order
        assert L["axis0"] == j
        k = L["axes"] - L["pair"]
        assert k >= 1 or (L["pair"] and k >= 0)
        j0 = j + L["pair"]
        if L["pair"]:
            assert i == 0 and problem == "hamming" and half_on
            assert axes[0] == 2 and axes[1] == 2 and init != 3
            assert L["inner"] == 2
        else:
            assert L["inner"] == math.prod(axes[:j])
        assert L["mid"] == math.prod(axes[j0:j0 + k])
        assert L["outer"] * L["inner"] * L["mid"] == space
        j += L["axes"]
        # ---- tiles
        W = L["W"]
        if L["inner"] >= 32:
            assert W in (16, 32) and L["Bo"] == 1
        else:
            assert W == L["inner"]
        assert L["tiles"] == (-(-L["outer"] // L["Bo"]) *
                              -(-L["inner"] // W))
        assert L["smem"] == smem_bytes(L, R1)
        assert L["smem"] <= MAX_SMEM
        if k > 1:
            assert L["smem"] <= budget_kb * 1024
        if L["kernel"] >= 0:
            assert L["round_axes"] == k and L["rounds"] >= 1
        else:
            assert L["rounds"] == 0 and not L["pack"] and not L["pipe"]
        assert L["skew"] == 0 or W == 1 or (L["pair"] and W == 2)
        # ---- sources, destinations, plane widths
        assert L["src"] == ((SRC_CODE if init == 0 else SRC_CNT) if i == 0
                            else SRC_LAYERS)
        assert L["dst"] == (final_dst if last else DST_LAYERS)
        assert L["in16"] == int(half_on and i > 0)
        assert L["out16"] == int(half_on and not last)
        if layered:
            assert L["lin"] == live_layers(problem, axes, L["axis0"], R)
            assert L["lout"] == (R1 if last and final_dst == DST_LAYERS
                                 else live_layers(problem, axes, j, R))
        else:
            assert L["lin"] == L["lout"] == 1
        # ---- packed pairs: 4-byte pair accesses, add-only recurrences
        if L["pack"]:
            q = axes[j0] if k else 2
            assert L["in16"] or L["pair"]
            assert L["inner"] % 2 == 0 and W % 2 == 0 and L["kernel"] >= 0
            assert problem == "lee" or (problem == "hamming" and q <= 3)
        # ---- prefetching: register kernels, never the staged code or the
        # pair group; over 16-bit planes only in the 16-byte packed form
        if L["pipe"]:
            assert L["kernel"] >= 0 and L["src"] != SRC_CODE
            assert not L["pair"]
            if L["in16"]:
                assert L["pack"] and W % 8 == 0 and L["inner"] % 8 == 0
        # ---- launch shape
        assert L["threads"] % 32 == 0 and 32 <= L["threads"] <= 512
        assert 1 <= L["grid"] <= max(1, L["tiles"])
        assert L["grid"] <= 148 * 32
    assert j == n


@pytest.mark.parametrize("problem,axes,R", GEOMETRIES,
                         ids=lambda v: str(v).replace(" ", ""))
def test_plans_cover_fit_and_align(problem, axes, R):
    layered = problem in ("hamming", "lee")
    for mode in MODES:
        if mode[1] == 3 and not layered:
            continue
        for budget, pipe in KNOBS:
            for half in (True, False):
                plan = plan_probe(problem, axes, R, *mode, budget_kb=budget,
                                  pipe=pipe, half=half)
                check_plan(plan, problem, axes, R, mode, budget, pipe, half)


def test_h2_26_3_groupings():
    """The five groupings the autotuner chooses among for H2(26,3)."""
    want = {(100, 1): [(0, 13), (13, 9), (22, 4)],
            (160, 1): [(0, 14), (14, 10), (24, 2)],
            (64, 1): [(0, 12), (12, 8), (20, 6)],
            (100, 2): [(0, 13), (13, 8), (21, 5)],
            (160, 2): [(0, 14), (14, 9), (23, 3)]}
    for (budget, pipe), groups in want.items():
        for mode in ((0, 2), (1, 1)):
            plan = plan_probe("hamming", [2] * 26, 3, *mode,
                              budget_kb=budget, pipe=pipe)
            assert [(L["axis0"], L["axes"]) for L in plan] == groups
            assert plan[0]["pair"] and all(L["pack"] for L in plan)


def test_wide_window_cells_have_no_groups_and_bad_args_raise():
    assert plan_probe("torus_linf", [2048, 2048], 1, 1, 1) == []
    with pytest.raises(RuntimeError):
        plan_probe("hamming", [2] * 4, 1, 1, 2)          # cnt out needs init 0
    with pytest.raises(RuntimeError):
        plan_probe("torus_linf", [5, 5], 1, 0, 3)        # no layers to output
    with pytest.raises(RuntimeError):
        plan_probe("hamming", [17, 2], 1, 1, 1)          # axis above 16
    with pytest.raises(RuntimeError):
        plan_probe("hamming", [2] * 4, 1, 1, 1, budget_kb=8)


N_FUZZ = 300


def test_planner_fuzz():
    """Seeded random geometries (mixed radix, every family, up to 2^34
    words): the same invariants on every plan."""
    rng = np.random.default_rng(2026)
    checked = 0
    for _ in range(N_FUZZ):
        problem = str(rng.choice(["hamming", "hamming", "lee", "torus_linf",
                                  "grid_linf"]))
        n = int(rng.integers(1, 13))
        if problem == "torus_linf":
            R = int(rng.integers(1, 3))
            axes = [int(a) for a in rng.integers(2 * R + 1, 17, n)]
        elif problem == "grid_linf":
            R = int(rng.integers(1, 4))
            axes = [int(a) for a in rng.integers(2, 17, n)]
        else:
            R = int(rng.integers(1, 8))
            q = int(rng.integers(2, 17))
            axes = ([q] * n if rng.random() < 0.6
                    else [int(a) for a in rng.integers(2, 17, n)])
        if math.prod(axes) > 1 << 34:
            continue
        layered = problem in ("hamming", "lee")
        modes = MODES if layered else [m for m in MODES if m[1] != 3]
        mode = modes[int(rng.integers(len(modes)))]
        budget, pipe = KNOBS[int(rng.integers(len(KNOBS)))]
        half = bool(rng.random() < 0.7)
        plan = plan_probe(problem, axes, R, *mode, budget_kb=budget,
                          pipe=pipe, half=half)
        check_plan(plan, problem, axes, R, mode, budget, pipe, half)
        checked += 1
    assert checked > N_FUZZ * 0.8


@pytest.mark.parametrize("axes,R", [([2] * 20, 2), ([3] * 12, 3),
                                    ([2, 3] * 6, 2)])
def test_lee_on_small_axes_plans_as_hamming(axes, R):
    """A Lee cell whose axes are all of size 2 or 3 gets the Hamming cell's
    launches (the distances are the same); one axis of size 4 keeps Lee."""
    for mode in MODES:
        assert plan_probe("lee", axes, R, *mode) == \
            plan_probe("hamming", axes, R, *mode)
    wider = [4] + axes[1:]
    assert plan_probe("lee", wider, R, 1, 1) != \
        plan_probe("hamming", wider, R, 1, 1)
