"""Out-of-core transforms on the host, without a GPU.

1. The two-phase plan (``plan_pieces``): a numpy executor copies each
   planned piece into a small "device" array, applies only that phase's
   axes there and copies it back; the result is the oracle's whole-space
   transform.
2. The engine's own piece plan (``dct_b200_ooc_plan``) is that rule.
3. The engine's schedule (``dct_b200_ooc_record``: every copy, fill,
   scatter and launch it would issue, in order) replayed on byte arrays:
   every access stays inside its buffer, each device piece is touched only
   by its own stream, 16-bit planes never overflow, and the map, cnt or
   layers it leaves equal the oracle's, for every family, init and output
   mode, with budgets that force many slabs and many ragged columns."""
from math import prod

import numpy as np
import pytest

from coldcore_b200 import build
from coldcore_b200 import outofcore as ooc
from coldcore_b200.outofcore import columns, plan_pieces, plan_stream, slabs
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
IDS = lambda v: str(v).replace(" ", "")                        # noqa: E731


def _code(o, seed):
    rng = np.random.default_rng(seed)
    return rng.choice(o.space.size, max(2, o.space.size // 30), replace=False)


@pytest.mark.parametrize("problem,axes,R", CELLS, ids=IDS)
@pytest.mark.parametrize("budget_words", [64, 200, 1000])
def test_streamed_transform_equals_the_whole_space(problem, axes, R,
                                                   budget_words):
    layered = problem in ("hamming", "lee")
    nl = R + 1 if layered else 1
    o = OracleBackend(axes, R, problem)
    code = _code(o, len(axes) * 10 + R)
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


# ------------------------------------------------------------ the engine
@pytest.fixture(scope="module")
def lib():
    build.build()
    return ooc._lib()


def _budget(R1, cap, out_mode, M):
    """The device budget whose piece capacity is ``cap`` words a plane."""
    per = 2 * (R1 * 4 + (2 if out_mode == 2 else 0))
    return (cap + 64) * per + 8 * M


def test_engine_plan_is_the_split_rule(lib):
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(400):
        problem = str(rng.choice(["hamming", "lee", "torus_linf",
                                  "grid_linf"]))
        n = int(rng.integers(2, 12))
        R = int(rng.integers(1, 4))
        lo = 2 * R + 1 if problem == "torus_linf" else 2
        axes = [int(a) for a in rng.integers(lo, 17, n)]
        if prod(axes) > 1 << 36:
            continue
        R1 = R + 1 if problem in ("hamming", "lee") else 1
        cap = int(rng.integers(8, 1 << 22))
        mw = int(rng.choice([0, 4, 32]))
        out_mode = int(rng.choice([1, 2]))
        try:
            want = plan_pieces(axes, cap, mw or 32)
        except ValueError:
            with pytest.raises(RuntimeError):
                ooc.ooc_plan(problem, axes, R, 0, out_mode,
                             _budget(R1, cap, out_mode, 0), min_width=mw)
            continue
        got = ooc.ooc_plan(problem, axes, R, 0, out_mode,
                           _budget(R1, cap, out_mode, 0), min_width=mw)
        assert got["cap"] == cap
        assert {k: got[k] for k in want} == want
        words = max(want["slab_rows"] * want["p_low"],
                    want["col_width"] * want["p_high"])
        assert words <= cap and got["plane"] == -(-words // 64) * 64
        assert got["device_bytes"] <= _budget(R1, cap, out_mode, 0)
        checked += 1
    assert checked > 300


def test_engine_plan_rejects_what_the_engine_rejects(lib):
    with pytest.raises(RuntimeError):                  # out 2 needs init 0
        ooc.ooc_plan("hamming", [2] * 8, 2, 1, 2, 1 << 20)
    with pytest.raises(RuntimeError):                  # no layers to output
        ooc.ooc_plan("torus_linf", [5] * 4, 1, 0, 3, 1 << 20)
    with pytest.raises(RuntimeError):                  # window-pass cell
        ooc.ooc_plan("torus_linf", [2048, 2048], 1, 0, 1, 1 << 30)
    # the counter rule: min(M, max multiplicity x |B|) <= 65535, |B| = 1351
    ooc.ooc_plan("hamming", [2] * 20, 3, 0, 1, 1 << 30, M=70000, maxmult=48)
    with pytest.raises(RuntimeError):
        ooc.ooc_plan("hamming", [2] * 20, 3, 0, 1, 1 << 30, M=70000,
                     maxmult=49)
    with pytest.raises(RuntimeError):                  # one axis: no split
        ooc.ooc_plan("hamming", [16], 1, 0, 1, 1 << 30)
    with pytest.raises(RuntimeError):                  # budget too small
        ooc.ooc_plan("hamming", [2] * 20, 3, 0, 1, 4096)
    with pytest.raises(RuntimeError):                  # word outside X
        ooc.ooc_record("hamming", [2] * 8, 2, 0, 1, 1 << 20, code=[256])


PRED = {1: lambda c, mu: (c == 0) if mu == 1 else (c < mu),
        2: lambda c, mu: (c == 1) if mu == 1 else ((c >= 1) & (c <= mu))}


def replay(rows, problem, axes, R, init_mode, out_mode, mu, info, code,
           cnt):
    """Run a recorded schedule on byte arrays; returns the output buffer
    (out 1/2) or the host planes (out 3)."""
    X, R1, P = prod(axes), info["R1"], info["plane"]
    s, p_low, p_high = info["split"], info["p_low"], info["p_high"]
    mem = {ooc.BUF_HOST: np.zeros(info["host_bytes"], np.uint8),
           ooc.BUF_PIECE0: np.zeros(R1 * P * 4, np.uint8),
           ooc.BUF_PIECE1: np.zeros(R1 * P * 4, np.uint8),
           ooc.BUF_STAGE0: np.zeros(P * 2, np.uint8),
           ooc.BUF_STAGE1: np.zeros(P * 2, np.uint8),
           ooc.BUF_CODE: np.sort(np.asarray(code, np.int64)).view(np.uint8),
           ooc.BUF_CNT: np.asarray(cnt, np.uint16).view(np.uint8),
           ooc.BUF_OUT: np.zeros(X * (4 if out_mode == 1 else 2), np.uint8)}
    owner = {ooc.BUF_PIECE0: 0, ooc.BUF_PIECE1: 1, ooc.BUF_STAGE0: 0,
             ooc.BUF_STAGE1: 1}
    joins = []

    def region(b, off, nbytes, st):
        assert 0 <= off and off + nbytes <= len(mem[b]), (b, off, nbytes)
        assert owner.get(b, st) == st, (b, st)
        return mem[b][off:off + nbytes]

    for r in rows:
        op, st = int(r[0]), int(r[1])
        if op == ooc.OP_COPY:
            db, doff, sb, soff, nb = (int(v) for v in r[2:7])
            region(db, doff, nb, st)[:] = region(sb, soff, nb, st)
        elif op == ooc.OP_COPY2D:
            db, doff, dp, sb, soff, sp, wb, h = (int(v) for v in r[2:10])
            assert wb <= dp <= ooc.MAX_PITCH and wb <= sp <= ooc.MAX_PITCH
            assert 0 < h and 0 < wb
            dst = region(db, doff, (h - 1) * dp + wb, st)
            src = region(sb, soff, (h - 1) * sp + wb, st)
            for k in range(h):
                dst[k * dp:k * dp + wb] = src[k * sp:k * sp + wb]
        elif op == ooc.OP_ZERO:
            b, off, nb = (int(v) for v in r[2:5])
            region(b, off, nb, st)[:] = 0
        elif op == ooc.OP_SCATTER:
            b, c0, n, x0 = (int(v) for v in r[2:6])
            words = mem[ooc.BUF_CODE].view(np.int64)[c0:c0 + n]
            assert c0 + n <= len(mem[ooc.BUF_CODE]) // 8
            local = words - x0
            assert (local >= 0).all() and (local < P).all()
            region(b, 0, 4 * P, st)
            np.add.at(mem[b].view(np.int32)[:P], local, 1)
        elif op == ooc.OP_LAUNCH:
            (b, plane, l16, src, dst, lin, lout, in16, out16, axis0, k,
             aux, space, phase, inner, mid, outer, pack) = (
                int(v) for v in r[2:20])
            assert plane == P and l16 == 4 * P and owner[b] == st
            sub = (list(axes[:s]) + [space // p_low] if phase == 1
                   else [space // p_high] + list(axes[s:]))
            assert prod(sub) == space <= P
            assert inner == prod(sub[:axis0])
            assert mid == prod(sub[axis0:axis0 + k])
            assert outer * inner * mid == space
            i32 = mem[b].view(np.int32)
            u16 = mem[b][l16:].view(np.uint16)
            if in16 or out16:
                assert l16 + R1 * P * 2 <= len(mem[b])
            A = np.zeros((R1, space), np.int64)
            if src == 0:
                for d in range(lin):
                    A[d] = (u16 if in16 else i32)[d * P:d * P + space]
            else:
                assert src == 1 and aux + space <= X
                c = mem[ooc.BUF_CNT].view(np.uint16)[aux:aux + space]
                A[0] = PRED[init_mode](c.astype(np.int64), mu)
            for j in range(axis0, axis0 + k):
                apply_axis(A, sub, j, problem, R)
            if dst == 0:
                for d in range(lout):
                    if out16:
                        assert A[d].max() <= 65535
                        u16[d * P:d * P + space] = A[d]
                    else:
                        i32[d * P:d * P + space] = A[d]
            elif dst == 1:
                i32[:space] = A.sum(axis=0)
            else:
                stage = ooc.BUF_STAGE0 + st
                mem[stage].view(np.uint16)[:space] = np.minimum(
                    A.sum(axis=0), 65535)
        elif op == ooc.OP_JOIN:
            joins.append(st)
        else:
            raise AssertionError(f"unknown op {op}")
    assert joins == [0, 1, 2]
    if out_mode == 1:
        return mem[ooc.BUF_OUT].view(np.int32)
    if out_mode == 2:
        return mem[ooc.BUF_OUT].view(np.uint16)
    return mem[ooc.BUF_HOST].view(np.int32).reshape(R1, X)


SCHEDULE_CELLS = CELLS + [("hamming", [2] * 11, 4), ("lee", [7] * 4, 5),
                          ("hamming", [4, 4, 4, 4, 4], 2)]
MODES = [(0, 1), (0, 2), (0, 3), (1, 1), (1, 3), (2, 1), (2, 3)]


@pytest.mark.parametrize("problem,axes,R", SCHEDULE_CELLS, ids=IDS)
@pytest.mark.parametrize("cap", [100, 400, 5000])
def test_engine_schedule_replays_to_the_oracle(lib, problem, axes, R, cap):
    layered = problem in ("hamming", "lee")
    R1 = R + 1 if layered else 1
    ran = 0
    for mu in (1, 2):
        o = OracleBackend(axes, R, problem, mu=mu)
        code = _code(o, cap + mu)
        code = np.concatenate([code, code[:3]])         # a multiset
        o.recount(code)
        cnt = o.cnt.copy()
        for init_mode, out_mode in MODES:
            if out_mode == 3 and not layered:
                continue
            if mu == 2 and init_mode == 0:
                continue
            M = len(code) if init_mode == 0 else 0
            budget = _budget(R1, cap, out_mode, M)
            try:
                info = ooc.ooc_plan(problem, axes, R, init_mode, out_mode,
                                    budget, M=M, maxmult=2, min_width=4)
            except RuntimeError:
                continue                                 # no split fits
            rows = ooc.ooc_record(problem, axes, R, init_mode, out_mode,
                                  budget, code=code, mu=mu, min_width=4)
            got = replay(rows, problem, axes, R, init_mode, out_mode, mu,
                         info, code, cnt)
            if init_mode == 0:
                o.recount(code)
                want = o.cnt
            elif init_mode == 1:
                o.gain_map()
                want = o.map
            else:
                o.loss_map()
                want = o.map
            if out_mode == 3:
                assert np.array_equal(got, o.layers()), (init_mode, mu)
            else:
                assert np.array_equal(got, want), (init_mode, out_mode, mu)
            ran += 1
    if cap >= 400:
        assert ran > 0


def test_schedule_pieces_and_traffic(lib):
    """H2(16,3) in 16-bit host planes: the row counts the plan implies and
    the bytes the copies move equal the plan's link bytes."""
    axes, R = [2] * 16, 3
    code = np.arange(0, 1 << 16, 97)
    budget = _budget(4, 3000, 1, len(code))
    info = ooc.ooc_plan("hamming", axes, R, 0, 1, budget, M=len(code),
                        maxmult=1, min_width=4)
    rows = ooc.ooc_record("hamming", axes, R, 0, 1, budget, code=code,
                          min_width=4)
    assert info["half"] == 1 and info["host_word_bytes"] == 2
    ops = rows[:, 0]
    assert (ops == ooc.OP_ZERO).sum() == info["n_slabs"]
    assert (ops == ooc.OP_COPY).sum() == info["n_slabs"] * info["live_mid"]
    c2 = rows[ops == ooc.OP_COPY2D]
    assert len(c2) == info["n_cols"] * (info["live_mid"] + 1)
    link = rows[ops == ooc.OP_COPY, 6].sum()
    h2d = c2[c2[:, 5] == ooc.BUF_HOST]
    link += (h2d[:, 8] * h2d[:, 9]).sum()
    assert link == info["link_bytes"]
    assert set(rows[ops == ooc.OP_LAUNCH, 1]) <= {0, 1}


def test_automatic_placement():
    """coldcore's placement rule on a B200 budget: HBM while the whole cell
    fits, else host layer planes (streamed) with cnt and the map in HBM,
    and managed cnt only when even those 6 bytes a word do not fit."""
    from coldcore_b200.gpu import placement
    assert placement(3 ** 16, 5, budget=160e9) == (0, 0)       # H3(16,4)
    assert placement(2 ** 34, 4, budget=160e9) == (1, 0)       # 309 GB
    assert placement(2 ** 34, 4, budget=320e9) == (0, 0)
    assert placement(10 ** 10, 6, budget=160e9) == (1, 0)      # K_10(10,5)
    assert placement(3 * 10 ** 10, 6, budget=160e9) == (1, 1)
    assert placement(1, 1, budget=0) == (1, 1)


def test_engine_schedule_fuzz(lib):
    """Seeded random cells (every family, mixed radix, up to 20,000 words),
    piece capacities, column widths, modes and multiplicities: each
    schedule that plans replays to the oracle's result."""
    rng = np.random.default_rng(2027)
    ran = 0
    for _ in range(80):
        problem = str(rng.choice(["hamming", "lee", "torus_linf",
                                  "grid_linf"]))
        R = int(rng.integers(1, 5))
        lo = 2 * R + 1 if problem == "torus_linf" else 2
        n = int(rng.integers(2, 8))
        axes = [int(a) for a in rng.integers(lo, 17, n)]
        if problem in ("hamming", "lee") and rng.random() < 0.5:
            axes = [axes[0]] * n
        X = prod(axes)
        if X > 20000 or X < 16:
            continue
        layered = problem in ("hamming", "lee")
        R1 = R + 1 if layered else 1
        modes = [m for m in MODES if layered or m[1] != 3]
        init_mode, out_mode = modes[int(rng.integers(len(modes)))]
        mu = 1 if init_mode == 0 else int(rng.integers(1, 4))
        o = OracleBackend(axes, R, problem, mu=mu)
        code = rng.choice(X, max(1, X // int(rng.integers(10, 60))),
                          replace=False)
        o.recount(code)
        cnt = o.cnt.copy()
        if cnt.max() > 65535:
            continue
        M = len(code) if init_mode == 0 else 0
        cap = int(rng.integers(16, X + 64))
        mw = int(rng.choice([1, 4, 8, 32]))
        budget = _budget(R1, cap, out_mode, M)
        try:
            info = ooc.ooc_plan(problem, axes, R, init_mode, out_mode, budget,
                                M=M, maxmult=1, min_width=mw)
        except RuntimeError:
            continue
        rows = ooc.ooc_record(problem, axes, R, init_mode, out_mode, budget,
                              code=code, mu=mu, min_width=mw)
        got = replay(rows, problem, axes, R, init_mode, out_mode, mu, info,
                     code, cnt)
        if init_mode == 1:
            o.gain_map()
        elif init_mode == 2:
            o.loss_map()
        want = (o.layers() if out_mode == 3
                else o.cnt if init_mode == 0 else o.map)
        assert np.array_equal(got, want), (problem, axes, R, init_mode,
                                           out_mode, mu, cap, mw)
        ran += 1
    assert ran >= 30


def test_pitch_limit_bounds_the_split(lib):
    """K_10(10,5), 10^10 words, on a 100 GB piece budget: P_low = 10^9
    would need a 4 GB row pitch (2-D copies take < 2^31 bytes), so the
    split stops at P_low = 10^8: 5 slabs of 20 rows, then 5 column blocks
    whose rows are 41 MB of 16-bit words."""
    axes, R = [10] * 10, 5
    info = ooc.ooc_plan("hamming", axes, R, 0, 2, 100 << 30, M=60000,
                        maxmult=1)
    assert info["p_low"] == 10 ** 8 and info["split"] == 8
    assert info["p_low"] * 4 <= ooc.MAX_PITCH
    assert info["half"] == 1 and info["live_mid"] == 6
    assert info["link_bytes"] == 2 * 10 ** 10 * 2 * 6
    assert info["device_bytes"] <= 100 << 30
    want = plan_pieces(axes, info["cap"])
    assert {k: info[k] for k in want} == want
    assert info["n_slabs"] == 5 and info["n_cols"] == 5
    assert info["col_width"] * 2 >= 32 << 20            # rows of >= 32 MB
