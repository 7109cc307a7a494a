"""GPU parity through the C-ABI (the GpuBackend binding): every field,
gather, update and query of the engine against the reference's own outputs
(golden fixtures) and the CPU oracle.  Integer work: bit-exact."""
import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend
from golden_data import (FAMILY_CELLS, TRANSFORM_CELLS, WIDE_CELLS, cell_id,
                         key, small)
from oracle.dp_oracle import OracleBackend

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("budget", ["100", "24"])
@pytest.mark.parametrize("axes,R,mu", TRANSFORM_CELLS)
def test_transform_cells(monkeypatch, axes, R, mu, budget):
    """Multiset codes; cnt, gain and loss over every word.  Two tile
    budgets change the axis grouping (one group vs several)."""
    monkeypatch.setenv("CC_SMEM_BUDGET_KB", budget)
    g = small()
    cid = cell_id("hamming", axes, R, mu)
    with GpuBackend(axes, R, mu=mu) as b:
        for k in range(3):
            b.recount(g[key(cid, k, "code")])
            assert np.array_equal(b.read_cnt(), g[key(cid, k, "cnt")])
            b.gain_map()
            assert np.array_equal(b.map_all(), g[key(cid, k, "gain")])
            b.loss_map()
            assert np.array_equal(b.map_all(), g[key(cid, k, "loss")])


@pytest.mark.parametrize("problem,axes,R,mu", FAMILY_CELLS + WIDE_CELLS)
def test_family_cells(problem, axes, R, mu):
    g = small()
    cid = cell_id(problem, axes, R, mu)
    code = g[key(cid, "code")]
    probe = g[key(cid, "probe")]
    with GpuBackend(axes, R, problem=problem, mu=mu) as b:
        b.recount(code)
        assert np.array_equal(b.read_cnt(), g[key(cid, "cnt")])
        assert [b.count_eq(t) for t in range(4)] == list(g[key(cid, "count_eq")])
        assert b.uncovered() == int(g[key(cid, "deficit")])
        b.gain_map()
        assert np.array_equal(b.map_all(), g[key(cid, "gain")])
        mx = b.map_max()
        assert mx == int(g[key(cid, "gain_max")])
        assert np.array_equal(b.map_hist(16, max(mx, 1)),
                              g[key(cid, "gain_hist")])
        thr = int(g[key(cid, "ext_thr")])
        idx, val, found = b.map_extract(thr)
        assert found == int(g[key(cid, "ext_found")])
        assert np.array_equal(np.sort(idx), g[key(cid, "ext_idx")])
        assert np.array_equal(val, g[key(cid, "gain")][idx])
        b.loss_map()
        assert np.array_equal(b.map_all(), g[key(cid, "loss")])
        assert np.array_equal(b.map_read_at(code), g[key(cid, "loss")][code])
        for t in (0, 1, 2):
            assert np.array_equal(b.ball_gather(probe, t),
                                  g[key(cid, "gather", t)])
        for w, s in zip(g[key(cid, "upd_words")], g[key(cid, "upd_signs")]):
            b.ball_update([w], int(s))
        assert np.array_equal(b.read_cnt(), g[key(cid, "upd_cnt")])
        assert np.array_equal(b.ball_gather(probe, 0),
                              g[key(cid, "upd_gather0")])
        assert np.array_equal(b.ball_gather(probe, 1),
                              g[key(cid, "upd_gather1")])


PIPE_PAIR_CELLS = [("hamming", [2] * 16, 3, 1), ("hamming", [2] * 15, 2, 2),
                   ("hamming", [2] * 17, 1, 1), ("lee", [4] * 8, 3, 1)]


@pytest.mark.parametrize("budget", ["16", "40"])
@pytest.mark.parametrize("problem,axes,R,mu", PIPE_PAIR_CELLS,
                         ids=lambda v: str(v))
def test_prefetch_in_pairs(monkeypatch, problem, axes, R, mu, budget):
    """Every group prefetching (CC_PIPE=2): the 16-bit layers of the packed
    launches are copied 16 bytes (4 packed lanes) at a time by cp.async.
    cnt, gain and loss equal the oracle's, and the plans hold that form."""
    monkeypatch.setenv("CC_PIPE", "2")
    monkeypatch.setenv("CC_SMEM_BUDGET_KB", budget)
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + 7 * R + mu)
    code = np.sort(rng.choice(size, size=max(4, size // 300), replace=False))
    o = OracleBackend(axes, R, problem, mu=mu)
    with GpuBackend(axes, R, problem=problem, mu=mu) as b:
        b.recount(code)
        o.recount(code)
        assert np.array_equal(b.read_cnt(), o.cnt)
        b.gain_map()
        o.gain_map()
        assert np.array_equal(b.map_all(), o.map)
        b.loss_map()
        o.loss_map()
        assert np.array_equal(b.map_all(), o.map)
        both = GpuBackend.PIPE | GpuBackend.PACK
        for mode in ((0, 2), (1, 1), (2, 1)):
            forms = b.plan_forms(*mode)
            assert any((f & both) == both for f in forms), forms.tolist()


@pytest.mark.parametrize("problem,axes,R", [("hamming", [2] * 16, 3),
                                            ("lee", [4] * 8, 3),
                                            ("hamming", [3] * 9, 2),
                                            ("hamming", [2, 3, 4, 5], 2)])
def test_plan_probe_matches_the_live_plan(monkeypatch, problem, axes, R):
    """The host-only plan probe gives the launches a live cell runs (cells
    below the autotuner's size, default knobs)."""
    from coldcore_b200.gpu import plan_probe
    monkeypatch.delenv("CC_PIPE", raising=False)
    monkeypatch.delenv("CC_SMEM_BUDGET_KB", raising=False)
    size = int(np.prod(axes))
    code = np.sort(np.random.default_rng(size).choice(size, size // 50,
                                                      replace=False))
    with GpuBackend(axes, R, problem=problem) as b:
        b.recount(code)
        for mode in ((0, 2), (1, 1), (2, 1)):
            live, forms = b.plan(*mode), b.plan_forms(*mode)
            probe = plan_probe(problem, axes, R, *mode)
            assert [(int(r[0]), int(r[1]), int(r[3])) for r in live] == \
                [(L["axis0"], L["axes"], L["kernel"]) for L in probe]
            assert forms.tolist() == [
                L["pipe"] | 2 * L["pack"] | 4 * L["in16"] | 8 * L["out16"] |
                16 * L["pair"] for L in probe]


def test_k3_8_2_config_with_100_updates():
    """K_3(8,2), 30 codewords (seed 0): full int32 count / gain / loss
    fields, then 100 seeded add/remove updates; cnt and count_eq(0..3) after
    every update against the reference's trace."""
    g = small()
    code = g[key("K3_8_2", "code")]
    with GpuBackend([3] * 8, 2) as b:
        b.recount(code)
        assert np.array_equal(b.read_cnt(), g[key("K3_8_2", "cnt")])
        b.gain_map()
        assert np.array_equal(b.map_all(), g[key("K3_8_2", "gain")])
        b.loss_map()
        assert np.array_equal(b.map_all(), g[key("K3_8_2", "loss")])
        tc, tq = g[key("K3_8_2", "trace_cnt")], g[key("K3_8_2", "trace_q")]
        for i, (w, s) in enumerate(zip(g[key("K3_8_2", "upd_words")],
                                       g[key("K3_8_2", "upd_signs")])):
            b.ball_update([w], int(s))
            assert np.array_equal(b.read_cnt(), tc[i])
            q = [b.count_eq(t) for t in range(4)] + [b.uncovered()]
            assert q == list(tq[i])
        b.gain_map()
        assert np.array_equal(b.map_all(), g[key("K3_8_2", "upd_gain")])
        b.loss_map()
        assert np.array_equal(b.map_all(), g[key("K3_8_2", "upd_loss")])


@pytest.mark.parametrize("problem,axes,R,mu", [
    ("hamming", [4] * 5, 2, 1), ("hamming", [3] * 5, 1, 2),
    ("lee", [5, 6, 7], 2, 1), ("torus_linf", [7, 9, 11], 2, 1),
    ("grid_linf", [4, 5, 6], 3, 1), ("grid_linf", [8, 8], 1, 2),
    ("torus_linf", [40, 33], 1, 1)])
def test_update_delta_and_swap_eval(problem, axes, R, mu):
    """ball_update_delta reports the change of uncovered(); swap_eval
    reproduces drop / gather / undo and leaves cnt untouched."""
    o = OracleBackend(axes, R, problem=problem, mu=mu)
    rng = np.random.default_rng(77)
    size = o.space.size
    code = np.sort(rng.choice(size, size=max(4, size // 40), replace=False))
    with GpuBackend(axes, R, problem=problem, mu=mu) as b:
        b.recount(code)
        o.recount(code)
        for w in (code[:1], code[1:4], rng.integers(0, size, 3)):
            w = np.asarray(w, dtype=np.int64)
            sign = -1 if np.isin(w, code).all() else +1
            dd = b.ball_update_delta(w, sign)
            assert dd == o.ball_update_delta(w, sign)
            assert b.uncovered() == o.uncovered()
            assert b.ball_update_delta(w, -sign) == o.ball_update_delta(w, -sign)
        k = 4
        drops = rng.choice(code, size=k, replace=False).astype(np.int64)
        cands = [rng.integers(0, size, size=int(rng.integers(0, 50)))
                 .astype(np.int64) for _ in range(k)]
        cnt0 = b.read_cnt().copy()
        loss, gains = b.swap_eval(drops, cands)
        assert np.array_equal(b.read_cnt(), cnt0)
        ol, og = o.swap_eval(drops, cands)
        assert np.array_equal(loss, ol)
        for a, c in zip(gains, og):
            assert np.array_equal(a, c)
        shared = rng.integers(0, size, size=30).astype(np.int64)
        loss2, g2 = b.swap_eval(drops, shared)
        ol2, og2 = o.swap_eval(drops, shared)
        assert np.array_equal(loss2, ol2) and np.array_equal(g2, og2)
        with pytest.raises(RuntimeError):       # an inactive drop is refused
            inactive = np.setdiff1d(np.arange(size), code)[:1]
            b.swap_eval(inactive, shared)


def test_counter_limit_is_exact_and_rejection_preserves_state():
    """The uint16 bound: accepted up to 65,535 occurrences on one word,
    rejected beyond, and every rejected call leaves cnt intact."""
    code = np.zeros(65535, dtype=np.int64)
    with GpuBackend([3, 3], 1, mu=65535) as g:
        g.recount(code)
        before = g.read_cnt().copy()
        assert before[0] == 65535
        for op in (lambda: g.recount(np.zeros(65536, dtype=np.int64)),
                   lambda: g.ball_update([0], +1),
                   lambda: g.ball_update([1], -1),
                   lambda: g.ball_update([0], 2),
                   lambda: g.recount([-1]),
                   lambda: g.recount([9])):
            with pytest.raises(RuntimeError):
                op()
            np.testing.assert_array_equal(g.read_cnt(), before)
        g.ball_update([0], -1)
        assert g.read_cnt(0, 1)[0] == 65534
        g.ball_update([0], +1)
        np.testing.assert_array_equal(g.read_cnt(), before)
        g.recount([8])
        before = g.read_cnt().copy()
        with pytest.raises(RuntimeError):
            g.ball_update([8, 8], -1)
        np.testing.assert_array_equal(g.read_cnt(), before)
        g.ball_update([8], -1)
        assert not g.read_cnt().any()


def test_distinct_overflow_rejected_exactly():
    """65,536 distinct centres all covering word 0 of H(12, R=6) would take
    cnt[0] past 65,535: rejected; 65,535 of them are accepted."""
    idx = np.arange(3 ** 12, dtype=np.int64)
    digits, weight = idx.copy(), np.zeros(len(idx), dtype=np.int16)
    for _ in range(12):
        weight += digits % 3 != 0
        digits //= 3
    code = idx[weight <= 6][:65536]
    with GpuBackend([3] * 12, 6, mu=65535) as g:
        g.recount(code[:-1])
        assert g.read_cnt(0, 1)[0] == 65535
        with pytest.raises(RuntimeError):
            g.recount(code)
        assert g.read_cnt(0, 1)[0] == 65535
        g.ball_update(code[:1], -1)
        assert g.read_cnt(0, 1)[0] == 65534


@pytest.mark.parametrize("problem,axes,R", [
    ("hamming", [3, 3], 1), ("lee", [5, 5], 1), ("torus_linf", [5, 5], 1),
    ("grid_linf", [5, 5], 1)])
@pytest.mark.parametrize("mu", [1, 2, 3])
def test_owner_loss_counts_every_critical_incidence(problem, axes, R, mu):
    code = np.array([0, 1, 2], dtype=np.int64)
    o = OracleBackend(axes, R, problem=problem, mu=mu)
    o.recount(code)
    base = o.uncovered()
    expected = []
    for i in range(len(code)):
        o.recount(np.delete(code, i))
        expected.append(o.uncovered() - base)
    with GpuBackend(axes, R, problem=problem, mu=mu, use_owner=True) as g:
        np.testing.assert_array_equal(g.loss_owner(code), expected)
        g.ball_update(code, -1)
        assert not g.read_cnt().any()


@pytest.mark.parametrize("cap", [1, 7, 100, 4096])
def test_extract_overflow_counts_exactly(cap):
    o = OracleBackend([5] * 6, 2)
    rng = np.random.default_rng(cap)
    code = np.sort(rng.choice(o.space.size, 30, replace=False))
    with GpuBackend([5] * 6, 2) as g:
        g.recount(code)
        o.recount(code)
        g.gain_map()
        o.gain_map()
        for thr in (1, 2, 5):
            idx, val, found = g.map_extract(thr, cap=cap)
            _, _, cf = o.map_extract(thr)
            assert found == cf and len(idx) == min(cap, cf)
            assert len(np.unique(idx)) == len(idx)
            assert (o.map[idx] == val).all() and (val >= thr).all()


def test_async_updates_then_reads():
    """Hundreds of back-to-back updates that return before the device
    finishes, then reads that must see all of them."""
    q, n, R = 3, 6, 1
    o = OracleBackend([q] * n, R)
    rng = np.random.default_rng(5)
    with GpuBackend([q] * n, R) as g:
        code = np.sort(rng.choice(o.space.size, 30, replace=False))
        g.recount(code)
        o.recount(code)
        live = list(code)
        for i in range(400):
            if i % 3 == 2 and live:
                w = np.array([live.pop(int(rng.integers(len(live))))])
                g.ball_update(w, -1)
                o.ball_update(w, -1)
            else:
                w = rng.integers(0, o.space.size, size=1 + i % 70)
                live.extend(int(x) for x in w)
                g.ball_update(w, +1)
                o.ball_update(w, +1)
            if i % 50 == 0:
                assert g.count_eq(0) == o.count_eq(0)
        assert np.array_equal(g.read_cnt(), o.read_cnt())
        g.gain_map()
        o.gain_map()
        assert np.array_equal(g.map_all(), o.map)


def test_large_batches_and_layers():
    """A 3,000-word update batch (staged path), and the exact distance
    layers N_0..N_R of a transform (out_mode 3) against the oracle."""
    axes, R = [4] * 6, 3
    o = OracleBackend(axes, R)
    rng = np.random.default_rng(9)
    code = rng.integers(0, o.space.size, size=60)
    extra = rng.integers(0, o.space.size, size=3000)
    with GpuBackend(axes, R) as g:
        g.recount(code)
        g.ball_update(extra, +1)
        o.recount(np.concatenate([code, extra]))
        assert np.array_equal(g.read_cnt(), o.read_cnt())
        g._set_code(code)
        g.layers_map(0)
        o.recount(code)
        for d in range(R + 1):
            assert np.array_equal(g.layer(d), o.layers()[d])
