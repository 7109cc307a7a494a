"""The learned ruin proposal on the B200: features against the brute-force
oracle, the move log, training, and LNS rounds chosen by the model."""
import numpy as np
import pytest

from oracle.dp_oracle import OracleBackend
from oracle.feature_oracle import features as oracle_features

pytestmark = pytest.mark.gpu

CELLS = [("hamming", [3] * 6, 1, 1), ("hamming", [3, 4, 5, 3], 2, 1),
         ("lee", [5, 5, 5], 1, 1), ("hamming", [3] * 5, 1, 2),
         ("hamming", [2] * 10, 3, 1)]


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from coldcore_b200 import gpu as g
    return g


@pytest.mark.parametrize("cell", CELLS, ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}")
def test_features_match_oracle(gpu, cell):
    from coldcore_b200.learned import RuinFeatures
    prob, axes, R, mu = cell
    size = int(np.prod(axes))
    rng = np.random.default_rng(size + R)
    code = np.sort(rng.choice(size, size=max(4, size // 20), replace=False))
    b = gpu.GpuBackend(axes, R, prob, mu=mu)
    try:
        b.recount(code)
        uncov = b.uncovered()
        got = RuinFeatures(b).compute(code, uncov)
    finally:
        b.close()
    want, wunc = oracle_features(OracleBackend(axes, R, prob, mu=mu), code)
    assert uncov == wunc
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-7)


def test_ball_hist_counts_every_ball_word(gpu):
    axes, R = [4] * 5, 2
    size = 4 ** 5
    b = gpu.GpuBackend(axes, R, "hamming")
    try:
        code = np.arange(0, size, 37, dtype=np.int64)
        b.recount(code)
        b.gain_map()
        h0 = b.ball_hist(code, 0, 8)
        h1 = b.ball_hist(code, 1, 8)
        assert (h0.sum(axis=1) == b.ball_len).all()
        assert (h1.sum(axis=1) == b.ball_len).all()
        ob = OracleBackend(axes, R, "hamming")
        ob.recount(code)
        for i, c in enumerate(code):
            ball = ob.ball_indices(c)
            want = np.bincount(np.minimum(ob.cnt[ball], 7), minlength=8)
            assert (h1[i] == want).all()
    finally:
        b.close()


def test_layers_at_reads_exact_layers(gpu):
    axes, R = [3] * 7, 3
    b = gpu.GpuBackend(axes, R, "hamming")
    try:
        rng = np.random.default_rng(5)
        code = np.sort(rng.choice(3 ** 7, 40, replace=False))
        b.stage_code(code)
        b.layers_map(0)
        idx = rng.integers(0, 3 ** 7, 300)
        got = b.layers_at(idx)
        for d in range(R + 1):
            assert (got[:, d] == b.layer(d)[idx]).all()
    finally:
        b.close()


def _solved_start(gpu, axes, R, seed):
    from coldcore_b200.search import Searcher
    b = gpu.GpuBackend(axes, R, "hamming")
    s = Searcher(b, seed=seed)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    s.peel()
    return b, s


def test_move_log_train_and_learned_lns(gpu):
    from coldcore_b200.learned import (LearnedRuin, MoveLog, RuinFeatures,
                                       train_scorer)
    from coldcore_b200.search import Searcher
    b, s = _solved_start(gpu, [3] * 7, 1, 3)
    try:
        feats = RuinFeatures(b)
        mlog = MoveLog(feats, cap=4000)
        start = s.code.copy()
        for seed in range(3):
            t = Searcher(b, seed=10 + seed, move_log=mlog)
            t.build_reserve_s = t.loop_reserve_s = 0.0
            t.load(start)
            t.ruin(3, "low")
            t.lns(len(start) - 2, round_budget_s=4.0, kmin=2, kmax=6,
                  log_every=0)
            assert t.verify_full() == t.uncov
        X, y, g = mlog.arrays()
        assert len(X) == len(y) == len(g) > 100
        assert set(np.unique(y)) <= {0.0, 1.0}
        sc = train_scorer(X, y, g, epochs=5)
        assert sc(X[:10]).shape == (10,)
        prop = LearnedRuin(sc, feats, auc_min=0.0, seed=1)
        t = Searcher(b, seed=99, proposer=prop)
        t.build_reserve_s = t.loop_reserve_s = 0.0
        t.load(start)
        t.ruin(3, "low")
        t.lns(len(start) - 2, round_budget_s=3.0, kmin=2, kmax=6,
              select="learned", log_every=0)
        assert t.stats["learned_rounds"] >= 1
        assert prop.stats["proposed"] == t.stats["learned_rounds"]
        # every round was scored exactly: the incremental count is the recount
        assert t.verify_full() == t.uncov
        assert len(np.unique(t.code)) == len(t.code)
    finally:
        b.close()


def test_gate_closes_on_low_auc(gpu):
    from coldcore_b200.learned import LearnedRuin, RuinFeatures

    class Flat:
        heldout_auc = 0.4

        def __call__(self, X):
            return np.zeros(len(X), np.float32)

    b, s = _solved_start(gpu, [3] * 6, 1, 2)
    try:
        prop = LearnedRuin(Flat(), RuinFeatures(b), auc_min=0.55)
        assert prop.propose(s, 4) is None
        assert prop.stats["gated_auc"] == 1
        Flat.heldout_auc = 0.9
        assert prop.propose(s, 4) is None          # flat scores: no opinion
        assert prop.stats["gated_flat"] == 1
    finally:
        b.close()


def test_learned_proposal_beats_plain_lns_on_k3_14_3(gpu):
    """On K_3(14,3) (4.78M words, R = 3), from the same greedy start per
    seed, descents whose ruins the trained model picks run in the same wall
    time as plain descents with the record mix, over three seeds: both arms
    end on verified covers, the model picks ruins, and the learned arm's
    best size stays within four words of the plain arm's in every seed.
    The device exact greedy repairs both arms (thousands of rounds a run),
    every size is a full recount, and the model is trained here on moves
    logged from plain runs on other seeds.  Which arm ends smaller in 20 s
    varies from run to run; the time-to-size comparison is the bench's
    five-seed LNS leg."""
    from coldcore_b200.learned import LearnedRuin, RuinFeatures, train_scorer
    from harness.lns_study import descent, greedy_start, log_moves
    b = gpu.GpuBackend([3] * 14, 3)
    try:
        feats = RuinFeatures(b)
        mlog = log_moves(b, feats, 30000, 60.0, 15.0, say=lambda *a: None,
                         repair="device")
        X, y, g = mlog.arrays()
        assert len(y) >= 10000 and 0 < y.mean() < 0.5
        sc = train_scorer(X, y, g, epochs=15)
        assert sc.heldout_auc > 0.6
        bests = []
        for seed in (7, 8, 9):
            start = greedy_start(b, seed)
            plain, _, ok_p = descent(b, start, seed, 20.0, "fixed",
                                     notch_s=10.0, repair="device")
            prop = LearnedRuin(sc, feats, seed=seed)
            learned, st, ok_l = descent(b, start, seed, 20.0, "learned",
                                        proposer=prop, notch_s=10.0,
                                        repair="device")
            assert ok_p and ok_l
            assert st["learned_rounds"] > 0
            bests.append((min(m for _, m in plain),
                          min(m for _, m in learned)))
        assert all(lv <= pv + 4 for pv, lv in bests), bests
    finally:
        b.close()
