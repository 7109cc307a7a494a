"""Host logic of the learned ruin proposal, on the CPU.

An oracle-backed stand-in supplies the three field queries the feature
builder needs (``ball_hist``, ``layers_map`` / ``layers_at``,
``stage_code``).  The feature slots assembled by
:class:`coldcore_b200.learned.RuinFeatures` must then equal the brute-force
restatement.  The move log and the AUC are checked here as well."""
import numpy as np
import pytest

from coldcore_b200.learned import (MoveLog, RuinFeatures, auc, grouped_auc,
                                   sphere_sizes)
from coldcore_b200.search import Searcher
from oracle.dp_oracle import OracleBackend
from oracle.feature_oracle import features as oracle_features


class FieldOracle(OracleBackend):
    """OracleBackend plus the feature queries, by their definitions."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self._staged = np.zeros(0, dtype=np.int64)

    def stage_code(self, idx):
        self._staged = np.asarray(idx, dtype=np.int64)

    def layers_map(self, init_mode=0):
        self._A[:] = 0
        if init_mode == 0:
            np.add.at(self._A[0], self._staged, 1)
        elif init_mode == 1:
            self._A[0] = self._deficient()
        else:
            self._A[0] = self._critical()
        self._transform(self.map)

    def layers_at(self, idx):
        return self._A[:, np.asarray(idx, dtype=np.int64)].T.astype(np.int32)

    def ball_hist(self, idx, src=0, nbins=8):
        out = np.zeros((len(idx), nbins), dtype=np.int32)
        for i, w in enumerate(np.asarray(idx, dtype=np.int64)):
            ball = self.ball_indices(w)
            if src == 0:
                v = self.map[ball]
                b = np.where(v <= 0, 0, np.minimum(
                    nbins - 1, np.floor(np.log2(np.maximum(v, 1))) + 1))
            else:
                b = np.minimum(self.cnt[ball], nbins - 1)
            out[i] = np.bincount(b.astype(int), minlength=nbins)[:nbins]
        return out


@pytest.mark.parametrize("cell", [("hamming", [3] * 5, 1, 1),
                                  ("hamming", [3, 4, 3, 2], 2, 1),
                                  ("lee", [5, 6, 5], 2, 1),
                                  ("hamming", [3] * 4, 1, 2)],
                         ids=lambda c: f"{c[0]}-{c[1]}-R{c[2]}-mu{c[3]}")
def test_feature_slots_match_brute_force(cell):
    prob, axes, R, mu = cell
    size = int(np.prod(axes))
    rng = np.random.default_rng(size)
    code = np.sort(rng.choice(size, size=max(4, size // 15), replace=False))
    fb = FieldOracle(axes, R, prob, mu=mu)
    fb.recount(code)
    got = RuinFeatures(fb).compute(code, fb.uncovered())
    want, _ = oracle_features(OracleBackend(axes, R, prob, mu=mu), code)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-7)


def test_sphere_sizes():
    assert sphere_sizes([3] * 14, 3, "hamming").tolist() == [1, 28, 364, 2912]
    assert sphere_sizes([5, 5], 2, "lee").tolist() == [1, 4, 8]
    assert sphere_sizes([4], 2, "lee").tolist() == [1, 2, 1]


def test_auc_matches_rank_definition():
    rng = np.random.default_rng(0)
    s = rng.normal(size=500).round(1)            # ties on purpose
    y = (rng.random(500) < 0.3).astype(float)
    pos, neg = s[y > 0.5], s[y < 0.5]
    want = ((pos[:, None] > neg[None, :]).sum() +
            0.5 * (pos[:, None] == neg[None, :]).sum()) / (len(pos) * len(neg))
    assert abs(auc(s, y) - want) < 1e-12
    assert auc(np.zeros(10), np.ones(10)) == 0.5


def test_grouped_auc_ignores_between_round_offsets():
    # within each round the score ranks perfectly; the rounds' base levels
    # are anti-correlated with their labels, which a pooled AUC would punish
    s = np.array([10.0, 11.0, 0.0, 1.0])
    y = np.array([0.0, 1.0, 0.0, 1.0])
    g = np.array([0, 0, 1, 1])
    assert grouped_auc(s, y, g) == 1.0
    assert grouped_auc(s, np.zeros(4), g) is None


def test_move_log_records_rounds():
    fb = FieldOracle([3] * 5, 1, "hamming")
    mlog = MoveLog(RuinFeatures(fb), cap=10 ** 6)
    s = Searcher(fb, seed=3, move_log=mlog)
    s.build_reserve_s = s.loop_reserve_s = 0.0
    s.load([])
    s.greedy_fill(10 ** 9)
    s.peel()
    s.ruin(3, "low")
    s.lns(len(s.code), round_budget_s=2.0, kmin=2, kmax=4, log_every=0)
    X, y, g = mlog.arrays()
    assert mlog.rounds == s.stats["rounds"] > 0
    assert X.shape[1] == 32 and len(X) == len(y) == len(g)
    assert set(np.unique(y)) <= {0.0, 1.0}


def test_move_log_labels_elements():
    """Label 1: the round improved and the repair did not put the removed
    incumbent back."""
    fb = FieldOracle([3] * 4, 1, "hamming")
    mlog = MoveLog(RuinFeatures(fb))

    class S:
        pass

    s = S()
    s.code = np.array([0, 10, 20, 30, 40, 50], dtype=np.int64)
    fb.recount(s.code)
    s.uncov = fb.uncovered()
    mlog(s, "pre", k=3, mode="low")
    mlog(s, "ruin", pick=np.array([1, 3, 4]))
    mlog(s, "repair", code=np.array([0, 20, 30, 50, 7, 8]))
    mlog(s, "post", pre=9, post=5, after=5, new_best=True)
    mlog(s, "pre", k=2, mode="hole")
    mlog(s, "ruin", pick=np.array([0, 5]))
    mlog(s, "repair", code=np.array([10, 20, 30, 40, 1, 2]))
    mlog(s, "post", pre=5, post=6, after=5, new_best=False)
    X, y, g = mlog.arrays()
    # round 0 removed 10, 30, 40 and re-added 30; round 1 did not improve
    assert y.tolist() == [1.0, 0.0, 1.0, 0.0, 0.0]
    assert g.tolist() == [0, 0, 0, 1, 1]
    assert mlog.mode == ["low"] * 3 + ["hole"] * 2


def test_heldout_rounds_keep_both_labels():
    from coldcore_b200.learned import heldout_rounds
    g = np.repeat(np.arange(200), 5)
    y = np.zeros(len(g), dtype=np.float32)
    y[g == 17] = 1.0                          # two rare positive rounds
    y[(g == 123) & (np.arange(len(g)) % 5 == 0)] = 1.0
    for seed in range(20):
        t = heldout_rounds(y, g, 0.1, np.random.default_rng(seed))
        assert (y[t] > 0.5).any() and (y[t] < 0.5).any()
        for r in np.unique(g[t]):             # whole rounds only
            assert t[g == r].all()


def test_time_to_size_target_and_bound():
    from harness.lns_study import summarize, time_to_size
    row = {"start_M": 100,
           "fixed": {"trace": [(0.0, 100)], "best": 100},
           "adaptive": {"trace": [(0.0, 100), (40.0, 99)], "best": 99},
           "learned": {"trace": [(0.0, 100), (5.0, 99), (9.0, 97)],
                       "best": 97}}
    r = time_to_size(row, ["fixed", "adaptive"], 60.0)
    assert r["target_M"] == 99 and r["t_plain"] == 40.0
    assert r["t_learned"] == 5.0 and abs(r["ratio"] - 0.125) < 1e-12
    row["adaptive"] = {"trace": [(0.0, 100)], "best": 100}
    r = time_to_size(row, ["fixed", "adaptive"], 60.0)
    assert r["target_M"] == 99 and r["t_plain"] is None
    assert r["ratio"] is None and abs(r["ratio_bound"] - 5.0 / 60) < 1e-12
    row.update(r)
    s = summarize([row])
    assert s["learned_reached"] == "1/1" and s["best_learned"] == [97]
