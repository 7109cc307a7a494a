"""Learned ruin proposal for the LNS of :mod:`coldcore_b200.search`.

The proposal plugs into the ruin choice of coldcore's LNS round
(src/coldcore/search.py:734-743): given the incumbent code, it chooses
which k incumbents to remove.  The exact repair and the exact counters
still score every round (search.py:744-754).

Pieces:

* :class:`RuinFeatures`: 32 features per incumbent c, read from exact
  fields the engine already builds:
  - the exact loss of c and its rank among the incumbents;
  - a log2 histogram of the gain map over B_R(c).  A word's gain counts
    the uncovered words of its own ball, so this histogram sees the
    uncovered words of B_2R(c);
  - a histogram of the coverage counts cnt over B_R(c);
  - the per-distance layer counts N_d(c) of the critical words (covered
    exactly mu times: the words c alone covers, by their distance from c)
    and of the code (d = 0..R, from ``layers_map`` + ``layers_at``), each
    scaled by the sphere size;
  - two ranks among the incumbents: the log-gain mass of the ball (how
    much uncovered territory lies within 2R), and the ball words of
    positive gain.
  Every feature describes c relative to the current state; none is
  constant across a round, so the model ranks incumbents rather than
  rounds.
* :class:`MoveLog`: a ``Searcher.move_log`` hook.  It records the features
  of every removed incumbent with a label.  The label is 1 when the round's
  repair covered more than the code before the ruin and did not put that
  incumbent back, 0 otherwise.
* :func:`train_scorer`: z-scores the features and fits the GPU MLP
  (:class:`coldcore_b200.mlp.GpuMlp`).  It reports the AUC on held-out
  rounds, pooled (the gate reads this) and within rounds.
* :class:`LearnedRuin`: the proposer that ``select="learned"`` calls.  It
  scores every incumbent and draws k of them without replacement with
  probabilities softmax(score / temperature) (the Gumbel top-k draw), or,
  with ``pick="anchor"``, draws one anchor that way and removes the k
  incumbents nearest it.  A confidence gate hands the round back to the
  bandit in two cases: the model's held-out AUC was below ``auc_min``, or
  the learned rounds' recent rewards fall below half of the fallback
  rounds'.
"""
import time

import numpy as np

from .mlp import N_IN, GpuMlp

N_FEATURES = N_IN
_HIST_BINS = 8
_MAX_D = 6          # layer slots per field (d = 0..5)


def sphere_sizes(axes, R, problem):
    """Words at each distance d = 0..R from a word (Hamming or Lee)."""
    poly = np.zeros(R + 1, dtype=np.float64)
    poly[0] = 1.0
    for a in axes:
        per = np.zeros(R + 1)
        for x in range(a):
            d = (1 if x else 0) if problem == "hamming" else min(x, a - x)
            if d <= R:
                per[d] += 1
        poly = np.convolve(poly, per)[:R + 1]
    return poly


def _rank(v):
    """Rank percentile in [0, 1], ties in order of position."""
    v = np.asarray(v, dtype=np.float64)
    return np.argsort(np.argsort(v, kind="stable")) / max(1, len(v) - 1)


class RuinFeatures:
    """Per-incumbent features from exact fields (GPU backend)."""

    def __init__(self, backend):
        b = self.b = backend
        self.layered = b.problem in ("hamming", "lee")
        self.R = int(b.R)
        self.ball = float(b.ball_len)
        self.sphere = (sphere_sizes(b.space.axes, self.R, b.problem)
                       if self.layered else None)
        self.seconds = 0.0
        self.calls = 0

    def compute(self, code, uncov):
        t0 = time.perf_counter()
        b, R, B = self.b, self.R, self.ball
        code = np.asarray(code, dtype=np.int64)
        m = len(code)
        f = np.zeros((m, N_FEATURES), dtype=np.float32)
        if m == 0:
            return f
        if self.layered:
            # the critical words by distance; their sum is the loss map
            b.layers_map(2)
            crit = b.layers_at(code)
            loss = crit.sum(axis=1).astype(np.float64)
        else:
            b.loss_map()
            loss = np.asarray(b.map_read_at(code), dtype=np.float64)
        f[:, 0] = loss / B
        f[:, 1] = _rank(loss)
        b.gain_map()
        gh = b.ball_hist(code, 0, _HIST_BINS)
        f[:, 2:10] = gh / B
        f[:, 10:18] = b.ball_hist(code, 1, _HIST_BINS) / B
        if self.layered:
            nd = min(R + 1, _MAX_D)
            sph = self.sphere[:nd][None, :]
            f[:, 18:18 + nd] = crit[:, :nd] / sph
            b.stage_code(code)
            b.layers_map(0)                    # the code by distance
            f[:, 24:24 + nd] = b.layers_at(code)[:, :nd] / sph
        f[:, 30] = _rank(gh @ np.arange(_HIST_BINS, dtype=np.float64))
        f[:, 31] = _rank(1.0 - f[:, 2].astype(np.float64))
        self.seconds += time.perf_counter() - t0
        self.calls += 1
        return f


class MoveLog:
    """``Searcher.move_log`` hook: (features, label) for every removal."""

    def __init__(self, features, cap=10 ** 5):
        self.features = features
        self.cap = int(cap)
        self.X, self.y, self.round_id, self.mode = [], [], [], []
        self._f = self._rows = self._words = self._kept = None
        self._mode = None
        self.rounds = 0

    def __len__(self):
        return sum(len(x) for x in self.X)

    @property
    def full(self):
        return len(self) >= self.cap

    def __call__(self, s, event, **info):
        if event == "pre":
            self._f = self.features.compute(s.code, s.uncov)
            self._mode = info.get("mode")
        elif event == "ruin":
            pick = np.asarray(info["pick"], dtype=np.int64)
            self._rows = self._f[pick]
            self._words = s.code[pick].copy()
        elif event == "repair" and self._rows is not None:
            self._kept = np.isin(self._words, info["code"])
        elif event == "post" and self._rows is not None:
            improved = info["post"] < info["pre"]
            label = np.where(self._kept, 0.0, 1.0 if improved else 0.0)
            self.X.append(self._rows)
            self.y.append(label.astype(np.float32))
            self.round_id.append(np.full(len(self._rows), self.rounds))
            self.mode.extend([self._mode] * len(self._rows))
            self.rounds += 1
            self._rows = self._kept = None

    def arrays(self):
        if not self.X:
            return (np.zeros((0, N_FEATURES), np.float32),
                    np.zeros(0, np.float32), np.zeros(0, np.int64))
        return (np.concatenate(self.X)[:self.cap],
                np.concatenate(self.y)[:self.cap],
                np.concatenate(self.round_id)[:self.cap])


def auc(scores, labels):
    """Area under the ROC curve (rank statistic, ties averaged)."""
    scores = np.asarray(scores, dtype=np.float64)
    labels = np.asarray(labels) > 0.5
    npos, nneg = int(labels.sum()), int((~labels).sum())
    if npos == 0 or nneg == 0:
        return 0.5
    order = np.argsort(scores, kind="stable")
    ranks = np.empty(len(scores))
    s = scores[order]
    i = 0
    while i < len(s):
        j = i
        while j + 1 < len(s) and s[j + 1] == s[i]:
            j += 1
        ranks[order[i:j + 1]] = 0.5 * (i + j) + 1.0
        i = j + 1
    return float((ranks[labels].sum() - npos * (npos + 1) / 2) / (npos * nneg))


def grouped_auc(scores, labels, groups):
    """Mean AUC within groups (rounds) that hold both labels, weighted by
    their number of (positive, negative) pairs."""
    scores, labels, groups = (np.asarray(scores), np.asarray(labels),
                              np.asarray(groups))
    num = den = 0.0
    for gid in np.unique(groups):
        sel = groups == gid
        y = labels[sel] > 0.5
        pairs = float(y.sum()) * float((~y).sum())
        if pairs:
            num += auc(scores[sel], labels[sel]) * pairs
            den += pairs
    return num / den if den else None


class Scorer:
    """z-scored features -> GPU MLP logit."""

    def __init__(self, mlp, mean, std, heldout_auc=None):
        self.mlp, self.mean, self.std = mlp, mean, std
        self.heldout_auc = heldout_auc
        self.within_auc = self.train_auc = None

    def __call__(self, X):
        return self.mlp.predict((np.asarray(X, np.float32) - self.mean) /
                                self.std)


def heldout_rounds(y, groups, holdout, rng):
    """Mask of the held-out moves: the same share of the rounds with a
    positive move and of those without, whole rounds only, so a rare label
    cannot leave the held-out slice one-sided."""
    ug, inv = np.unique(groups, return_inverse=True)
    pos_g = np.zeros(len(ug), dtype=bool)
    np.logical_or.at(pos_g, inv, np.asarray(y) > 0.5)
    picked = []
    for part in (ug[pos_g], ug[~pos_g]):
        if len(part) >= 2:
            picked.append(rng.choice(part, size=max(1, int(len(part) *
                                                           holdout)),
                                     replace=False))
    return np.isin(groups, np.concatenate(picked) if picked else [])


def train_scorer(X, y, groups=None, epochs=30, batch=512, lr=2e-3, seed=0,
                 holdout=0.1):
    """Fit the MLP on logged moves.  The held-out slice is split by round
    (``groups``), so the moves of one round never straddle the split.
    Returns a :class:`Scorer` whose ``heldout_auc`` is the pooled AUC of
    the held-out rounds (``within_auc``: the AUC within those rounds)."""
    X = np.asarray(X, dtype=np.float32)
    y = np.asarray(y, dtype=np.float32)
    groups = np.arange(len(y)) if groups is None else np.asarray(groups)
    test = heldout_rounds(y, groups, holdout, np.random.default_rng(seed))
    mean = X[~test].mean(axis=0)
    std = X[~test].std(axis=0) + 1e-3
    mlp = GpuMlp(seed=seed)
    mlp.train((X[~test] - mean) / std, y[~test], epochs=epochs, batch=batch,
              lr=lr, seed=seed)
    sc = Scorer(mlp, mean.astype(np.float32), std.astype(np.float32))
    if not (y > 0.5).any():
        sc.heldout_auc = 0.0           # nothing to learn from: gate closed
    elif test.any():
        st = sc(X[test])
        sc.heldout_auc = auc(st, y[test])
        sc.within_auc = grouped_auc(st, y[test], groups[test])
    sc.train_auc = auc(sc(X[~test][:20000]), y[~test][:20000])
    return sc


class LearnedRuin:
    """The ``select="learned"`` proposer, with its confidence gate."""

    def __init__(self, scorer, features, auc_min=0.6, temperature=0.5,
                 score_weight=1.0, decay=0.9, seed=0, pick="topk",
                 scale="raw"):
        if pick not in ("topk", "anchor"):
            raise ValueError(f"unknown pick rule {pick!r}")
        if scale not in ("raw", "std"):
            raise ValueError(f"unknown score scale {scale!r}")
        self.pick, self.scale = pick, scale
        self.scorer, self.features = scorer, features
        self.auc_min = float(auc_min)
        self.temperature = float(temperature)
        self.score_weight = float(score_weight)
        self.decay = float(decay)
        self.rng = np.random.default_rng(seed)
        self.ema = {"learned": 1.0, "fallback": 1.0}
        self.stats = {"proposed": 0, "gated_auc": 0, "gated_reward": 0,
                      "gated_flat": 0}

    def gate_open(self):
        auc_ok = (self.scorer.heldout_auc is None or
                  self.scorer.heldout_auc >= self.auc_min)
        if not auc_ok:
            self.stats["gated_auc"] += 1
            return False
        if (self.ema["learned"] < 0.5 * self.ema["fallback"]
                and self.rng.random() > 0.1):
            self.stats["gated_reward"] += 1
            return False
        return True

    def propose(self, s, k):
        if k <= 0 or not self.gate_open():
            return None
        f = self.features.compute(s.code, s.uncov)
        z = np.asarray(self.scorer(f), dtype=np.float64)
        if z.std() < 1e-4:
            self.stats["gated_flat"] += 1
            return None
        self.stats["proposed"] += 1
        if self.pick == "topk":
            # Gumbel top-k: k draws without replacement, P ~ exp(z / T);
            # scale="std" measures T in units of this round's score spread
            zt = z if self.scale == "raw" else (z - z.mean()) / z.std()
            gumbel = -np.log(-np.log(self.rng.random(len(z)) + 1e-300))
            return np.argsort(-(zt / self.temperature + gumbel))[:k]
        p = np.exp((z - z.max()) / self.temperature)
        p /= p.sum()
        anchor = int(self.rng.choice(len(z), p=p))
        digs = s.b.index_word(s.code).astype(np.int16)
        d = (digs != digs[anchor][None, :]).sum(axis=1).astype(np.float64)
        zr = (z - z.mean()) / (z.std() + 1e-9)
        key = (d - self.score_weight * 0.25 * np.tanh(zr) +
               0.5 * self.rng.random(len(z)))
        return np.argsort(key)[:k]

    def observe(self, s, mode, pre, post, new_best):
        from .search import OperatorBandit
        r = OperatorBandit.tier(new_best, pre, post)
        arm = "learned" if mode == "learned" else "fallback"
        self.ema[arm] = self.decay * self.ema[arm] + (1 - self.decay) * r
