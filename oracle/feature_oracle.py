"""Brute-force restatement of the learned ruin proposal's features.

Test infrastructure only: the GPU features of
``coldcore_b200.learned.RuinFeatures`` are checked against this on small
cells.  Everything here is read off explicit distances between words; there
are no transforms.
"""
import numpy as np


def _distance(problem, axes, a, B):
    """Distance from word digits ``a`` (n,) to every row of ``B`` (m, n)."""
    if problem == "hamming":
        return (B != a[None, :]).sum(axis=1)
    ax = np.asarray(axes)[None, :]
    d = np.abs(B - a[None, :])
    return np.minimum(d, ax - d).sum(axis=1)


def features(ob, code, n_features=32, bins=8, max_d=6):
    """Features of every incumbent over an ``OracleBackend`` ``ob``.

    The slots are: loss/|B|; loss rank/(m-1); log2 gain histogram/|B| (8);
    cnt histogram/|B| (8); critical words at distance d / |S_d| (6);
    codewords at distance d / |S_d| (6); the rank of the ball's log-gain
    mass (sum of bin index x count); the rank of the ball words of positive
    gain."""
    code = np.asarray(code, dtype=np.int64)
    m, B = len(code), float(ob.ball_len)
    R, axes, prob = ob.R, ob.axes, ob.problem
    ob.recount(code)
    cnt = ob.cnt.copy()
    uncov = int(np.maximum(ob.mu - cnt, 0).sum())
    words = ob.space.digits(np.arange(ob.space.size))
    deficient = cnt < ob.mu
    critical = (cnt >= 1) & (cnt <= ob.mu)
    # gain of every word: its deficient ball words
    gain = np.zeros(ob.space.size, dtype=np.int64)
    loss = np.zeros(m, dtype=np.int64)
    sphere = np.zeros(R + 1)
    d0 = _distance(prob, axes, words[0], words)
    for d in range(R + 1):
        sphere[d] = (d0 == d).sum()
    for x in range(ob.space.size):
        gain[x] = deficient[ob.ball_indices(x)].sum()
    f = np.zeros((m, n_features), dtype=np.float64)
    crit_words = words[critical]
    code_words = words[code]
    mass = np.zeros(m)
    for i, c in enumerate(code):
        ball = ob.ball_indices(c)
        loss[i] = critical[ball].sum()
        g = gain[ball]
        gb = np.where(g <= 0, 0, np.minimum(
            bins - 1, np.floor(np.log2(np.maximum(g, 1))) + 1))
        f[i, 2:2 + bins] = np.bincount(gb.astype(int), minlength=bins)[:bins]
        mass[i] = f[i, 2:2 + bins] @ np.arange(bins)
        cb = np.minimum(cnt[ball], bins - 1)
        f[i, 10:10 + bins] = np.bincount(cb.astype(int), minlength=bins)[:bins]
        if prob in ("hamming", "lee"):
            nd = min(R + 1, max_d)
            dk = _distance(prob, axes, words[c], crit_words)
            dc = _distance(prob, axes, words[c], code_words)
            for d in range(nd):
                f[i, 18 + d] = (dk == d).sum() / sphere[d]
                f[i, 24 + d] = (dc == d).sum() / sphere[d]
    f[:, 2:18] /= B
    f[:, 0] = loss / B

    def rank(v):
        return np.argsort(np.argsort(v, kind="stable")) / max(1, m - 1)

    f[:, 1] = rank(loss)
    f[:, 30] = rank(mass)
    f[:, 31] = rank(1.0 - f[:, 2].astype(np.float32).astype(np.float64))
    return f.astype(np.float32), uncov
