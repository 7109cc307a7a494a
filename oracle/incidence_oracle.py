"""CPU restatement of coldcore's explicit-incidence backends (plugin ABI 2).

Test infrastructure only: the checker of the ABI-2 engine
(``coldcore_b200/csrc/sparse/sparse_abi.cu``), never part of the product path.

Restates, with the same integer semantics:

* ``SparseIncidenceBackend`` (coldcore ``src/coldcore/incidence.py:89-298``):
  n_cand candidates, each covering the d universe elements of one row of
  an ``(n_cand, d)`` matrix.  ``recount`` scatters the solution's rows into
  ``cnt`` (:189-191), ``gain_map`` / ``loss_map`` count deficient
  (``cnt < mu``) / critical (``1 <= cnt <= mu``) elements per candidate
  (:193-197, roles :180-187), ``ball_update`` adds ``delta`` per incidence
  (:200-201), ``ball_gather`` answers the role counts for listed
  candidates, any other target being the literal ``cnt == target``
  (:203-220);
* ``WeightedIncidenceBackend`` (``incidence.py:301-419``): CSR rows with
  per-incidence weights ``w >= 1`` and universe weights ``uw >= 1``; an
  update adds ``delta * w``; the fields are the exact weighted marginals
  (:374-384): gain ``uw * min(w, max(0, mu - cnt))``, loss
  ``uw * (max(0, mu - cnt + w) - max(0, mu - cnt))`` where ``cnt >= w``,
  other targets literal and unweighted; ``uncovered`` is
  ``sum uw * max(0, mu - cnt)`` (:407-409);
* the shared queries of ``DenseFieldBackend`` (``src/coldcore/protocol.py``):
  ``count_eq`` literal over the universe, ``map_max`` (0 for an empty or
  non-positive map), ``map_hist`` (positive v in bin
  ``(v - 1) * nbins // vmax``, clipped to the last), ``map_extract``
  (every candidate with ``map >= thr``, the true count even past the cap).

Pinned against the reference's own backends by ``tests/golden/
incidence_golden.npz`` (``tests/golden/make_incidence_golden.py``) and
against the dict-of-lists brute force below.
"""
import numpy as np


class _OneAxis:
    """The one-axis index set a search core walks (incidence.py:48-86)."""

    def __init__(self, size):
        self.size, self.n, self.axes = int(size), 1, [int(size)]

    def index_word(self, idx):
        return np.asarray(idx, dtype=np.int64).reshape(-1, 1)

    def word_index(self, words):
        return np.asarray(words, dtype=np.int64).reshape(-1)


class IncidenceOracle:
    """Dense (n_cand, d) incidence rows, with the backend protocol the
    search core asks (fields, gathers, updates, map queries)."""

    indep_dist = None

    def __init__(self, inc, n_univ, mu=1, extract_cap=1 << 22):
        self.inc = np.ascontiguousarray(inc, dtype=np.int64)
        self.n_cand, self.d = self.inc.shape
        self.n_univ, self.mu = int(n_univ), int(mu)
        self.cnt = np.zeros(self.n_univ, dtype=np.int64)
        self.map = np.zeros(self.n_cand, dtype=np.int64)
        self.space = _OneAxis(self.n_cand)
        self.extract_cap = int(extract_cap)

    def index_word(self, idx):
        return self.space.index_word(idx)

    def word_index(self, words):
        return self.space.word_index(words)

    def map_read_at(self, idx):
        return self.map[np.atleast_1d(np.asarray(idx, dtype=np.int64))]

    def map_all(self):
        return self.map

    def read_cnt(self, off=0, length=None):
        length = self.n_univ - off if length is None else length
        return self.cnt[off:off + length].astype(np.uint16)

    def deficient_universe(self, limit, rng=None):
        """Up to ``limit`` universe elements with cnt < mu, sorted; a random
        subset of them when ``rng`` is given (incidence.py:232-238)."""
        u = np.flatnonzero(self.cnt < self.mu)
        if rng is not None and len(u) > limit:
            u = np.sort(rng.choice(u, size=int(limit), replace=False))
        return u[:limit].astype(np.int64)

    def verify(self, idx):
        c = np.zeros(self.n_univ, dtype=np.int64)
        np.add.at(c, self.rows_of(idx).ravel(), 1)
        return bool((c >= self.mu).all())

    # ---- roles (incidence.py:180-187)
    def role(self, c, target):
        if target == 0:
            return c < self.mu
        if target == 1:
            return (c >= 1) & (c <= self.mu)
        return c == target

    def rows_of(self, idx):
        return self.inc[np.asarray(idx, dtype=np.int64).ravel()]

    def recount(self, idx):
        self.cnt[:] = 0
        self.ball_update(idx, 1)

    def ball_update(self, idx, delta):
        np.add.at(self.cnt, self.rows_of(idx).ravel(), int(delta))

    def ball_gather(self, idx, target):
        rows = self.rows_of(idx)
        return self.role(self.cnt[rows], int(target)).sum(axis=1)

    def field(self, target):
        self.map[:] = self.ball_gather(np.arange(self.n_cand), target)

    def gain_map(self):
        self.field(0)

    def loss_map(self):
        self.field(1)

    def uncovered(self):
        return int(np.maximum(self.mu - self.cnt, 0).sum())

    # ---- queries shared by both forms
    def count_eq(self, target):
        return int((self.cnt == target).sum())

    def map_max(self):
        return int(max(0, self.map.max(initial=0)))

    def map_hist(self, nbins, vmax):
        v = self.map[self.map > 0]
        b = np.minimum((v - 1) * nbins // vmax, nbins - 1)
        return np.bincount(b, minlength=nbins)[:nbins]

    def map_extract(self, thr, cap=None):
        """Ascending candidates with map >= thr, the first min(found, cap)
        of them, and the true count (protocol.py:201-208 without the
        optional shuffle)."""
        cap = min(cap or self.extract_cap, self.extract_cap)
        idx = np.flatnonzero(self.map >= thr)
        return idx[:cap], self.map[idx[:cap]], len(idx)


class WeightedIncidenceOracle(IncidenceOracle):
    """CSR rows with incidence weights w and universe weights uw."""

    def __init__(self, indptr, indices, w, n_univ, uw=None, mu=1):
        self.indptr = np.asarray(indptr, dtype=np.int64)
        self.indices = np.asarray(indices, dtype=np.int64)
        self.w = np.asarray(w, dtype=np.int64)
        self.n_cand = len(self.indptr) - 1
        self.n_univ, self.mu = int(n_univ), int(mu)
        self.uw = (np.ones(self.n_univ, dtype=np.int64) if uw is None
                   else np.asarray(uw, dtype=np.int64))
        self.cnt = np.zeros(self.n_univ, dtype=np.int64)
        self.map = np.zeros(self.n_cand, dtype=np.int64)
        self.space = _OneAxis(self.n_cand)
        self.extract_cap = 1 << 22

    def _row(self, c):
        s, e = self.indptr[c], self.indptr[c + 1]
        return self.indices[s:e], self.w[s:e]

    def ball_update(self, idx, delta):
        for c in np.asarray(idx, dtype=np.int64).ravel():
            u, w = self._row(int(c))
            np.add.at(self.cnt, u, w * int(delta))

    def values(self, u, w, target):
        """Per-incidence contributions (incidence.py:374-384)."""
        c = self.cnt[u]
        if target == 0:
            return self.uw[u] * np.minimum(w, np.maximum(0, self.mu - c))
        if target == 1:
            return (self.uw[u] * (np.maximum(0, self.mu - c + w)
                                  - np.maximum(0, self.mu - c)) * (c >= w))
        return (c == target).astype(np.int64)

    def ball_gather(self, idx, target):
        out = []
        for c in np.asarray(idx, dtype=np.int64).ravel():
            u, w = self._row(int(c))
            out.append(int(self.values(u, w, int(target)).sum()))
        return np.asarray(out, dtype=np.int64)

    def uncovered(self):
        return int((self.uw * np.maximum(self.mu - self.cnt, 0)).sum())


def brute_cnt(rows, n_univ, sol):
    """Multiplicities by explicit loops over the solution's rows."""
    c = [0] * n_univ
    for s in sol:
        for u in rows[int(s)]:
            c[int(u)] += 1
    return np.asarray(c, dtype=np.int64)


def brute_gather(rows, cnt, mu, cands, target):
    """Role counts by explicit loops (incidence.py:180-187)."""
    def role(c):
        if target == 0:
            return c < mu
        if target == 1:
            return 1 <= c <= mu
        return c == target
    return np.asarray([sum(role(int(cnt[int(u)])) for u in rows[int(w)])
                       for w in cands], dtype=np.int64)


def colex_rank(subset):
    """Colex rank of a sorted subset: sum_j C(s_j, j + 1)
    (coldcore ``problems/covering_design.py:59-73``)."""
    from math import comb
    return sum(comb(int(s), j + 1) for j, s in enumerate(sorted(subset)))


def design_incidence(v, k, t):
    """The C(v,k,t) incidence in coldcore's layout
    (``problems/covering_design.py:95-135``): rows in colex order of the
    blocks, columns the block's t-subsets by lex order of their positions,
    entries their colex ranks.  Plain loops: small designs only."""
    from itertools import combinations
    blocks = sorted(combinations(range(v), k), key=colex_rank)
    subs = list(combinations(range(k), t))
    return np.array([[colex_rank([b[p] for p in s]) for s in subs]
                     for b in blocks], dtype=np.int64)


class DesignOracle(IncidenceOracle):
    """A covering design C(v,k,t) (mu-fold) with the block metric of
    coldcore's design backend (``problems/covering_design.py:200-229``):
    distance k - |A n B|, removal independence beyond k - t."""

    def __init__(self, v, k, t, mu=1):
        from itertools import combinations
        from math import comb
        super().__init__(design_incidence(v, k, t), comb(v, t), mu=mu)
        self.v, self.k, self.t = v, k, t
        self.blocks = np.array(sorted(combinations(range(v), k),
                                      key=colex_rank), dtype=np.int64)
        self.indep_dist = k - t

    def universe_distance(self, idx, univ):
        """t - |B n T|: 0 exactly where block covers the t-subset
        (covering_design.py:221-229)."""
        from itertools import combinations
        if not hasattr(self, "_tsets"):
            self._tsets = np.array(sorted(combinations(range(self.v), self.t),
                                          key=colex_rank), dtype=np.int64)
        B = self.blocks[np.atleast_1d(np.asarray(idx, dtype=np.int64))]
        T = self._tsets[np.atleast_1d(np.asarray(univ, dtype=np.int64))]
        shared = (B[:, None, :, None] == T[None, :, None, :]).any(
            axis=-1).sum(axis=-1)
        return (self.t - shared).astype(np.int64)

    def distance(self, a, b):
        A = self.blocks[np.asarray(a, dtype=np.int64)]
        B = self.blocks[np.asarray(b, dtype=np.int64)]
        shared = (A[..., :, None] == B[..., None, :]).any(axis=-1).sum(axis=-1)
        return (self.k - shared).astype(np.int64)
