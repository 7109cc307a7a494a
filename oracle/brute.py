"""Brute-force coverage oracle for tiny spaces (test infrastructure only).

Restates the reference's brute-force backends
(``src/coldcore/reference/base.py:22-97`` and the four ``_covers``
predicates in ``covering.py:16``, ``lee.py:22``, ``torus.py:22``,
``grid.py:23``): every field is a direct count over the coverage relation,
O(|X|^2 n), capped at 2^16 words like the reference (``base.py:19,31``).
"""
import numpy as np

from .dp_oracle import Space

MAX_SPACE = 1 << 16


def covers(problem, axes, R, a, b):
    """dist(a, b) <= R for broadcastable digit arrays (..., n)."""
    if problem == "hamming":
        return (a != b).sum(axis=-1) <= R
    d = np.abs(a.astype(np.int64) - b.astype(np.int64))
    if problem == "grid_linf":
        return d.max(axis=-1) <= R
    d = np.minimum(d, np.asarray(axes, dtype=np.int64) - d)
    if problem == "torus_linf":
        return d.max(axis=-1) <= R
    if problem == "lee":
        return d.sum(axis=-1) <= R
    raise ValueError(problem)


class BruteBackend:
    def __init__(self, axes, R, problem="hamming", mu=1):
        self.problem, self.R, self.mu = problem, int(R), int(mu)
        self.space = Space(axes)
        if self.space.size > MAX_SPACE:
            raise ValueError("brute-force oracle: space too large")
        self.axes = self.space.axes
        self._digs = self.space.digits(np.arange(self.space.size))
        self.cnt = np.zeros(self.space.size, dtype=np.int64)
        self.map = np.zeros(self.space.size, dtype=np.int64)

    def ball_indices(self, w):
        m = covers(self.problem, self.axes, self.R, self._digs,
                   self._digs[int(w)][None, :])
        return np.flatnonzero(m)

    def recount(self, idx):
        self.cnt[:] = 0
        for w in np.atleast_1d(np.asarray(idx, dtype=np.int64)):
            self.cnt[self.ball_indices(w)] += 1

    def _role(self, target):
        if target == 0:
            return self.cnt < self.mu
        if target == 1:
            return (self.cnt >= 1) & (self.cnt <= self.mu)
        return self.cnt == target

    def _field(self, mask):
        sel = np.flatnonzero(mask)
        self.map[:] = 0
        if not len(sel):
            return
        m = covers(self.problem, self.axes, self.R, self._digs[:, None, :],
                   self._digs[None, sel, :])
        self.map[:] = m.sum(axis=1)

    def gain_map(self):
        self._field(self._role(0))

    def loss_map(self):
        self._field(self._role(1))

    def ball_update(self, idx, delta):
        for w in np.atleast_1d(np.asarray(idx, dtype=np.int64)):
            self.cnt[self.ball_indices(w)] += delta

    def ball_gather(self, idx, target):
        mask = self._role(target)
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        return np.array([int(mask[self.ball_indices(w)].sum()) for w in idx],
                        dtype=np.int32)

    def count_eq(self, t):
        return int((self.cnt == t).sum())

    def uncovered(self):
        return int(np.maximum(self.mu - self.cnt, 0).sum())
