"""numpy restatement of the reference's axis-DP CPU backend (test oracle).

Follows coldcore ``src/coldcore/dp.py`` (class ``NumpyDPBackend``) and the
dense-field query semantics of ``src/coldcore/protocol.py:143-219``.  Two
deliberate differences, both for the checker's sake:

* digits are int64 (the reference's ``ProductSpace.index_word`` returns
  uint8, ``src/coldcore/space.py:34-36``, which breaks its ball walks on axes
  wider than 255 — the king 2048x2048 torus needs them);
* the ball is enumerated straight from the metric's per-axis admissible
  shifts (``src/coldcore/patterns.py:34-68``) as (position, delta) columns,
  with no nibble packing, so axes of any width work.

Everything else — the per-axis recurrences, the predicates, the map queries
and ``map_extract``'s ascending order — is the reference's CPU semantics.
"""
from itertools import combinations

import numpy as np

PROBLEMS = ("hamming", "torus_linf", "lee", "grid_linf")


# ------------------------------------------------------------------ space
class Space:
    """Little-endian mixed radix: x = sum_j d_j * prod_{i<j} a_i
    (``src/coldcore/space.py:10-45``), with int64 digits."""

    def __init__(self, axes):
        self.axes = [int(a) for a in axes]
        self.n = len(self.axes)
        self.pow = np.ones(self.n, dtype=np.int64)
        for j in range(1, self.n):
            self.pow[j] = self.pow[j - 1] * self.axes[j - 1]
        self.size = int(self.pow[-1] * self.axes[-1])
        self.pow_q = self.pow                # the reference's name

    def digits(self, idx):
        idx = np.asarray(idx, dtype=np.int64).ravel()
        out = np.empty((len(idx), self.n), dtype=np.int64)
        x = idx.copy()
        for j, a in enumerate(self.axes):
            out[:, j] = x % a
            x //= a
        return out

    def index(self, digs):
        return np.asarray(digs, dtype=np.int64) @ self.pow


# ------------------------------------------------------------------ ball
def delta_sets(axes, R, problem):
    """Admissible circular shifts per axis (``patterns.py:34-50``)."""
    if problem == "hamming":
        return [list(range(1, a)) for a in axes]
    if problem == "torus_linf":
        return [list(range(1, R + 1)) + list(range(a - R, a)) for a in axes]
    if problem == "grid_linf":
        return [sorted({d for d in range(1, a) if d <= R or a - d <= R})
                for a in axes]
    if problem == "lee":
        return [[d for d in range(1, a) if min(d, a - d) <= R] for a in axes]
    raise ValueError(problem)


def max_weight(n, R, problem):
    """Most positions one support pattern changes (``patterns.py:53-59``)."""
    if problem == "hamming":
        return min(R, n)
    if problem == "lee":
        return min(n, R)
    return n


def ball_columns(axes, R, problem):
    """The support table as (L, w) position and delta columns; unused slots
    have delta 0.  Row 0 is the centre.  Same enumeration as the reference
    (subsets of positions in lexicographic order, Cartesian product of the
    per-position shift sets, Lee's total-weight coupling)."""
    n = len(axes)
    ds = delta_sets(axes, R, problem)
    w = max_weight(n, R, problem)
    pos_rows = [np.zeros((1, max(w, 1)), dtype=np.int64)]
    del_rows = [np.zeros((1, max(w, 1)), dtype=np.int64)]
    for k in range(1, w + 1):
        for subs in combinations(range(n), k):
            sets = [np.asarray(ds[p], dtype=np.int64) for p in subs]
            if any(len(s) == 0 for s in sets):
                continue
            grid = np.meshgrid(*sets, indexing="ij")
            d = np.stack([g.ravel() for g in grid], axis=1)
            if problem == "lee":
                wt = sum(np.minimum(d[:, i], axes[p] - d[:, i])
                         for i, p in enumerate(subs))
                d = d[wt <= R]
            if not len(d):
                continue
            P = np.zeros((len(d), max(w, 1)), dtype=np.int64)
            D = np.zeros((len(d), max(w, 1)), dtype=np.int64)
            P[:, :k] = np.asarray(subs, dtype=np.int64)[None, :]
            D[:, :k] = d
            pos_rows.append(P)
            del_rows.append(D)
    return np.concatenate(pos_rows), np.concatenate(del_rows)


# ------------------------------------------------------------------ backend
class OracleBackend:
    """One cell on the CPU: the reference's ``NumpyDPBackend`` semantics."""

    def __init__(self, axes, R, problem="hamming", mu=1, extract_cap=1 << 22,
                 dtype=np.int64):
        if problem not in PROBLEMS:
            raise ValueError(problem)
        self.problem, self.R, self.mu = problem, int(R), int(mu)
        self.space = Space(axes)
        self.axes, self.n = self.space.axes, self.space.n
        if problem == "torus_linf" and any(2 * R + 1 > a for a in self.axes):
            raise ValueError("need 2R+1 <= ax_j on every axis")
        self.extract_cap = extract_cap
        self.dtype = np.dtype(dtype)
        self.nlayers = 1 if problem in ("torus_linf", "grid_linf") else R + 1
        size = self.space.size
        self.cnt = np.zeros(size, dtype=self.dtype)
        self.map = np.zeros(size, dtype=self.dtype)
        self._A = np.zeros((self.nlayers, size), dtype=self.dtype)
        self.bpos, self.bdel = ball_columns(self.axes, self.R, problem)
        self.ball_len = len(self.bpos)
        # search-protocol attributes (dp.py:97-98)
        self.indep_dist = 2 * R if problem in ("hamming", "lee") else None
        self.supports_hist = True

    def index_word(self, idx):
        return self.space.digits(np.atleast_1d(np.asarray(idx, np.int64)))

    def word_index(self, digs):
        return self.space.index(np.asarray(digs, dtype=np.int64))

    # ------------------------------------------------ axis passes
    def _fibres(self, j):
        s = int(self.space.pow[j])
        q = self.axes[j]
        return self._A.reshape(self.nlayers, self.space.size // (q * s), q, s)

    def _axis_hamming(self, j):
        # dp.py:239-243: newA_d[a] = A_d[a] + T_{d-1} - A_{d-1}[a]
        v = self._fibres(j)
        tot = v.sum(axis=2)
        for d in range(self.nlayers - 1, 0, -1):
            v[d] += tot[d - 1][:, None, :] - v[d - 1]

    def _axis_lee(self, j):
        # dp.py:245-254: circulant grades, antipode once on even axes
        v = self._fibres(j)
        q = self.axes[j]
        half = q // 2
        for d in range(self.nlayers - 1, 0, -1):
            for w in range(1, min(d, half) + 1):
                v[d] += np.roll(v[d - w], w, axis=1)
                if not (q % 2 == 0 and w == half):
                    v[d] += np.roll(v[d - w], -w, axis=1)

    def _axis_torus(self, j):
        # dp.py:256-262: circular window of radius R
        v = self._fibres(j)
        acc = np.zeros_like(v[0])
        for e in range(-self.R, self.R + 1):
            acc += np.roll(v[0], -e, axis=1)
        v[0] = acc

    def _axis_grid(self, j):
        # dp.py:264-273: window clamped to [0, Q)
        v = self._fibres(j)
        h, q, s = v.shape[1:]
        cs = np.zeros((h, q + 1, s), dtype=self.dtype)
        np.cumsum(v[0], axis=1, out=cs[:, 1:, :])
        a = np.arange(q)
        lo = np.maximum(a - self.R, 0)
        hi = np.minimum(a + self.R, q - 1) + 1
        v[0] = cs[:, hi, :] - cs[:, lo, :]

    def _transform(self, out):
        step = {"hamming": self._axis_hamming, "lee": self._axis_lee,
                "torus_linf": self._axis_torus,
                "grid_linf": self._axis_grid}[self.problem]
        for j in range(self.n):
            step(j)
        if self.nlayers == 1:
            out[:] = self._A[0]
        else:
            np.sum(self._A, axis=0, out=out)

    def layers(self):
        """The (nlayers, |X|) stack left by the last transform."""
        return self._A

    # ------------------------------------------------ fields
    def recount(self, idx):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        self._A[:] = 0
        if idx.size:
            np.add.at(self._A[0], idx, 1)
        self._transform(self.cnt)

    def _deficient(self):
        return self.cnt < self.mu

    def _critical(self):
        return (self.cnt >= 1) & (self.cnt <= self.mu)

    def _role(self, values, target):
        if target == 0:
            return values < self.mu
        if target == 1:
            return (values >= 1) & (values <= self.mu)
        return values == target

    def gain_map(self):
        self._A[:] = 0
        self._A[0] = self._deficient()
        self._transform(self.map)

    def loss_map(self):
        self._A[:] = 0
        self._A[0] = self._critical()
        self._transform(self.map)

    # ------------------------------------------------ balls
    def balls(self, idx):
        """(m, L) ball word indices per centre and an in-board mask
        (None unless the open grid rejects some patterns)."""
        idx = np.asarray(idx, dtype=np.int64).ravel()
        digs = self.space.digits(idx)
        off = np.zeros((len(idx), self.ball_len), dtype=np.int64)
        good = None
        if self.problem == "grid_linf":
            good = np.ones((len(idx), self.ball_len), dtype=bool)
        for k in range(self.bpos.shape[1]):
            p = self.bpos[:, k]
            dl = self.bdel[:, k]
            used = dl > 0
            a = np.asarray(self.axes, dtype=np.int64)[p]
            base = digs[:, p]                               # (m, L)
            sh = (base + dl[None, :]) % a[None, :] - base
            sh = np.where(used[None, :], sh, 0)
            off += sh * self.space.pow[p][None, :]
            if good is not None:
                good &= np.abs(sh) <= self.R
        off += idx[:, None]
        return off, good

    def ball_indices(self, w):
        off, good = self.balls([int(w)])
        out = off[0] if good is None else off[0][good[0]]
        return np.sort(out)

    def _chunk(self):
        return max(1, (1 << 22) // max(1, self.ball_len))

    def ball_update(self, idx, delta):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        step = self._chunk()
        for lo in range(0, len(idx), step):
            off, good = self.balls(idx[lo:lo + step])
            for k in range(len(off)):
                row = off[k] if good is None else off[k][good[k]]
                self.cnt[row] += delta

    def ball_gather(self, idx, target):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        out = np.empty(len(idx), dtype=np.int32)
        step = self._chunk()
        for lo in range(0, len(idx), step):
            off, good = self.balls(idx[lo:lo + step])
            hit = self._role(self.cnt[off], target)
            if good is not None:
                hit &= good
            out[lo:lo + step] = hit.sum(axis=1)
        return out

    # ------------------------------------------------ queries
    def count_eq(self, target):
        return int((self.cnt == target).sum())

    def uncovered(self):
        return int(np.maximum(self.mu - self.cnt, 0).sum(dtype=np.int64))

    def map_max(self):
        return int(self.map.max(initial=0))

    def map_hist(self, nbins, vmax):
        out = np.zeros(nbins, dtype=np.int32)
        v = np.asarray(self.map[self.map > 0], dtype=np.int64)
        if len(v) and vmax > 0:
            b = np.minimum((v - 1) * nbins // vmax, nbins - 1)
            np.add.at(out, b, 1)
        return out

    def map_extract(self, thr, cap=None):
        cap = min(cap or self.extract_cap, self.extract_cap)
        idx = np.flatnonzero(self.map >= thr).astype(np.int64)
        found = len(idx)
        idx = idx[:cap]
        return idx, self.map[idx].astype(np.int32), found

    def map_read_at(self, idx):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        return self.map[idx].astype(np.int32)

    def read_cnt(self, off=0, length=None):
        length = self.space.size - off if length is None else length
        return self.cnt[off:off + length].astype(np.uint16)

    # ------------------------------------------------ composed forms
    def ball_update_delta(self, idx, delta):
        """Update plus the change of the total deficit it caused
        (``src/coldcore/gpu.py:167-173``)."""
        u0 = self.uncovered()
        self.ball_update(idx, delta)
        return self.uncovered() - u0

    def swap_eval(self, drops, cands):
        """Per drop: loss = gather role 1; gains = role-0 gathers with that
        drop removed (``src/coldcore/gpu.py:132-164``); cnt is restored."""
        drops = np.atleast_1d(np.asarray(drops, dtype=np.int64))
        shared = not isinstance(cands, (list, tuple))
        parts = ([np.atleast_1d(np.asarray(cands, dtype=np.int64))]
                 * len(drops) if shared else
                 [np.atleast_1d(np.asarray(c, dtype=np.int64)) for c in cands])
        loss = np.empty(len(drops), dtype=np.int32)
        gains = []
        for i, w in enumerate(drops.tolist()):
            wa = np.array([w], dtype=np.int64)
            loss[i] = int(self.ball_gather(wa, 1)[0])
            if len(parts[i]):
                self.ball_update(wa, -1)
                gains.append(self.ball_gather(parts[i], 0))
                self.ball_update(wa, +1)
            else:
                gains.append(np.zeros(0, dtype=np.int32))
        if shared:
            return loss, (np.stack(gains) if gains else
                          np.zeros((0, len(parts[0]) if parts else 0),
                                   dtype=np.int32))
        return loss, gains


def exact_greedy(oracle, code, max_add):
    """The exact greedy the device repair runs, by brute force: from the
    counts of ``code`` (already loaded into ``oracle``), repeatedly place
    the word outside ``code`` and outside the words placed so far with the
    largest gain (deficient words in its ball), ties to the smallest index;
    stop at zero deficit, no positive gain, or ``max_add`` words.  Returns
    (placed words in order, deficit left)."""
    taken = set(np.asarray(code, dtype=np.int64).tolist())
    placed = []
    while len(placed) < max_add and oracle.uncovered() > 0:
        oracle.gain_map()
        g = oracle.map.astype(np.int64).copy()
        if taken:
            g[np.fromiter(taken, dtype=np.int64)] = np.iinfo(np.int64).min
        w = int(np.argmax(g))
        if g[w] <= 0:
            break
        oracle.ball_update(np.array([w]), +1)
        placed.append(w)
        taken.add(w)
    return np.array(placed, dtype=np.int64), oracle.uncovered()


def owner_losses(oracle, code):
    """Exact per-codeword deficit increase of removing that one copy — what
    the reference's owner-trick loss pass returns
    (``src/plugins/covering/dct_hc.cu:997-1022``)."""
    return oracle.ball_gather(np.asarray(code, dtype=np.int64), 1)
