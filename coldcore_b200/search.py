"""Ruin-and-recreate search over a covering backend.

This module restates the part of coldcore's search core
(src/coldcore/search.py) that the learned ruin proposal plugs into:

* ``greedy_fill``: the exact lazy greedy repair (search.py:260-360);
* ``ruin``: the four proven ruin operators low / hole / cluster / random
  (search.py:536-618);
* ``peel``: zero-loss removal in independent batches (search.py:621-670);
* ``lns``: fixed-M LNS with ``select="fixed"`` (the record mix) or
  ``"adaptive"`` (:class:`OperatorBandit`), search.py:672-784;
* ``descend``: the notch ladder, v0.2 schedule (search.py:1757-1918).

The swap polish (``anneal``, ``two_swap``) is not restated: it is a caller
of the engine's ``swap_eval`` / ``ball_update_delta`` fast paths, and
coldcore's own ``Searcher`` drives those unchanged.

The random draws happen in the reference's order, so with a backend whose
``map_extract`` returns ascending indices (the CPU backends) a seeded run
makes the same moves as the reference's.

One repair rule is added: ``repair="device"`` runs the exact greedy on
the GPU (``GpuBackend.greedy_fill_device``): the word of largest exact
gain, ties to the smallest index, placed one after another without a host
round trip.  The default stays the Python lazy greedy.

One selection rule is added: ``select="learned"`` asks a *proposer* (see
:mod:`coldcore_b200.learned`) for the k incumbents to remove.  When its
confidence gate is closed the round falls back to the bandit.  Every round
is still scored by the exact repair and the exact counters, whichever rule
picked the ruin.

The searcher is backend-blind.  It calls only the protocol methods
(``recount``, ``gain_map``, ``loss_map``, ``uncovered``, ``map_max``,
``map_hist``, ``map_extract``, ``map_read_at``, ``ball_gather``,
``ball_update``, ``index_word``) and the attributes ``extract_cap`` and
``indep_dist``.
"""
import heapq
import time

import numpy as np

#: the proven ruin operators and their prior weights (search.py:54-55)
RUIN_OPS = ("low", "hole", "cluster", "random")
RUIN_PRIOR = {"low": 1.0, "hole": 2.0, "cluster": 1.0, "random": 1.0}
#: fixed selection: a uniform draw from this list (search.py:65)
FIXED_DRAW = ("low", "hole", "hole", "cluster", "random")
SELECTIONS = ("fixed", "adaptive", "learned")
#: the opt-in deficit-targeted operator (``lns(..., deficit=True)``):
#: weighted like ``hole`` in both the prior and the fixed list
#: (search.py:57-66)
RUIN_OPS_EXT = RUIN_OPS + ("deficit",)
RUIN_PRIOR_EXT = dict(RUIN_PRIOR, deficit=2.0)
FIXED_DRAW_DEFICIT = FIXED_DRAW + ("deficit", "deficit")
#: uncovered words the deficit operator aims at, and counters read per
#: scan of cnt (search.py:80-81)
DEFICIT_WORDS = 4
SCAN_CHUNK = 1 << 24
def _rng_for(seed):
    return np.random.default_rng(seed * 1000003 + 12345)


class OperatorBandit:
    """Adaptive ruin-operator choice (coldcore ``search.py:96-167``).

    State per operator: ``score``, an exponential moving average of the
    rewards its rounds earned (weight ``1 - decay`` on the newest), which
    starts at the prior mix rescaled to mean 1.  A draw mixes the score
    shares with a uniform ``floor``: P(op) = floor / n + (1 - floor) *
    score / total.  A hint ``{op: factor}`` multiplies one operator's score,
    first raised to at least the floor, for that draw only.  Rewards are
    tiered: a new global best 3, better than the round's start 1, equal
    0.3, worse 0."""

    REWARD_BEST, REWARD_BETTER, REWARD_EQUAL, REWARD_WORSE = 3.0, 1.0, 0.3, 0.0

    def __init__(self, rng, ops=RUIN_OPS, floor=0.15, decay=0.9,
                 prior=RUIN_PRIOR):
        self.rng = rng
        self.ops = list(ops)
        self._slot = {op: i for i, op in enumerate(self.ops)}
        self.floor = float(floor)
        self.decay = float(decay)
        n = len(self.ops)
        start = np.fromiter((float(prior.get(op, 1.0)) for op in self.ops),
                            dtype=np.float64, count=n)
        self.score = start * (n / start.sum())
        self.uses = np.zeros(n, dtype=np.int64)
        self.reward = np.zeros(n, dtype=np.float64)

    def probabilities(self, boost=None):
        n = len(self.ops)
        w = np.clip(self.score, 0.0, None)
        for op, factor in (boost or {}).items():
            i = self._slot.get(op)
            if i is not None:
                w[i] = max(w[i], self.floor) * float(factor)
        total = w.sum()
        if not total > 0:
            return np.full(n, 1.0 / n)
        return self.floor / n + (1.0 - self.floor) * w / total

    def select(self, boost=None):
        i = int(self.rng.choice(len(self.ops), p=self.probabilities(boost)))
        self.uses[i] += 1
        return self.ops[i]

    def update(self, op, reward):
        i = self._slot[op]
        self.reward[i] += reward
        keep = self.decay
        self.score[i] = keep * self.score[i] + (1.0 - keep) * reward

    @classmethod
    def tier(cls, new_best, pre, post):
        """Reward of one round from its outcome."""
        if new_best:
            return cls.REWARD_BEST
        if post != pre:
            return cls.REWARD_BETTER if post < pre else cls.REWARD_WORSE
        return cls.REWARD_EQUAL

    def summary(self):
        p = self.probabilities()
        mean = self.reward / np.maximum(self.uses, 1)
        return {op: {"uses": int(self.uses[i]), "reward": float(mean[i]),
                     "p": float(p[i])} for op, i in self._slot.items()}


class Searcher:
    """LNS driver for one cell on one backend.

    ``proposer``: an object with ``propose(searcher, k) -> positions or
    None`` and ``observe(searcher, mode, pre, post, new_best)``; used by
    ``select="learned"``.  ``move_log``: called once per LNS round as
    ``move_log(searcher, event, **info)`` with event ``"pre"`` (before the
    ruin, with ``k`` and ``mode``), ``"ruin"`` (with the removed positions),
    ``"repair"`` (after the greedy repair, with the repaired ``code``) and
    ``"post"`` (after the accept/reject rule, with ``pre``, ``post`` (the
    repaired count), ``after`` and ``new_best``)."""

    def __init__(self, backend, seed=1, deadline=None, on_log=None,
                 on_solved=None, proposer=None, move_log=None,
                 repair="exact"):
        if repair not in ("exact", "device"):
            raise ValueError(f"unknown repair mode: {repair!r}")
        if repair == "device" and not hasattr(backend, "greedy_fill_device"):
            raise ValueError("repair='device' needs a GPU backend")
        self.repair = repair
        self.b = backend
        self.rng = _rng_for(seed)
        self.deadline = deadline
        self.on_log = on_log or (lambda s: None)
        self.on_solved = on_solved or (lambda m, idx: None)
        self.proposer = proposer
        self.move_log = move_log
        self.code = np.zeros(0, dtype=np.int64)
        self.uncov = None
        self.best_code = None
        self.best_uncov = None
        self.loop_reserve_s = 10.0
        self.build_reserve_s = 5.0
        self.stats = {"transforms": 0, "placements": 0, "removals": 0,
                      "rounds": 0, "recounts": 0, "accepts": 0,
                      "learned_rounds": 0, "fallback_rounds": 0}
        self._scan_off = 0                 # rotating start of the cnt scan
        self._deficit_cache = (None, None)

    # ------------------------------------------------ state
    def time_left(self):
        return np.inf if self.deadline is None else self.deadline - time.time()

    def load(self, code):
        code = np.asarray(code)
        if code.ndim == 2:
            code = self.b.word_index(code.astype(np.int64))
        self.code = (np.unique(code.astype(np.int64)) if code.size
                     else np.zeros(0, dtype=np.int64))
        self.b.recount(self.code)
        self.stats["transforms"] += 1
        self.uncov = self.b.uncovered()
        self._snapshot()

    def _snapshot(self):
        better = self.best_uncov is None or self.uncov < self.best_uncov
        tie_smaller = (self.uncov == self.best_uncov and (
            self.best_code is None or len(self.code) < len(self.best_code)))
        if better or tie_smaller:
            self.best_uncov = self.uncov
            self.best_code = self.code.copy()

    def verify_full(self):
        """Recount from scratch; returns the exact uncovered count."""
        self.b.recount(self.code)
        self.stats["transforms"] += 1
        self.stats["recounts"] += 1
        self.uncov = self.b.uncovered()
        return self.uncov

    def _digits(self, idx):
        return self.b.index_word(np.asarray(idx, dtype=np.int64)).astype(
            np.int16)

    # ------------------------------------------------ repair
    def _threshold(self, cap):
        """Smallest gain threshold whose extraction fits ~90% of ``cap``,
        read off a 1024-bin histogram of the gain map (search.py:294-304)."""
        b = self.b
        mx = b.map_max()
        thr = 1
        if mx > 1 and getattr(b, "supports_hist", True):
            hist = np.asarray(b.map_hist(1024, mx), dtype=np.int64)
            tail = np.cumsum(hist[::-1])[::-1]        # entries at bin >= i
            fits = np.flatnonzero(tail <= cap * 0.9)
            first = int(fits[0]) if len(fits) else 1023
            thr = max(1, first * mx // 1024 + 1)
        return mx, thr

    def _candidate_heap(self, cap, codeset):
        """(mx, thr, heap) from a fresh gain map: the extracted candidates
        as (-gain, index) in stable descending-gain order, incumbents
        dropped."""
        b = self.b
        b.gain_map()
        self.stats["transforms"] += 1
        mx, thr = self._threshold(cap)
        if mx <= 0:
            return mx, thr, None
        idx, val, found = b.map_extract(thr, cap=cap)
        while found > cap and thr < mx:
            thr = min(mx, thr + max(1, (mx - thr) // 2))
            idx, val, found = b.map_extract(thr, cap=cap)
        val = np.asarray(val, dtype=np.int64)
        order = np.argsort(-val, kind="stable")
        keys = (-val[order]).tolist()
        words = np.asarray(idx, dtype=np.int64)[order].tolist()
        heap = [e for e in zip(keys, words) if e[1] not in codeset]
        heapq.heapify(heap)
        return mx, thr, heap

    def greedy_fill(self, target_m, batch=64, refresh_every=512):
        """Exact lazy greedy until covered, ``target_m`` points, or the
        deadline.  Stale gains from the last gain map bound a max-heap; a
        batch of the best bounds is re-scored exactly with ``ball_gather``
        and the best is placed when it is at least the next stale bound and
        the extraction threshold (search.py:260-360)."""
        b = self.b
        if self.repair == "device":
            return self._device_fill(target_m)
        cap = min(b.extract_cap, 1 << 18)
        codeset = set(self.code.tolist())
        heap, thr, since = [], 1, refresh_every
        while self.uncov > 0 and len(codeset) < target_m:
            if self.time_left() < self.build_reserve_s:
                break
            if since >= refresh_every or not heap:
                mx, thr, heap = self._candidate_heap(cap, codeset)
                if mx <= 0:
                    break
                since = 0
                if not heap:
                    if thr > 1:              # nothing new above thr: retry at 1
                        since, thr = refresh_every, 1
                        continue
                    break
            cand = []
            while heap and len(cand) < batch:
                key, w = heapq.heappop(heap)
                if w not in codeset:
                    cand.append(w)
            if not cand:
                since = refresh_every
                continue
            widx = np.array(cand, dtype=np.int64)
            exact = np.asarray(b.ball_gather(widx, 0))
            bi = int(np.argmax(exact))
            bg = int(exact[bi])
            gains = exact.tolist()
            bound = -heap[0][0] if heap else 0
            if bg < 1:
                since = refresh_every
                continue
            placed = bg >= bound and bg >= thr
            if placed:
                w = cand[bi]
                b.ball_update(np.array([w], dtype=np.int64), +1)
                codeset.add(w)
                self.uncov -= bg
                self.stats["placements"] += 1
                since += 1
            for g, w in zip(gains, cand):
                if g > 0 and not (placed and w == cand[bi]):
                    heapq.heappush(heap, (-g, w))
            if not placed and bg < thr:
                since = refresh_every
        self.code = np.array(sorted(codeset), dtype=np.int64)
        return self.uncov

    def _device_fill(self, target_m):
        """The exact greedy on the GPU, up to ``target_m`` points."""
        need = int(target_m) - len(self.code)
        if need > 0 and self.uncov > 0:
            placed, deficit = self.b.greedy_fill_device(need)
            if len(placed):
                self.code = np.sort(np.concatenate([self.code, placed]))
                self.stats["placements"] += len(placed)
            self.stats["transforms"] += 1
            self.uncov = deficit
        return self.uncov

    # ------------------------------------------------ ruin
    def losses(self):
        """Exact loss of every incumbent (words only it covers)."""
        self.b.loss_map()
        self.stats["transforms"] += 1
        return self.b.map_read_at(self.code)

    def _near(self, centre):
        """Jittered distance of every incumbent to the word ``centre``: the
        backend's own metric when it has one (the locality hook of
        coldcore's protocol, e.g. the block metric of a covering design,
        search.py:581-583), else the digit-Hamming distance."""
        dist = getattr(self.b, "distance", None)
        if dist is not None:
            d = np.asarray(dist(self.code, int(centre)), dtype=np.int64)
        else:
            c = self._digits(np.array([centre]))[0]
            d = (self._digits(self.code) != c[None, :]).sum(axis=1)
        return d + self.rng.random(len(self.code))

    # ------------------------------------------------ the deficit itself
    def supports_deficit(self):
        """The backend can hand back cnt (search.py:471-478)."""
        return hasattr(self.b, "read_cnt")

    def uncovered_words(self, limit=DEFICIT_WORDS, chunk=SCAN_CHUNK,
                        scan_cap=None):
        """Up to ``limit`` currently deficient words (coldcore
        ``search.py:480-528``), ascending.  A backend with its own
        ``deficient_universe`` answers directly; otherwise cnt is read in
        chunks from a rotating cursor (so repeated calls at one state see
        different deficient words), the cursor moving past the last hit and
        back to 0 after a scan that came up short.  A non-empty answer is
        memoised for the solution that produced it.  Empty means none was
        found within ``scan_cap`` words, not that nothing is uncovered."""
        if self.uncov == 0 or not self.supports_deficit():
            return np.zeros(0, dtype=np.int64)
        direct = getattr(self.b, "deficient_universe", None)
        if direct is not None:
            return np.asarray(direct(limit, self.rng), dtype=np.int64)
        state = (len(self.code), self.uncov,
                 hash(np.ascontiguousarray(self.code).tobytes()))
        memo_state, memo = self._deficit_cache
        if (memo_state == state and memo is not None
                and len(memo) >= min(limit, self.uncov)):
            return memo[:limit]
        n = self.b.space.size
        mu = getattr(self.b, "mu", 1)
        step = max(1, int(chunk))
        left = n if scan_cap is None else min(n, int(scan_cap))
        cursor = int(self._scan_off) % n
        hits = np.zeros(0, dtype=np.int64)
        while left > 0 and len(hits) < limit:
            span = min(step, n - cursor, left)
            low = np.flatnonzero(np.asarray(self.b.read_cnt(cursor, span))
                                 < mu)[:limit - len(hits)]
            if len(low):
                hits = np.concatenate([hits, low.astype(np.int64) + cursor])
                self._scan_off = (int(hits[-1]) + 1) % n
            left -= span
            cursor = (cursor + span) % n
        if len(hits) < limit:
            self._scan_off = 0
        hits = np.sort(hits)
        if len(hits):
            self._deficit_cache = (state, hits)
        return hits

    def _pick(self, k, mode, deficit_pool=3):
        """Positions (into ``self.code``) that ``mode`` removes."""
        m = len(self.code)
        if mode == "deficit":
            # k incumbents drawn from the ~3k nearest to the words that are
            # actually uncovered (search.py:552-576); none found: ``hole``
            tgt = self.uncovered_words()
            if not len(tgt):
                return self._pick(k, "hole")
            self.stats["deficit_ruins"] = self.stats.get("deficit_ruins",
                                                         0) + 1
            udist = getattr(self.b, "universe_distance", None)
            if udist is not None:
                d = np.asarray(udist(self.code, tgt), dtype=np.int64).min(
                    axis=1)
            else:
                digs, tw = self._digits(self.code), self._digits(tgt)
                d = np.full(m, np.iinfo(np.int32).max, dtype=np.int64)
                for t in tw:
                    np.minimum(d, (digs != t[None, :]).sum(axis=1), out=d)
            order = np.argsort(d + self.rng.random(m))
            near = order[:min(m, max(deficit_pool * k, k + 8))]
            return self.rng.choice(near, size=k, replace=False)
        if mode == "random":
            return self.rng.choice(m, size=k, replace=False)
        if mode == "cluster":
            centre = int(self.code[self.rng.integers(m)])
            return np.argsort(self._near(centre))[:k]
        if mode == "hole":
            self.b.gain_map()
            self.stats["transforms"] += 1
            mx = self.b.map_max()
            if mx > 0:
                oi, _ov, _found = self.b.map_extract(max(1, mx // 2), cap=4096)
                if len(oi):
                    anchor = int(oi[self.rng.integers(len(oi))])
                    return np.argsort(self._near(anchor))[:k]
            mode = "low"                         # no hole: fall back
        lo = np.asarray(self.losses(), dtype=np.float64)
        jit = self.rng.exponential(scale=max(1.0, lo.mean() * 0.15), size=m)
        return np.argsort(lo + jit)[:k]

    def ruin(self, k, mode="low", pick=None):
        """Remove k incumbents chosen by ``mode`` (or at the given
        positions); returns the removed words (search.py:536-618)."""
        m = len(self.code)
        k = min(k, m - 1)
        if k <= 0:
            return np.zeros(0, dtype=np.int64)
        if pick is None:
            pick = self._pick(k, mode)
        pick = np.asarray(pick, dtype=np.int64)[:k]
        removed = self.code[pick]
        self.b.ball_update(removed, -1)
        self.code = np.delete(self.code, pick)
        self.uncov = self.b.uncovered()
        self.stats["removals"] += len(pick)
        return removed

    # ------------------------------------------------ peel
    def peel(self):
        """Remove zero-loss incumbents to a fixpoint, in batches whose
        members are pairwise more than ``indep_dist`` apart, so removing
        all of them together keeps every word covered (search.py:621-670)."""
        b = self.b
        total = 0
        while self.time_left() >= self.build_reserve_s:
            lo = np.asarray(self.losses())
            zeros = np.flatnonzero(lo == 0)
            if not len(zeros):
                break
            zeros = zeros[np.asarray(b.ball_gather(self.code[zeros], 1)) == 0]
            if not len(zeros):
                break
            self.rng.shuffle(zeros)
            sep = b.indep_dist
            dist = getattr(b, "distance", None)
            if sep is not None and (dist is not None or sep < self.b.space.n):
                cand = self.code[zeros]
                digs = None if dist is not None else self._digits(cand)
                keep = [0]
                for i in range(1, len(zeros)):
                    if dist is not None:        # the backend's own metric
                        d = np.asarray(dist(cand[np.array(keep)], cand[i]))
                    else:
                        d = (digs[keep] != digs[i][None, :]).sum(axis=1)
                    if (d > sep).all():
                        keep.append(i)
                pick = zeros[np.array(keep)]
            else:
                pick = zeros[:1]
            b.ball_update(self.code[pick], -1)
            self.code = np.delete(self.code, pick)
            total += len(pick)
            self.stats["removals"] += len(pick)
        if total:
            self.uncov = self.b.uncovered()
        return total

    # ------------------------------------------------ LNS at fixed M
    def lns(self, M, round_budget_s, kmin=8, kmax=None, select="fixed",
            log_every=20, stall_s=None, deficit=False, deficit_hint=3,
            deficit_boost=4.0):
        """Ruin/recreate rounds at fixed M until feasible or out of budget
        (search.py:672-784).  A round that ends worse than it started is
        rejected (the best snapshot is restored) except with probability
        0.1.  ``deficit=True`` adds the deficit-targeted ruin to the
        selection and, within ``deficit_hint`` of feasible, favours it
        (half the fixed draws; a ``deficit_boost`` hint to the bandit).
        Returns the final uncovered count (0 = solved)."""
        if select not in SELECTIONS:
            raise ValueError(f"unknown ruin selection: {select!r}")
        if select == "learned" and self.proposer is None:
            raise ValueError("select='learned' needs a proposer")
        t0 = time.time()
        t_best = t0
        kmax = kmax or max(kmin + 1, M // 20)
        self.best_uncov = self.best_code = None
        if len(self.code) < M:
            self.greedy_fill(M)
        self._snapshot()
        modes = FIXED_DRAW_DEFICIT if deficit else FIXED_DRAW
        if select == "fixed":
            bandit = None
        elif deficit:
            bandit = OperatorBandit(self.rng, ops=RUIN_OPS_EXT,
                                    prior=RUIN_PRIOR_EXT)
        else:
            bandit = OperatorBandit(self.rng)
        hint = {"deficit": deficit_boost} if deficit else None
        r = 0
        while self.uncov > 0:
            now = time.time()
            if (now - t0 > round_budget_s
                    or self.time_left() < self.loop_reserve_s):
                break
            if stall_s is not None and now - t_best > stall_s:
                break
            pre, pre_best = self.uncov, self.best_uncov
            k = int(self.rng.integers(kmin, kmax + 1))
            near = deficit and self.uncov <= deficit_hint
            pick = None
            if select == "fixed":
                if near and self.rng.random() < 0.5:
                    mode = "deficit"
                else:
                    mode = modes[int(self.rng.integers(len(modes)))]
            else:
                mode = None
                if select == "learned":
                    pick = self.proposer.propose(self, min(k, len(self.code) - 1))
                    if pick is not None:
                        mode = "learned"
                        self.stats["learned_rounds"] += 1
                    else:
                        self.stats["fallback_rounds"] += 1
                if mode is None:
                    mode = bandit.select(hint if near else None)
            if self.move_log is not None:
                self.move_log(self, "pre", k=k, mode=mode)
            if mode == "learned" or self.move_log is not None:
                # resolve the positions first, so the log sees them
                if pick is None:
                    kk = min(k, len(self.code) - 1)
                    pick = self._pick(kk, mode) if kk > 0 else np.zeros(
                        0, dtype=np.int64)
                if self.move_log is not None:
                    self.move_log(self, "ruin", pick=np.asarray(pick))
            self.ruin(k, mode, pick=pick)
            self.greedy_fill(M)
            if self.move_log is not None:
                self.move_log(self, "repair", code=self.code)
            self.stats["rounds"] += 1
            r += 1
            post = self.uncov
            if self.uncov > pre and self.rng.random() > 0.10:
                self.code = self.best_code.copy()
                self.b.recount(self.code)
                self.stats["transforms"] += 1
                self.uncov = self.b.uncovered()
            else:
                self.stats["accepts"] += 1
                self._snapshot()
            new_best = self.best_uncov < pre_best
            if new_best:
                t_best = time.time()
            # rewards read the state after the accept/reject rule
            after = self.uncov
            if self.move_log is not None:
                self.move_log(self, "post", pre=pre, post=post, after=after,
                              new_best=new_best)
            if select == "learned":
                self.proposer.observe(self, mode, pre, after, new_best)
            if bandit is not None and mode != "learned":
                bandit.update(mode, bandit.tier(new_best, pre, after))
            if bandit is not None:
                self.stats["ops"] = bandit.summary()
            if log_every and r % log_every == 0:
                self.on_log(f"lns M={M} round={r} uncov={self.uncov} "
                            f"best={self.best_uncov} k={k} "
                            f"({time.time() - t0:.1f}s)")
            if r % 50 == 0:
                inc = self.uncov
                if self.verify_full() != inc:
                    self.on_log(f"drift: incremental {inc} != recount "
                                f"{self.uncov}; adopting the recount")
        if self.uncov == 0:
            self._snapshot()
        elif self.best_code is not None and self.best_uncov < self.uncov:
            self.code = self.best_code.copy()
            self.b.recount(self.code)
            self.uncov = self.b.uncovered()
        return self.uncov

    # ------------------------------------------------ notch descent
    def descend(self, floor=1, notch_budget_s=300.0, step0=4, step_cap=1024,
                kmin=8, kmax=None, select="fixed", deficit=False,
                reserve_s=30.0,
                min_notch_s=20.0, fail_limit=3):
        """From a feasible solution, try M - step; halve the step on a
        failed notch, double it on a success in under a quarter of the
        notch budget.  Each verified solution fires ``on_solved(M, code)``
        (search.py:1757-1918, v0.2 schedule).  Returns the final M."""
        if self.uncov != 0:
            raise RuntimeError("descend requires a feasible starting solution")
        self.peel()
        if self.verify_full() != 0:
            raise RuntimeError("peel broke feasibility")
        solved = self.code.copy()
        M = len(solved)
        self.on_solved(M, solved)
        step, fails_at_1 = step0, 0
        while self.time_left() > 0 and M > floor and fails_at_1 < fail_limit:
            target = M - step
            t0 = time.time()
            nominal = notch_budget_s * (2 ** min(fails_at_1, 2))
            budget = min(nominal, max(0.0, self.time_left() - reserve_s))
            if budget < min(min_notch_s, notch_budget_s):
                break
            self.ruin(len(self.code) - target, "low")
            unc = self.lns(target, budget, kmin=kmin, kmax=kmax,
                           select=select, log_every=0, deficit=deficit)
            if unc == 0 and self.verify_full() == 0:
                self.peel()
                if self.verify_full() != 0:
                    self.load(solved)
                    break
                solved = self.code.copy()
                M = len(solved)
                dt = time.time() - t0
                self.on_log(f"solved M={M} in {dt:.1f}s (step={step})")
                self.on_solved(M, solved)
                fails_at_1 = 0
                if dt < budget * 0.25:
                    step = min(step * 2, step_cap)
            else:
                self.on_log(f"notch M={target} failed (best uncov="
                            f"{self.best_uncov}, step={step})")
                if step == 1:
                    fails_at_1 += 1
                step = max(1, step // 2)
                self.load(solved)
        return M
