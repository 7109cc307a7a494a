"""Ruin-and-recreate search over a covering backend.

This module restates the part of coldcore's search core
(src/coldcore/search.py) that the learned ruin proposal plugs into:

* ``greedy_fill``: the exact lazy greedy repair (search.py:260-360);
* ``ruin``: the four proven ruin operators low / hole / cluster / random
  (search.py:536-618);
* ``peel``: zero-loss removal in independent batches (search.py:621-670);
* ``lns``: fixed-M LNS with ``select="fixed"`` (the record mix) or
  ``"adaptive"`` (:class:`OperatorBandit`), search.py:672-784;
* ``descend``: the notch ladder, v0.2 schedule (search.py:1757-1918);
* ``anneal``: the swap-neighbourhood polish at fixed M (LAHC or
  Metropolis), over the "pool" or the local "shell" neighbourhood,
  costed exactly by the backend's ``swap_eval`` (search.py:787-1360).

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
#: shell-polish defaults (search.py:70-90): sampled distance-2 words,
#: top-of-gain draws and uniform draws per move, the cheapest incumbents
#: a move drops from, the top-gain pool cap and the pool-neighbourhood cap
SHELL2, SHELL_TOP, SHELL_RAND, SHELL_TOPK = 128, 48, 8, 24
SHELL_POOL_CAP = 4096
POOL_CAP = 1 << 14


def _rng_for(seed):
    return np.random.default_rng(seed * 1000003 + 12345)


class OperatorBandit:
    """Roulette-wheel ruin-operator choice with a uniform floor
    (search.py:96-167).

    Each operator's score is an exponential moving average of the reward
    of its rounds.  The draw is ``floor / k + (1 - floor) * score / sum``.
    Scores start at the prior mix, scaled to mean 1."""

    REWARD_BEST, REWARD_BETTER, REWARD_EQUAL, REWARD_WORSE = 3.0, 1.0, 0.3, 0.0

    def __init__(self, rng, ops=RUIN_OPS, floor=0.15, decay=0.9,
                 prior=RUIN_PRIOR):
        self.ops = list(ops)
        self.rng = rng
        self.floor, self.decay = float(floor), float(decay)
        w = np.array([float(prior.get(o, 1.0)) for o in self.ops])
        self.score = w * (len(w) / w.sum())
        self.uses = np.zeros(len(self.ops), dtype=np.int64)
        self.reward = np.zeros(len(self.ops))

    def probabilities(self, boost=None):
        """``boost``: optional {op: factor} hint applied to the scores
        (lifted to the floor first, so a crushed score can come back)
        before normalising (search.py:131-149)."""
        w = np.maximum(self.score, 0.0)
        k = len(self.ops)
        if boost:
            w = w.copy()
            for op, f in boost.items():
                if op in self.ops:
                    i = self.ops.index(op)
                    w[i] = max(w[i], self.floor) * float(f)
        if w.sum() <= 0:
            return np.full(k, 1.0 / k)
        return self.floor / k + (1.0 - self.floor) * w / w.sum()

    def select(self, boost=None):
        i = int(self.rng.choice(len(self.ops), p=self.probabilities(boost)))
        self.uses[i] += 1
        return self.ops[i]

    def update(self, op, reward):
        i = self.ops.index(op)
        self.reward[i] += reward
        self.score[i] = self.decay * self.score[i] + (1 - self.decay) * reward

    @classmethod
    def tier(cls, new_best, pre, post):
        """Reward of a round: new global best > better > sideways > worse."""
        if new_best:
            return cls.REWARD_BEST
        if post < pre:
            return cls.REWARD_BETTER
        return cls.REWARD_EQUAL if post == pre else cls.REWARD_WORSE

    def summary(self):
        p = self.probabilities()
        return {o: {"uses": int(self.uses[i]),
                    "reward": float(self.reward[i] / max(1, self.uses[i])),
                    "p": float(p[i])} for i, o in enumerate(self.ops)}


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
        self._sh1 = None                   # per-axis shell displacements
        self.stats.update({"moves": 0})

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
        """Up to ``limit`` currently deficient words (search.py:480-528):
        the backend's own ``deficient_universe`` when it has one, else a
        chunked scan of cnt from a rotating offset, cached against the
        solution that produced it.  Empty means none found within the cap,
        never that nothing is uncovered."""
        if not self.supports_deficit() or self.uncov == 0:
            return np.zeros(0, dtype=np.int64)
        exact = getattr(self.b, "deficient_universe", None)
        if exact is not None:
            return np.asarray(exact(limit, self.rng), dtype=np.int64)
        key = (len(self.code), self.uncov,
               hash(np.ascontiguousarray(self.code).tobytes()))
        ckey, cval = self._deficit_cache
        if ckey == key and cval is not None and len(cval) >= min(
                limit, self.uncov):
            return cval[:limit]
        size = self.b.space.size
        mu = getattr(self.b, "mu", 1)
        chunk = max(1, int(chunk))
        budget = size if scan_cap is None else min(size, int(scan_cap))
        found = []
        off = int(self._scan_off) % size
        read = 0
        while read < budget and len(found) < limit:
            take = min(chunk, size - off, budget - read)
            hit = np.flatnonzero(np.asarray(self.b.read_cnt(off, take)) < mu)
            if len(hit):
                got = hit[:limit - len(found)] + off
                found.extend(int(v) for v in got)
                self._scan_off = (int(got[-1]) + 1) % size
            read += take
            off = (off + take) % size
        if len(found) < limit:
            self._scan_off = 0                 # exhausted: restart the sweep
        out = np.array(sorted(found), dtype=np.int64)
        if len(out):
            self._deficit_cache = (key, out)
        return out

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

    # ------------------------------------------------ polish at fixed M
    def _rng_pass(self, seed):
        """The stream a pass draws from: the searcher's own, or a fresh
        one for an explicit seed (search.py:214-229)."""
        return self.rng if seed is None else _rng_for(seed)

    def _gain_pool(self):
        """Every word of positive exact gain, up to the pool cap
        (search.py:787-799)."""
        self.b.gain_map()
        self.stats["transforms"] += 1
        if self.b.map_max() <= 0:
            return np.zeros(0, dtype=np.int64)
        cap = min(POOL_CAP, self.b.extract_cap)
        idx, _v, _f = self.b.map_extract(1, cap=cap)
        return np.asarray(idx, dtype=np.int64)

    def _top_gain_pool(self, work, cap=SHELL_POOL_CAP):
        """The top of the gain map, at the histogram threshold that keeps
        about ``cap`` words, minus the incumbents (search.py:871-902)."""
        b = self.b
        b.gain_map()
        self.stats["transforms"] += 1
        mx = b.map_max()
        if mx <= 0:
            return np.zeros(0, dtype=np.int64)
        thr = 1
        if mx > 1 and getattr(b, "supports_hist", True):
            hist = b.map_hist(1024, mx)
            csum = np.cumsum(hist[::-1])[::-1]
            good = np.flatnonzero(csum <= cap)
            if len(good):
                thr = max(1, int(good[0]) * mx // 1024 + 1)
        idx, _v, _f = b.map_extract(thr, cap=min(cap, b.extract_cap))
        idx = np.asarray(idx, dtype=np.int64)
        return idx[~np.isin(idx, work)] if len(idx) else idx

    def _shell1(self, idx):
        """Every word at digit distance 1 from ``idx`` (one coordinate to
        every other value), or the backend's own radius-1 neighbours
        (search.py:818-852)."""
        nb = getattr(self.b, "neighbours", None)
        if nb is not None:
            return np.asarray(nb(int(idx), 1), dtype=np.int64)
        sp = self.b.space
        if self._sh1 is None:
            self._sh1 = []
            for p in range(sp.n):
                a, pw = int(sp.axes[p]), int(sp.pow_q[p])
                v = np.arange(a, dtype=np.int64)
                self._sh1.append(np.stack([(v[v != d] - d) * pw
                                           for d in range(a)]))
        d = (idx // np.asarray(sp.pow_q)) % np.asarray(sp.axes, dtype=np.int64)
        out = [idx + self._sh1[p][d[p]] for p in range(sp.n)]
        return np.concatenate(out) if out else np.zeros(0, dtype=np.int64)

    def _shell_k(self, idx, k, m, rng):
        """``m`` sampled words at digit distance <= k (search.py:854-869)."""
        nb = getattr(self.b, "neighbours", None)
        if nb is not None:
            return np.asarray(nb(int(idx), k, m, rng), dtype=np.int64)
        sp = self.b.space
        if m <= 0 or k <= 0 or k > sp.n:
            return np.zeros(0, dtype=np.int64)
        ax = np.asarray(sp.axes, dtype=np.int64)
        pw = np.asarray(sp.pow_q, dtype=np.int64)
        movable = np.flatnonzero(ax > 1)
        if not len(movable):
            return np.zeros(0, dtype=np.int64)
        out = np.full(m, idx, dtype=np.int64)
        for _ in range(k):
            p = movable[rng.integers(0, len(movable), size=m)]
            a = ax[p]
            v = rng.integers(0, a - 1)
            cur = (out // pw[p]) % a
            v = v + (v >= cur)                   # skip the current digit
            out = out + (v - cur) * pw[p]
        return out

    def _polish_start(self, M):
        """Trim or fill to M words and reset the best snapshot."""
        if len(self.code) > M:
            self.ruin(len(self.code) - M, "low")
        if len(self.code) < M and self.uncov > 0:
            self.greedy_fill(M)
        self.best_uncov = self.best_code = None
        self._snapshot()

    def anneal(self, M, budget_s, mode="lahc", t0=1.0, t_end=0.05,
               lahc_len=50, pool_refresh=64, sample=8, seed=None,
               log_every=0, neighbourhood="pool", n_shell2=SHELL2,
               n_top=SHELL_TOP, n_rand=SHELL_RAND, w_topk=SHELL_TOPK,
               w_random_p=0.25, greedy_p=0.5, loss_refresh=48,
               restart_stale=15000, verify_every=1):
        """Swap-neighbourhood polish at fixed M that accepts regressions
        (search.py:1091-1235).  A move drops one incumbent and adds one
        candidate, costed exactly: uncov + loss(w) - gain(v | w removed).
        ``mode`` "lahc" (late acceptance over ``lahc_len`` moves) or
        "anneal" (Metropolis, geometric cooling ``t0`` -> ``t_end`` over
        the budget).  ``neighbourhood`` "pool": the cheapest of ``sample``
        random incumbents against the best of ``sample`` draws from the
        positive-gain pool; "shell": one of the ``w_topk`` cheapest
        incumbents against its whole distance-1 shell, sampled distance-2
        words, top-of-gain and uniform draws, all costed in one
        ``swap_eval``.  Returns the final uncovered count."""
        if mode not in ("anneal", "lahc"):
            raise ValueError(f"unknown polish mode: {mode!r}")
        if neighbourhood not in ("pool", "shell"):
            raise ValueError(f"unknown neighbourhood: {neighbourhood!r}")
        if int(pool_refresh) < 1:
            raise ValueError("pool_refresh must be >= 1")
        saved = self.rng
        self.rng = rng = self._rng_pass(seed)
        try:
            self.stats["polish_neighbourhood"] = neighbourhood
            if neighbourhood == "shell":
                return self._shift_anneal(
                    M, budget_s, mode, t0, t_end, lahc_len,
                    int(pool_refresh), log_every, rng, n_shell2, n_top,
                    n_rand, w_topk, w_random_p, greedy_p, loss_refresh,
                    restart_stale, verify_every)
            return self._pool_anneal(M, budget_s, mode, t0, t_end, lahc_len,
                                     int(pool_refresh), sample, log_every,
                                     rng)
        finally:
            self.rng = saved

    def _accept_many(self, costs, uncov, bound, mode, t0, t_end, elapsed,
                     budget_s, rng):
        if mode == "lahc":
            return np.flatnonzero(costs <= max(bound, uncov))
        temp = t0 * (t_end / t0) ** min(1.0, elapsed / max(budget_s, 1e-9))
        dl = (costs - uncov).astype(np.float64)
        return np.flatnonzero((dl <= 0) | (rng.random(len(dl)) < np.exp(
            -np.maximum(dl, 0.0) / max(temp, 1e-9))))

    def _pool_anneal(self, M, budget_s, mode, t0, t_end, lahc_len, period,
                     sample, log_every, rng):
        """The "pool" neighbourhood (search.py:1237-1360)."""
        b = self.b
        self._polish_start(M)
        if self.uncov == 0 or not len(self.code):
            return self.uncov
        work = np.asarray(self.code, dtype=np.int64).copy()
        codeset = set(work.tolist())
        pool = np.zeros(0, dtype=np.int64)
        since_refresh, starved = period, 0
        hist = [float(self.uncov)] * max(1, int(lahc_len))
        t_start = time.time()
        i = moves = accepts = 0
        while self.uncov > 0:
            elapsed = time.time() - t_start
            if elapsed > budget_s or self.time_left() < self.loop_reserve_s:
                break
            if since_refresh >= period or not len(pool):
                self.code = work
                pool = self._gain_pool()
                exact = b.uncovered()
                if exact != self.uncov:
                    self.on_log(f"WARNING drift: incremental {self.uncov} "
                                f"!= field {exact}; adopting field")
                    self.uncov = exact
                since_refresh = 0
                if not len(pool):
                    break
            # drop: the cheapest of `sample` random incumbents
            ns = min(sample, len(work))
            ridx = rng.choice(len(work), size=ns, replace=False)
            loss = b.ball_gather(work[ridx], 1).astype(np.float64)
            j = int(np.argmin(loss + rng.random(ns)))
            slot = int(ridx[j])
            w = int(work[slot])
            wa = np.array([w], dtype=np.int64)
            b.ball_update(wa, -1)
            codeset.discard(w)
            # add: the best of `sample` pool draws, exact gains
            ns = min(sample, len(pool))
            draw = pool[rng.integers(0, len(pool), size=ns)]
            cand = np.array([c for c in draw.tolist()
                             if c != w and c not in codeset], dtype=np.int64)
            if not len(cand):                    # stale pool exhausted
                b.ball_update(wa, +1)
                codeset.add(w)
                since_refresh = period
                pool = np.zeros(0, dtype=np.int64)
                starved += 1
                if starved > 2:
                    break
                continue
            starved = 0
            gain = b.ball_gather(cand, 0).astype(np.float64)
            g = int(np.argmax(gain + rng.random(len(gain))))
            v = int(cand[g])
            b.ball_update(np.array([v], dtype=np.int64), +1)
            cost = self.uncov + int(loss[j]) - int(gain[g])
            moves += 1
            if mode == "lahc":
                ok = cost <= hist[i % len(hist)] or cost <= self.uncov
            else:
                delta = cost - self.uncov
                temp = t0 * (t_end / t0) ** min(
                    1.0, elapsed / max(budget_s, 1e-9))
                ok = delta <= 0 or rng.random() < np.exp(
                    -delta / max(temp, 1e-9))
            if ok:
                work[slot] = v
                codeset.add(v)
                self.uncov = cost
                accepts += 1
                since_refresh += 1
                self.code = work
                self._snapshot()
            else:
                b.ball_update(np.array([v], dtype=np.int64), -1)
                b.ball_update(wa, +1)
                codeset.add(w)
            if mode == "lahc":
                hist[i % len(hist)] = float(self.uncov)
            i += 1
            if log_every and i % log_every == 0:
                self.on_log(f"{mode} M={M} move={i} acc={accepts} "
                            f"uncov={self.uncov} best={self.best_uncov}")
        self.stats["moves"] += moves
        self.stats["accepts"] += accepts
        return self._polish_end(np.sort(work))

    def _polish_end(self, code):
        """Adopt the final or the best state, recounted exactly."""
        self.code = code
        if self.uncov == 0:
            self._snapshot()
        elif self.best_code is not None and self.best_uncov < self.uncov:
            self.code = np.sort(self.best_code)
            self.b.recount(self.code)
            self.stats["transforms"] += 1
            self.uncov = self.b.uncovered()
        return self.uncov

    def _shift_anneal(self, M, budget_s, mode, t0, t_end, lahc_len, period,
                      log_every, rng, n_shell2, n_top, n_rand, w_topk,
                      w_random_p, greedy_p, loss_refresh, restart_stale,
                      verify_every):
        """The "shell" neighbourhood (search.py:904-1089)."""
        from .gpu import swap_eval_generic
        b = self.b
        swap_eval = getattr(b, "swap_eval", None) or (
            lambda d, c: swap_eval_generic(b, d, c))
        self._polish_start(M)
        if self.uncov == 0 or not len(self.code):
            return self.uncov
        work = np.sort(np.asarray(self.code, dtype=np.int64)).copy()
        M = len(work)
        self.code = work
        uncov = int(self.uncov)
        best_u, best_code = uncov, work.copy()
        losses = self.losses().astype(np.int64)
        pool = self._top_gain_pool(work)
        t_start = time.time()
        since_pool = since_loss = 0
        hist = [float(uncov)] * max(1, int(lahc_len))
        i = moves = accepts = drift = stale = 0
        last_slot = -1
        while uncov > 0:
            elapsed = time.time() - t_start
            if elapsed > budget_s or self.time_left() < self.loop_reserve_s:
                break
            # the word to move: one of the cheapest by exact loss, or now
            # and then a uniform one
            if rng.random() < w_random_p or len(losses) != M:
                slot = int(rng.integers(M))
            else:
                k = min(int(w_topk), M)
                cheap = np.argpartition(losses, k - 1)[:k]
                slot = int(cheap[rng.integers(k)])
            if slot == last_slot and M > 1:
                slot = int(rng.integers(M))
            w = int(work[slot])
            wa = np.array([w], dtype=np.int64)
            # candidates that can plug the hole w would leave
            parts = [self._shell1(w)]
            if n_shell2:
                parts.append(self._shell_k(w, 2, int(n_shell2), rng))
            if n_top and len(pool):
                parts.append(pool[rng.integers(0, len(pool),
                                               size=min(int(n_top),
                                                        len(pool)))])
            if n_rand:
                parts.append(rng.integers(0, b.space.size, size=int(n_rand))
                             .astype(np.int64))
            cand = np.unique(np.concatenate(parts))
            cand = cand[(cand != w) & ~np.isin(cand, work)]
            if not len(cand):
                i += 1
                continue
            # the drop and the whole batch, costed in one read-only call
            lw_a, g_l = swap_eval(wa, [cand])
            lw = int(lw_a[0])
            gains = np.asarray(g_l[0]).astype(np.int64)
            costs = uncov + lw - gains
            moves += 1
            ok = self._accept_many(costs, uncov, hist[i % len(hist)], mode,
                                   t0, t_end, elapsed, budget_s, rng)
            if len(ok):
                if rng.random() < greedy_p:
                    sub = ok[costs[ok] == costs[ok].min()]
                    pick = int(sub[rng.integers(len(sub))])
                else:
                    pick = int(ok[rng.integers(len(ok))])
                v = int(cand[pick])
                b.ball_update(wa, -1)
                b.ball_update(np.array([v], dtype=np.int64), +1)
                work[slot] = v
                uncov = int(costs[pick])
                accepts += 1
                since_pool += 1
                since_loss += 1
                last_slot = slot
                if verify_every and accepts % verify_every == 0:
                    exact = b.uncovered()
                    if exact != uncov:
                        drift += 1
                        uncov = exact
                if uncov < best_u:
                    best_u, best_code = uncov, work.copy()
                    stale = 0
                    self.code, self.uncov = work, uncov
                    self._snapshot()
                    if uncov == 0:
                        break
            else:
                last_slot = -1
            if mode == "lahc":
                hist[i % len(hist)] = float(uncov)
            i += 1
            stale += 1
            if restart_stale and stale >= restart_stale:
                # back to the best state, acceptance history restarted
                work = best_code.copy()
                b.recount(work)
                self.stats["transforms"] += 1
                uncov = b.uncovered()
                hist = [float(uncov)] * len(hist)
                losses = self.losses().astype(np.int64)
                pool = self._top_gain_pool(work)
                since_pool = since_loss = stale = 0
                last_slot = -1
                continue
            if since_pool >= period:
                pool = self._top_gain_pool(work)
                since_pool = 0
            if since_loss >= loss_refresh:
                self.code = work
                losses = self.losses().astype(np.int64)
                since_loss = 0
            if log_every and i % log_every == 0:
                self.on_log(f"shift M={M} move={i} acc={accepts} "
                            f"uncov={uncov} best={best_u}")
        self.stats["moves"] += moves
        self.stats["accepts"] += accepts
        self.stats["shift_drift"] = self.stats.get("shift_drift", 0) + drift
        self.code = np.sort(best_code if best_u < uncov else work)
        b.recount(self.code)
        self.stats["transforms"] += 1
        self.uncov = b.uncovered()
        self._snapshot()
        return self.uncov
