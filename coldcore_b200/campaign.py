"""A campaign of searches on the batched engine: one search per cell, every
cell's transforms in one persistent graph launch per tick.

coldcore runs a campaign as one process per cell, each with its own
singleton plugin context (``src/coldcore/campaign.py:88-221``: ``run_job``
per cell, ``run_campaign`` over a process pool).  Here every cell of the
campaign sits in one ``BatchEngine``; each cell's search runs in its own
host thread against a :class:`BatchCellBackend`, the search protocol on
that cell.  The per-cell calls (updates, gathers, extraction, counts) go to
the device at once; a transform request (recount, gain map, loss map)
blocks its thread until a TICK: the driver waits until every live search
is blocked on a transform, uploads the codes that changed, runs the one
graph launch that recounts every cell and rebuilds every gain and loss map,
and releases them all.  So N searches cost one launch per transform step
instead of N.

A cell's counters are recounted from its code at every tick, so the
adapter keeps the code as a multiset that follows its updates; between
ticks no search is inside a transform, and no launch races a cell's
incremental updates.

``run_campaign(jobs)`` returns one record per job, like ``run_job``: the
cell, seed, final size M, the uncovered count (0 = a verified cover), the
solution trace and the search's counters.
"""
import sys
import threading
import time
import traceback
from collections import Counter

import numpy as np

from .batch import BatchEngine
from .patterns import wide_table
from .space import ProductSpace


class Ticker:
    """Lock-step transform ticks over the live searches of one batch."""

    def __init__(self, engine, cells):
        self.engine = engine
        self.cells = cells
        self.cv = threading.Condition()
        self.live = 0
        self.waiting = 0
        self.tick = 0
        self.scalars = None
        self.ticks = 0
        self.error = None
        self.greedy_req = {}            # cell -> words it may place
        self.greedy_out = {}            # cell -> (placed, deficit)
        self.greedy_calls = 0

    def join(self):
        with self.cv:
            self.live += 1

    def leave(self):
        with self.cv:
            self.live -= 1
            self.cv.notify_all()

    def request(self, greedy_cell=None, max_add=0):
        """Block until the next tick has run (every cell recounted from
        its code, every gain and loss map rebuilt).  With ``greedy_cell``,
        that cell's exact greedy repair (up to ``max_add`` words) runs in
        the same tick, beside every other cell asking for one; returns its
        (placed words, deficit)."""
        with self.cv:
            t = self.tick
            if greedy_cell is not None:
                self.greedy_req[greedy_cell] = int(max_add)
            self.waiting += 1
            self.cv.notify_all()
            while self.tick == t and self.error is None:
                self.cv.wait()
            if self.error is not None:
                raise RuntimeError(f"batched tick failed: {self.error}")
            if greedy_cell is not None:
                return self.greedy_out.pop(greedy_cell)
            return None

    def serve(self):
        """The driver loop: run a tick whenever every live search waits;
        returns when no search is left."""
        with self.cv:
            while True:
                while self.live and self.waiting < self.live:
                    self.cv.wait()
                if not self.live:
                    return
                try:
                    for c in self.cells:
                        c.sync_code()
                    self.engine.run(0)
                    self.scalars = self.engine.scalars()
                    self.ticks += 1
                    if self.greedy_req:
                        ids = sorted(self.greedy_req)
                        # each placement serves a deficient word: no cell
                        # places more words than its deficit
                        adds = [max(0, min(self.greedy_req[k],
                                           int(self.scalars[k, 0])))
                                for k in ids]
                        res = self.engine.greedy(ids, adds)
                        self.greedy_out.update(zip(ids, res))
                        self.greedy_req.clear()
                        self.greedy_calls += 1
                except Exception as e:          # noqa: BLE001
                    self.error = repr(e)
                self.waiting = 0
                self.tick += 1
                self.cv.notify_all()
                if self.error is not None:
                    return


class BatchCellBackend:
    """The search protocol on cell ``i`` of a batch (the methods coldcore's
    ``Searcher`` calls, ``src/coldcore/protocol.py:60-140``)."""

    def __init__(self, engine, ticker, i, problem, axes, R, mu=1,
                 extract_cap=1 << 18):
        self.engine, self.ticker, self.i = engine, ticker, int(i)
        self.problem, self.R, self.mu = problem, int(R), int(mu)
        self.space = ProductSpace(axes)
        self.extract_cap = int(extract_cap)
        self.indep_dist = 2 * R if problem in ("hamming", "lee") else None
        self.supports_hist = False
        self.code = Counter()           # the multiset the counters follow
        self._dirty = True
        self.field = 1                  # map the last transform left

    # ---------------- the code behind the counters
    def sync_code(self):
        if self._dirty:
            words = np.fromiter(self.code.elements(), dtype=np.int64,
                                count=sum(self.code.values()))
            self.engine.set_code(self.i, np.sort(words))
            self._dirty = False

    def word_index(self, words):
        return self.space.word_index(words)

    def index_word(self, idx):
        return self.space.index_word(idx)

    # ---------------- transforms (one tick each)
    def recount(self, idx):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        self.code = Counter(idx.tolist())
        self._dirty = True
        self.ticker.request()

    def gain_map(self):
        self.ticker.request()
        self.field = 1

    def loss_map(self):
        self.ticker.request()
        self.field = 2

    def greedy_fill_device(self, max_add):
        """Exact greedy repair on the device, batched with every other
        cell's in one tick: (placed words in order, deficit left)."""
        placed, deficit = self.ticker.request(self.i, max_add)
        if len(placed):
            self.code.update(placed.tolist())
            self._dirty = True
        return placed, deficit

    # ---------------- incremental / exact
    def ball_update(self, idx, delta):
        idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
        if not len(idx):
            return
        if delta < 0:
            for w in idx.tolist():
                if self.code[w] <= 0:
                    raise RuntimeError(f"ball_update removes absent {w}")
                self.code[w] -= 1
                if not self.code[w]:
                    del self.code[w]
        else:
            self.code.update(idx.tolist())
        self._dirty = True
        self.engine.update(self.i, idx, int(delta))

    def ball_gather(self, idx, target):
        return self.engine.gather(self.i, idx, int(target))

    # ---------------- queries
    def count_eq(self, target):
        return self.engine.count(self.i, 0, int(target))

    def uncovered(self):
        if self.mu == 1:
            return self.engine.count(self.i, 0, 0)
        return self.engine.count(self.i, 1)

    def map_max(self):
        sc = self.ticker.scalars
        return int(sc[self.i, self.field]) if sc is not None else 0

    def map_extract(self, thr, cap=None):
        cap = min(cap or self.extract_cap, self.extract_cap)
        idx, val, found = self.engine.extract(self.i, self.field, int(thr),
                                              cap)
        return idx, val, found

    def map_read_at(self, idx):
        return self.engine.read_at(self.i, self.field, idx)

    def read_cnt(self, off=0, length=None):
        length = self.space.size - off if length is None else length
        return self.engine.read_range(self.i, 0, off, length)


class _LockedEngine:
    """The batch's per-cell calls under one lock: they share the batch's
    stream and staging buffers, and ctypes releases the GIL during them."""

    _CALLS = ("set_code", "update", "gather", "count", "extract", "read_at",
              "read_range", "greedy")

    def __init__(self, engine, lock):
        self._e, self._lock = engine, lock

    def __getattr__(self, name):
        f = getattr(self._e, name)
        if name not in self._CALLS:
            return f

        def locked(*a, **kw):
            with self._lock:
                return f(*a, **kw)
        return locked


def _cell_spec(job):
    return (job.get("problem", "hamming"), tuple(int(a) for a in job["axes"]),
            int(job["R"]), int(job.get("mu", 1)))


def _label(job):
    p, a, R, mu = _cell_spec(job)
    return job.get("label") or (
        f"{p}:{'x'.join(map(str, a))}:R{R}" + (f":mu{mu}" if mu > 1 else ""))


def run_job(job, backend):
    """One cell's search on a protocol backend, to the job's budget: a
    greedy cover from empty, then (mode "descend") the notch descent; the
    record of coldcore's ``run_job`` (``campaign.py:88-179``) without its
    files.  Never raises: an error is recorded."""
    from .search import Searcher
    t0 = time.time()
    budget = float(job.get("budget_s", 30.0))
    rec = {"label": _label(job), "cell": _cell_spec(job),
           "seed": int(job.get("seed", 1)), "budget_s": budget, "M": None,
           "uncov": None, "solutions": [], "stats": {}, "error": None}

    def on_solved(M, idx):
        rec["M"] = int(M)
        rec["solutions"].append([round(time.time() - t0, 3), int(M)])

    try:
        s = Searcher(backend, seed=rec["seed"], deadline=t0 + budget,
                     on_solved=on_solved,
                     repair=job.get("repair", "exact"))
        s.build_reserve_s = s.loop_reserve_s = 0.0
        s.load(np.zeros(0, dtype=np.int64))
        s.greedy_fill(10 ** 9)
        if s.uncov == 0:
            s.peel()
            if s.verify_full() == 0:
                on_solved(len(s.code), s.code)
            if job.get("mode", "build") == "descend" and s.uncov == 0:
                s.descend(floor=int(job.get("floor", 1)),
                          notch_budget_s=float(job.get("notch_s", 5.0)),
                          reserve_s=0.0, min_notch_s=0.5,
                          step0=int(job.get("step0", 2)))
        rec["uncov"] = int(s.uncov)
        rec["M"] = rec["M"] if rec["M"] is not None else len(s.code)
        rec["code"] = np.asarray(s.best_code if s.uncov and s.best_code
                                 is not None else s.code).tolist()
        rec["stats"] = {k: v for k, v in s.stats.items()
                        if isinstance(v, (int, float))}
    except Exception:                                   # noqa: BLE001
        rec["error"] = traceback.format_exc()
    rec["secs"] = round(time.time() - t0, 3)
    return rec


def run_campaign(jobs, plugin_path=None, tile_kb=0, engine=None,
                 switch_s=5e-5):
    """Every job's search on one batched engine (see the module text);
    returns one record per job, in job order, and the number of ticks.
    ``engine``: a stand-in with BatchEngine's methods (host tests)."""
    eng = engine if engine is not None else BatchEngine(plugin_path)
    try:
        specs = [_cell_spec(j) for j in jobs]
        for p, a, R, mu in specs:
            eng.add(p, a, R, np.zeros(0, dtype=np.int64), mu)
        eng.build(tile_kb)
        lock = threading.Lock()
        locked = _LockedEngine(eng, lock)
        cells = []
        ticker = Ticker(locked, cells)
        for k, (p, a, R, mu) in enumerate(specs):
            eng.set_table(k, wide_table(a, R, p))
            cells.append(BatchCellBackend(locked, ticker, k, p, a, R, mu))
        recs = [None] * len(jobs)

        def work(k):
            try:
                recs[k] = run_job(jobs[k], cells[k])
            finally:
                ticker.leave()

        for _ in jobs:
            ticker.join()
        threads = [threading.Thread(target=work, args=(k,), daemon=True)
                   for k in range(len(jobs))]
        # a search thread returning from a device call waits for the GIL;
        # hand it over often, or every call waits out the default 5 ms
        switch = sys.getswitchinterval()
        sys.setswitchinterval(switch_s)
        try:
            for t in threads:
                t.start()
            ticker.serve()
            for t in threads:
                t.join()
        finally:
            sys.setswitchinterval(switch)
        return recs, ticker.ticks
    finally:
        eng.close()


def run_serial(jobs, plugin_path=None):
    """The same jobs one after another, each on its own singleton cell
    context (coldcore's one-context-per-cell campaign, in one process)."""
    from .gpu import GpuBackend
    recs = []
    for j in jobs:
        p, a, R, mu = _cell_spec(j)
        with GpuBackend(list(a), R, problem=p, mu=mu,
                        plugin_path=plugin_path) as b:
            recs.append(run_job(j, b))
    return recs
