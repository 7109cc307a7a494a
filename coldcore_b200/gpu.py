"""ctypes binding of the B200 covering engine (plugin ABI v1).

Mirrors coldcore's ``src/coldcore/gpu.py`` (``GpuBackend``,
``load_plugin``, ``default_plugin_path``, ``locality_order`` and the two
``*_generic`` reference forms): same constructor arguments, method names,
return types and ``RuntimeError`` on a negative return code, so a search
core written against the reference's backend runs on this one unchanged.
The library is ``coldcore_b200/libcoldcore_covering.so`` (built by
``python -m coldcore_b200.build``); there is no fallback — a missing or
unloadable library raises.

Additions: cells with axes wider than 16 (king 2048x2048) go through
``dct_init3w`` with the engine's wide support table; ``layer(d)`` reads
the exact distance layers after ``layers_map()``; ``stream`` is the
engine's CUDA stream handle for host-side timing.
"""
import ctypes
import os

import numpy as np

from .patterns import PROBLEM_IDS, locality_key, v1_table, wide_table
from .space import ProductSpace

_libs = {}

# HBM budget of the automatic placement (bytes): COLDCORE_HBM_BUDGET, as in
# coldcore (src/coldcore/gpu.py:31-33), defaulting to most of a B200's
# 180 GB with room for tables, staging and other tenants.
HBM_BUDGET = int(float(os.environ.get("COLDCORE_HBM_BUDGET", 160e9)))

_LL = ctypes.c_longlong
_I32P = ctypes.POINTER(ctypes.c_int32)
_LLP = ctypes.POINTER(_LL)

REQUIRED = ("dct_init3", "dct_free", "dct_set_code", "dct_transform",
            "dct_ball_update", "dct_ball_gather", "dct_count_eq",
            "dct_map_max", "dct_map_extract", "dct_map_extract64",
            "dct_map_read_at", "dct_read_cnt")


def _rc_msg(rc):
    if rc <= -100:
        return f"rc={rc} (CUDA error {-(rc + 100)})"
    return f"rc={rc}"


def _check(name, rc):
    if rc != 0:
        raise RuntimeError(f"{name} {_rc_msg(rc)}")


def _bind(path):
    lib = ctypes.CDLL(path)
    missing = [f for f in REQUIRED if not hasattr(lib, f)]
    if missing:
        raise RuntimeError(f"{path} lacks required symbols {missing}")
    I, P64 = ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)
    sig = {
        "dct_init3": (I, [I, I, ctypes.POINTER(I), I, P64, _LL, I, _LLP, I, I,
                          I]),
        "dct_init3w": (I, [I, I, ctypes.POINTER(I), I, _I32P, I, _LL, I,
                           _LLP]),
        "dct_b200_init3wm": (I, [I, I, ctypes.POINTER(I), I, _I32P, I, _LL,
                                 I, _LLP, I, I]),
        "dct_init2": (I, [I, I, I, P64, _LL, I, _LLP, I, I, I]),
        "dct_init": (I, [I, I, I, P64, _LL, I, _LLP]),
        "dct_free": (I, []),
        "dct_host_bytes": (_LL, []),
        "dct_set_code": (I, [_LLP, I]),
        "dct_transform": (I, [I, I]),
        "dct_set_mu": (I, [I]),
        "dct_get_mu": (I, []),
        "dct_ball_update": (I, [_LLP, I, I]),
        "dct_ball_gather": (I, [_LLP, I, I, _I32P]),
        "dct_ball_gather_mu": (I, [_LLP, I, I, _I32P]),
        "dct_loss_owner": (I, [_LLP, I, _I32P]),
        "dct_ball_update_delta": (I, [_LLP, I, I, _LLP]),
        "dct_swap_eval": (I, [_LLP, I, _LLP, _LLP, _I32P, _I32P]),
        "dct_stats": (I, [_LLP, I]),
        "dct_count_eq": (_LL, [I]),
        "dct_count_deficit": (_LL, []),
        "dct_map_max": (I, [_I32P]),
        "dct_map_hist": (I, [I, ctypes.c_int32, _I32P]),
        "dct_map_extract": (_LL, [ctypes.c_int32,
                                  ctypes.POINTER(ctypes.c_uint32), _I32P, I]),
        "dct_map_extract64": (_LL, [ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int64), _I32P, I]),
        "dct_map_read_at": (I, [_LLP, I, _I32P]),
        "dct_read_cnt": (I, [_LL, _LL, ctypes.POINTER(ctypes.c_uint16)]),
        "dct_set_tbl2": (I, [ctypes.POINTER(ctypes.c_uint16), P64, _LL]),
        "dct_use_fmt": (I, [I]),
        "dct_b200_stream": (_LL, []),
        "dct_b200_plan": (I, [I, I, _LLP, I]),
        "dct_b200_plan_forms": (I, [I, I, _I32P, I]),
        "dct_b200_plan_probe": (I, [I, I, ctypes.POINTER(ctypes.c_int), I, I,
                                    I, I, I, I, _LLP, I]),
        "dct_b200_read_layer": (I, [I, _LL, _LL, _I32P]),
        "dct_b200_read_map": (I, [_LL, _LL, _I32P]),
        "dct_b200_set_timing": (I, [I]),
        "dct_b200_ball_hist": (I, [_LLP, I, I, I, _I32P]),
        "dct_b200_layers_at": (I, [_LLP, I, _I32P]),
        "dct_b200_greedy_fill": (I, [I, _LLP, _LLP]),
        "dct_b200_last_timings": (I, [ctypes.POINTER(ctypes.c_float), I]),
        "dct_b200_ooc_plan": (I, [I, I, ctypes.POINTER(I), I, I, I, _LL, _LL,
                                  _LL, I, _LLP, I]),
        "dct_b200_ooc_record": (_LL, [I, I, ctypes.POINTER(I), I, I, I, I,
                                      _LLP, _LL, _LL, I, _LLP, _LL]),
        "dct_b200_ooc_transform": (I, [I, I, ctypes.POINTER(I), I, I, I, I,
                                       _LLP, _LL, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, _LL,
                                       _LL, I,
                                       ctypes.POINTER(ctypes.c_float)]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    return lib


def placement(size, nlayers, budget=None):
    """(layers_mode, cnt_mode) for a cell of ``size`` words: everything in
    HBM when ``size * (4 * nlayers + 2)`` bytes fit the budget, else the
    layer planes in host memory, streamed (mode 1); cnt stays in HBM while
    it and the device map plane (6 bytes a word) fit, else managed.  The
    rule of coldcore's policy (``src/coldcore/gpu.py:253-260``) with the
    map plane counted, since a streamed cell keeps it on the device."""
    budget = HBM_BUDGET if budget is None else budget
    layers_mode = 0 if size * (4 * nlayers + 2) <= budget else 1
    cnt_mode = 0 if layers_mode == 0 or size * 6 <= budget else 1
    return layers_mode, cnt_mode


def default_plugin_path():
    """``COLDCORE_PLUGIN_PATH`` if set, else the in-tree library."""
    env = os.environ.get("COLDCORE_PLUGIN_PATH")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "libcoldcore_covering.so")


def load_plugin(path=None):
    """Load (and cache) the engine library; raises when it is missing."""
    path = os.path.abspath(path or default_plugin_path())
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(
                f"engine library not built: {path} "
                "(run `python -m coldcore_b200.build`)")
        _libs[path] = _bind(path)
    return _libs[path]


PLAN_FIELDS = ("axis0", "axes", "pair", "W", "mid", "Bo", "inner", "outer",
               "tiles", "kernel", "pipe", "pack", "in16", "out16", "smem",
               "threads", "lin", "lout", "skew", "grid", "src", "dst",
               "rounds", "round_axes")


def plan_probe(problem, axes, R, init_mode, out_mode, budget_kb=100, pipe=1,
               half=True, plugin_path=None):
    """The launches the planner gives a geometry, without a cell or a GPU:
    one dict per launch (``PLAN_FIELDS``), [] for window passes."""
    lib = load_plugin(plugin_path)
    ax = (ctypes.c_int * len(axes))(*[int(a) for a in axes])
    rows = np.zeros(24 * 64, dtype=np.int64)
    n = lib.dct_b200_plan_probe(PROBLEM_IDS[problem], len(axes), ax, int(R),
                                int(init_mode), int(out_mode), int(budget_kb),
                                int(pipe), 1 if half else 0, _p(rows),
                                len(rows))
    if n < 0:
        _check("plan_probe", n)
    return [dict(zip(PLAN_FIELDS, (int(v) for v in rows[24 * i:24 * i + 24])))
            for i in range(n)]


def ball_order():
    """True unless ``COLDCORE_BALL_ORDER=native`` asks for the builder's
    table order (coldcore ``gpu.py:119``, an A/B switch: the walks are
    order-free, so only the memory traffic changes)."""
    return os.environ.get("COLDCORE_BALL_ORDER", "locality") != "native"


def locality_order(pats, axes):
    """Sort a v1 table by unwrapped offset so that neighbouring walk threads
    touch neighbouring words (coldcore ``gpu.py:106-129``); order-free walks
    make this a pure traffic optimisation.  Entry 0 stays the centre."""
    if not ball_order():
        return pats
    pats = np.ascontiguousarray(pats, dtype=np.uint64)
    n = len(axes)
    pos = np.zeros((len(pats), 8), dtype=np.int64)
    dlt = np.zeros((len(pats), 8), dtype=np.int64)
    for k in range(8):
        b = ((pats >> np.uint64(8 * k)) & np.uint64(255)).astype(np.int64)
        pos[:, k] = np.minimum(b >> 4, n - 1)
        dlt[:, k] = b & 15
    return np.ascontiguousarray(
        pats[np.argsort(locality_key(pos, dlt, axes), kind="stable")])


def _swap_inputs(drops, cands):
    """Normalise swap_eval's arguments: (drops int64[k], one candidate
    array per drop, the length of the array every drop shares, or None
    when each drop has its own)."""
    drops = np.ascontiguousarray(np.atleast_1d(drops), dtype=np.int64)
    if isinstance(cands, (list, tuple)):
        if len(cands) != len(drops):
            raise ValueError("need one candidate array per drop")
        return drops, [np.ascontiguousarray(np.atleast_1d(c), dtype=np.int64)
                       for c in cands], None
    one = np.ascontiguousarray(np.atleast_1d(cands), dtype=np.int64)
    return drops, [one] * len(drops), len(one)


def _swap_output(loss, gains, shared):
    """Shared candidates come back as a (k, shared) array, else a list."""
    if shared is None:
        return loss, gains
    return loss, (np.stack(gains) if gains
                  else np.zeros((0, shared), dtype=np.int32))


def swap_eval_generic(backend, drops, cands):
    """``swap_eval`` composed from the protocol for any backend (the form
    of coldcore ``gpu.py:132-164``): per drop word its role-1 gather, then,
    with the word taken out, the role-0 gathers of its candidates; the
    word is put back, so cnt ends as it started."""
    drops, parts, shared = _swap_inputs(drops, cands)
    loss = np.zeros(len(drops), dtype=np.int32)
    gains = []
    for i, (w, cand) in enumerate(zip(drops.tolist(), parts)):
        one = np.array([w], dtype=np.int64)
        loss[i] = int(backend.ball_gather(one, 1)[0])
        g = np.zeros(0, dtype=np.int32)
        if cand.size:
            backend.ball_update(one, -1)
            try:
                g = np.asarray(backend.ball_gather(cand, 0), dtype=np.int32)
            finally:
                backend.ball_update(one, +1)
        gains.append(g)
    return _swap_output(loss, gains, shared)


def ball_update_delta_generic(backend, idx, delta):
    """Update plus the change of ``uncovered()`` (coldcore ``gpu.py:167``)."""
    u0 = backend.uncovered()
    backend.ball_update(idx, delta)
    return backend.uncovered() - u0


def _p(a, t=_LL):
    return a.ctypes.data_as(ctypes.POINTER(t))


class GpuBackend:
    """One problem cell resident on the B200 (coldcore ``gpu.py:207-537``).

    problem: "hamming", "torus_linf", "lee" or "grid_linf"; mu: covering
    multiplicity; layers_mode: 0 = HBM, 1 = pinned host planes streamed
    through the device by each transform (cells of two or more axes up to
    16; others fall back to managed memory), 2 = managed memory; cnt_mode:
    0 = HBM, 1 / 2 = managed memory.  None picks both by ``placement``
    (HBM whenever the cell fits ``COLDCORE_HBM_BUDGET``); cells that take
    the wide table (more than 16 axes, or axes above 16) get theirs through
    ``dct_b200_init3wm``.
    """

    def __init__(self, axes, R, problem="hamming", plugin_path=None,
                 extract_cap=1 << 22, layers_mode=None, cnt_mode=None,
                 use_owner=False, mu=1):
        if problem not in PROBLEM_IDS:
            raise ValueError(f"unknown problem {problem!r}")
        self.problem = problem
        self.R = int(R)
        self.mu = mu = int(mu)
        if not 1 <= mu <= 65535:
            raise ValueError("mu must be in 1..65535")
        self.space = ProductSpace(axes)
        self.extract_cap = int(extract_cap)
        self.indep_dist = 2 * R if problem in ("hamming", "lee") else None
        self.supports_hist = True
        self._lib = lib = load_plugin(plugin_path)
        self._ext_bufs = None
        self._closed = True
        axes = self.space.axes
        auto_l, auto_c = placement(
            self.space.size,
            1 if problem in ("torus_linf", "grid_linf") else self.R + 1)
        layers_mode = auto_l if layers_mode is None else layers_mode
        cnt_mode = auto_c if cnt_mode is None else cnt_mode
        self.layers_mode, self.cnt_mode = layers_mode, cnt_mode
        by = _LL(0)
        ax = (ctypes.c_int * self.space.n)(*axes)
        pid = PROBLEM_IDS[problem]
        if max(axes) <= 16 and self.space.n <= 16 and (
                problem in ("hamming", "lee") or self.space.n <= 8):
            pats = v1_table(axes, R, problem, order=ball_order())
            self.ball_len = len(pats)
            rc = lib.dct_init3(pid, self.space.n, ax, self.R,
                               _p(pats, ctypes.c_uint64), len(pats),
                               self.extract_cap, ctypes.byref(by),
                               layers_mode or 0, cnt_mode or 0,
                               1 if use_owner else 0)
        else:
            tbl = wide_table(axes, R, problem, order=ball_order())
            self.ball_len = len(tbl)
            if layers_mode or cnt_mode:
                rc = lib.dct_b200_init3wm(
                    pid, self.space.n, ax, self.R, _p(tbl, ctypes.c_int32),
                    tbl.shape[1], len(tbl), self.extract_cap,
                    ctypes.byref(by), int(layers_mode), int(cnt_mode))
            else:
                rc = lib.dct_init3w(pid, self.space.n, ax, self.R,
                                    _p(tbl, ctypes.c_int32), tbl.shape[1],
                                    len(tbl), self.extract_cap,
                                    ctypes.byref(by))
        _check("init", rc)
        self._closed = False
        _check("set_mu", lib.dct_set_mu(mu))
        self.gpu_bytes = by.value
        self.host_bytes = int(lib.dct_host_bytes())

    # ---------------- lifecycle
    def close(self):
        if not self._closed:
            self._lib.dct_free()
            self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def word_index(self, words):
        return self.space.word_index(words)

    def index_word(self, idx):
        return self.space.index_word(idx)

    @property
    def stream(self):
        return int(self._lib.dct_b200_stream())

    # ---------------- fields
    def _set_code(self, idx):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        _check("set_code", self._lib.dct_set_code(_p(idx), len(idx)))

    def stage_code(self, idx):
        """Upload a code for ``layers_map(0)`` without touching cnt."""
        self._set_code(idx)

    def recount(self, idx):
        self._set_code(idx)
        _check("transform(code->cnt)", self._lib.dct_transform(0, 2))

    def gain_map(self):
        _check("transform(uncov->gain)", self._lib.dct_transform(1, 1))

    def loss_map(self):
        _check("transform(cnt1->loss)", self._lib.dct_transform(2, 1))

    def layers_map(self, init_mode=0):
        """Transform into the exact distance layers N_0..N_R (Hamming, Lee):
        init_mode 0 = the staged code, 1 = deficient words, 2 = critical."""
        _check("transform(layers)", self._lib.dct_transform(init_mode, 3))

    def layer(self, d, off=0, length=None):
        length = self.space.size - off if length is None else length
        out = np.empty(length, dtype=np.int32)
        _check("read_layer", self._lib.dct_b200_read_layer(
            d, off, length, _p(out, ctypes.c_int32)))
        return out

    def set_timing(self, on):
        self._lib.dct_b200_set_timing(1 if on else 0)

    def last_timings(self):
        """Device milliseconds of each launch of the last transform."""
        buf = (ctypes.c_float * 64)()
        n = self._lib.dct_b200_last_timings(buf, 64)
        return [float(buf[i]) for i in range(min(n, 64))]

    def ball_hist(self, idx, src=0, nbins=8):
        """Per word, a histogram over its ball: src 0 = the current map in
        log2 bins (0: v <= 0, 1: v == 1, 2: 2..3, ...), src 1 = cnt in
        linear bins; the last bin takes everything above."""
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.zeros((len(idx), nbins), dtype=np.int32)
        if len(idx):
            _check("ball_hist", self._lib.dct_b200_ball_hist(
                _p(idx), len(idx), int(src), int(nbins),
                _p(out, ctypes.c_int32)))
        return out

    def layers_at(self, idx):
        """(k, R+1) exact distance layers at k words, after layers_map()."""
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.zeros((len(idx), self.R + 1), dtype=np.int32)
        if len(idx):
            _check("layers_at", self._lib.dct_b200_layers_at(
                _p(idx), len(idx), _p(out, ctypes.c_int32)))
        return out

    def greedy_fill_device(self, max_add):
        """Exact greedy repair on the GPU: places up to ``max_add`` words of
        largest exact gain (ties: smallest index), non-active words only;
        returns (placed words in order, deficit left).  Every placement
        serves a deficient word, so at most the deficit is placed."""
        max_add = min(int(max_add), self.uncovered())
        placed = np.zeros(max(1, int(max_add)), dtype=np.int64)
        deficit = _LL(0)
        n = self._lib.dct_b200_greedy_fill(int(max_add), _p(placed),
                                           ctypes.byref(deficit))
        if n < 0:
            _check("greedy_fill", n)
        return placed[:n].copy(), int(deficit.value)

    def plan(self, init_mode, out_mode):
        """Launches of one transform: rows (first axis, axes, bytes, kernel)."""
        buf = np.zeros(4 * 64, dtype=np.int64)
        n = self._lib.dct_b200_plan(init_mode, out_mode, _p(buf), len(buf))
        if n < 0:
            _check("plan", n)
        return buf[:4 * n].reshape(n, 4)

    PIPE, PACK, IN16, OUT16, PAIR, STREAMED, BYTE8 = 1, 2, 4, 8, 16, 32, 64

    def plan_forms(self, init_mode, out_mode):
        """Schedule form of each group launch of one transform, as bit flags
        (PIPE prefetching kernel, PACK word pairs, IN16 / OUT16 16-bit
        layers, PAIR axis 0 inside each pair, STREAMED a streamed form,
        BYTE8 8-bit layers read or written)."""
        buf = np.zeros(64, dtype=np.int32)
        n = self._lib.dct_b200_plan_forms(init_mode, out_mode,
                                          _p(buf, ctypes.c_int32), len(buf))
        if n < 0:
            _check("plan_forms", n)
        return buf[:n].copy()

    # ---------------- incremental / exact
    def ball_update(self, idx, delta):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        _check("ball_update", self._lib.dct_ball_update(
            _p(idx), len(idx), int(delta)))

    def ball_gather(self, idx, target):
        """Exact per-candidate count of ball words by coverage role:
        0 deficient (cnt < mu), 1 critical (1 <= cnt <= mu), else the
        literal cnt == target (coldcore ``gpu.py:323-348``)."""
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.empty(len(idx), dtype=np.int32)
        if not len(idx):
            return out
        if self.mu == 1 or target not in (0, 1):
            _check("ball_gather", self._lib.dct_ball_gather(
                _p(idx), len(idx), int(target), _p(out, ctypes.c_int32)))
        else:
            _check("ball_gather_mu", self._lib.dct_ball_gather_mu(
                _p(idx), len(idx), int(target), _p(out, ctypes.c_int32)))
        return out

    def ball_update_delta(self, idx, delta):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        dd = _LL(0)
        _check("ball_update_delta", self._lib.dct_ball_update_delta(
            _p(idx), len(idx), int(delta), ctypes.byref(dd)))
        return int(dd.value)

    #: most drops, and most candidates, one dct_swap_eval call takes (the
    #: ABI's 65,535-occurrence word check applies to both)
    SWAP_CAP = (1 << 16) - 1

    def swap_eval(self, drops, cands):
        """Exact costs of many swaps without changing state (coldcore
        ``gpu.py:368-440``): ``(loss, gains)``.  Drops are sent in runs
        that stay within ``SWAP_CAP`` drops and ``SWAP_CAP`` candidates."""
        drops, parts, shared = _swap_inputs(drops, cands)
        k, cap = len(drops), self.SWAP_CAP
        ends = np.zeros(k + 1, dtype=np.int64)
        np.cumsum([len(p) for p in parts], out=ends[1:])
        loss = np.zeros(k, dtype=np.int32)
        gains = []
        lo = 0
        while lo < k:
            # the longest run [lo, hi) within both caps
            hi = min(k, lo + cap,
                     int(np.searchsorted(ends, ends[lo] + cap, "right")) - 1)
            if hi <= lo:
                raise ValueError(f"over {cap} candidates for one drop")
            base = ends[lo:hi + 1] - ends[lo]
            flat = (np.concatenate(parts[lo:hi]) if base[-1]
                    else np.zeros(1, dtype=np.int64))
            g = np.zeros(max(int(base[-1]), 1), dtype=np.int32)
            run = np.ascontiguousarray(drops[lo:hi])
            _check("swap_eval", self._lib.dct_swap_eval(
                _p(run), hi - lo, _p(flat), _p(np.ascontiguousarray(base)),
                _p(g, ctypes.c_int32), _p(loss[lo:hi], ctypes.c_int32)))
            gains.extend(g[base[t]:base[t + 1]].copy()
                         for t in range(hi - lo))
            lo = hi
        return _swap_output(loss, gains, shared)

    def loss_owner(self, idx):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.empty(len(idx), dtype=np.int32)
        _check("loss_owner", self._lib.dct_loss_owner(
            _p(idx), len(idx), _p(out, ctypes.c_int32)))
        return out

    def gpu_stats(self):
        buf = (_LL * 8)()
        self._lib.dct_stats(buf, 8)
        keys = ("gather_set_side", "gather_walk", "set_scans",
                "set_overflows", "swap_eval_fast", "swap_eval_fallback",
                "count_eq0_listed", "gather_set_tiled")
        return {k: int(v) for k, v in zip(keys, buf)}

    # ---------------- queries
    def count_eq(self, target):
        r = int(self._lib.dct_count_eq(int(target)))
        if r < 0:
            _check("count_eq", r)
        return r

    def uncovered(self):
        """Total deficit sum_x max(0, mu - cnt(x)) (mu = 1: uncovered)."""
        if self.mu == 1:
            return self.count_eq(0)
        r = int(self._lib.dct_count_deficit())
        if r < 0:
            _check("count_deficit", r)
        return r

    def map_max(self):
        v = ctypes.c_int32(0)
        _check("map_max", self._lib.dct_map_max(ctypes.byref(v)))
        return int(v.value)

    def map_hist(self, nbins, vmax):
        out = np.zeros(nbins, dtype=np.int32)
        _check("map_hist", self._lib.dct_map_hist(
            int(nbins), int(vmax), _p(out, ctypes.c_int32)))
        return out

    def map_extract(self, thr, cap=None):
        cap = min(cap or self.extract_cap, self.extract_cap)
        wide = self.space.size > 2 ** 32 - 2
        oi = np.empty(max(cap, 1), dtype=np.int64 if wide else np.uint32)
        ov = np.empty(max(cap, 1), dtype=np.int32)
        if wide:
            found = self._lib.dct_map_extract64(
                int(thr), _p(oi, ctypes.c_int64), _p(ov, ctypes.c_int32), cap)
        else:
            found = self._lib.dct_map_extract(
                int(thr), _p(oi, ctypes.c_uint32), _p(ov, ctypes.c_int32), cap)
        if found < 0:
            _check("map_extract", int(found))
        m = min(int(found), cap)
        return oi[:m].astype(np.int64), ov[:m].copy(), int(found)

    def map_all(self):
        """The whole map field in one device-to-host copy."""
        out = np.empty(self.space.size, dtype=np.int32)
        _check("read_map", self._lib.dct_b200_read_map(
            0, self.space.size, _p(out, ctypes.c_int32)))
        return out

    def map_read_at(self, idx):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.empty(len(idx), dtype=np.int32)
        if len(idx):
            _check("map_read_at", self._lib.dct_map_read_at(
                _p(idx), len(idx), _p(out, ctypes.c_int32)))
        return out

    def read_cnt(self, off=0, length=None):
        length = self.space.size - off if length is None else length
        out = np.empty(length, dtype=np.uint16)
        _check("read_cnt", self._lib.dct_read_cnt(
            off, length, _p(out, ctypes.c_uint16)))
        return out


class GpuCoveringBackend(GpuBackend):
    """Homogeneous covering-code cell K_q(n,R)."""

    def __init__(self, q, n, R, **kw):
        super().__init__([q] * n, R, problem="hamming", **kw)
        self.q, self.n = q, n
