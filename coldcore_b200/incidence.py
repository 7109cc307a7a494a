"""Explicit-incidence cells on the B200: the Python side of plugin ABI 2.

Mirrors coldcore's ``src/coldcore/incidence_gpu.py`` (the ctypes binding of
``sparse_*``) with the same classes, arguments, methods and errors, over
this engine's ``libcoldcore_sparse.so``:

* :class:`GpuIncidenceBackend` — dense rows, ``incidence_gpu.py:98-283``;
* :class:`GpuWeightedIncidenceBackend` — weighted CSR rows,
  ``incidence_gpu.py:286-360``;
* :class:`IncidenceSpace` — the one-axis stand-in for a product space that
  the search core reads (``src/coldcore/incidence.py:48-86``).

Placement: ``cnt``, ``map`` and the query buffers are in HBM.  The
incidence goes to HBM when the cell fits the budget (``hbm_budget``, else
env ``COLDCORE_HBM_BUDGET``, default 160 GB of the B200's 180), else to
managed memory that prefers the host (``inc_mode=1``; reported as 2).
"""
import ctypes
import os

import numpy as np

from .gpu import _check

_libs = {}

_LL = ctypes.c_longlong
_I32P = ctypes.POINTER(ctypes.c_int32)
_I64P = ctypes.POINTER(ctypes.c_int64)
_LLP = ctypes.POINTER(_LL)

PLUGIN_NAME = "libcoldcore_sparse.so"
HBM_BUDGET = int(os.environ.get("COLDCORE_HBM_BUDGET", 160 * 10 ** 9))


def _bind(path):
    lib = ctypes.CDLL(path)
    if not hasattr(lib, "sparse_init") or lib.sparse_abi_version() != 2:
        raise RuntimeError(f"{path} is not a plugin of ABI 2")
    I = ctypes.c_int
    sig = {
        "sparse_abi_version": (I, []),
        "sparse_init": (I, [_LL, I, _LL, _I32P, I, I, _LLP, _LLP]),
        "sparse_init_csr": (I, [_LL, _LL, _LL, _I64P, _I32P, _I32P, _I32P, I,
                                I, _LLP, _LLP]),
        "sparse_free": (I, []),
        "sparse_set_mu": (I, [I]),
        "sparse_get_mu": (I, []),
        "sparse_inc_mode": (I, []),
        "sparse_is_csr": (I, []),
        "sparse_field": (I, [I]),
        "sparse_recount": (I, [_LLP, _LL]),
        "sparse_ball_update": (I, [_LLP, _LL, I]),
        "sparse_ball_gather": (I, [_LLP, _LL, I, _I32P]),
        "sparse_map_read_at": (I, [_LLP, _LL, _I32P]),
        "sparse_read_cnt": (I, [_LL, _LL, _I32P]),
        "sparse_map_max": (I, [_I32P]),
        "sparse_map_hist": (I, [I, ctypes.c_int32, _I32P]),
        "sparse_map_extract": (_LL, [ctypes.c_int32, _I64P, _I32P, I]),
        "sparse_count_eq": (_LL, [I]),
        "sparse_count_deficit": (_LL, []),
        "sparse_dev_bytes": (_LL, []),
        "sparse_host_bytes": (_LL, []),
        "sparse_b200_stream": (_LL, []),
        "sparse_b200_row_lanes": (I, []),
        "sparse_b200_init_design": (I, [I, I, I, I, I, _LLP, _LLP]),
        "sparse_b200_read_rows": (I, [_LL, _LL, _I32P]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(lib, name):
            if name.startswith("sparse_b200_"):
                continue                # this engine's additions only
            raise RuntimeError(f"{path} lacks {name}")
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def default_sparse_plugin_path():
    """``COLDCORE_SPARSE_PLUGIN_PATH`` if set, else the in-tree library."""
    env = os.environ.get("COLDCORE_SPARSE_PLUGIN_PATH")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        PLUGIN_NAME)


def load_sparse_plugin(path=None):
    """Load (and cache) the ABI-2 library; raises when it is missing."""
    path = os.path.abspath(path or default_sparse_plugin_path())
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(
                f"engine library not built: {path} "
                "(run `python -m coldcore_b200.build`)")
        _libs[path] = _bind(path)
    return _libs[path]


class IncidenceSpace:
    """One axis of ``size`` candidates standing in for a product space: a
    "word" is a one-digit row ``(idx,)`` (coldcore ``incidence.py:48-86``)."""

    def __init__(self, size):
        self.size = int(size)
        if self.size < 1:
            raise ValueError("IncidenceSpace needs at least one candidate")
        self.n = 1
        self.axes = [self.size]
        self.q = self.size
        self.pow_q = np.array([1], dtype=np.int64)

    def word_index(self, words):
        return np.asarray(words, dtype=np.int64).reshape(-1)

    def index_word(self, idx):
        return np.asarray(idx, dtype=np.int64).reshape(-1, 1)

    def all_words(self):
        return np.arange(self.size, dtype=np.int64)[:, None]

    def __repr__(self):
        return f"IncidenceSpace({self.size})"


def _ll(name, r):
    if r < 0:
        raise RuntimeError(f"{name} rc={r}")
    return int(r)


class GpuIncidenceBackend:
    """One dense explicit-incidence cell resident on the B200.

    inc: (n_cand, d) integer array, entries in [0, n_univ), uploaded at
    init; n_univ, mu, extract_cap as for coldcore's host backend;
    inc_mode None | 0 | 1 (None: by size against the HBM budget)."""

    indep_dist = None
    supports_hist = True

    def __init__(self, inc, n_univ, mu=1, extract_cap=1 << 22, inc_mode=None,
                 plugin_path=None, hbm_budget=None):
        inc = np.asarray(inc)
        if inc.ndim != 2 or not np.issubdtype(inc.dtype, np.integer):
            raise ValueError("inc must be a 2-D integer array (n_cand, d)")
        self.n_univ = int(n_univ)
        if not (1 <= self.n_univ <= np.iinfo(np.int32).max):
            raise ValueError("n_univ must be in 1..2^31-1 (int32 indices)")
        if inc.size and (int(inc.min()) < 0 or int(inc.max()) >= self.n_univ):
            raise ValueError("incidence entries must lie in [0, n_univ)")
        inc = np.ascontiguousarray(inc, dtype=np.int32)
        self.n_cand, self.d = (int(x) for x in inc.shape)
        self.mu = int(mu)
        if self.mu < 1:
            raise ValueError("mu must be >= 1")
        self.space = IncidenceSpace(self.n_cand)
        self.extract_cap = int(extract_cap)
        budget = HBM_BUDGET if hbm_budget is None else int(hbm_budget)
        inc_bytes = self.n_cand * self.d * 4
        other = (self.n_cand + self.n_univ) * 4 + self.extract_cap * 12
        if inc_mode is None:
            inc_mode = 0 if inc_bytes + other <= budget else 1
        if inc_mode not in (0, 1):
            raise ValueError("inc_mode must be 0 (HBM) or 1 (pinned host)")
        self._lib = lib = load_sparse_plugin(plugin_path)
        bd, bh = _LL(0), _LL(0)
        self._closed = True
        _check("sparse_init", lib.sparse_init(
            self.n_cand, self.d, self.n_univ, inc.ctypes.data_as(_I32P),
            int(inc_mode), self.extract_cap, ctypes.byref(bd),
            ctypes.byref(bh)))
        self._closed = False
        self._after_init(bd, bh)

    def _after_init(self, bd, bh):
        _check("sparse_set_mu", self._lib.sparse_set_mu(self.mu))
        self.inc_mode = int(self._lib.sparse_inc_mode())
        self.gpu_bytes = bd.value
        self.host_bytes = bh.value

    def close(self):
        if not self._closed:
            self._lib.sparse_free()
            self._closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _idx(idx):
        return np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64).ravel()

    # ---- the index set the search core walks (coldcore protocol.py:83-87)
    def word_index(self, words):
        return self.space.word_index(words)

    def index_word(self, idx):
        return self.space.index_word(idx)

    # ---- fields
    def recount(self, idx):
        idx = self._idx(idx)
        _check("sparse_recount", self._lib.sparse_recount(
            idx.ctypes.data_as(_LLP), len(idx)))

    def gain_map(self):
        _check("sparse_field(gain)", self._lib.sparse_field(0))

    def loss_map(self):
        _check("sparse_field(loss)", self._lib.sparse_field(1))

    # ---- incremental
    def ball_update(self, idx, delta):
        idx = self._idx(idx)
        _check("sparse_ball_update", self._lib.sparse_ball_update(
            idx.ctypes.data_as(_LLP), len(idx), int(delta)))

    def ball_gather(self, idx, target):
        """target is a coverage ROLE: 0 = deficient (cnt < mu), 1 =
        critical (1 <= cnt <= mu), anything else = literal cnt == target."""
        idx = self._idx(idx)
        out = np.empty(len(idx), dtype=np.int32)
        _check("sparse_ball_gather", self._lib.sparse_ball_gather(
            idx.ctypes.data_as(_LLP), len(idx), int(target),
            out.ctypes.data_as(_I32P)))
        return out

    # ---- queries
    def count_eq(self, target):
        return _ll("sparse_count_eq", self._lib.sparse_count_eq(int(target)))

    def uncovered(self):
        """Total deficit sum max(0, mu - cnt) (x uw when weighted)."""
        return _ll("sparse_count_deficit", self._lib.sparse_count_deficit())

    def map_max(self):
        v = ctypes.c_int32(0)
        _check("sparse_map_max", self._lib.sparse_map_max(ctypes.byref(v)))
        return int(v.value)

    def map_hist(self, nbins, vmax):
        out = np.zeros(nbins, dtype=np.int32)
        _check("sparse_map_hist", self._lib.sparse_map_hist(
            int(nbins), int(vmax), out.ctypes.data_as(_I32P)))
        return out

    def map_extract(self, thr, cap=None):
        cap = min(cap or self.extract_cap, self.extract_cap)
        oi = np.empty(max(cap, 1), dtype=np.int64)
        ov = np.empty(max(cap, 1), dtype=np.int32)
        found = _ll("sparse_map_extract", self._lib.sparse_map_extract(
            int(thr), oi.ctypes.data_as(_I64P), ov.ctypes.data_as(_I32P),
            cap))
        m = min(found, cap)
        return oi[:m], ov[:m], found

    def map_read_at(self, idx):
        idx = self._idx(idx)
        out = np.empty(len(idx), dtype=np.int32)
        _check("sparse_map_read_at", self._lib.sparse_map_read_at(
            idx.ctypes.data_as(_LLP), len(idx), out.ctypes.data_as(_I32P)))
        return out

    def map_all(self):
        return self.map_read_at(np.arange(self.n_cand, dtype=np.int64))

    def read_cnt(self, off=0, length=None):
        """A range of cnt over the universe, clipped like a numpy slice."""
        off = max(0, int(off))
        hi = (self.n_univ if length is None
              else min(self.n_univ, off + int(length)))
        n = max(0, hi - off)
        out = np.empty(n, dtype=np.int32)
        if n:
            _check("sparse_read_cnt", self._lib.sparse_read_cnt(
                off, n, out.ctypes.data_as(_I32P)))
        return out.astype(np.uint16)

    def deficient_universe(self, limit, rng=None):
        """Up to ``limit`` universe elements with cnt < mu (sorted, or a
        random subset when ``rng`` is given)."""
        cnt = np.empty(self.n_univ, dtype=np.int32)
        _check("sparse_read_cnt", self._lib.sparse_read_cnt(
            0, self.n_univ, cnt.ctypes.data_as(_I32P)))
        u = np.flatnonzero(cnt < self.mu)
        if rng is not None and len(u) > limit:
            u = np.sort(rng.choice(u, size=int(limit), replace=False))
        return u[:limit].astype(np.int64)

    def verify(self, idx):
        """Feasibility of ``idx`` from a fresh device recount (overwrites
        cnt)."""
        self.recount(idx)
        return self.uncovered() == 0

    def __repr__(self):
        return (f"{type(self).__name__}(n_cand={self.n_cand}, d={self.d}, "
                f"n_univ={self.n_univ}, mu={self.mu}, "
                f"inc_mode={getattr(self, 'inc_mode', None)})")


class GpuWeightedIncidenceBackend(GpuIncidenceBackend):
    """A weighted CSR cell (coldcore ``WeightedIncidenceBackend`` on the
    GPU): the exact weighted marginals, ``uncovered`` the weighted
    deficiency."""

    def __init__(self, indptr, indices, w, n_univ, uw=None, mu=1,
                 extract_cap=1 << 22, inc_mode=None, plugin_path=None,
                 hbm_budget=None):
        indptr = np.ascontiguousarray(indptr, dtype=np.int64).ravel()
        indices = np.ascontiguousarray(indices, dtype=np.int32).ravel()
        w = np.ascontiguousarray(w, dtype=np.int32).ravel()
        self.n_univ = int(n_univ)
        if not (1 <= self.n_univ <= np.iinfo(np.int32).max):
            raise ValueError("n_univ must be in 1..2^31-1 (int32 indices)")
        if len(indptr) < 2 or indptr[0] != 0 or indptr[-1] != len(indices) or (
                np.diff(indptr) < 0).any():
            raise ValueError("indptr is not a valid CSR offset array")
        if len(w) != len(indices) or (w < 1).any():
            raise ValueError("w must match indices and be >= 1")
        if indices.size and (int(indices.min()) < 0
                             or int(indices.max()) >= self.n_univ):
            raise ValueError("indices must lie in [0, n_univ)")
        uw = (np.ones(self.n_univ, dtype=np.int32) if uw is None
              else np.ascontiguousarray(uw, dtype=np.int32).ravel())
        if len(uw) != self.n_univ or (uw < 1).any():
            raise ValueError("uw must have n_univ entries >= 1")
        self.n_cand = len(indptr) - 1
        self.nnz = len(indices)
        self.d = None
        self.row_len = np.diff(indptr)
        self.mu = int(mu)
        if self.mu < 1:
            raise ValueError("mu must be >= 1")
        self.space = IncidenceSpace(self.n_cand)
        self.extract_cap = int(extract_cap)
        budget = HBM_BUDGET if hbm_budget is None else int(hbm_budget)
        inc_bytes = self.nnz * 8 + (self.n_cand + 1) * 8
        other = (self.n_cand + 2 * self.n_univ) * 4 + self.extract_cap * 12
        if inc_mode is None:
            inc_mode = 0 if inc_bytes + other <= budget else 1
        if inc_mode not in (0, 1):
            raise ValueError("inc_mode must be 0 (HBM) or 1 (pinned host)")
        self._lib = lib = load_sparse_plugin(plugin_path)
        bd, bh = _LL(0), _LL(0)
        self._closed = True
        _check("sparse_init_csr", lib.sparse_init_csr(
            self.n_cand, self.n_univ, self.nnz, indptr.ctypes.data_as(_I64P),
            indices.ctypes.data_as(_I32P), w.ctypes.data_as(_I32P),
            uw.ctypes.data_as(_I32P), int(inc_mode), self.extract_cap,
            ctypes.byref(bd), ctypes.byref(bh)))
        self._closed = False
        self._after_init(bd, bh)

    def __repr__(self):
        return (f"{type(self).__name__}(n_cand={self.n_cand}, nnz={self.nnz}, "
                f"n_univ={self.n_univ}, mu={self.mu}, "
                f"inc_mode={getattr(self, 'inc_mode', None)})")


# ------------------------------------------------ covering-design helpers
def _binomials(v, r):
    """C[a, b] for 0 <= a <= v, 0 <= b <= r, saturating at 2^62 (only
    ranks below C(v, k) are ever unranked, and those fit)."""
    C = np.zeros((v + 1, r + 1), dtype=np.int64)
    C[:, 0] = 1
    sat = np.int64(1) << 62
    for a in range(1, v + 1):
        C[a, 1:] = np.minimum(C[a - 1, :-1] + C[a - 1, 1:], sat)
    return C


def design_blocks(v, k, idx):
    """The k-subsets of {0..v-1} with colex ranks ``idx``: an (m, k)
    int64 array of sorted elements.  Position j from the top is the
    largest a with C(a, j+1) <= the remaining rank (the combinatorial
    number system; coldcore ``problems/covering_design.py:76-92``)."""
    idx = np.atleast_1d(np.asarray(idx, dtype=np.int64))
    C = _binomials(v, k)
    rem = idx.ravel().copy()
    out = np.empty((len(rem), k), dtype=np.int64)
    for j in range(k - 1, -1, -1):
        col = C[:, j + 1]
        a = np.searchsorted(col, rem, side="right") - 1
        out[:, j] = a
        rem -= col[a]
    return out.reshape(idx.shape + (k,))


def subset_ranks(S):
    """Colex ranks of sorted subsets (rows of S): sum_j C(s_j, j+1)."""
    S = np.asarray(S, dtype=np.int64)
    C = _binomials(int(S.max(initial=0)) + 1, S.shape[-1])
    return sum(C[S[..., j], j + 1] for j in range(S.shape[-1]))


def _shared(A, B):
    """|A n B| for broadcastable rows of distinct elements."""
    return (A[..., :, None] == B[..., None, :]).any(axis=-1).sum(axis=-1)


def block_distance(v, k, a, b):
    """k - |A n B| for blocks of colex ranks a, b (broadcast): the block
    metric of coldcore's covering designs (covering_design.py:206-219)."""
    A, B = design_blocks(v, k, a), design_blocks(v, k, b)
    return (k - _shared(A, B)).astype(np.int64)


def universe_distance(v, k, t, idx, univ):
    """t - |B n T| for every block in idx and t-subset in univ,
    (len(idx), len(univ)); 0 exactly when the block covers the t-subset
    (covering_design.py:221-229)."""
    B = design_blocks(v, k, np.atleast_1d(idx))[:, None, :]
    T = design_blocks(v, t, np.atleast_1d(univ))[None, :, :]
    return (t - _shared(B, T)).astype(np.int64)


def block_neighbours(v, k, idx, radius=1, m=None, rng=None):
    """Blocks at block distance ``radius`` from block ``idx``
    (covering_design.py:231-257): every one of the k (v-k) single swaps
    at radius 1 (``m`` of them sampled when given), and a sample of up to
    ``m`` (default 64) distinct ``radius``-fold swaps beyond that."""
    B = design_blocks(v, k, [int(idx)])[0]
    outside = np.setdiff1d(np.arange(v, dtype=np.int64), B)
    r = int(radius)
    if r < 1 or r > min(k, v - k):
        return np.zeros(0, dtype=np.int64)
    if r == 1:
        n = k * (v - k)
        rows = np.repeat(B[None, :], n, axis=0)
        rows[np.arange(n), np.repeat(np.arange(k), v - k)] = np.tile(outside,
                                                                     k)
        res = subset_ranks(np.sort(rows, axis=1))
        if m is not None and int(m) < n:
            rng = np.random.default_rng() if rng is None else rng
            res = rng.choice(res, size=int(m), replace=False)
        return res
    m = 64 if m is None else int(m)
    if m <= 0:
        return np.zeros(0, dtype=np.int64)
    rng = np.random.default_rng() if rng is None else rng
    drop = np.argsort(rng.random((m, k)), axis=1)[:, :r]
    add = np.argsort(rng.random((m, v - k)), axis=1)[:, :r]
    rows = np.repeat(B[None, :], m, axis=0)
    rows[np.arange(m)[:, None], drop] = outside[add]
    return np.unique(subset_ranks(np.sort(rows, axis=1)))


def candidates_covering(v, k, t, univ_idx):
    """Every block containing the t-subset ``univ_idx``, sorted: its
    C(v-t, k-t) completions (covering_design.py:259-269)."""
    from itertools import combinations
    T = design_blocks(v, t, [int(univ_idx)])[0]
    rest = np.setdiff1d(np.arange(v, dtype=np.int64), T)
    tails = np.array(list(combinations(rest.tolist(), k - t)),
                     dtype=np.int64).reshape(-1, k - t)
    rows = np.concatenate([np.repeat(T[None, :], len(tails), axis=0), tails],
                          axis=1)
    return np.sort(subset_ranks(np.sort(rows, axis=1)))


class GpuCoveringDesignBackend(GpuIncidenceBackend):
    """A covering design C(v,k,t) (mu-fold) whose incidence is built on the
    B200 (``sparse_b200_init_design``), in the layout of coldcore's
    ``problems.covering_design.build_incidence``: candidates are the
    k-subsets of {0..v-1} by colex rank, universe elements the t-subsets,
    row c the ranks of block c's t-subsets.  The host never holds the
    C(v,k) x C(k,t) matrix."""

    def __init__(self, v, k, t, mu=1, extract_cap=1 << 22, inc_mode=0,
                 plugin_path=None):
        from math import comb
        self.v, self.k, self.t = int(v), int(k), int(t)
        if not (1 <= self.t <= self.k <= self.v):
            raise ValueError("need 1 <= t <= k <= v")
        self.mu = int(mu)
        if self.mu < 1:
            raise ValueError("mu must be >= 1")
        if inc_mode not in (0, 1):
            raise ValueError("inc_mode must be 0 (HBM) or 1 (pinned host)")
        self.n_cand = comb(self.v, self.k)
        self.d = comb(self.k, self.t)
        self.n_univ = comb(self.v, self.t)
        self.space = IncidenceSpace(self.n_cand)
        self.extract_cap = int(extract_cap)
        self._lib = lib = load_sparse_plugin(plugin_path)
        if not hasattr(lib, "sparse_b200_init_design"):
            raise RuntimeError("the loaded ABI-2 library builds no designs")
        bd, bh = _LL(0), _LL(0)
        self._closed = True
        _check("sparse_b200_init_design", lib.sparse_b200_init_design(
            self.v, self.k, self.t, int(inc_mode), self.extract_cap,
            ctypes.byref(bd), ctypes.byref(bh)))
        self._closed = False
        self._after_init(bd, bh)

    # ---- locality hooks the search core uses when present (coldcore
    # problems/covering_design.py:206-229): the block metric
    @property
    def indep_dist(self):
        """Blocks farther apart than k - t share no t-subset."""
        return self.k - self.t

    def distance(self, a, b):
        return block_distance(self.v, self.k, a, b)

    def universe_distance(self, idx, univ):
        return universe_distance(self.v, self.k, self.t, idx, univ)

    def rank_block(self, idx):
        """Candidate indices -> (m, k) sorted 0-based blocks."""
        return design_blocks(self.v, self.k, np.ravel(idx))

    def block_rank(self, blocks):
        """(m, k) 0-based blocks (any element order) -> candidates."""
        S = np.sort(np.atleast_2d(np.asarray(blocks, dtype=np.int64)), axis=1)
        if S.shape[1] != self.k or (S.size and (S.min() < 0
                                                or S.max() >= self.v)):
            raise ValueError(f"blocks must be (m, {self.k}) with elements "
                             f"in 0..{self.v - 1}")
        return subset_ranks(S)

    def neighbours(self, idx, radius=1, m=None, rng=None):
        return block_neighbours(self.v, self.k, idx, radius, m, rng)

    def candidates_covering(self, univ_idx):
        return candidates_covering(self.v, self.k, self.t, univ_idx)

    def rows(self, c0=0, n=None):
        """Incidence rows [c0, c0 + n) as an (n, d) int32 array."""
        n = self.n_cand - c0 if n is None else int(n)
        out = np.empty((n, self.d), dtype=np.int32)
        _check("sparse_b200_read_rows", self._lib.sparse_b200_read_rows(
            int(c0), n, out.ctypes.data_as(_I32P)))
        return out

    def __repr__(self):
        return (f"{type(self).__name__}(C({self.v},{self.k},{self.t}), "
                f"mu={self.mu}, n_cand={self.n_cand}, d={self.d}, "
                f"n_univ={self.n_univ})")


def CoveringDesignBackend(v, k, t, mu=1, device="gpu", **kw):
    """coldcore's constructor name for a design cell
    (``problems/covering_design.py:174-191``).  This engine serves the
    device form only: ``device="gpu"`` gives a
    :class:`GpuCoveringDesignBackend`; the reference's host forms ("cpu",
    "ref") are its numpy backends, which this package does not ship."""
    if device != "gpu":
        raise ValueError(f"device {device!r}: this engine has the GPU form "
                         "only (the host forms are coldcore's own numpy "
                         "backends)")
    kw.pop("keep_host", None)
    return GpuCoveringDesignBackend(v, k, t, mu=mu, **kw)
