"""Batched campaign engine: many independent cells, one persistent launch.

The reference's campaign runs one process per cell (coldcore
``src/coldcore/campaign.py:186-221``) because its plugin ABI is a
per-process singleton.  ``BatchEngine`` holds many cells in one device
arena and computes, for every cell, cnt from its code, the deficit
(uncovered count at mu = 1), the gain map and its maximum and the loss map
and its maximum, in one persistent kernel launch replayed from a CUDA graph
(``dct_batch_*`` in ``include/coldcore_b200/plugin.h``).
"""
import ctypes

import numpy as np

from .gpu import _check, load_plugin
from .patterns import PROBLEM_IDS

_LL = ctypes.c_longlong


def _bind(lib):
    if getattr(lib, "_batch_bound", False):
        return lib
    I = ctypes.c_int
    lib.dct_batch_create.restype = _LL
    lib.dct_batch_create.argtypes = []
    lib.dct_batch_add.restype = I
    lib.dct_batch_add.argtypes = [_LL, I, I, ctypes.POINTER(I), I, I,
                                  ctypes.POINTER(_LL), I]
    lib.dct_batch_build.restype = I
    lib.dct_batch_build.argtypes = [_LL, I]
    lib.dct_batch_run.restype = I
    lib.dct_batch_run.argtypes = [_LL, I]
    lib.dct_batch_read.restype = I
    lib.dct_batch_read.argtypes = [_LL, I, I, _LL, _LL, ctypes.c_void_p]
    lib.dct_batch_scalars.restype = I
    lib.dct_batch_scalars.argtypes = [_LL, ctypes.POINTER(_LL), I]
    lib.dct_batch_info.restype = I
    lib.dct_batch_info.argtypes = [_LL, ctypes.POINTER(_LL), I]
    lib.dct_batch_free.restype = I
    lib.dct_batch_free.argtypes = [_LL]
    I32P = ctypes.POINTER(ctypes.c_int32)
    lib.dct_batch_set_code.restype = I
    lib.dct_batch_set_code.argtypes = [_LL, I, ctypes.POINTER(_LL), I]
    lib.dct_batch_set_table.restype = I
    lib.dct_batch_set_table.argtypes = [_LL, I, I32P, I, _LL]
    lib.dct_batch_update.restype = I
    lib.dct_batch_update.argtypes = [_LL, I, ctypes.POINTER(_LL), I, I]
    lib.dct_batch_gather.restype = I
    lib.dct_batch_gather.argtypes = [_LL, I, ctypes.POINTER(_LL), I, I, I32P]
    lib.dct_batch_extract.restype = _LL
    lib.dct_batch_extract.argtypes = [_LL, I, I, ctypes.c_int32,
                                      ctypes.POINTER(_LL), I32P, I]
    lib.dct_batch_count.restype = _LL
    lib.dct_batch_count.argtypes = [_LL, I, I, I]
    lib.dct_batch_read_at.restype = I
    lib.dct_batch_read_at.argtypes = [_LL, I, I, ctypes.POINTER(_LL), I,
                                      I32P]
    IP = ctypes.POINTER(I)
    lib.dct_batch_greedy.restype = I
    lib.dct_batch_greedy.argtypes = [_LL, IP, I, IP, ctypes.POINTER(_LL), I,
                                     IP, ctypes.POINTER(_LL)]
    lib._batch_bound = True
    return lib


class BatchEngine:
    """Cells are added, then ``build()`` allocates and schedules them (tile
    size autotuned unless ``tile_kb`` is given); each ``run()`` recomputes
    every cell's fields."""

    def __init__(self, plugin_path=None):
        self._lib = _bind(load_plugin(plugin_path))
        self.h = int(self._lib.dct_batch_create())
        if self.h <= 0:
            raise RuntimeError("dct_batch_create failed")
        self.cells = []

    def add(self, problem, axes, R, code, mu=1):
        axes = [int(a) for a in axes]
        code = np.ascontiguousarray(np.atleast_1d(code), dtype=np.int64)
        ax = (ctypes.c_int * len(axes))(*axes)
        rc = self._lib.dct_batch_add(
            self.h, PROBLEM_IDS[problem], len(axes), ax, int(R), int(mu),
            code.ctypes.data_as(ctypes.POINTER(_LL)), len(code))
        if rc < 0:
            _check("batch_add", rc)
        self.cells.append((problem, tuple(axes), int(R), int(mu)))
        return rc

    def build(self, tile_kb=0):
        _check("batch_build", self._lib.dct_batch_build(self.h, int(tile_kb)))

    def run(self, mode=0):
        _check("batch_run", self._lib.dct_batch_run(self.h, int(mode)))

    def run_rc(self, mode):
        return int(self._lib.dct_batch_run(self.h, int(mode)))

    def read(self, cell, field):
        size = int(np.prod(self.cells[cell][1]))
        out = np.empty(size, dtype=np.uint16 if field == 0 else np.int32)
        _check("batch_read", self._lib.dct_batch_read(
            self.h, int(cell), int(field), 0, size,
            out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def cnt(self, cell):
        return self.read(cell, 0)

    def gain(self, cell):
        return self.read(cell, 1)

    def loss(self, cell):
        return self.read(cell, 2)

    def scalars(self):
        """(cells, 3) int64: deficit, gain maximum, loss maximum."""
        buf = np.zeros(3 * len(self.cells), dtype=np.int64)
        n = self._lib.dct_batch_scalars(
            self.h, buf.ctypes.data_as(ctypes.POINTER(_LL)), len(buf))
        if n < 0:
            _check("batch_scalars", n)
        return buf.reshape(-1, 3)

    # ---------------- per cell, between runs
    def set_code(self, cell, code):
        """Replace a cell's code; the next run recounts from it."""
        code = np.ascontiguousarray(np.atleast_1d(code), dtype=np.int64)
        _check("batch_set_code", self._lib.dct_batch_set_code(
            self.h, int(cell), code.ctypes.data_as(ctypes.POINTER(_LL)),
            len(code)))

    def set_table(self, cell, tbl):
        """The cell's support table: (len, slots) int32 slots as
        ``patterns.wide_table`` builds them."""
        tbl = np.ascontiguousarray(tbl, dtype=np.int32)
        _check("batch_set_table", self._lib.dct_batch_set_table(
            self.h, int(cell),
            tbl.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            tbl.shape[1], tbl.shape[0]))

    def update(self, cell, words, delta):
        words = np.ascontiguousarray(np.atleast_1d(words), dtype=np.int64)
        for lo in range(0, len(words), 1 << 16):
            part = np.ascontiguousarray(words[lo:lo + (1 << 16)])
            _check("batch_update", self._lib.dct_batch_update(
                self.h, int(cell), part.ctypes.data_as(ctypes.POINTER(_LL)),
                len(part), int(delta)))

    def gather(self, cell, words, role):
        words = np.ascontiguousarray(np.atleast_1d(words), dtype=np.int64)
        out = np.zeros(len(words), dtype=np.int32)
        for lo in range(0, len(words), 1 << 16):
            part = np.ascontiguousarray(words[lo:lo + (1 << 16)])
            o = np.zeros(len(part), dtype=np.int32)
            _check("batch_gather", self._lib.dct_batch_gather(
                self.h, int(cell), part.ctypes.data_as(ctypes.POINTER(_LL)),
                len(part), int(role),
                o.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
            out[lo:lo + len(part)] = o
        return out

    def extract(self, cell, field, thr, cap):
        idx = np.zeros(max(1, cap), dtype=np.int64)
        val = np.zeros(max(1, cap), dtype=np.int32)
        found = int(self._lib.dct_batch_extract(
            self.h, int(cell), int(field), int(thr),
            idx.ctypes.data_as(ctypes.POINTER(_LL)),
            val.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(cap)))
        if found < 0:
            _check("batch_extract", found)
        n = min(found, cap)
        return idx[:n].copy(), val[:n].copy(), found

    def greedy(self, cells, max_add):
        """Exact greedy on several cells at once (dct_batch_greedy):
        returns per cell (placed words in order, deficit left)."""
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        adds = np.ascontiguousarray(max_add, dtype=np.int32)
        n = len(cells)
        cap = max(1, int(adds.max()) if n else 1)
        placed = np.zeros(n * cap, dtype=np.int64)
        nplaced = np.zeros(n, dtype=np.int32)
        deficit = np.zeros(n, dtype=np.int64)
        IP = ctypes.POINTER(ctypes.c_int)
        _check("batch_greedy", self._lib.dct_batch_greedy(
            self.h, cells.ctypes.data_as(IP), n, adds.ctypes.data_as(IP),
            placed.ctypes.data_as(ctypes.POINTER(_LL)), cap,
            nplaced.ctypes.data_as(IP),
            deficit.ctypes.data_as(ctypes.POINTER(_LL))))
        return [(placed[k * cap:k * cap + nplaced[k]].copy(), int(deficit[k]))
                for k in range(n)]

    def count(self, cell, mode, target=0):
        r = int(self._lib.dct_batch_count(self.h, int(cell), int(mode),
                                          int(target)))
        if r < 0:
            _check("batch_count", r)
        return r

    def read_at(self, cell, field, idx):
        idx = np.ascontiguousarray(np.atleast_1d(idx), dtype=np.int64)
        out = np.zeros(len(idx), dtype=np.int32)
        for lo in range(0, len(idx), 1 << 16):
            part = np.ascontiguousarray(idx[lo:lo + (1 << 16)])
            o = np.zeros(len(part), dtype=np.int32)
            _check("batch_read_at", self._lib.dct_batch_read_at(
                self.h, int(cell), int(field),
                part.ctypes.data_as(ctypes.POINTER(_LL)), len(part),
                o.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
            out[lo:lo + len(part)] = o
        return out

    def read_range(self, cell, field, off, length):
        out = np.empty(length, dtype=np.uint16 if field == 0 else np.int32)
        _check("batch_read", self._lib.dct_batch_read(
            self.h, int(cell), int(field), int(off), int(length),
            out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def info(self):
        """Plan facts of the built batch; ``step_bytes`` is one step's
        algorithmic HBM bytes (every launch's source read once and its
        destination written once, plus the deficit count and the two map
        maxima), ``big_bytes`` those of the cells with their own launches."""
        buf = (_LL * 8)()
        _check("batch_info", 0 if self._lib.dct_batch_info(self.h, buf, 8) == 8
               else -1)
        keys = ("cells", "passes", "items", "tile_kb", "grid", "tuned_us",
                "step_bytes", "big_bytes")
        return {k: int(v) for k, v in zip(keys, buf)}

    def close(self):
        if self.h > 0:
            self._lib.dct_batch_free(self.h)
            self.h = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
