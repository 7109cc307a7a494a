"""ctypes wrapper of the C restatement of the axis DP (``dp.c``).

Test infrastructure and the timed CPU baseline only.  ``build()`` compiles
``dp.c`` with gcc (-O3, OpenMP) into ``oracle/cport/libccport.so``.
"""
import ctypes
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "dp.c")
LIB = os.path.join(HERE, "libccport.so")
PROBLEMS = {"hamming": 0, "torus_linf": 1, "lee": 2, "grid_linf": 3}
_lib = None


def build():
    if (not os.path.exists(LIB)
            or os.path.getmtime(LIB) < os.path.getmtime(SRC)):
        subprocess.run(["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC",
                        "-shared", "-o", LIB, SRC], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        _lib.cc_transform.argtypes = [ctypes.c_int, ctypes.c_int, P,
                                      ctypes.c_int, P, P, P]
        _lib.cc_seed_pred.argtypes = [P, ctypes.c_longlong, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, P]
        _lib.cc_seed_code.argtypes = [P, ctypes.c_longlong, ctypes.c_longlong,
                                      P]
        _lib.cc_inc_field.argtypes = [P, ctypes.c_longlong, ctypes.c_int, P,
                                      ctypes.c_int, ctypes.c_int, P]
    return _lib


def inc_field(inc, cnt, target, mu=1, out=None):
    """Field over dense incidence rows on the host threads (the reference's
    SparseIncidenceBackend field, incidence.py:160-197)."""
    inc = np.ascontiguousarray(inc, dtype=np.int32)
    cnt = np.ascontiguousarray(cnt, dtype=np.int32)
    out = np.empty(len(inc), dtype=np.int32) if out is None else out
    lib().cc_inc_field(inc.ctypes.data, len(inc), inc.shape[1],
                       cnt.ctypes.data, int(target), int(mu), out.ctypes.data)
    return out


class CPortCell:
    """One cell on the host cores: recount / gain / loss as the reference's
    CPU backend computes them."""

    def __init__(self, axes, R, problem="hamming", mu=1):
        self.axes = np.asarray(axes, dtype=np.int32)
        self.n, self.R, self.mu = len(axes), int(R), int(mu)
        self.pid = PROBLEMS[problem]
        self.size = int(np.prod(self.axes.astype(np.int64)))
        nl = R + 1 if problem in ("hamming", "lee") else 1
        self.A = np.zeros((nl, self.size), dtype=np.int32)
        self.cnt = np.zeros(self.size, dtype=np.uint16)
        self.map = np.zeros(self.size, dtype=np.int32)
        self._l = lib()

    def _run(self, out_map, out_cnt):
        self._l.cc_transform(self.pid, self.n, self.axes.ctypes.data, self.R,
                             self.A.ctypes.data,
                             out_map.ctypes.data if out_map is not None else None,
                             out_cnt.ctypes.data if out_cnt is not None else None)

    def recount(self, code):
        code = np.ascontiguousarray(code, dtype=np.int64)
        self._l.cc_seed_code(code.ctypes.data, len(code), self.size,
                             self.A.ctypes.data)
        self._run(None, self.cnt)

    def _pred(self, mode, target):
        self._l.cc_seed_pred(self.cnt.ctypes.data, self.size, mode, target,
                             self.mu, self.A.ctypes.data)

    def gain_map(self):
        self._pred(1, 0)
        self._run(self.map, None)

    def loss_map(self):
        self._pred(2, 0)
        self._run(self.map, None)


# ------------------------------------------------------------ campaign pool
def _one_thread():
    """Pool initializer: one OpenMP thread per worker process (set before
    the worker first loads the library)."""
    os.environ["OMP_NUM_THREADS"] = "1"


def _warm(seconds):
    lib()
    time.sleep(seconds)
    return os.getpid()


def cell_step(item):
    """One campaign step of one cell on one host core: recount, deficit,
    gain map and its maximum, loss map and its maximum.  Returns seconds."""
    problem, axes, R, code = item
    t0 = time.perf_counter()
    c = CPortCell(list(axes), R, problem)
    c.recount(code)
    int(np.maximum(c.mu - c.cnt.astype(np.int64), 0).sum())
    c.gain_map()
    int(c.map.max())
    c.loss_map()
    int(c.map.max())
    return time.perf_counter() - t0


def campaign_rate(cells, workers=None):
    """A campaign step over `cells` ((problem, axes, R, code) tuples) on a
    pool of single-threaded worker processes, the way coldcore's campaign
    runs one cell per process: largest cells first, the pool started (and
    every worker's library loaded) outside the timed region.  Returns
    (instances/s, wall seconds, summed cell seconds, workers)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    workers = workers or os.cpu_count() or 1
    order = sorted(cells, key=lambda c: -int(np.prod(c[1])))
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn"),
                             initializer=_one_thread) as ex:
        list(ex.map(_warm, [0.3] * workers))
        t0 = time.perf_counter()
        per = list(ex.map(cell_step, order, chunksize=1))
        wall = time.perf_counter() - t0
    return len(cells) / wall, wall, float(sum(per)), workers
