"""ctypes wrapper of the C restatement of the axis DP (``dp.c``).

Test infrastructure and the timed CPU baseline only.  ``build()`` compiles
``dp.c`` with gcc (-O3, OpenMP) into ``oracle/cport/libccport.so``.
"""
import ctypes
import os
import subprocess

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
    return _lib


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
