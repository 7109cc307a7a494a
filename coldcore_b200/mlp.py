"""The learned ruin proposal's scorer on the GPU: a 32-128-128-1 ReLU MLP
trained and evaluated by the engine's own BF16 / FP32-accumulate kernels
(``dct_mlp_*``, ``csrc/mlp.cu``)."""
import ctypes

import numpy as np

from .gpu import _check, load_plugin

N_IN, N_HID = 32, 128
N_PARAMS = N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID + 1

_F = ctypes.POINTER(ctypes.c_float)


def _bind(lib):
    if getattr(lib, "_mlp_bound", False):
        return lib
    LL, I = ctypes.c_longlong, ctypes.c_int
    lib.dct_mlp_create.restype = LL
    lib.dct_mlp_create.argtypes = [ctypes.c_ulonglong]
    lib.dct_mlp_params.restype = I
    lib.dct_mlp_params.argtypes = [LL, _F, _F]
    lib.dct_mlp_grad.restype = I
    lib.dct_mlp_grad.argtypes = [LL, _F, _F, I, _F]
    lib.dct_mlp_train.restype = I
    lib.dct_mlp_train.argtypes = [LL, _F, _F, I, I, I, ctypes.c_float,
                                  ctypes.c_ulonglong]
    lib.dct_mlp_predict.restype = I
    lib.dct_mlp_predict.argtypes = [LL, _F, I, _F]
    lib.dct_mlp_free.restype = I
    lib.dct_mlp_free.argtypes = [LL]
    lib._mlp_bound = True
    return lib


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


class GpuMlp:
    def __init__(self, seed=0, plugin_path=None):
        self._lib = _bind(load_plugin(plugin_path))
        self.h = int(self._lib.dct_mlp_create(seed))
        if self.h <= 0:
            raise RuntimeError("dct_mlp_create failed")

    def params(self):
        out = np.empty(N_PARAMS, dtype=np.float32)
        n = self._lib.dct_mlp_params(self.h, out.ctypes.data_as(_F), None)
        if n != N_PARAMS:
            _check("mlp_params", -1)
        return out

    def set_params(self, p):
        p = _f32(p)
        assert p.size == N_PARAMS
        n = self._lib.dct_mlp_params(self.h, None, p.ctypes.data_as(_F))
        if n != N_PARAMS:
            _check("mlp_params", -1)

    def grad(self, X, T):
        X, T = _f32(X, (-1, N_IN)), _f32(T)
        out = np.empty(N_PARAMS, dtype=np.float32)
        n = self._lib.dct_mlp_grad(self.h, X.ctypes.data_as(_F),
                                   T.ctypes.data_as(_F), len(T),
                                   out.ctypes.data_as(_F))
        if n != N_PARAMS:
            _check("mlp_grad", n if n < 0 else -1)
        return out

    def train(self, X, T, epochs=10, batch=512, lr=1e-3, seed=0):
        X, T = _f32(X, (-1, N_IN)), _f32(T)
        _check("mlp_train", self._lib.dct_mlp_train(
            self.h, X.ctypes.data_as(_F), T.ctypes.data_as(_F), len(T),
            int(epochs), int(batch), float(lr), int(seed)))

    def predict(self, X):
        X = _f32(X, (-1, N_IN))
        out = np.empty(len(X), dtype=np.float32)
        _check("mlp_predict", self._lib.dct_mlp_predict(
            self.h, X.ctypes.data_as(_F), len(X), out.ctypes.data_as(_F)))
        return out

    def close(self):
        if self.h > 0:
            self._lib.dct_mlp_free(self.h)
            self.h = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
