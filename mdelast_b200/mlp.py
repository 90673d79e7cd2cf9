"""The warm-start network on the device, through the C-ABI (mdelast_mlp_* of
include/mdelast.h): a small FP32 MLP with GELU hidden layers trained by the library's own
forward, backward and Adam kernels."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                            "libmdelast_cuda.so")
        L = C.CDLL(path)
        P, F = C.c_void_p, C.POINTER(C.c_float)
        L.mdelast_mlp_create.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.c_uint64, C.c_int32,
                                         C.POINTER(P)]
        L.mdelast_mlp_destroy.argtypes = [P]
        L.mdelast_mlp_destroy.restype = None
        L.mdelast_mlp_n_params.argtypes = [P, C.POINTER(C.c_int64)]
        L.mdelast_mlp_get_params.argtypes = [P, F]
        L.mdelast_mlp_set_params.argtypes = [P, F]
        L.mdelast_mlp_forward.argtypes = [P, F, C.c_int32, F]
        L.mdelast_mlp_gradients.argtypes = [P, F, F, C.c_int32, F, F]
        L.mdelast_mlp_train.argtypes = [P, F, F, C.c_int32, C.c_int32, C.c_float, F]
        L.mdelast_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().mdelast_last_error().decode())


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """Fully connected network of the given widths (inputs, hidden..., outputs)."""

    def __init__(self, widths, seed=0, device=0):
        self.widths = [int(w) for w in widths]
        w = (C.c_int32 * len(self.widths))(*self.widths)
        h = C.c_void_p()
        _check(lib().mdelast_mlp_create(len(self.widths) - 1, w, seed, device, C.byref(h)))
        self._h = h
        n = C.c_int64()
        _check(lib().mdelast_mlp_n_params(self._h, C.byref(n)))
        self.n_params = int(n.value)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.mdelast_mlp_destroy(self._h)
            self._h = None

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().mdelast_mlp_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    @params.setter
    def params(self, p):
        p, ptr = _f(p)
        assert p.size == self.n_params
        _check(lib().mdelast_mlp_set_params(self._h, ptr))

    def __call__(self, x) -> np.ndarray:
        x, px = _f(x)
        n = x.shape[0]
        y = np.zeros((n, self.widths[-1]), dtype=np.float32)
        _check(lib().mdelast_mlp_forward(self._h, px, n, y.ctypes.data_as(C.POINTER(C.c_float))))
        return y

    def gradients(self, x, y):
        x, px = _f(x)
        y, py = _f(y)
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().mdelast_mlp_gradients(self._h, px, py, x.shape[0],
                                           loss.ctypes.data_as(C.POINTER(C.c_float)),
                                           g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss[0]), g

    def train(self, x, y, steps, lr=1e-3) -> float:
        x, px = _f(x)
        y, py = _f(y)
        loss = np.zeros(1, dtype=np.float32)
        _check(lib().mdelast_mlp_train(self._h, px, py, x.shape[0], int(steps), float(lr),
                                       loss.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss[0])
