"""Host side of the calibration surrogate (include/dem_surrogate.h,
libdem_surrogate.so): a tensor-core MLP from contact parameters
(sliding friction, rolling friction, restitution, PSD width) to heap
responses (angle of repose, packing fraction, settle time).

There is no CPU fallback: constructing a Surrogate fails if the library is
missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdem_surrogate.so")
NI, NH, NO = 4, 256, 3
NPARAMS = 133635

_pf = C.POINTER(C.c_float)
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        sig = {
            "dem_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
            "dem_mlp_set_normalisation": (C.c_int, [C.c_void_p, _pf, _pf, _pf, _pf]),
            "dem_mlp_get_params": (C.c_int, [C.c_void_p, _pf]),
            "dem_mlp_set_params": (C.c_int, [C.c_void_p, _pf]),
            "dem_mlp_forward": (C.c_int, [C.c_void_p, _pf, C.c_int, _pf]),
            "dem_mlp_gradients": (C.c_int, [C.c_void_p, _pf, _pf, C.c_int, _pf, _pf]),
            "dem_mlp_train_step": (C.c_int, [C.c_void_p, _pf, _pf, C.c_int, C.c_float, _pf]),
            "dem_mlp_time_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _pf]),
            "dem_mlp_last_error": (C.c_char_p, [C.c_void_p]),
            "dem_mlp_destroy": (None, [C.c_void_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _f32(a, shape=None):
    out = np.ascontiguousarray(a, dtype=np.float32)
    return out.reshape(shape) if shape is not None else out


def _p(a):
    return a.ctypes.data_as(_pf)


class SurrogateError(RuntimeError):
    pass


class Surrogate:
    """One network on one GPU; batches of up to `capacity` rows."""

    def __init__(self, capacity: int = 65536, seed: int = 0, device: int = 0):
        self._h = C.c_void_p()
        rc = lib().dem_mlp_create(device, capacity, seed, C.byref(self._h))
        if rc:
            raise SurrogateError(f"dem_mlp_create failed ({rc})")
        self.capacity = capacity
        self.norm = (np.zeros(NI), np.ones(NI), np.zeros(NO), np.ones(NO))

    def _check(self, rc):
        if rc:
            raise SurrogateError(f"{rc}: {lib().dem_mlp_last_error(self._h).decode()}")

    def close(self):
        if self._h:
            lib().dem_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_normalisation(self, in_mean, in_std, out_mean, out_std):
        a = [_f32(v) for v in (in_mean, in_std, out_mean, out_std)]
        self._check(lib().dem_mlp_set_normalisation(self._h, *[_p(v) for v in a]))
        self.norm = tuple(np.asarray(v, np.float64) for v in a)

    def fit_normalisation(self, x, y):
        x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
        self.set_normalisation(x.mean(0), np.maximum(x.std(0), 1e-6), y.mean(0), np.maximum(y.std(0), 1e-6))

    def params(self) -> np.ndarray:
        out = np.zeros(NPARAMS, np.float32)
        self._check(lib().dem_mlp_get_params(self._h, _p(out)))
        return out

    def set_params(self, p):
        p = _f32(p)
        self._check(lib().dem_mlp_set_params(self._h, _p(p)))

    def predict(self, x) -> np.ndarray:
        x = _f32(x, (-1, NI))
        out = np.zeros((len(x), NO), np.float32)
        for a in range(0, len(x), self.capacity):
            b = min(len(x), a + self.capacity)
            xs = np.ascontiguousarray(x[a:b])
            ys = np.zeros((b - a, NO), np.float32)
            self._check(lib().dem_mlp_forward(self._h, _p(xs), b - a, _p(ys)))
            out[a:b] = ys
        return out

    def time_forward(self, n: int, reps: int = 20) -> float:
        """Device milliseconds of one forward pass of n rows already on the device."""
        ms = C.c_float(0)
        self._check(lib().dem_mlp_time_forward(self._h, n, reps, C.byref(ms)))
        return float(ms.value)

    def gradients(self, x, t):
        x, t = _f32(x, (-1, NI)), _f32(t, (-1, NO))
        loss = C.c_float(0)
        g = np.zeros(NPARAMS, np.float32)
        self._check(lib().dem_mlp_gradients(self._h, _p(x), _p(t), len(x), C.byref(loss), _p(g)))
        return float(loss.value), g

    def train_step(self, x, t, lr: float = 1e-3) -> float:
        x, t = _f32(x, (-1, NI)), _f32(t, (-1, NO))
        loss = C.c_float(0)
        self._check(lib().dem_mlp_train_step(self._h, _p(x), _p(t), len(x), lr, C.byref(loss)))
        return float(loss.value)

    def fit(self, x, y, epochs: int = 200, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> list:
        """Adam over shuffled mini-batches; returns the mean loss per epoch."""
        x, y = _f32(x, (-1, NI)), _f32(y, (-1, NO))
        rng = np.random.default_rng(seed)
        hist = []
        for _ in range(epochs):
            order = rng.permutation(len(x))
            losses = []
            for a in range(0, len(x), batch):
                idx = order[a:a + batch]
                losses.append(self.train_step(x[idx], y[idx], lr))
            hist.append(float(np.mean(losses)))
        return hist
