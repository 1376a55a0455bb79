"""The learned revaluation surrogate: a 16 -> 128 -> 128 -> 128 -> 1 SiLU perceptron with BF16 weights and
FP32 accumulation, trained and evaluated on the GPU's tensor cores by this package's kernels (zk_surrogate_*).

Parameters flatten as W1[128][16] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4 (PARAMS floats);
the scaling as input mean[16], input 1/sd[16], target mean, target sd.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._native import check, lib

IN, HID = 16, 128
PARAMS = HID * IN + HID + 2 * (HID * HID + HID) + HID + 1
LAYOUT = (("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)),
          ("w4", (HID,)), ("b4", (1,)))


def unflatten(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n]).reshape(shape)
        o += n
    return out


class Surrogate:
    def __init__(self, ctx, seed: int = 1):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().zk_surrogate_create(ctx.handle, seed, C.byref(h)), ctx.handle)
        self.handle = h

    def close(self) -> None:
        if self.handle:
            lib().zk_surrogate_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _xy(x, y=None):
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 2 or x.shape[1] != IN:
            raise ValueError(f"inputs must be [n][{IN}]")
        if y is not None:
            y = np.ascontiguousarray(y, np.float32).reshape(-1)
            if y.size != x.shape[0]:
                raise ValueError("one target per input row")
        return x, y

    def train(self, x, y, epochs: int = 10, batch: int = 8192, lr: float = 1e-3, weight_decay: float = 0.0) -> np.ndarray:
        """Adam over `epochs` passes; returns the mean squared error (standardised units) of every pass."""
        x, y = self._xy(x, y)
        losses = np.zeros(max(epochs, 1), np.float32)
        check(lib().zk_surrogate_train(self.handle, x.ctypes.data, y.ctypes.data, x.shape[0], epochs, batch, lr, weight_decay,
                                       losses.ctypes.data), self.ctx.handle)
        return losses[:epochs]

    def predict(self, x) -> np.ndarray:
        x, _ = self._xy(x)
        out = np.zeros(x.shape[0], np.float32)
        check(lib().zk_surrogate_predict(self.handle, x.ctypes.data, x.shape[0], out.ctypes.data), self.ctx.handle)
        return out

    def gradients(self, x, y):
        """(loss, gradient of the mean squared error over all rows) at the current parameters."""
        x, y = self._xy(x, y)
        g = np.zeros(PARAMS, np.float32)
        loss = C.c_float()
        check(lib().zk_surrogate_gradients(self.handle, x.ctypes.data, y.ctypes.data, x.shape[0], C.byref(loss), g.ctypes.data),
              self.ctx.handle)
        return float(loss.value), g

    def params(self):
        p = np.zeros(PARAMS, np.float32)
        sc = np.zeros(34, np.float32)
        check(lib().zk_surrogate_params(self.handle, p.ctypes.data, None, sc.ctypes.data, None), self.ctx.handle)
        return p, sc

    def set_params(self, p: Optional[np.ndarray] = None, scaling: Optional[np.ndarray] = None) -> None:
        pp = None if p is None else np.ascontiguousarray(p, np.float32)
        ss = None if scaling is None else np.ascontiguousarray(scaling, np.float32)
        check(lib().zk_surrogate_params(self.handle, None, None if pp is None else pp.ctypes.data, None,
                                        None if ss is None else ss.ctypes.data), self.ctx.handle)
