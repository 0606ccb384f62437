"""The learned smoother's network (mgsb_mlp_* in the C ABI): a per-vertex MLP
9 -> 64 -> 64 -> 3 with GELU, BF16 weights on the tensor cores, trained on
the GPU by the library's own forward/backward kernels and Adam."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

NUM_PARAMS = 4995


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = L.load()
        h = C.c_void_p()
        st = self._lib.mgsb_mlp_create(device, seed, C.byref(h))
        if st != 0:
            raise RuntimeError(f"mgsb_mlp_create failed: {L.STATUS.get(st, st)}")
        self.h = h

    def _check(self, st):
        if st != 0:
            msg = self._lib.mgsb_mlp_last_error(self.h)
            raise RuntimeError(f"{L.STATUS.get(st, st)}: {msg.decode() if msg else ''}")

    def close(self):
        if self.h:
            self._lib.mgsb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.empty(NUM_PARAMS, np.float32)
        self._check(self._lib.mgsb_mlp_get_params(self.h, _fp(out), NUM_PARAMS))
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._lib.mgsb_mlp_set_params(self.h, _fp(p), p.shape[0]))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        y = np.empty((x.shape[0], 3), np.float32)
        self._check(self._lib.mgsb_mlp_forward(self.h, _fp(x), x.shape[0], _fp(y)))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, 3)
        g = np.empty(NUM_PARAMS, np.float32)
        loss = np.empty(1, np.float32)
        self._check(self._lib.mgsb_mlp_loss_grad(self.h, _fp(x), _fp(t), x.shape[0], _fp(g), _fp(loss)))
        return float(loss[0]), g

    def train(self, x, t, steps: int = 20000, batch: int = 4096, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, 3)
        losses = np.empty(steps, np.float32)
        self._check(self._lib.mgsb_mlp_train(self.h, _fp(x), _fp(t), x.shape[0], steps, batch, lr, seed, _fp(losses)))
        return losses
