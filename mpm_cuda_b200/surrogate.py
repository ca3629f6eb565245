"""Learned stress surrogate: a BF16 MLP 10 -> 64 -> 64 -> 9 (SiLU) trained and
run on the GPU by the library's own tensor-core kernels.

The network predicts the residual of sqrt(B), B = F F^T, beyond its
second-order series in X = B - I; the fixed-corotated Kirchhoff stress of the
reference (MPMCUDA.cu:229-264, there from an SVD) is then
``tau = mu (X + X^2/4 - 2 sym(r)) + lambda J (J - 1) I``.  See
``csrc/mpm_mlp.cuh`` for the layout and ``csrc/mpm_surrogate.cu`` for the
training kernels.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L

META_FIELDS = ("in_scale", "out_scale", "env_c", "env_jlo", "env_jhi", "skew_tol", "tau_floor", "pad")
# packed parameter layout (include/mpm_b200.h)
IN, IN_PAD, HID, OUT, OUT_PAD = 10, 16, 64, 9, 16
OFF_W1 = 0
OFF_W2 = OFF_W1 + HID * IN_PAD
OFF_W3 = OFF_W2 + HID * HID
OFF_B1 = OFF_W3 + OUT_PAD * HID
OFF_B2 = OFF_B1 + HID
OFF_B3 = OFF_B2 + HID
N_PARAMS = OFF_B3 + OUT_PAD


def unpack_params(p: np.ndarray) -> dict:
    """Packed FP32 parameters -> W1 [64x10], W2 [64x64], W3 [9x64], b1, b2, b3 (real rows / columns)."""
    return {
        "W1": p[OFF_W1:OFF_W2].reshape(HID, IN_PAD)[:, :IN],
        "W2": p[OFF_W2:OFF_W3].reshape(HID, HID),
        "W3": p[OFF_W3:OFF_B1].reshape(OUT_PAD, HID)[:OUT],
        "b1": p[OFF_B1:OFF_B2], "b2": p[OFF_B2:OFF_B3], "b3": p[OFF_B3:OFF_B3 + OUT],
    }


def train_options(**kw) -> L.SurrogateTrainOptions:
    o = L.SurrogateTrainOptions()
    L.load().mpm_surrogate_default_train_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class StressSurrogate:
    """One network on one device (``mpm_surrogate*``)."""

    def __init__(self, device: int = 0, seed: int = 1234, _handle: Optional[C.c_void_p] = None):
        self._lib = L.load()
        if _handle is not None:
            self._h = _handle
        else:
            self._h = C.c_void_p()
            L.check(self._lib.mpm_surrogate_create(device, seed, C.byref(self._h)))
        self.device = device

    @classmethod
    def load(cls, path: str, device: int = 0) -> "StressSurrogate":
        h = C.c_void_p()
        L.check(L.load().mpm_surrogate_load(path.encode(), device, C.byref(h)))
        return cls(device, _handle=h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mpm_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train(self, F_seed: np.ndarray, **options) -> float:
        """Trains from deformation gradients F_seed (n, 3, 3); returns the last epoch's loss."""
        F = np.ascontiguousarray(F_seed, np.float32).reshape(-1, 9)
        loss = C.c_float()
        o = train_options(**options)
        L.check(self._lib.mpm_surrogate_train(self._h, L.fptr(F), F.shape[0], C.byref(o), C.byref(loss)))
        return loss.value

    def eval(self, F: np.ndarray, lam_over_mu: float):
        """(tau_pred / mu, tau_ref / mu, accepted) of deformation gradients F (n, 3, 3)."""
        F = np.ascontiguousarray(F, np.float32).reshape(-1, 9)
        n = F.shape[0]
        tp = np.empty((n, 3, 3), np.float32)
        tr = np.empty((n, 3, 3), np.float32)
        ok = np.empty(n, np.uint8)
        L.check(self._lib.mpm_surrogate_eval(self._h, L.fptr(F), n, float(lam_over_mu), L.fptr(tp), L.fptr(tr),
                                             ok.ctypes.data_as(C.POINTER(C.c_uint8))))
        return tp, tr, ok.astype(bool)

    def gradients(self, x: np.ndarray, y: np.ndarray):
        """(packed parameter gradient, loss) of the mean squared error of a batch
        of network inputs x (n, 10) and targets y (n, 9), n a multiple of 128."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.empty(N_PARAMS, np.float32)
        loss = C.c_float()
        L.check(self._lib.mpm_surrogate_gradients(self._h, L.fptr(x), L.fptr(y), x.shape[0], L.fptr(g),
                                                  C.byref(loss)))
        return g, loss.value

    def params(self):
        p = np.empty(N_PARAMS, np.float32)
        m = np.empty(len(META_FIELDS), np.float32)
        L.check(self._lib.mpm_surrogate_get_params(self._h, L.fptr(p), L.fptr(m)))
        return p, dict(zip(META_FIELDS, m.tolist()))

    def set_params(self, params: Optional[np.ndarray] = None, meta: Optional[dict] = None):
        m = None
        if meta is not None:
            cur = self.params()[1]
            cur.update(meta)
            m = np.array([cur[k] for k in META_FIELDS], np.float32)
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        L.check(self._lib.mpm_surrogate_set_params(self._h, L.fptr(p), L.fptr(m)))

    def save(self, path: str):
        L.check(self._lib.mpm_surrogate_save(self._h, path.encode()))


def harvest_F(sim, scene: int = 0) -> np.ndarray:
    """Deformation gradients (n, 3, 3) of a scene's particles (training seeds)."""
    return sim.get_state(scene)["F"]
