"""ctypes wrapper of the reference's own CUDA substep -- TEST INFRASTRUCTURE.

_ref/libmpm_ref.so is the reference's src/simulator/MPMCUDA.cu compiled
unmodified for sm_100a and linked with ref_harness.cu (see oracle/Makefile).
It runs the reference MPMSimulator::step() on FP64 AoS state.  Its physical
constants are the reference's hard-coded ones: gravity -9.8 on y, a 10h slip
band at every wall, xi = 10, snow clamp [1 - 8e-2, 1 + 2e-2], water
p = 2.51 (J^-7 - 1), grid origin 0.  Needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libmpm_ref.so")
_DP = C.POINTER(C.c_double)

# boundary of the reference build expressed in the project's terms:
# a node is a wall node when its index i satisfies i <= 10 or i >= n - 10
REF_BC_LO, REF_BC_HI = 11, 10
REF_GRAVITY = (0.0, -9.8, 0.0)
REF_MASS_EPS = 2.220446049250313e-16

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB_PATH)
        lib.mpmref_create.restype = C.c_void_p
        lib.mpmref_create.argtypes = [C.c_double, C.c_double, C.c_uint, C.c_uint, C.c_uint]
        lib.mpmref_destroy.argtypes = [C.c_void_p]
        lib.mpmref_add_group.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_uint, _DP, _DP, _DP, _DP, _DP, _DP]
        lib.mpmref_step.argtypes = [C.c_void_p, C.c_int]
        lib.mpmref_time_steps.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float)]
        lib.mpmref_get_group.argtypes = [C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP]
        lib.mpmref_get_grid.argtypes = [C.c_void_p, _DP, _DP]
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else np.ascontiguousarray(a, np.float64).ctypes.data_as(_DP)


class RefSim:
    """The reference simulator with groups added from arrays."""

    def __init__(self, h: float, dt: float, n):
        self.lib = load()
        self.h, self.dt, self.n = h, dt, tuple(n)
        self.s = self.lib.mpmref_create(h, dt, *self.n)
        if not self.s:
            raise RuntimeError("mpmref_create failed")
        self.sizes = []
        self.types = []

    def add_group(self, type_: int, E: float, nu: float, rho: float, p_mass: float, p_vol: float,
                  x, v, F, Fp=None, J=None, C_=None):
        n = x.shape[0]
        keep = [np.ascontiguousarray(a, np.float64) if a is not None else None for a in (x, v, F, Fp, J, C_)]
        rc = self.lib.mpmref_add_group(self.s, type_, E, nu, rho, p_mass, p_vol, n,
                                       *[k.ctypes.data_as(_DP) if k is not None else None for k in keep])
        if rc != 0:
            raise RuntimeError("mpmref_add_group failed")
        self.sizes.append(n)
        self.types.append(type_)

    def step(self, n: int = 1):
        if self.lib.mpmref_step(self.s, n) != 0:
            raise RuntimeError("reference step failed")

    def time_steps(self, n: int) -> float:
        ms = C.c_float()
        if self.lib.mpmref_time_steps(self.s, n, C.byref(ms)) != 0:
            raise RuntimeError("reference step failed")
        return ms.value

    def get_group(self, g: int) -> dict:
        n = self.sizes[g]
        out = {"x": np.empty((n, 3)), "v": np.empty((n, 3)), "F": np.empty((n, 3, 3)), "C": np.empty((n, 3, 3))}
        Fp = np.empty((n, 3, 3)) if self.types[g] == 1 else None
        J = np.empty(n) if self.types[g] == 2 else None
        rc = self.lib.mpmref_get_group(self.s, g, out["x"].ctypes.data_as(_DP), out["v"].ctypes.data_as(_DP),
                                       out["F"].ctypes.data_as(_DP),
                                       Fp.ctypes.data_as(_DP) if Fp is not None else None,
                                       J.ctypes.data_as(_DP) if J is not None else None,
                                       out["C"].ctypes.data_as(_DP))
        if rc != 0:
            raise RuntimeError("mpmref_get_group failed")
        if Fp is not None:
            out["Fp"] = Fp
        if J is not None:
            out["J"] = J
        return out

    def close(self):
        if self.s:
            self.lib.mpmref_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
