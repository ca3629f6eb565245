"""ctypes wrapper of the FP64 CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

The substep it runs restates MPMSimulator::step() (MPMCUDA.cu:793-925) in 3D
and the Taichi substep() (MPMJello.py:31-120, MPMSnow.py:78-150,
MPMWater.py:71-138) in 2D; see mpm_oracle.c for the line-by-line map.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

JELLO, SNOW, WATER = 0, 1, 2
BC_STICKY, BC_SLIP, BC_SEPARATE = 0, 1, 2
ERR_OUT_OF_GRID, ERR_NONFINITE, ERR_DET, ERR_WEIGHTS = 1, 2, 4, 8

_DP = C.POINTER(C.c_double)


class OrcGrid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3), ("h", C.c_double), ("origin", C.c_double * 3),
                ("dt", C.c_double), ("gravity", C.c_double * 3), ("bc_type", C.c_int),
                ("bc_lo", C.c_int), ("bc_hi", C.c_int), ("mass_eps", C.c_double), ("ref_band", C.c_double)]


class OrcGroup(C.Structure):
    _fields_ = [("type", C.c_int), ("mu", C.c_double), ("lambda_", C.c_double), ("xi", C.c_double),
                ("theta_c", C.c_double), ("theta_s", C.c_double), ("bulk_k", C.c_double),
                ("gamma", C.c_double), ("p_mass", C.c_double), ("p_vol", C.c_double)]


class OrcParticles(C.Structure):
    _fields_ = [("n", C.c_int), ("x", _DP), ("v", _DP), ("C", _DP), ("F", _DP), ("Fp", _DP),
                ("J", _DP), ("group", C.POINTER(C.c_int))]


_lib = None


def build():
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        lib.orc_substep.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcGroup), C.POINTER(OrcParticles),
                                    _DP, _DP, C.c_int]
        lib.orc_p2g.argtypes = lib.orc_substep.argtypes
        lib.orc_grid_update.argtypes = [C.POINTER(OrcGrid), _DP, _DP]
        lib.orc_g2p.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcGroup), C.POINTER(OrcParticles), _DP, C.c_int]
        lib.orc_kirchhoff_fcr.argtypes = [C.c_int, _DP, C.c_double, C.c_double, _DP]
        lib.orc_polar_svd.argtypes = [C.c_int, _DP, _DP, _DP, _DP]
        lib.orc_seed.argtypes = [C.c_int, _DP, _DP, _DP, C.POINTER(C.c_float), C.c_long, C.POINTER(C.c_int),
                                 C.c_long, C.c_int, C.c_double, _DP, C.c_int, C.c_ulonglong,
                                 C.POINTER(C.c_float), C.c_long, C.POINTER(C.c_long)]
        lib.orc_bspline.argtypes = [C.c_double]
        lib.orc_bspline.restype = C.c_double
        lib.orc_bspline_deriv.argtypes = [C.c_double]
        lib.orc_bspline_deriv.restype = C.c_double
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


@dataclass
class OGroup:
    type: int
    mu: float
    lam: float
    p_mass: float
    p_vol: float
    xi: float = 10.0
    theta_c: float = 8e-2
    theta_s: float = 2e-2
    bulk_k: float = 2.51
    gamma: float = 7.0


class OracleSim:
    """FP64 state + grid of one scene, stepped by the C oracle.

    State arrays (float64): x (N,3), v (N,3), C (N,3,3), F (N,3,3), Fp (N,3,3),
    J (N,), group (N,) int32.  2D scenes use the leading 2 components."""

    def __init__(self, dim: int, n: Sequence[int], h: float, dt: float, groups: List[OGroup],
                 x, v, C_, F, aux, group=None, origin=(0, 0, 0), gravity=(0, -9.8, 0),
                 bc_type=BC_SLIP, bc_lo=3, bc_hi=3, mass_eps=2.220446049250313e-16, ref_band=0.0):
        self.lib = load()
        self.dim = dim
        N = x.shape[0]
        self.N = N
        self.x = np.zeros((N, 3))
        self.v = np.zeros((N, 3))
        self.C = np.zeros((N, 3, 3))
        self.F = np.zeros((N, 3, 3))
        self.Fp = np.zeros((N, 3, 3))
        self.J = np.ones(N)
        d = dim
        self.x[:, :d] = x
        self.v[:, :d] = v
        self.C[:, :d, :d] = C_
        self.F[:, :d, :d] = F
        self.group = np.zeros(N, np.int32) if group is None else np.ascontiguousarray(group, np.int32)
        # aux: det Fp for snow (Fp stored as diag(aux^(1/d))), J for water
        for gi, g in enumerate(groups):
            m = self.group == gi
            if g.type == SNOW:
                s = np.asarray(aux)[m] ** (1.0 / d)
                Fp = np.zeros((m.sum(), 3, 3))
                for a in range(d):
                    Fp[:, a, a] = s
                self.Fp[m] = Fp
            elif g.type == WATER:
                self.J[m] = np.asarray(aux)[m]
        nn = list(n) + [1] * (3 - len(n))
        self.grid = OrcGrid(dim, (C.c_int * 3)(*nn[:3]), h, (C.c_double * 3)(*list(origin)[:3]), dt,
                            (C.c_double * 3)(*(list(gravity) + [0, 0, 0])[:3]), bc_type, bc_lo, bc_hi,
                            mass_eps, ref_band)
        self.groups = (OrcGroup * len(groups))(*[
            OrcGroup(g.type, g.mu, g.lam, g.xi, g.theta_c, g.theta_s, g.bulk_k, g.gamma, g.p_mass, g.p_vol)
            for g in groups])
        G = int(np.prod(nn))
        self.nn = nn
        self.mass = np.zeros(G)
        self.mom = np.zeros(3 * G)

    def _parts(self):
        return OrcParticles(self.N, _dp(self.x), _dp(self.v), _dp(self.C), _dp(self.F), _dp(self.Fp),
                            _dp(self.J), self.group.ctypes.data_as(C.POINTER(C.c_int)))

    def step(self, n: int = 1, threads: int = 1) -> int:
        err = 0
        p = self._parts()
        for _ in range(n):
            err |= self.lib.orc_substep(C.byref(self.grid), self.groups, C.byref(p), _dp(self.mass),
                                        _dp(self.mom), threads)
        return err

    def aux(self) -> np.ndarray:
        """det Fp for snow particles, J for water, 1 for jello (as the CUDA path stores)."""
        out = np.ones(self.N)
        d = self.dim
        for gi in range(len(self.groups)):
            m = self.group == gi
            if self.groups[gi].type == SNOW:
                out[m] = np.linalg.det(self.Fp[m][:, :d, :d])
            elif self.groups[gi].type == WATER:
                out[m] = self.J[m]
        return out

    def grid_update(self, mass: np.ndarray, mom: np.ndarray) -> np.ndarray:
        """The oracle's grid update (MPMCUDA.cu:435-472) on given node masses
        and momenta of this scene's grid; returns the node velocities (G, 3)."""
        m = np.ascontiguousarray(mass, np.float64).copy()
        v = np.ascontiguousarray(mom, np.float64).reshape(-1).copy()
        self.lib.orc_grid_update(C.byref(self.grid), _dp(m), _dp(v))
        return v.reshape(-1, 3)

    def grid_mass(self):
        return self.mass.reshape(self.nn[::-1]) if self.dim == 3 else self.mass.reshape(self.nn[1], self.nn[0])

    def state(self):
        d = self.dim
        return {"x": self.x[:, :d].copy(), "v": self.v[:, :d].copy(), "C": self.C[:, :d, :d].copy(),
                "F": self.F[:, :d, :d].copy(), "aux": self.aux()}


def kirchhoff_fcr(F: np.ndarray, mu: float, lam: float) -> np.ndarray:
    d = F.shape[0]
    F3 = np.zeros((3, 3))
    F3[:d, :d] = F
    tau = np.zeros((3, 3))
    load().orc_kirchhoff_fcr(d, _dp(F3), mu, lam, _dp(tau))
    return tau[:d, :d]


def polar_svd(F: np.ndarray):
    d = F.shape[0]
    F3 = np.zeros((3, 3))
    F3[:d, :d] = F
    U, s, V = np.zeros((3, 3)), np.zeros(3), np.zeros((3, 3))
    load().orc_polar_svd(d, _dp(F3), _dp(U), _dp(s), _dp(V))
    return U[:d, :d], s[:d], V[:d, :d]


def bspline(x: float) -> float:
    return load().orc_bspline(x)


def bspline_deriv(x: float) -> float:
    return load().orc_bspline_deriv(x)


SEED_SHAPES = {"cube": 0, "sphere": 1, "cylinder": 2, "mesh": 3}


def seed_positions(shape: str, h: float, ppc: int, *, translation=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0),
                   rot=None, origin=(0.0, 0.0, 0.0), dim: int = 3, seed_value: int = 1234, vertices=None,
                   triangles=None) -> np.ndarray:
    """The CPU restatement of the GPU seeding (orc_seed): positions (n, dim)
    float32 in cell order, bit for bit what mpm_seed returns."""
    lib = load()
    R = np.ascontiguousarray(np.eye(3) if rot is None else rot, np.float64).ravel()
    S = np.ascontiguousarray(list(scale) + [1.0] * (3 - len(scale)), np.float64)[:3]
    T = np.ascontiguousarray(list(translation) + [0.0] * (3 - len(translation)), np.float64)[:3]
    O = np.ascontiguousarray(list(origin) + [0.0] * (3 - len(origin)), np.float64)[:3]
    v = t = None
    nv = nt = 0
    if shape == "mesh":
        v = np.ascontiguousarray(vertices, np.float32)
        t = np.ascontiguousarray(triangles, np.int32)
        nv, nt = v.shape[0], t.shape[0]
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
    ip = t.ctypes.data_as(C.POINTER(C.c_int)) if t is not None else None
    n = C.c_long()
    args = (SEED_SHAPES[shape], _dp(R), _dp(S), _dp(T), fp(v), nv, ip, nt, dim, h, _dp(O), ppc, seed_value)
    if lib.orc_seed(*args, None, 0, C.byref(n)) != 0:
        raise ValueError("orc_seed: bad argument")
    out = np.empty((n.value, dim), np.float32)
    if n.value and lib.orc_seed(*args, fp(out), out.size, C.byref(n)) != 0:
        raise ValueError("orc_seed failed")
    return out
