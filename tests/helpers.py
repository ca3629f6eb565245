"""Shared helpers of the parity tests: build the same scene for the CUDA
path (through the C ABI) and for the FP64 oracle, and compare states."""
from __future__ import annotations

import numpy as np

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200.sim import Group, MaterialParams, Scene, Simulation
from oracle import cpu as ocpu

# FP32 path vs FP64 oracle, one substep: errors are reported relative to the
# field's largest magnitude (max |a - b| / max |b|), positions absolutely.
TOL_STEP = {"x": 2e-6, "v": 1e-4, "C": 1e-4, "F": 1e-5, "aux": 1e-5}

# Against the reference build's golden fixtures (tests/golden/ref3d_*.npz).
# The reference computes stress and the snow SVD in FP32 with an
# approximate-Jacobi SVD whose singular vectors are ill-conditioned for
# near-equal singular values; the bound is max relative 1e-4 per substep.
TOL_REF = {1: {"x": 1e-6, "v": 1e-4, "C": 1e-4, "F": 1e-4, "aux": 1e-4},
           10: {"x": 5e-6, "v": 1e-3, "C": 1e-3, "F": 1e-3, "aux": 1e-3}}
TOL_REF_MEDIAN = {1: 2e-6, 10: 2e-5}


def group_from_arrays(mat: MaterialParams, h: float, ppc: int, x, v, C, F, aux) -> Group:
    d = x.shape[1]
    vol = h ** d / ppc
    return Group(material=mat, p_mass=mat.rho * vol, p_vol=vol, x=np.float32(x), v=np.float32(v),
                 C=np.float32(C), F=np.float32(F), aux=np.float32(aux))


def oracle_group(g: Group) -> ocpu.OGroup:
    m = g.material
    return ocpu.OGroup(m.type, m.mu, m.lam, g.p_mass, g.p_vol, m.xi, m.theta_c, m.theta_s, m.bulk_k, m.gamma)


def oracle_for(scene: Scene) -> ocpu.OracleSim:
    d = scene.dim
    xs, vs, Cs, Fs, auxs, grp = [], [], [], [], [], []
    for gi, g in enumerate(scene.groups):
        n = g.n
        xs.append(np.float64(np.float32(g.x)))
        vs.append(np.float64(np.float32(g.v)) if g.v is not None else np.tile(np.float64(np.float32(g.init_v[:d])), (n, 1)))
        Cs.append(np.float64(np.float32(g.C)) if g.C is not None else np.zeros((n, d, d)))
        Fs.append(np.float64(np.float32(g.F)) if g.F is not None else np.tile(np.eye(d), (n, 1, 1)))
        auxs.append(np.float64(np.float32(g.aux)) if g.aux is not None else np.ones(n))
        grp.append(np.full(n, gi, np.int32))
    cat = lambda a: np.concatenate(a, axis=0)
    return ocpu.OracleSim(d, scene.n, scene.h, scene.dt, [oracle_group(g) for g in scene.groups], cat(xs),
                          cat(vs), cat(Cs), cat(Fs), cat(auxs), group=cat(grp), origin=scene.origin,
                          gravity=scene.gravity, bc_type=scene.bc_type, bc_lo=scene.bc_lo, bc_hi=scene.bc_hi,
                          mass_eps=scene.mass_eps)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


def compare(gpu_state: dict, ref_state: dict, tol: dict, fields=("x", "v", "C", "F", "aux"),
            skip_F: bool = False):
    errs = {}
    for k in fields:
        if skip_F and k == "F":
            continue
        if k == "x":
            errs[k] = float(np.abs(np.float64(gpu_state[k]) - ref_state[k]).max())
        else:
            errs[k] = rel_err(gpu_state[k], ref_state[k])
    bad = {k: e for k, e in errs.items() if e > tol[k]}
    assert not bad, f"errors above tolerance: {bad} (all: {errs})"
    return errs
