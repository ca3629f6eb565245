"""Independent NumPy restatement of the MPM substep -- TEST INFRASTRUCTURE.

Written separately from mpm_oracle.c (vectorised over particles, NumPy's
LAPACK SVD instead of Jacobi) so the two CPU oracles check each other.  It
follows the 2D Taichi scripts (MPMJello.py:31-120, MPMSnow.py:78-150,
MPMWater.py:71-138) and, for dim 3, the reference kernels
(MPMCUDA.cu:310-741), which are the same algorithm.  Only for small cases.
"""
from __future__ import annotations

import numpy as np

JELLO, SNOW, WATER = 0, 1, 2
BC_STICKY, BC_SLIP, BC_SEPARATE = 0, 1, 2


def _signed_svd(F):
    """F = U diag(s) V^T with det U = det V = 1 (last s may be negative)."""
    U, s, Vh = np.linalg.svd(F)
    V = np.swapaxes(Vh, -1, -2).copy()
    s = s.copy()
    neg = np.linalg.det(U) < 0
    U[neg, :, -1] *= -1
    s[neg, -1] *= -1
    neg = np.linalg.det(V) < 0
    V[neg, :, -1] *= -1
    s[neg, -1] *= -1
    return U, s, V


def _weights(x, o, h, n):
    """base index, weights (N,3,d) and derivatives (N,3,d) along each axis."""
    g = (x - o) / h
    base = np.maximum(0, np.floor(g - 0.5).astype(np.int64))
    fx = g - base
    w = np.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2], axis=1)
    dw = np.stack([fx - 1.5, -2.0 * (fx - 1.0), fx - 0.5], axis=1)
    return base, fx, w, dw


def substep(scene: dict, st: dict) -> dict:
    """One substep.  scene: dim, n, h, origin, dt, gravity, bc_type, bc_lo,
    bc_hi, mass_eps, groups[list of dict(type, mu, lam, xi, theta_c, theta_s,
    bulk_k, gamma, p_mass, p_vol)].  st: x (N,d), v, C (N,d,d), F, aux (N,)
    (det Fp for snow, J for water), group (N,).  Returns the new state."""
    d = scene["dim"]
    n = np.array(scene["n"][:d])
    h, dt = scene["h"], scene["dt"]
    o = np.array(scene.get("origin", (0, 0, 0))[:d], dtype=np.float64)
    x, v, C, F, aux = (np.array(st[k], dtype=np.float64) for k in ("x", "v", "C", "F", "aux"))
    grp = np.asarray(st["group"])
    N = x.shape[0]
    G = int(np.prod(n))
    mass = np.zeros(G)
    mom = np.zeros((G, d))

    typ = np.array([scene["groups"][g]["type"] for g in grp])
    par = lambda key: np.array([scene["groups"][g][key] for g in grp], dtype=np.float64)
    mu, lam, pm, pv = par("mu"), par("lam"), par("p_mass"), par("p_vol")

    # ---- stress (Kirchhoff), MPMCUDA.cu:329-354
    tau = np.zeros((N, d, d))
    solid = typ != WATER
    if solid.any():
        hard = np.where(typ == SNOW, np.exp(par("xi") * (1.0 - aux)), 1.0)
        Fs = F[solid]
        U, s, V = _signed_svd(Fs)
        R = U @ np.swapaxes(V, -1, -2)
        J = np.linalg.det(Fs)
        t = 2.0 * (mu * hard)[solid, None, None] * (Fs - R) @ np.swapaxes(Fs, -1, -2)
        t += ((lam * hard)[solid] * J * (J - 1.0))[:, None, None] * np.eye(d)
        tau[solid] = t
    wat = typ == WATER
    if wat.any():
        Jw = aux[wat]
        p = par("bulk_k")[wat] * (Jw ** (-par("gamma")[wat]) - 1.0)
        tau[wat] = -(p * Jw)[:, None, None] * np.eye(d)

    base, fx, w, dw = _weights(x, o, h, n)
    offsets = np.stack(np.meshgrid(*([np.arange(3)] * d), indexing="ij"), -1).reshape(-1, d)

    def node_terms(off):
        wk = np.ones(N)
        gw = np.ones((N, d))
        for a in range(d):
            wk = wk * w[np.arange(N), off[a], a]
            for b in range(d):
                gw[:, b] *= (dw if a == b else w)[np.arange(N), off[a], a]
        gw /= h
        idx = base + off
        lin = np.zeros(N, dtype=np.int64)
        stride = 1
        for a in range(d):
            lin += idx[:, a] * stride
            stride *= n[a]
        dpos = (off - fx) * h
        return wk, gw, lin, dpos

    # ---- P2G
    for off in offsets:
        wk, gw, lin, dpos = node_terms(off)
        np.add.at(mass, lin, wk * pm)
        mv = (wk * pm)[:, None] * (v + np.einsum("nab,nb->na", C, dpos))
        force = -pv[:, None] * np.einsum("nab,nb->na", tau, gw)
        np.add.at(mom, lin, mv + dt * force)

    # ---- grid update
    act = mass > scene.get("mass_eps", 0.0)
    vel = np.zeros_like(mom)
    vel[act] = mom[act] / mass[act, None] + dt * np.array(scene["gravity"][:d])
    ids = np.stack(np.unravel_index(np.arange(G), tuple(n[::-1]))[::-1], axis=1)
    lo_w = ids < scene["bc_lo"]
    hi_w = ids >= n - scene["bc_hi"]
    bc = scene["bc_type"]
    if bc == BC_STICKY:
        vel[np.any(lo_w | hi_w, axis=1)] = 0.0
    elif bc == BC_SLIP:
        vel[lo_w | hi_w] = 0.0
    else:
        vel[lo_w & (vel < 0)] = 0.0
        vel[hi_w & (vel > 0)] = 0.0
    vel[~act] = 0.0

    # ---- G2P
    vp = np.zeros((N, d))
    Cn = np.zeros((N, d, d))
    gv = np.zeros((N, d, d))
    for off in offsets:
        wk, gw, lin, dpos = node_terms(off)
        vi = vel[lin]
        vp += wk[:, None] * vi
        Cn += 4.0 / (h * h) * wk[:, None, None] * np.einsum("na,nb->nab", vi, dpos)
        gv += np.einsum("na,nb->nab", vi, gw)
    L = np.eye(d) + dt * gv
    Fn = F.copy()
    auxn = aux.copy()
    jel = typ == JELLO
    Fn[jel] = L[jel] @ F[jel]
    sn = typ == SNOW
    if sn.any():
        Ft = L[sn] @ F[sn]
        U, s, V = _signed_svd(Ft)
        s = np.clip(s, 1.0 - par("theta_c")[sn, None], 1.0 + par("theta_s")[sn, None])
        Fe = U @ (s[:, :, None] * np.swapaxes(V, -1, -2))
        Fp_ratio = np.linalg.det(Ft) / np.linalg.det(Fe)
        Fn[sn] = Fe
        auxn[sn] = aux[sn] * Fp_ratio
    if wat.any():
        auxn[wat] = (1.0 + dt * np.trace(gv[wat], axis1=1, axis2=2)) * aux[wat]
    return {"x": x + dt * vp, "v": vp, "C": Cn, "F": Fn, "aux": auxn, "group": grp,
            "grid_mass": mass, "grid_vel": vel}
