"""FP64 CPU restatement of the learned stress surrogate (test infrastructure).

Checks the library's tensor-core training kernels (csrc/mpm_surrogate.cu)
and its stress formula (csrc/mpm_mlp.cuh):

* ``forward_backward`` -- the MLP 10 -> 64 -> 64 -> 9 with SiLU and its exact
  gradient of the mean squared error, in FP64.  With ``bf16_ops=True`` it
  rounds the same operands to bfloat16 as the GPU kernels do (inputs, weights,
  the hidden activations, which the kernels compute on packed bf16 pairs, the
  output and hidden deltas fed to the backward products), still accumulating
  in FP64.
* ``residual_target`` / ``tau_from_residual`` -- sqrt(B) beyond its
  second-order series and the Kirchhoff stress rebuilt from it; with the exact
  residual they reproduce the fixed-corotated stress of the reference
  (MPMCUDA.cu:229-264, tau = 2 mu (F - R) F^T + lambda J (J - 1) I).
* ``fcr_tau`` -- that stress from an FP64 SVD (numpy).

The reference has no learned stress, so this oracle is pinned by those
identities and by finite differences, not by reference outputs.
Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

IN, IN_PAD, HID, OUT, OUT_PAD = 10, 16, 64, 9, 16
OFF_W1 = 0
OFF_W2 = OFF_W1 + HID * IN_PAD
OFF_W3 = OFF_W2 + HID * HID
OFF_B1 = OFF_W3 + OUT_PAD * HID
OFF_B2 = OFF_B1 + HID
OFF_B3 = OFF_B2 + HID
N_PARAMS = OFF_B3 + OUT_PAD


def bf16(a) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, np.float64)
    return {
        "W1": p[OFF_W1:OFF_W2].reshape(HID, IN_PAD)[:, :IN],
        "W2": p[OFF_W2:OFF_W3].reshape(HID, HID),
        "W3": p[OFF_W3:OFF_B1].reshape(OUT_PAD, HID)[:OUT],
        "b1": p[OFF_B1:OFF_B2], "b2": p[OFF_B2:OFF_B3], "b3": p[OFF_B3:OFF_B3 + OUT],
    }


def pack(g: dict) -> np.ndarray:
    p = np.zeros(N_PARAMS, np.float64)
    p[OFF_W1:OFF_W2].reshape(HID, IN_PAD)[:, :IN] = g["W1"]
    p[OFF_W2:OFF_W3] = g["W2"].ravel()
    p[OFF_W3:OFF_B1].reshape(OUT_PAD, HID)[:OUT] = g["W3"]
    p[OFF_B1:OFF_B2] = g["b1"]
    p[OFF_B2:OFF_B3] = g["b2"]
    p[OFF_B3:OFF_B3 + OUT] = g["b3"]
    return p


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_bf16(z):
    """SiLU as the kernels evaluate it on packed bfloat16 pairs: z rounded to
    bf16, then z * (1/2 + tanh(z/2)/2) with every operation rounded to bf16
    (tanh exact here, the hardware's approximation there)."""
    zb = bf16(z)
    t = bf16(np.tanh(bf16(0.5 * zb)))
    s = bf16(0.5 * t + 0.5)
    return bf16(zb * s)


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s + z * s * (1.0 - s)


def forward(params, x, bf16_ops: bool = False):
    w = unpack(params)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    act = silu_bf16 if bf16_ops else silu
    W1, W2, W3 = r(w["W1"]), r(w["W2"]), r(w["W3"])
    z1 = r(x) @ W1.T + w["b1"]
    h1 = act(z1)
    z2 = h1 @ W2.T + w["b2"]
    h2 = act(z2)
    return h2 @ W3.T + w["b3"]


def forward_backward(params, x, y, bf16_ops: bool = False):
    """(loss, packed gradient) of mean((f(x) - y)^2) over the n x 9 outputs."""
    w = unpack(params)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    act = silu_bf16 if bf16_ops else silu
    x = r(x)
    y = np.asarray(y, np.float64)
    W1, W2, W3 = r(w["W1"]), r(w["W2"]), r(w["W3"])
    z1 = x @ W1.T + w["b1"]
    h1 = act(z1)
    z2 = h1 @ W2.T + w["b2"]
    h2 = act(z2)
    o = h2 @ W3.T + w["b3"]
    n = x.shape[0]
    d = o - y
    loss = float(np.mean(d * d))
    dO = 2.0 * d / (n * OUT)
    dOr = r(dO)
    g = {"W3": dOr.T @ h2, "b3": dO.sum(0)}
    dz2 = (dOr @ W3) * silu_grad(z2)
    dz2r = r(dz2)
    g["W2"] = dz2r.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2r @ W2) * silu_grad(z1)
    g["W1"] = r(dz1).T @ x
    g["b1"] = dz1.sum(0)
    return loss, pack(g)


# ------------------------------------------------------------ stress --

def strain_b(F):
    """X = F F^T - I of F (..., 3, 3)."""
    F = np.asarray(F, np.float64)
    return F @ np.swapaxes(F, -1, -2) - np.eye(3)


def residual_target(F):
    """r = sqrt(B) - I - X/2 + X^2/8, B = F F^T = I + X, from an eigendecomposition."""
    X = strain_b(F)
    lam, Q = np.linalg.eigh(X + np.eye(3))
    sq = (Q * np.sqrt(np.maximum(lam, 0.0))[..., None, :]) @ np.swapaxes(Q, -1, -2)
    return sq - np.eye(3) - 0.5 * X + 0.125 * (X @ X)


def tau_from_residual(F, r, mu, lam):
    """tau = mu (X + X^2/4 - 2 sym(r)) + lambda J (J - 1) I."""
    X = strain_b(F)
    J = np.linalg.det(np.asarray(F, np.float64))
    rs = 0.5 * (r + np.swapaxes(r, -1, -2))
    return mu * (X + 0.25 * (X @ X) - 2.0 * rs) + (lam * J * (J - 1.0))[..., None, None] * np.eye(3)


def fcr_tau(F, mu, lam):
    """Fixed-corotated Kirchhoff stress 2 mu (F - R) F^T + lambda J (J - 1) I
    with R = U V^T from an FP64 SVD (det F > 0)."""
    F = np.asarray(F, np.float64)
    U, s, Vt = np.linalg.svd(F)
    R = U @ Vt
    J = np.linalg.det(F)
    return 2.0 * mu * (F - R) @ np.swapaxes(F, -1, -2) + (lam * J * (J - 1.0))[..., None, None] * np.eye(3)


def features(F, in_scale: float):
    """Network input (n, 10): X / in_scale (9 entries), (J - 1) / in_scale."""
    F = np.asarray(F, np.float64)
    X = strain_b(F).reshape(-1, 9)
    J = np.linalg.det(F).reshape(-1, 1)
    return np.concatenate([X, J - 1.0], axis=1) / in_scale
