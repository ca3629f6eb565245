"""Seeded synthetic scenes: the benchmark workloads and small parity scenes.

The reference seeds particles from .obj meshes with ``rand()`` jitter
(MPMSimulator.cpp:239-260).  No meshes or datasets ship with it, so every
workload here is an analytic shape (box, sphere, column) filled with
``ppc`` uniformly jittered samples per grid cell from a seeded generator
(seed = 1234 + scene id), keeping the samples inside the shape.  Particle
volume is h^dim / ppc and mass rho * volume.
"""
from __future__ import annotations

import math
from typing import Callable, List, Sequence

import numpy as np

from . import _lib as L
from .sim import Group, MaterialParams, Scene


def jitter_fill(lo: Sequence[float], hi: Sequence[float], h: float, ppc: int,
                inside: Callable[[np.ndarray], np.ndarray], rng: np.random.Generator) -> np.ndarray:
    """ppc uniform samples in every cell overlapping [lo, hi], kept if inside."""
    d = len(lo)
    i0 = [int(math.floor(lo[a] / h)) for a in range(d)]
    i1 = [int(math.ceil(hi[a] / h)) for a in range(d)]
    axes = [np.arange(i0[a], i1[a], dtype=np.int64) for a in range(d)]
    cells = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, d)
    cells = np.repeat(cells, ppc, axis=0)
    x = (cells + rng.random(cells.shape)) * h
    return x[inside(x)].astype(np.float32)


def box(lo, hi):
    lo, hi = np.asarray(lo), np.asarray(hi)
    return lambda x: np.all((x >= lo) & (x < hi), axis=1)


def sphere(c, r):
    c = np.asarray(c)
    return lambda x: np.sum((x - c) ** 2, axis=1) < r * r


def jello(E=5e4, nu=0.3, rho=1000.0) -> MaterialParams:
    return MaterialParams(L.JELLO, E, nu, rho)


def snow(E=1.4e5, nu=0.2, rho=400.0, theta_c=2.5e-2, theta_s=7.5e-3, xi=10.0) -> MaterialParams:
    return MaterialParams(L.SNOW, E, nu, rho, xi=xi, theta_c=theta_c, theta_s=theta_s)


def water(K=1e4, rho=1000.0, gamma=7.0) -> MaterialParams:
    # E, nu are unused by the water model but must pass the Material range checks
    return MaterialParams(L.WATER, 0.0, 0.0, rho, bulk_k=K, gamma=gamma)


def make_group(mat: MaterialParams, x: np.ndarray, h: float, ppc: int, v0) -> Group:
    d = x.shape[1]
    vol = h ** d / ppc
    return Group(material=mat, p_mass=mat.rho * vol, p_vol=vol, x=x, init_v=tuple(v0))


# ---------------------------------------------------------------- workloads

def c0_jello2d(seed: int = 1234, E: float = 1e3) -> Scene:
    """2D jello as MPMJello.py: 128^2, dx = 1/128, N = 9000 uniform in a 0.2
    square centred at (0.5, 0.6), v = (0, -1), nu = 0.2, rho = 1,
    p_vol = (dx/2)^2, dt = 1e-4, gravity -9.8, 3-cell wall as
    MPMJello.py:92-95 (zero the wall-normal velocity moving into the wall).

    E defaults to the script's 1e3 (MPMJello.py:12).  E = 1e4 with rho = 1
    gives an elastic wave speed of 100 m/s and a CFL number
    dt sqrt(E / rho) / dx = 1.28 > 1: the substep diverges (the FP64 oracle
    within ~45 substeps)."""
    rng = np.random.default_rng(seed)
    n_grid, dx = 128, 1.0 / 128
    x = (rng.random((9000, 2)) * 0.2 + np.array([0.4, 0.5])).astype(np.float32)
    mat = MaterialParams(L.JELLO, E, 0.2, 1.0)
    vol = (dx * 0.5) ** 2
    g = Group(material=mat, p_mass=vol * 1.0, p_vol=vol, x=x, init_v=(0.0, -1.0))
    return Scene(dim=2, n=(n_grid, n_grid), h=dx, dt=1e-4, groups=[g], gravity=(0.0, -9.8),
                 bc_type=L.BC_SEPARATE, bc_lo=3, bc_hi=2, mass_eps=0.0, name="c0_jello2d")


def c1_jello3d(seed: int = 1234, n_grid: int = 128, edge: float = 0.3) -> Scene:
    """3D jello: 128^3 on the unit cube, 0.3 cube centred at (0.5, 0.6, 0.5),
    8 ppc, v = (0, -2, 0), E = 5e4, nu = 0.3, rho = 1000, dt = 1e-4,
    gravity -9.8, slip walls 3 cells wide."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n_grid
    c = np.array([0.5, 0.6, 0.5])
    lo, hi = c - edge / 2, c + edge / 2
    x = jitter_fill(lo, hi, h, 8, box(lo, hi), rng)
    g = make_group(jello(), x, h, 8, (0.0, -2.0, 0.0))
    return Scene(dim=3, n=(n_grid,) * 3, h=h, dt=1e-4, groups=[g], bc_type=L.BC_SLIP, bc_lo=3,
                 bc_hi=3, name=f"c1_jello3d_{n_grid}")


def c2_snow3d(seed: int = 1234, n_grid: int = 256) -> Scene:
    """3D snow: 256^3, spheres r = 0.12 at (0.3, 0.5, 0.5) and (0.7, 0.52, 0.5)
    at 8 ppc moving toward each other at 3 m/s, Stomakhin plasticity
    E0 = 1.4e5, nu = 0.2, theta_c = 2.5e-2, theta_s = 7.5e-3, xi = 10,
    rho = 400, dt = 5e-5, slip walls 3 cells wide."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n_grid
    groups = []
    for c, v in (((0.3, 0.5, 0.5), (3.0, 0.0, 0.0)), ((0.7, 0.52, 0.5), (-3.0, 0.0, 0.0))):
        c = np.array(c)
        x = jitter_fill(c - 0.12, c + 0.12, h, 8, sphere(c, 0.12), rng)
        groups.append(make_group(snow(), x, h, 8, v))
    return Scene(dim=3, n=(n_grid,) * 3, h=h, dt=5e-5, groups=groups, bc_type=L.BC_SLIP, bc_lo=3,
                 bc_hi=3, name=f"c2_snow3d_{n_grid}")


def c3_jello3d(seed: int = 1234, edge: float = 0.245) -> Scene:
    """The c1 scene rescaled to 256^3.  edge = 0.245 gives ~2.0M particles at
    8 ppc; the literal 0.45 edge gives ~12.2M."""
    s = c1_jello3d(seed=seed, n_grid=256, edge=edge)
    s.name = f"c3_jello3d_256_edge{edge}"
    return s


def c4_batched(seed: int = 1234, n_scenes: int = 64) -> List[Scene]:
    """64 independent scenes, N log-uniform in [1e4, 5e5], grid side matched
    to N in [64, 192], materials cycled jello / snow / water (dam-break column
    0.3 x 0.6 x 0.3 scaled to N, K = 1e4, rho = 1000), dt = 1e-4, 8 ppc."""
    rng = np.random.default_rng(seed)
    scenes = []
    ppc = 8
    for i in range(n_scenes):
        srng = np.random.default_rng(seed + i)
        n_target = float(np.exp(rng.uniform(math.log(1e4), math.log(5e5))))
        t = (math.log(n_target) - math.log(1e4)) / (math.log(5e5) - math.log(1e4))
        side = int(round((64 + t * 128) / 8.0)) * 8
        h = 1.0 / side
        kind = i % 3
        if kind == 0:
            vol0 = 0.3 ** 3
            s = (n_target / (vol0 * side ** 3 * ppc)) ** (1 / 3)
            e = 0.3 * s
            c = np.array([0.5, 0.55, 0.5])
            x = jitter_fill(c - e / 2, c + e / 2, h, ppc, box(c - e / 2, c + e / 2), srng)
            g = make_group(jello(), x, h, ppc, (0.0, -1.0, 0.0))
        elif kind == 1:
            vol0 = 4.0 / 3.0 * math.pi * 0.12 ** 3
            s = (n_target / (vol0 * side ** 3 * ppc)) ** (1 / 3)
            r = 0.12 * s
            c = np.array([0.5, 0.5, 0.5])
            x = jitter_fill(c - r, c + r, h, ppc, sphere(c, r), srng)
            g = make_group(snow(), x, h, ppc, (0.0, -2.0, 0.0))
        else:
            vol0 = 0.3 * 0.6 * 0.3
            s = (n_target / (vol0 * side ** 3 * ppc)) ** (1 / 3)
            ext = np.array([0.3, 0.6, 0.3]) * s
            lo = np.array([0.1, 0.1, 0.5 - ext[2] / 2])
            x = jitter_fill(lo, lo + ext, h, ppc, box(lo, lo + ext), srng)
            g = make_group(water(), x, h, ppc, (0.0, 0.0, 0.0))
        scenes.append(Scene(dim=3, n=(side,) * 3, h=h, dt=1e-4, groups=[g], bc_type=L.BC_SLIP,
                            bc_lo=3, bc_hi=3, name=f"c4_{i}_{['jello', 'snow', 'water'][kind]}"))
    return scenes


WORKLOADS = {
    "c0": c0_jello2d,
    "c1": c1_jello3d,
    "c2": c2_snow3d,
    "c3": c3_jello3d,
}


# ------------------------------------------------------------ parity scenes

def perturbed_blob(dim: int, mat: MaterialParams, n_grid: int = 48, h: float = 1.0 / 64,
                   ppc: int = 2, radius_cells: float = 6.0, seed: int = 7, amp_F: float = 0.05,
                   amp_C: float = 2.0, v0=(0.3, -0.5, 0.2), center=None):
    """A small sphere of particles with random velocities, affine matrices and
    deformation gradients near identity (so one substep exercises every term
    of P2G, the stress and G2P).  Returns (x, v, C, F, aux) float64 arrays."""
    rng = np.random.default_rng(seed)
    if center is None:
        center = np.full(dim, n_grid * h / 2)
    center = np.asarray(center, dtype=np.float64)
    r = radius_cells * h
    x = jitter_fill(center - r, center + r, h, ppc, sphere(center, r), rng).astype(np.float64)
    n = x.shape[0]
    v = np.asarray(v0[:dim]) + 0.2 * rng.standard_normal((n, dim))
    C = amp_C * rng.standard_normal((n, dim, dim))
    F = np.eye(dim) + amp_F * rng.standard_normal((n, dim, dim))
    if mat.type == L.SNOW:
        aux = 1.0 + 0.02 * rng.standard_normal(n)
    elif mat.type == L.WATER:
        aux = 1.0 + 0.01 * rng.standard_normal(n)
    else:
        aux = np.ones(n)
    return x, v, C, F, aux
