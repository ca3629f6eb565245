"""Particle seeding on the GPU (mpm_seed): jittered samples per lattice cell
kept inside a unit shape or a closed triangle mesh placed in the world."""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

SHAPES = {"cube": L.SHAPE_CUBE, "sphere": L.SHAPE_SPHERE, "cylinder": L.SHAPE_CYLINDER, "mesh": L.SHAPE_MESH}


def rotation(axis: Sequence[float] = (0.0, 1.0, 0.0), degrees: float = 0.0) -> np.ndarray:
    """Rodrigues rotation about `axis` by `degrees` (the reference's
    glm::rotate, model.cpp:202-207)."""
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    t = math.radians(degrees)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(t) * K + (1 - math.cos(t)) * (K @ K)


def seed(shape: str, h: float, ppc: int, *, translation=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0),
         rot: Optional[np.ndarray] = None, origin=(0.0, 0.0, 0.0), dim: int = 3, seed_value: int = 1234,
         vertices: Optional[np.ndarray] = None, triangles: Optional[np.ndarray] = None,
         device: int = 0) -> np.ndarray:
    """Positions (n, dim) float32 of one seeded object, in cell order."""
    lib = L.load()
    obj = L.SeedObject()
    obj.shape = SHAPES[shape]
    R = np.eye(3) if rot is None else np.asarray(rot, np.float64)
    obj.rotation = (C.c_double * 9)(*R.ravel().tolist())
    obj.scale = (C.c_double * 3)(*[float(v) for v in scale])
    obj.translation = (C.c_double * 3)(*[float(v) for v in list(translation) + [0.0] * (3 - len(translation))])
    keep = []
    if shape == "mesh":
        v = np.ascontiguousarray(vertices, np.float32)
        t = np.ascontiguousarray(triangles, np.int32)
        keep += [v, t]
        obj.vertices = L.fptr(v)
        obj.n_vertices = v.shape[0]
        obj.triangles = t.ctypes.data_as(C.POINTER(C.c_int32))
        obj.n_triangles = t.shape[0]
    org = (C.c_double * 3)(*[float(o) for o in list(origin) + [0.0] * (3 - len(origin))])
    n = C.c_int64()
    L.check(lib.mpm_seed(C.byref(obj), dim, h, org, ppc, seed_value, device, None, 0, C.byref(n)))
    out = np.empty((n.value, dim), np.float32)
    if n.value:
        L.check(lib.mpm_seed(C.byref(obj), dim, h, org, ppc, seed_value, device, L.fptr(out), out.size,
                             C.byref(n)))
    return out
