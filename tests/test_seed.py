"""Particle seeding on the GPU (mpm_seed): counts follow the object's volume,
every sample lies inside the object and inside its lattice cell, output is
deterministic for a seed, a triangle mesh of a shape seeds like the analytic
shape, and the positions equal the CPU restatement's (oracle.cpu.seed_positions)
bit for bit."""
import ctypes as C

import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L


def _obj(shape=L.SHAPE_CUBE):
    o = L.SeedObject()
    o.shape = shape
    o.rotation = (C.c_double * 9)(1, 0, 0, 0, 1, 0, 0, 0, 1)
    o.scale = (C.c_double * 3)(1, 1, 1)
    return o


def test_argument_checks_run_on_the_host():
    lib = L.load()
    n = C.c_int64()
    o = _obj()
    assert lib.mpm_seed(C.byref(o), 3, 0.01, None, 0, 1, 0, None, 0, C.byref(n)) == L.ERR_INVALID   # ppc
    assert lib.mpm_seed(C.byref(o), 4, 0.01, None, 8, 1, 0, None, 0, C.byref(n)) == L.ERR_INVALID   # dim
    assert lib.mpm_seed(C.byref(o), 3, 0.0, None, 8, 1, 0, None, 0, C.byref(n)) == L.ERR_INVALID    # h
    o.scale = (C.c_double * 3)(1, 0, 1)
    assert lib.mpm_seed(C.byref(o), 3, 0.01, None, 8, 1, 0, None, 0, C.byref(n)) == L.ERR_INVALID   # scale
    m = _obj(L.SHAPE_MESH)
    v = np.zeros((3, 3), np.float32)
    t = np.array([[0, 1, 7]], np.int32)
    m.vertices, m.n_vertices = L.fptr(v), 3
    m.triangles, m.n_triangles = t.ctypes.data_as(C.POINTER(C.c_int32)), 1
    assert lib.mpm_seed(C.byref(m), 3, 0.01, None, 8, 1, 0, None, 0, C.byref(n)) == L.ERR_INVALID   # index


def local_of(p, R, S, T):
    return ((p - np.asarray(T)) / np.asarray(S)) @ R  # R^T q, row vectors


@pytest.mark.gpu
def test_cube_sphere_cylinder_counts_and_containment(gpu):
    from mpm_cuda_b200.seed import rotation, seed
    h, ppc = 1.0 / 128, 8
    R = rotation((1.0, 2.0, 0.5), 30.0)
    T, S = (0.5, 0.6, 0.5), (0.3, 0.2, 0.25)
    for shape, vol, inside in (
            ("cube", 1.0, lambda l: np.all(np.abs(l) <= 0.5 + 1e-6, axis=1)),
            ("sphere", np.pi / 6, lambda l: np.sum(l * l, axis=1) <= 0.25 + 1e-6),
            ("cylinder", np.pi / 4, lambda l: (l[:, 0] ** 2 + l[:, 2] ** 2 <= 0.25 + 1e-6) &
                                             (np.abs(l[:, 1]) <= 0.5 + 1e-6))):
        p = seed(shape, h, ppc, translation=T, scale=S, rot=R, seed_value=7)
        expect = vol * np.prod(S) / h ** 3 * ppc
        assert abs(len(p) - expect) < 0.01 * expect, (shape, len(p), expect)
        assert inside(local_of(p.astype(np.float64), R, S, T)).all(), shape
        # cell order: the lattice cell index never decreases along the output
        cell = np.floor(p.astype(np.float64) / h).astype(np.int64)
        lin = (cell[:, 0] * 4096 + cell[:, 1]) * 4096 + cell[:, 2]
        assert np.all(np.diff(lin) >= 0), shape
        assert np.max(np.bincount(lin - lin.min())) <= ppc
        q = seed(shape, h, ppc, translation=T, scale=S, rot=R, seed_value=7)
        assert np.array_equal(p, q)
        assert not np.array_equal(p[:100], seed(shape, h, ppc, translation=T, scale=S, rot=R, seed_value=8)[:100])


def cube_mesh():
    v = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = np.array([[a, b, c] for a, b, c, d in quads] + [[a, c, d] for a, b, c, d in quads], np.int32)
    return v, t


@pytest.mark.gpu
def test_mesh_seeds_like_the_analytic_shape(gpu):
    from mpm_cuda_b200.seed import rotation, seed
    h, ppc = 1.0 / 96, 4
    R = rotation((0.3, 1.0, 0.2), 17.0)
    kw = dict(translation=(0.5, 0.5, 0.5), scale=(0.4, 0.3, 0.35), rot=R, seed_value=3)
    v, t = cube_mesh()
    a = seed("cube", h, ppc, **kw)
    m = seed("mesh", h, ppc, vertices=v, triangles=t, **kw)
    assert len(a) > 10000
    assert len(m) == len(a) and np.array_equal(m, a)


@pytest.mark.gpu
def test_tetrahedron_mesh(gpu):
    from mpm_cuda_b200.seed import seed
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32) - 0.25
    t = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    h, ppc = 1.0 / 128, 8
    p = seed("mesh", h, ppc, vertices=v, triangles=t, translation=(0.5, 0.5, 0.5), scale=(0.5, 0.5, 0.5))
    l = (p.astype(np.float64) - 0.5) / 0.5 + 0.25
    assert np.all(l >= -1e-6) and np.all(l.sum(axis=1) <= 1.0 + 1e-6)
    expect = (1 / 6) * 0.125 / h ** 3 * ppc
    assert abs(len(p) - expect) < 0.01 * expect


@pytest.mark.gpu
def test_2d_square(gpu):
    from mpm_cuda_b200.seed import seed
    p = seed("cube", 1.0 / 128, 4, translation=(0.5, 0.6), scale=(0.2, 0.2, 1.0), dim=2)
    assert p.shape[1] == 2
    assert np.all(np.abs(p - np.array([0.5, 0.6], np.float32)) <= 0.1 + 1e-6)
    assert abs(len(p) - 0.04 * 128 ** 2 * 4) < 0.01 * 0.04 * 128 ** 2 * 4


# ------------------------------------------------- against the CPU restatement

def _cases():
    from mpm_cuda_b200.seed import rotation
    R = rotation((1.0, 2.0, 0.5), 30.0)
    v, t = cube_mesh()
    tv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32) - 0.25
    tt = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    return [
        ("cube", dict(h=1.0 / 128, ppc=8, translation=(0.5, 0.6, 0.5), scale=(0.3, 0.2, 0.25), rot=R, seed_value=7)),
        ("sphere", dict(h=1.0 / 100, ppc=8, translation=(0.45, 0.5, 0.55), scale=(0.3, 0.3, 0.3), rot=R,
                        seed_value=9, origin=(0.01, -0.02, 0.0))),
        ("cylinder", dict(h=1.0 / 96, ppc=4, translation=(0.5, 0.5, 0.5), scale=(0.2, 0.4, 0.2), rot=R, seed_value=3)),
        ("mesh", dict(h=1.0 / 96, ppc=4, translation=(0.5, 0.5, 0.5), scale=(0.4, 0.3, 0.35),
                      rot=rotation((0.3, 1.0, 0.2), 17.0), seed_value=3, vertices=v, triangles=t)),
        ("mesh", dict(h=1.0 / 128, ppc=8, translation=(0.5, 0.5, 0.5), scale=(0.5, 0.5, 0.5), seed_value=5,
                      vertices=tv, triangles=tt)),
        ("cube", dict(h=1.0 / 128, ppc=4, translation=(0.5, 0.6), scale=(0.2, 0.2, 1.0), dim=2, seed_value=11)),
    ]


def test_restatement_counts_and_containment():
    """The CPU restatement alone: counts follow the volume, samples lie in
    the object and in their lattice cell, cell order."""
    from oracle import cpu as ocpu
    for shape, kw in _cases():
        p = ocpu.seed_positions(shape, **kw).astype(np.float64)
        d = kw.get("dim", 3)
        h, ppc = kw["h"], kw["ppc"]
        S = np.asarray(kw["scale"], np.float64)[:d]
        vol = {"cube": 1.0, "sphere": np.pi / 6, "cylinder": np.pi / 4}.get(shape)
        if vol is None:  # meshes: the unit cube or the tetrahedron of volume 1/6
            vol = 1.0 if len(kw["vertices"]) == 8 else 1.0 / 6
        expect = vol * np.prod(S) / h ** d * ppc
        assert abs(len(p) - expect) < 0.015 * expect, (shape, len(p), expect)
        org = np.asarray(kw.get("origin", (0.0, 0.0, 0.0)), np.float64)[:d]
        cell = np.floor((p - org) / h).astype(np.int64)
        lin = cell[:, 0] * (1 << 40) + cell[:, 1] * (1 << 20) + (cell[:, 2] if d == 3 else 0)
        assert np.all(np.diff(lin) >= 0), shape


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(6))
def test_gpu_seeding_is_bit_identical_to_the_restatement(gpu, case):
    from mpm_cuda_b200.seed import seed
    from oracle import cpu as ocpu
    shape, kw = _cases()[case]
    got = seed(shape, **kw)
    want = ocpu.seed_positions(shape, **kw)
    assert len(got) > 1000
    assert got.shape == want.shape and np.array_equal(got.view(np.uint32), want.view(np.uint32)), shape
