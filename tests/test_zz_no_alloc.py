"""mpm_step_noalloc: substeps for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc: plug-in hosts that hand
out a fixed device memory budget, real-time loops that forbid allocator calls
after start-up.  mpm_step_noalloc serves them: it steps a scene whose particle state
lives in device memory the caller already owns, and keeps the grid in a fixed
scratch array compiled into the library.  These tests check it against the
handle-based entry point (mpm_create + mpm_step) and the FP64 oracle on two
calls in a row, a call of two substeps (the grid is cleared between the
substeps of one call), that a particle outside the grid sets the error word,
and that grids larger than the scratch are refused.

This file is collected last, so a run that stops at the first failure has run
every other test before it; it also passes when run alone in a new process.
"""
import ctypes as C

import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200.sim import Scene, Simulation, scene_descs

from helpers import TOL_STEP, compare, group_from_arrays, oracle_for

MATS = {"jello": S.jello(), "snow": S.snow(), "water": S.water()}


def _scene(d, name, seed, n_grid=32):
    h = 1.0 / n_grid
    x, v, Cm, F, aux = S.perturbed_blob(d, MATS[name], n_grid=n_grid, h=h, ppc=2, radius_cells=5.0, seed=seed,
                                        center=np.full(d, n_grid / 2 * h))
    g = group_from_arrays(MATS[name], h, 2, x, v, Cm, F, aux)
    grav = (0.0, -9.8, 0.0) if d == 3 else (0.0, -9.8)
    return Scene(dim=d, n=(n_grid,) * d, h=h, dt=1e-4, groups=[g], gravity=grav)


def _to_planes(g, d):
    """The handle's device plane layout: x[d], v[d], C[d*d], F[d*d], aux."""
    n = g.n
    cols = [g.x.reshape(n, d), g.v.reshape(n, d), g.C.reshape(n, d * d), g.F.reshape(n, d * d),
            g.aux.reshape(n, 1)]
    return np.ascontiguousarray(np.concatenate(cols, axis=1).T.astype(np.float32))


def _from_planes(p, d):
    n = p.shape[1]
    o = 0
    out = {}
    for key, k, shape in (("x", d, (n, d)), ("v", d, (n, d)), ("C", d * d, (n, d, d)), ("F", d * d, (n, d, d)),
                          ("aux", 1, (n,))):
        out[key] = p[o:o + k].T.reshape(shape).copy()
        o += k
    return out


def _caller_state(sc, d):
    import torch
    return torch.from_numpy(_to_planes(sc.groups[0], d)).to("cuda:0").contiguous()


def _call(lib, sc, dev, n_substeps):
    descs, keep = scene_descs([sc])
    import torch
    stream = torch.cuda.current_stream(0).cuda_stream
    n = sc.groups[0].n
    return lib.mpm_step_noalloc(descs, C.c_void_p(dev.data_ptr()), n, n, n_substeps, C.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("d,name", [(3, "jello"), (3, "snow"), (3, "water"), (2, "jello"), (2, "snow"),
                                    (2, "water")])
def test_noalloc_matches_handle_entry_point_on_two_calls_in_a_row(gpu, d, name):
    sc = _scene(d, name, seed=100 + d)
    orc = oracle_for(sc)
    with Simulation([sc]) as sim:
        sim.step(1)
        ref1 = sim.get_state(0)
        sim.step(1)
        ref2 = sim.get_state(0)

    # the caller owns the particle state on the device
    dev = _caller_state(sc, d)
    lib = L.load()
    for ref in (ref1, ref2):
        rc = _call(lib, sc, dev, 1)
        assert rc == L.OK, L.last_error()
        got = _from_planes(dev.cpu().numpy(), d)
        compare(got, ref, TOL_STEP)
        # and directly against the FP64 oracle, substep by substep
        assert orc.step(1) == 0
        compare(got, orc.state(), TOL_STEP)


@pytest.mark.gpu
@pytest.mark.parametrize("d,name", [(3, "jello"), (2, "snow")])
def test_noalloc_two_substeps_in_one_call(gpu, d, name):
    sc = _scene(d, name, seed=200 + d)
    with Simulation([sc]) as sim:
        sim.step(2)
        ref = sim.get_state(0)
    dev = _caller_state(sc, d)
    rc = _call(L.load(), sc, dev, 2)
    assert rc == L.OK, L.last_error()
    compare(_from_planes(dev.cpu().numpy(), d), ref, TOL_STEP)


@pytest.mark.gpu
def test_noalloc_particle_outside_the_grid_sets_the_error_word(gpu):
    # a particle placed outside the grid on the host: the kernels' own stencil
    # check skips it and records the out-of-grid bit, which the call reports
    sc = _scene(3, "jello", seed=7)
    sc.groups[0].x[0] = np.float32([2.0, 0.5, 0.5])
    dev = _caller_state(sc, 3)
    rc = _call(L.load(), sc, dev, 1)
    assert rc == L.ERR_SIM
    msg = L.last_error()
    bits = int(msg.rsplit("0x", 1)[1].split()[0], 16)
    assert bits & L.DEVERR_OUT_OF_GRID, msg
    # the next call starts from a cleared error word
    sc2 = _scene(3, "jello", seed=8)
    dev2 = _caller_state(sc2, 3)
    assert _call(L.load(), sc2, dev2, 1) == L.OK, L.last_error()


def test_noalloc_rejects_grids_larger_than_its_scratch():
    # 128^3 nodes need 2,097,152 nodes; the scratch holds 262,144.  The check
    # runs before any CUDA call, so this needs no GPU.
    sc = S.c1_jello3d(n_grid=128, edge=0.1)
    descs, keep = scene_descs([sc])
    lib = L.load()
    rc = lib.mpm_step_noalloc(descs, None, 0, 0, 1, None)
    assert rc == L.ERR_INVALID
    msg = L.last_error()
    assert "2097152" in msg and "262144" in msg
