"""Paged grid (mpm_options.grid_pool_blocks > 0): the grid arrays are a pool of
64-node blocks assigned on the device to the blocks particles reach and
returned when nothing is active near them.  The CUDA path with a paged grid
tracks the FP64 oracle like the dense one, follows the dense grid over many
substeps, keeps its pages near the particles as they move, and reports a pool
that runs out instead of touching memory outside it."""
import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200.sim import Scene, Simulation

from helpers import TOL_STEP, compare, group_from_arrays, oracle_for

pytestmark = pytest.mark.gpu

MATS = {"jello": S.jello(), "snow": S.snow(), "water": S.water()}


def blob(d, name, seed=3, n_grid=32, v0=(0.3, -0.5, 0.2)):
    h = 1.0 / n_grid
    mat = MATS[name]
    x, v, C, F, aux = S.perturbed_blob(d, mat, n_grid=n_grid, h=h, ppc=2, radius_cells=5.0, seed=seed,
                                       center=np.full(d, n_grid / 2 * h), v0=v0)
    g = group_from_arrays(mat, h, 2, x, v, C, F, aux)
    return Scene(dim=d, n=(n_grid,) * d, h=h, dt=1e-4, groups=[g], bc_type=L.BC_SLIP, bc_lo=3, bc_hi=3,
                 gravity=(0.0, -9.8, 0.0)[:d] if d == 3 else (0.0, -9.8))


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("name", ["jello", "snow", "water"])
def test_paged_grid_tracks_the_oracle(gpu, d, name):
    sc = blob(d, name)
    orc = oracle_for(sc)
    with Simulation([sc], grid_pool_blocks=256, rebin_interval=3) as sim:
        sim.step(1)
        one = sim.get_state(0)
        assert orc.step(1) == 0
        compare(one, orc.state(), TOL_STEP)
        sim.step(19)
        got = sim.get_state(0)
        assert sim.device_errors() == 0
        cap, used = sim.grid_pool()
    assert orc.step(19) == 0
    compare(got, orc.state(), {"x": 1e-5, "v": 2e-3, "C": 2e-3, "F": 1e-4, "aux": 1e-4})
    blocks = (32 // 4) ** 3 if d == 3 else (32 // 8) ** 2
    assert cap == min(256, blocks) and 0 < used <= cap


def test_every_paged_configuration_tracks_the_oracle(gpu):
    import ctypes as C
    lib = L.load()
    sc = blob(3, "jello", seed=24)
    orc = oracle_for(sc)
    assert orc.step(6) == 0
    ref = orc.state()
    for k in range(lib.mpm_num_kernel_configs()):
        cm, sg = C.c_int(), C.c_int()
        assert lib.mpm_kernel_config_scatter(k, C.byref(cm), C.byref(sg)) == L.OK
        if sg.value:
            with pytest.raises(L.MPMError) as e:
                Simulation([sc], kernel_config=k, grid_pool_blocks=256)
            assert e.value.code == L.ERR_UNSUPPORTED
            continue
        with Simulation([sc], kernel_config=k, rebin_interval=3, grid_pool_blocks=256) as sim:
            sim.step(6)
            compare(sim.get_state(0), ref, {"x": 5e-6, "v": 6e-4, "C": 6e-4, "F": 4e-5, "aux": 4e-5})


def test_paged_grid_follows_the_dense_grid(gpu):
    # 300 substeps of the 64^3 jello scene: the two grids differ only in the
    # order of float atomics; the grid itself reads back the same
    sc = S.c1_jello3d(n_grid=64, edge=0.3)
    with Simulation([sc]) as dense, Simulation([sc], grid_pool_blocks=4096) as paged:
        dense.step(300)
        paged.step(300)
        a, b = dense.get_state(0), paged.get_state(0)
        ma, va = dense.get_grid(0)
        mb, vb = paged.get_grid(0)
        assert paged.device_errors() == 0
        cap, used = paged.grid_pool()
        assert dense.grid_pool()[0] == 16 ** 3
    assert float(np.abs(a["x"] - b["x"]).max()) < 1e-5
    assert float(np.abs(a["v"] - b["v"]).max()) < 1e-3
    assert np.allclose(ma, mb, rtol=1e-4, atol=1e-9)
    # momentum, not velocity: a node with little mass divides round-off by it
    pa, pb = ma[:, None] * va, mb[:, None] * vb
    assert float(np.abs(pa - pb).max()) <= 1e-3 * float(np.abs(pa).max())
    assert used < 16 ** 3 // 2, used  # the cube and its surroundings, not the domain


def test_pages_follow_a_moving_object(gpu):
    # a blob crossing the domain at 15 m/s: blocks behind it are returned, so
    # the pages in use stay near the count the blob needs
    sc = blob(3, "jello", n_grid=64, v0=(15.0, 0.0, 0.0))
    for g in sc.groups:
        g.x[:, 0] -= np.float32(0.3)
    sc.gravity = (0.0, 0.0, 0.0)
    with Simulation([sc], grid_pool_blocks=600) as sim:
        sim.step(2)
        _, first = sim.grid_pool()
        x0 = sim.get_state(0)["x"][:, 0].mean()
        peak = first
        for _ in range(12):
            sim.step(16)
            peak = max(peak, sim.grid_pool()[1])
        x1 = sim.get_state(0)["x"][:, 0].mean()
        assert sim.device_errors() == 0
    assert x1 - x0 > 0.25  # moved across a quarter of the domain (16 blocks)
    assert peak < 2.5 * first, (first, peak)


def test_a_pool_that_runs_out_is_reported(gpu):
    sc = blob(3, "jello")
    with Simulation([sc], grid_pool_blocks=4) as sim:
        assert sim.step_status(2) == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_POOL
        cap, used = sim.grid_pool()
        assert cap == 4 and used == 4


def test_paged_grid_refuses_dense_paths(gpu):
    sc = blob(3, "jello")
    with Simulation([sc], grid_pool_blocks=256) as sim:
        for mode in (L.P2G_DIRECT, L.P2G_DETERMINISTIC):
            with pytest.raises(L.MPMError) as e:
                sim.set_p2g_mode(mode)
            assert e.value.code == L.ERR_UNSUPPORTED


def test_paged_grid_with_the_learned_stress_kernel(gpu):
    # an untrained network: every particle falls back to the decomposition,
    # so the learned-stress kernel must match the plain kernel on a paged grid
    from mpm_cuda_b200.surrogate import StressSurrogate
    sur = StressSurrogate(seed=1)
    sc = blob(3, "jello", seed=5)
    with Simulation([sc], grid_pool_blocks=256) as plain, Simulation([sc], grid_pool_blocks=256) as sim:
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        plain.step(3)
        sim.step(3)
        compare(sim.get_state(0), plain.get_state(0), TOL_STEP)
    sur.close()
