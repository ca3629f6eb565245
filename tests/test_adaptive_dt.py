"""Adaptive dt (MPM_P2G_ATOMIC): the next substep's dt is chosen on the device
from the CFL bound of the fastest signal (|v| + material wave speed)."""
import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def test_stiff_2d_jello_stays_bounded(gpu):
    # E = 1e4 at rho = 1, dx = 1/128 has wave speed ~105 m/s: the fixed
    # dt = 1e-4 breaks the CFL bound (the FP64 oracle diverges, see
    # test_oracle.py); with adaptive dt the substeps shrink and stay bounded
    sc = S.c0_jello2d(E=1e4)
    with Simulation([sc], adaptive_dt=True, cfl=0.5) as sim:
        t0, dt0 = sim.scene_time(0)
        assert t0 == 0.0 and dt0 < 1e-4
        assert sim.step_status(400) == L.OK
        st = sim.get_state(0)
        t, dt = sim.scene_time(0)
    c = np.sqrt((1e4 * 0.2 / (1.2 * 0.6) + 2 * 1e4 / 2.4) / 1.0)
    assert dt <= 0.5 * sc.h / c * 1.0001
    assert 0 < t < 400 * 1e-4
    assert np.isfinite(st["x"]).all() and float(np.abs(st["v"]).max()) < 10.0


def test_matches_fixed_dt_when_the_bound_does_not_bind(gpu):
    # E = 1e3: cfl h / (|v| + c) > 1e-4, so every substep takes dt_max and the
    # run follows the fixed-dt run (up to the order of float atomics)
    sc = S.c0_jello2d()
    with Simulation([sc]) as fixed, Simulation([sc], adaptive_dt=True) as sim:
        fixed.step(30)
        sim.step(30)
        t, dt = sim.scene_time(0)
        a, b = fixed.get_state(0), sim.get_state(0)
    assert dt == np.float32(1e-4)
    assert abs(t - 30 * float(np.float32(1e-4))) < 1e-12
    assert float(np.abs(a["x"] - b["x"]).max()) < 1e-5
    assert float(np.abs(a["v"] - b["v"]).max()) < 1e-3


def test_fast_particles_shrink_dt_and_time_adds_up(gpu):
    sc = S.c1_jello3d(n_grid=64, edge=0.2)
    sc.groups[0].init_v = (0.0, -40.0, 0.0)
    with Simulation([sc], adaptive_dt=True, cfl=0.4) as sim:
        _, dt0 = sim.scene_time(0)
        assert dt0 < 0.4 * sc.h / 40.0
        total = 0.0
        for _ in range(5):
            t, dt = sim.scene_time(0)
            sim.step(1)
            total += dt
        t, _ = sim.scene_time(0)
        assert abs(t - total) < 1e-9
        assert sim.time()[0] == t


def test_adaptive_needs_the_binned_path(gpu):
    sc = S.c0_jello2d()
    with pytest.raises(L.MPMError) as e:
        Simulation([sc], p2g_mode=L.P2G_DIRECT, adaptive_dt=True)
    assert e.value.code == L.ERR_UNSUPPORTED
    with Simulation([sc], adaptive_dt=True) as sim:
        with pytest.raises(L.MPMError) as e:
            sim.set_p2g_mode(L.P2G_DETERMINISTIC)
        assert e.value.code == L.ERR_UNSUPPORTED


@pytest.mark.parametrize("d", [2, 3])
def test_the_chosen_dt_sequence_replays_through_the_fp64_oracle(gpu, d):
    """The dt the device chose for every substep (read between substeps),
    fed to the FP64 oracle substep by substep, reproduces the state: the
    adaptive path differs from a fixed-dt run only in its dt sequence.  The
    scene is a blob with perturbed v, C and F of a stiff, light jello, so the
    wave speed binds dt below the scene's dt and the particles' speeds move it."""
    from mpm_cuda_b200.sim import Scene
    from helpers import compare, group_from_arrays, oracle_for
    mat = S.jello(E=5e4, nu=0.3, rho=1.0)
    h, n_grid = 1.0 / 32, 32
    x, v, C_, F, aux = S.perturbed_blob(d, mat, n_grid=n_grid, h=h, ppc=2, radius_cells=5.0, seed=31,
                                        center=np.full(d, 0.5))
    sc = Scene(dim=d, n=(n_grid,) * d, h=h, dt=1e-4, groups=[group_from_arrays(mat, h, 2, x, v, C_, F, aux)],
               bc_type=L.BC_SLIP, bc_lo=3, bc_hi=3, gravity=(0.0, -9.8, 0.0)[:d] if d == 3 else (0.0, -9.8))
    orc = oracle_for(sc)
    dts = []
    with Simulation([sc], adaptive_dt=True, cfl=0.5, rebin_interval=4) as sim:
        for _ in range(24):
            dts.append(sim.scene_time(0)[1])
            assert sim.step_status(1) == L.OK
        got = sim.get_state(0)
    assert len(set(dts)) > 1 and max(dts) < 1e-4, dts  # the bound binds and varies
    for dt in dts:
        orc.grid.dt = dt
        assert orc.step(1) == 0
    compare(got, orc.state(), {"x": 1e-5, "v": 2e-3, "C": 2e-3, "F": 1e-4, "aux": 1e-4})
