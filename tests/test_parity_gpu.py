"""GPU parity of the CUDA substep (through the C ABI) against the FP64 CPU
oracle and the reference build's golden fixtures."""
import glob
import os

import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200.sim import Scene, Simulation

from helpers import (TOL_REF, TOL_STEP, check_snow_f_percentile, compare, golden_tolerance, group_from_arrays,
                     oracle_for, rel_err)

pytestmark = pytest.mark.gpu

MATS = {"jello": S.jello(), "snow": S.snow(), "water": S.water()}
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def blob_scene(d, name, bc=L.BC_SLIP, seed=3, n_grid=32, h=1.0 / 32, ppc=2, radius=5.0, **kw):
    mat = MATS[name]
    x, v, C, F, aux = S.perturbed_blob(d, mat, n_grid=n_grid, h=h, ppc=ppc, radius_cells=radius, seed=seed,
                                       center=np.full(d, n_grid / 2 * h))
    g = group_from_arrays(mat, h, ppc, x, v, C, F, aux)
    return Scene(dim=d, n=(n_grid,) * d, h=h, dt=1e-4, groups=[g], bc_type=bc, bc_lo=3, bc_hi=3,
                 gravity=(0.0, -9.8, 0.0)[:d] if d == 3 else (0.0, -9.8), **kw)


MODES = [L.P2G_ATOMIC, L.P2G_DIRECT, L.P2G_DETERMINISTIC]
MODE_IDS = ["binned", "direct", "deterministic"]


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("name", ["jello", "snow", "water"])
def test_one_substep_matches_oracle(gpu, d, name, mode):
    sc = blob_scene(d, name)
    orc = oracle_for(sc)
    with Simulation([sc], p2g_mode=mode) as sim:
        sim.step(1)
        got = sim.get_state(0)
    assert orc.step(1) == 0
    compare(got, orc.state(), TOL_STEP)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("bc", [L.BC_STICKY, L.BC_SLIP, L.BC_SEPARATE])
def test_boundaries_match_oracle(gpu, d, bc, mode):
    # blob pushed into the lower x wall band so every boundary branch runs
    sc = blob_scene(d, "jello", bc=bc, seed=4)
    g = sc.groups[0]
    g.x[:, 0] -= np.float32(10 * sc.h)
    g.v[:, 0] = -np.abs(g.v[:, 0]) - 1.0
    sc.bc_lo, sc.bc_hi = 8, 3
    orc = oracle_for(sc)
    with Simulation([sc], p2g_mode=mode) as sim:
        sim.step(1)
        got = sim.get_state(0)
        mass, vel = sim.get_grid(0)
    assert orc.step(1) == 0
    compare(got, orc.state(), TOL_STEP)
    ref_vel = orc.mom.reshape(-1, 3)[:, :d]
    assert rel_err(vel, ref_vel) < 1e-4
    assert rel_err(mass, orc.mass) < 1e-5


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_grid_matches_oracle(gpu, mode):
    sc = blob_scene(3, "snow", seed=8)
    orc = oracle_for(sc)
    with Simulation([sc], p2g_mode=mode) as sim:
        sim.step(1)
        mass, vel = sim.get_grid(0)
        active = sim.count_active_nodes(0)
    orc.step(1)
    assert rel_err(mass, orc.mass) < 1e-5
    assert rel_err(vel, orc.mom.reshape(-1, 3)) < 1e-4
    assert active == int((orc.mass > 0).sum())


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("name", ["jello", "snow", "water"])
def test_twenty_substeps_track_oracle(gpu, name, mode):
    sc = blob_scene(3, name, seed=21)
    orc = oracle_for(sc)
    with Simulation([sc], p2g_mode=mode, rebin_interval=4) as sim:
        sim.step(20)
        got = sim.get_state(0)
    assert orc.step(20) == 0
    tol = {"x": 1e-5, "v": 2e-3, "C": 2e-3, "F": 1e-4, "aux": 1e-4}
    compare(got, orc.state(), tol)


@pytest.mark.parametrize("d,name", [(3, "jello"), (3, "snow"), (3, "water"), (2, "jello")])
def test_every_kernel_config_tracks_oracle(gpu, d, name):
    """Every launch configuration of the fused kernel, including those whose
    threads take two particles of a chunk in turn, gives the oracle's state."""
    import ctypes as C
    lib = L.load()
    sc = blob_scene(d, name, seed=24, ppc=4)  # 3D: ~250 particles per block: partial second rounds
    orc = oracle_for(sc)
    assert orc.step(6) == 0
    ref = orc.state()
    rounds_seen = set()
    for k in range(lib.mpm_num_kernel_configs()):
        rd = C.c_int()
        assert lib.mpm_kernel_config_info(k, None, None, C.byref(rd)) == L.OK
        rounds_seen.add(rd.value)
        with Simulation([sc], kernel_config=k, rebin_interval=3) as sim:
            sim.step(6)
            assert sim.kernel_config() == k
            compare(sim.get_state(0), ref, {"x": 5e-6, "v": 6e-4, "C": 6e-4, "F": 4e-5, "aux": 4e-5})
    assert rounds_seen >= {1, 2}


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_multi_scene_batch_matches_single(gpu, mode):
    scs = [blob_scene(3, "jello", seed=30), blob_scene(3, "snow", seed=31, n_grid=40, h=1.0 / 40),
           blob_scene(3, "water", seed=32, n_grid=24, h=1.0 / 24)]
    with Simulation(scs, p2g_mode=mode, rebin_interval=2) as sim:
        sim.step(3)
        batched = [sim.get_state(i) for i in range(3)]
    for i, sc in enumerate(scs):
        orc = oracle_for(sc)
        assert orc.step(3) == 0
        compare(batched[i], orc.state(), {"x": 5e-6, "v": 5e-4, "C": 5e-4, "F": 3e-5, "aux": 3e-5})


def test_deterministic_batch_equals_single_scenes_bitwise(gpu):
    # deterministic P2G sums every node in an order fixed by the sort (global
    # node keys, stable in creation order) and the stencil offsets, so a scene
    # batched with others gives bitwise the same state and grid as alone
    scs = [blob_scene(3, "jello", seed=33), blob_scene(3, "snow", seed=34, n_grid=40, h=1.0 / 40),
           blob_scene(3, "water", seed=35, n_grid=24, h=1.0 / 24)]
    with Simulation(scs, p2g_mode=L.P2G_DETERMINISTIC) as sim:
        sim.step(4)
        batched = [(sim.get_state(i), sim.get_grid(i)) for i in range(3)]
    for i, sc in enumerate(scs):
        with Simulation([sc], p2g_mode=L.P2G_DETERMINISTIC) as one:
            one.step(4)
            st, gr = one.get_state(0), one.get_grid(0)
        for k in ("x", "v", "C", "F", "aux"):
            assert np.array_equal(batched[i][0][k], st[k]), (i, k)
        assert np.array_equal(batched[i][1][0], gr[0]) and np.array_equal(batched[i][1][1], gr[1]), i


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_mixed_groups_in_one_grid(gpu, mode):
    a = blob_scene(3, "jello", seed=40)
    b = blob_scene(3, "water", seed=41)
    for g in b.groups:
        g.x[:, 0] += np.float32(3 * a.h)
    a.groups += b.groups
    orc = oracle_for(a)
    with Simulation([a], p2g_mode=mode) as sim:
        sim.step(2)
        got = sim.get_state(0)
    assert orc.step(2) == 0
    compare(got, orc.state(), {"x": 5e-6, "v": 3e-4, "C": 3e-4, "F": 2e-5, "aux": 2e-5})


def test_graph_and_stream_paths_agree(gpu):
    sc = blob_scene(3, "jello", seed=50)
    with Simulation([sc], use_graph=True) as a, Simulation([sc], use_graph=False) as b:
        a.step(5)
        b.step(5)
        sa, sb = a.get_state(0), b.get_state(0)
    for k in ("x", "v", "C", "F"):
        assert rel_err(sa[k], sb[k]) < 1e-5


def test_set_get_state_roundtrip(gpu):
    sc = blob_scene(3, "snow", seed=60)
    with Simulation([sc]) as sim:
        st = sim.get_state(0)
        g = sc.groups[0]
        assert np.array_equal(st["x"], g.x)
        assert np.array_equal(st["F"], g.F)
        st["x"][:, 1] += np.float32(0.01)
        sim.set_state(0, x=st["x"])
        st2 = sim.get_state(0)
        assert np.array_equal(st2["x"], st["x"])
        assert np.array_equal(st2["C"], g.C)
        assert np.array_equal(sim.positions(0), st["x"])


def test_out_of_grid_particle_sets_error_word(gpu):
    sc = blob_scene(3, "jello", seed=70)
    sc.groups[0].x[0] = np.float32([0.995, 0.5, 0.5])
    with Simulation([sc]) as sim:
        rc = sim.step_status(1)
        assert rc == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_OUT_OF_GRID
        sim.clear_device_errors()
        assert sim.device_errors() == 0


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_far_outside_particle_sets_error_word(gpu, mode):
    # coordinates beyond the int range of node indices: the stencil check
    # must reject them without overflowing (base saturates to INT_MAX/INT_MIN)
    sc = blob_scene(3, "jello", seed=73)
    sc.groups[0].x[0] = np.float32([3e9, 0.5, 0.5])
    sc.groups[0].x[1] = np.float32([0.5, -3e9, 0.5])
    with Simulation([sc], p2g_mode=mode) as sim:
        assert sim.step_status(2) == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_OUT_OF_GRID
        st = sim.get_state(0)
    assert np.isfinite(st["x"][2:]).all()


def test_nan_particle_sets_error_word(gpu):
    sc = blob_scene(3, "jello", seed=71)
    sc.groups[0].x[3, 1] = np.float32(np.nan)
    with Simulation([sc]) as sim:
        assert sim.step_status(1) == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_NONFINITE


def test_inverted_water_sets_det_error(gpu):
    sc = blob_scene(3, "water", seed=72)
    sc.groups[0].aux[5] = np.float32(-0.5)
    with Simulation([sc]) as sim:
        assert sim.step_status(1) == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_DET


def test_write_bgeo_roundtrip(gpu, tmp_path):
    from test_bgeo import read_bgeo
    sc = blob_scene(3, "jello", seed=80)
    with Simulation([sc]) as sim:
        sim.step(2)
        p = str(tmp_path / "Frame000001.bgeo")
        sim.write_bgeo(p, 0)
        pos = sim.positions(0)
    assert np.array_equal(read_bgeo(p), pos)


# ------------------------------------------------ reference golden fixtures

def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref3d_*.npz")))


def golden_scene(z):
    h, dt, n = float(z["h"]), float(z["dt"]), int(z["n_grid"])
    groups = []
    for gi in range(int(z["n_groups"])):
        p = f"g{gi}_"
        t = int(z[p + "type"])
        if t == L.JELLO:
            mat = S.jello(E=float(z[p + "E"]), nu=float(z[p + "nu"]), rho=float(z[p + "rho"]))
        elif t == L.SNOW:
            mat = S.snow(E=float(z[p + "E"]), nu=float(z[p + "nu"]), rho=float(z[p + "rho"]), theta_c=8e-2,
                         theta_s=2e-2, xi=10.0)
        else:
            mat = S.water(K=2.51, rho=float(z[p + "rho"]), gamma=7.0)
        from mpm_cuda_b200.sim import Group
        groups.append(Group(material=mat, p_mass=float(z[p + "p_mass"]), p_vol=float(z[p + "p_vol"]),
                            x=z[p + "in_x"], v=z[p + "in_v"], C=z[p + "in_C"], F=z[p + "in_F"],
                            aux=z[p + "in_aux"]))
    # the reference build's constants: its 10h slip band (FP64 position test),
    # gravity -9.8 on y
    return Scene(dim=3, n=(n, n, n), h=h, dt=dt, groups=groups, bc_type=L.BC_SLIP, ref_band=10.0,
                 gravity=(0.0, -9.8, 0.0), mass_eps=2.220446049250313e-16)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("path", _golden_files(), ids=lambda p: os.path.basename(p))
def test_matches_reference_build_golden(gpu, path, mode):
    z = np.load(path)
    sc = golden_scene(z)
    with Simulation([sc], p2g_mode=mode, rebin_interval=3) as sim:
        done = 0
        for k in (1, 10):
            sim.step(k - done)
            done = k
            st = sim.get_state(0)
            off = 0
            for gi in range(int(z["n_groups"])):
                n = z[f"g{gi}_in_x"].shape[0]
                ref = {f: z[f"g{gi}_s{k}_{f}"] for f in ("x", "v", "C", "F", "aux")}
                got = {f: st[f][off:off + n] for f in st}
                gtype = int(z[f"g{gi}_type"])
                compare(got, ref, golden_tolerance(gtype, k))
                if gtype == L.SNOW:
                    check_snow_f_percentile(got["F"], ref["F"], k)
                off += n


def test_fast_particles_cross_blocks_between_rebinnings(gpu):
    """Particles moving ~0.4 cells per substep with re-binning only every 32
    substeps leave their block's tile: those gathers and scatters go to
    global memory and the result still tracks the oracle."""
    sc = blob_scene(3, "jello", seed=90)
    g = sc.groups[0]
    g.v[:] = np.float32([1.2, -0.8, 0.6]) * np.float32(0.4 * sc.h / sc.dt / 1.2)
    g.C[:] = 0
    orc = oracle_for(sc)
    with Simulation([sc], rebin_interval=32) as sim:
        sim.step(12)
        got = sim.get_state(0)
        fallbacks, rebins = sim.bin_stats()
    assert orc.step(12) == 0
    compare(got, orc.state(), {"x": 2e-5, "v": 2e-3, "C": 5e-3, "F": 1e-4, "aux": 1e-4})
    assert fallbacks > 0
    assert rebins == 1  # the prologue's


def test_switching_modes_keeps_state(gpu):
    sc = blob_scene(3, "snow", seed=91)
    orc = oracle_for(sc)
    with Simulation([sc]) as sim:
        sim.step(3)
        sim.set_p2g_mode(L.P2G_DIRECT)
        sim.step(3)
        sim.set_p2g_mode(L.P2G_ATOMIC)
        sim.step(3)
        got = sim.get_state(0)
    assert orc.step(9) == 0
    compare(got, orc.state(), {"x": 5e-6, "v": 1e-3, "C": 1e-3, "F": 5e-5, "aux": 5e-5})


@pytest.mark.parametrize("d,n", [(3, 30), (2, 44)])
def test_grid_not_a_multiple_of_the_block_near_its_upper_edge(gpu, d, n):
    # the last block row reaches past the grid; windows near the upper edge
    # load nodes outside it (zero), and the linear velocity layout of a
    # single-scene run must not let the padding nodes of one row spill into
    # the next
    mat = MATS["jello"]
    h = 1.0 / n
    x, v, C, F, aux = S.perturbed_blob(d, mat, n_grid=n, h=h, ppc=2, radius_cells=3.5, seed=95,
                                       center=np.full(d, (n - 8.5) * h))
    g = group_from_arrays(mat, h, 2, x, v, C, F, aux)
    sc = Scene(dim=d, n=(n,) * d, h=h, dt=1e-4, groups=[g], bc_type=L.BC_SLIP, bc_lo=3, bc_hi=3,
               gravity=(0.0, -9.8, 0.0)[:d] if d == 3 else (0.0, -9.8))
    orc = oracle_for(sc)
    assert orc.step(6) == 0
    ref = orc.state()
    with Simulation([sc], rebin_interval=3) as sim:
        sim.step(6)
        compare(sim.get_state(0), ref, {"x": 5e-6, "v": 6e-4, "C": 6e-4, "F": 4e-5, "aux": 4e-5})
    with Simulation([sc, blob_scene(d, "water", seed=96)], rebin_interval=3) as sim:  # blocked layout
        sim.step(6)
        compare(sim.get_state(0), ref, {"x": 5e-6, "v": 6e-4, "C": 6e-4, "F": 4e-5, "aux": 4e-5})


def test_grid_read_back_follows_the_velocity_layout(gpu):
    # a single-scene dense run keeps grid velocities in the linear layout; a
    # change of P2G path before the next substep leaves them so, and the grid
    # read-back must still see the same values
    sc = blob_scene(3, "jello", seed=93)
    with Simulation([sc]) as sim:
        sim.step(5)
        m1, v1 = sim.get_grid(0)
        sim.set_p2g_mode(L.P2G_DETERMINISTIC)
        m2, v2 = sim.get_grid(0)
        assert np.array_equal(v1, v2)
        sim.step(1)  # the deterministic path's grid update writes the blocked layout
        _, v3 = sim.get_grid(0)
        assert np.abs(v3).max() > 0
    with Simulation([sc, blob_scene(3, "jello", seed=94)]) as batch:  # two scenes: blocked layout
        batch.step(5)
        _, vb = batch.get_grid(0)
    assert np.allclose(v1, vb, rtol=1e-4, atol=1e-6 * np.abs(vb).max())


def test_set_state_mid_run_binned(gpu):
    sc = blob_scene(3, "jello", seed=92)
    with Simulation([sc], rebin_interval=5) as sim:
        sim.step(7)
        st = sim.get_state(0)
        st["v"][:, 0] += np.float32(0.5)
        sim.set_state(0, v=st["v"])
        sim.step(2)
        got = sim.get_state(0)
    sc2 = blob_scene(3, "jello", seed=92)
    g = sc2.groups[0]
    g.x, g.v, g.C, g.F, g.aux = st["x"], st["v"], st["C"], st["F"], st["aux"]
    orc = oracle_for(sc2)
    assert orc.step(2) == 0
    compare(got, orc.state(), {"x": 5e-6, "v": 5e-4, "C": 5e-4, "F": 3e-5, "aux": 3e-5})


def test_dense_scene_fills_the_chunk_lists(gpu):
    """A small grid filled at 8 particles per cell needs the most chunks per
    block (here ~2,200 64-particle chunks for 512 blocks); the configurations
    with the smallest and with two-round chunks both track the oracle."""
    h, n = 1.0 / 32, 32
    lo, hi = [4 * h] * 3, [28 * h] * 3
    x = S.jitter_fill(lo, hi, h, 8, S.box(lo, hi), np.random.default_rng(7))
    g = S.make_group(S.water(), x, h, 8, (0.0, 0.0, 0.0))
    sc = Scene(dim=3, n=(n,) * 3, h=h, dt=1e-4, groups=[g], bc_type=L.BC_SLIP, bc_lo=3, bc_hi=3,
               gravity=(0.0, -9.8, 0.0))
    orc = oracle_for(sc)
    assert orc.step(2) == 0
    ref = orc.state()
    for k in (3, 10):  # 64 threads x 1 round, 64 threads x 2 rounds
        with Simulation([sc], kernel_config=k) as sim:
            sim.step(2)
            assert sim.device_errors() == 0
            compare(sim.get_state(0), ref, {"x": 5e-6, "v": 5e-4, "C": 5e-4, "F": 3e-5, "aux": 3e-5})


def test_deferred_v_and_c_read_back_and_kept(gpu):
    """The fused substep writes v and C lazily: reading the state rebuilds them
    (a second read gives the same bits), an upload of x alone keeps the last
    substep's v and C, and the run continues as the oracle's."""
    sc = blob_scene(3, "jello", seed=93)
    orc = oracle_for(sc)
    with Simulation([sc], rebin_interval=4) as sim:
        sim.step(5)
        a = sim.get_state(0)
        b = sim.get_state(0)
        for k in ("x", "v", "C", "F", "aux"):
            assert np.array_equal(a[k], b[k]), k
        sim.set_state(0, x=a["x"])
        c = sim.get_state(0)
        assert np.array_equal(c["v"], a["v"]) and np.array_equal(c["C"], a["C"])
        sim.step(3)
        got = sim.get_state(0)
    assert orc.step(8) == 0
    compare(got, orc.state(), {"x": 5e-6, "v": 6e-4, "C": 6e-4, "F": 4e-5, "aux": 4e-5})


def _mixed_scene(seed):
    a = blob_scene(3, "jello", seed=seed)
    for name, shift in (("snow", 4), ("water", -4)):
        b = blob_scene(3, name, seed=seed + shift)
        for g in b.groups:
            g.x[:, 1] += np.float32(shift * a.h)
        a.groups += b.groups
    return a


def test_deterministic_mode_is_bitwise_reproducible(gpu):
    results = []
    for _ in range(2):
        with Simulation([_mixed_scene(110)], p2g_mode=L.P2G_DETERMINISTIC) as sim:
            sim.step(12)
            results.append((sim.get_state(0), sim.get_grid(0)))
    (s0, g0), (s1, g1) = results
    for k in ("x", "v", "C", "F", "aux"):
        assert np.array_equal(s0[k], s1[k]), k
    assert np.array_equal(g0[0], g1[0]) and np.array_equal(g0[1], g1[1])


@pytest.mark.parametrize("d", [2, 3])
def test_deterministic_out_of_grid_particle_is_left_out_exactly(gpu, d):
    # a particle whose stencil leaves the grid gets the sort key past the last
    # node: it sorts after every run, starts none, and adds nothing, so the
    # other particles and the grid come out bitwise equal to a run without it
    sc = blob_scene(d, "jello", seed=71)
    g = sc.groups[0]
    extra = blob_scene(d, "jello", seed=71)
    eg = extra.groups[0]
    out = np.float32([0.999] + [0.5] * (d - 1))
    for k in ("x", "v", "C", "F", "aux"):
        a = getattr(eg, k)
        setattr(eg, k, np.concatenate([a, a[:1]], axis=0))
    eg.x[-1] = out
    with Simulation([sc], p2g_mode=L.P2G_DETERMINISTIC) as ref, \
            Simulation([extra], p2g_mode=L.P2G_DETERMINISTIC) as sim:
        ref.step(3)
        want, want_grid = ref.get_state(0), ref.get_grid(0)
        assert sim.step_status(3) == L.ERR_SIM
        assert sim.device_errors() & L.DEVERR_OUT_OF_GRID
        got, got_grid = sim.get_state(0), sim.get_grid(0)
    n = g.n
    for k in ("x", "v", "C", "F", "aux"):
        assert np.array_equal(got[k][:n], want[k]), k
    assert np.array_equal(got["x"][n], out)  # left where it was
    assert np.array_equal(got_grid[0], want_grid[0]) and np.array_equal(got_grid[1], want_grid[1])


def test_deterministic_after_binned_steps_is_reproducible(gpu):
    # binned steps permute the particles (atomically ranked sort keys); the
    # deterministic mode first restores creation order, so two handles whose
    # storage orders differ agree bitwise once they hold the same state
    with Simulation([_mixed_scene(120)]) as sim:
        sim.step(3)
        st = sim.get_state(0)
    outs = []
    for _ in range(2):
        with Simulation([_mixed_scene(120)], rebin_interval=2) as sim:
            sim.step(5)
            sim.set_p2g_mode(L.P2G_DETERMINISTIC)
            sim.set_state(0, x=st["x"], v=st["v"], C_=st["C"], F=st["F"], aux=st["aux"])
            sim.step(6)
            outs.append(sim.get_state(0))
    for k in ("x", "v", "C", "F", "aux"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_async_positions_match_synchronous_reads(gpu):
    # deterministic P2G: two handles stepping the same state agree bitwise, so
    # the pipelined reads (substep k+1 enqueued before step k's copy is waited
    # for, more copies in flight than staging slots) must equal blocking reads
    sc = blob_scene(3, "jello", seed=90)
    n_steps = 6
    with Simulation([sc], p2g_mode=L.P2G_DETERMINISTIC) as ref, \
            Simulation([sc], p2g_mode=L.P2G_DETERMINISTIC) as sim:
        want = []
        for _ in range(n_steps):
            ref.step(1)
            want.append(ref.positions(0).copy())
        n = sim.num_particles(0)
        outs = [np.empty((n, 3), np.float32) for _ in range(n_steps)]
        tickets = []
        for k in range(n_steps):
            sim.step_async(1)
            tickets.append(sim.positions_async(outs[k], scene=0))
        for k in reversed(range(n_steps)):
            sim.wait_positions(tickets[k])
            assert np.array_equal(outs[k], want[k]), k
        with pytest.raises(L.MPMError) as e:
            sim.wait_positions(tickets[-1] + 1)
        assert e.value.code == L.ERR_INVALID


def test_async_positions_of_all_scenes(gpu):
    scenes = [blob_scene(3, "jello", seed=91), blob_scene(3, "snow", seed=92)]
    with Simulation(scenes) as sim:
        sim.step(2)
        sync = np.concatenate([sim.positions(0), sim.positions(1)])
        out = np.empty_like(sync)
        sim.wait_positions(sim.positions_async(out, scene=-1))
        assert np.array_equal(out, sync)
