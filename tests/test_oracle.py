"""CPU tests of the FP64 oracle: its building blocks, its invariants, and a
cross-check against the independent NumPy restatement (2D and 3D, every
material)."""
import numpy as np
import pytest

from oracle import cpu as ocpu
from oracle import numpy_mpm as onp

from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200 import _lib as L


def test_bspline_partition_of_unity():
    # sum_k N(fx - k) = 1 and sum_k N'(fx - k) = 0 for fx in [0.5, 1.5)
    # (the reference asserts |sum w - 1| < 1e-3 / 1e-4, MPMCUDA.cu:431,546)
    for fx in np.linspace(0.5, 1.5, 41)[:-1]:
        w = sum(ocpu.bspline(fx - k) for k in range(3))
        dw = sum(ocpu.bspline_deriv(fx - k) for k in range(3))
        assert abs(w - 1.0) < 1e-14
        assert abs(dw) < 1e-14


def test_bspline_values():
    assert ocpu.bspline(0.0) == 0.75
    assert ocpu.bspline(1.0) == 0.125
    assert ocpu.bspline(1.5) == 0.0
    assert ocpu.bspline_deriv(0.25) == -0.5
    assert ocpu.bspline_deriv(1.0) == -0.5
    assert ocpu.bspline_deriv(-1.0) == 0.5


@pytest.mark.parametrize("d", [2, 3])
def test_polar_svd_reconstruction(d):
    rng = np.random.default_rng(0)
    for _ in range(200):
        F = np.eye(d) + 0.5 * rng.standard_normal((d, d))
        U, s, V = ocpu.polar_svd(F)
        assert np.allclose(U @ np.diag(s) @ V.T, F, atol=1e-12)
        assert np.allclose(U.T @ U, np.eye(d), atol=1e-12)
        assert np.allclose(V.T @ V, np.eye(d), atol=1e-12)
        assert np.linalg.det(U) > 0 and np.linalg.det(V) > 0
        assert np.all(s[:-1] >= 0)
        assert np.sign(s[-1]) == np.sign(np.linalg.det(F)) or abs(s[-1]) < 1e-12
        assert np.all(np.diff(np.abs(s)) <= 1e-12)


@pytest.mark.parametrize("d", [2, 3])
def test_fcr_zero_at_identity_and_rotations(d):
    rng = np.random.default_rng(1)
    assert np.allclose(ocpu.kirchhoff_fcr(np.eye(d), 10.0, 20.0), 0.0, atol=1e-12)
    for _ in range(20):
        A = rng.standard_normal((d, d))
        Q, _ = np.linalg.qr(A)
        if np.linalg.det(Q) < 0:
            Q[:, 0] *= -1
        assert np.allclose(ocpu.kirchhoff_fcr(Q, 10.0, 20.0), 0.0, atol=1e-10)


@pytest.mark.parametrize("d", [2, 3])
def test_fcr_rotation_covariance(d):
    # tau(Q F) = Q tau(F) Q^T
    rng = np.random.default_rng(2)
    for _ in range(20):
        F = np.eye(d) + 0.2 * rng.standard_normal((d, d))
        Q, _ = np.linalg.qr(rng.standard_normal((d, d)))
        if np.linalg.det(Q) < 0:
            Q[:, 0] *= -1
        t1 = ocpu.kirchhoff_fcr(Q @ F, 3.0, 5.0)
        t2 = Q @ ocpu.kirchhoff_fcr(F, 3.0, 5.0) @ Q.T
        assert np.allclose(t1, t2, atol=1e-10)


def _groups_for(mat, h, ppc, d):
    vol = h ** d / ppc
    return ocpu.OGroup(mat.type, mat.mu, mat.lam, mat.rho * vol, vol, mat.xi, mat.theta_c, mat.theta_s,
                       mat.bulk_k, mat.gamma)


def _scene_dict(d, n, h, dt, g, bc_type, bc_lo, bc_hi, gravity, mass_eps):
    return {"dim": d, "n": n, "h": h, "dt": dt, "gravity": gravity, "bc_type": bc_type, "bc_lo": bc_lo,
            "bc_hi": bc_hi, "mass_eps": mass_eps,
            "groups": [{"type": g.type, "mu": g.mu, "lam": g.lam, "xi": g.xi, "theta_c": g.theta_c,
                        "theta_s": g.theta_s, "bulk_k": g.bulk_k, "gamma": g.gamma, "p_mass": g.p_mass,
                        "p_vol": g.p_vol}]}


MATS = {"jello": S.jello(), "snow": S.snow(), "water": S.water()}


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("name", ["jello", "snow", "water"])
@pytest.mark.parametrize("bc", [L.BC_STICKY, L.BC_SLIP, L.BC_SEPARATE])
def test_c_oracle_matches_numpy_oracle(d, name, bc):
    mat = MATS[name]
    n_grid, h, dt = 24, 1.0 / 32, 1e-4
    x, v, C, F, aux = S.perturbed_blob(d, mat, n_grid=n_grid, h=h, ppc=2, radius_cells=5.0, seed=3,
                                       center=np.full(d, 12 * h))
    # put part of the blob inside the wall band so the boundary code runs
    x[:, 0] -= 6 * h
    g = _groups_for(mat, h, 2, d)
    n = (n_grid,) * d
    sim = ocpu.OracleSim(d, n, h, dt, [g], x, v, C, F, aux, bc_type=bc, bc_lo=7, bc_hi=3)
    err = sim.step(1)
    assert err == 0
    st = {"x": x, "v": v, "C": C, "F": F, "aux": aux, "group": np.zeros(len(x), int)}
    ref = onp.substep(_scene_dict(d, n, h, dt, g, bc, 7, 3, (0, -9.8, 0), 2.22e-16), st)
    out = sim.state()
    assert np.allclose(out["x"], ref["x"], rtol=0, atol=1e-13)
    assert np.allclose(out["v"], ref["v"], rtol=1e-10, atol=1e-10)
    assert np.allclose(out["C"], ref["C"], rtol=1e-9, atol=1e-8)
    assert np.allclose(out["F"], ref["F"], rtol=1e-10, atol=1e-12)
    assert np.allclose(out["aux"], ref["aux"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("d", [2, 3])
def test_p2g_conserves_mass_and_momentum(d):
    # P2G alone: total grid mass = sum m_p, total grid momentum = sum m_p v_p
    # + dt * sum of internal forces (which sum to zero: sum_i grad w_ip = 0)
    import ctypes as C
    mat = S.jello()
    h, dt = 1.0 / 32, 1e-4
    x, v, Cm, F, aux = S.perturbed_blob(d, mat, n_grid=24, h=h, ppc=2, radius_cells=4, seed=5,
                                        center=np.full(d, 12 * h))
    g = _groups_for(mat, h, 2, d)
    sim = ocpu.OracleSim(d, (24,) * d, h, dt, [g], x, v, Cm, F, aux)
    lib = ocpu.load()
    p = sim._parts()
    err = lib.orc_p2g(C.byref(sim.grid), sim.groups, C.byref(p), ocpu._dp(sim.mass), ocpu._dp(sim.mom), 1)
    assert err == 0
    assert np.isclose(sim.mass.sum(), g.p_mass * len(x), rtol=1e-12)
    mom = sim.mom.reshape(-1, 3)[:, :d].sum(axis=0)
    assert np.allclose(mom, g.p_mass * v.sum(axis=0), rtol=1e-9, atol=1e-12)


def test_out_of_grid_sets_error():
    mat = S.jello()
    h = 1.0 / 32
    x = np.array([[0.99, 0.5, 0.5]])
    sim = ocpu.OracleSim(3, (24,) * 3, h, 1e-4, [_groups_for(mat, h, 2, 3)], x, np.zeros((1, 3)),
                         np.zeros((1, 3, 3)), np.eye(3)[None], np.ones(1))
    assert sim.step(1) & ocpu.ERR_OUT_OF_GRID


def test_openmp_matches_serial():
    mat = S.snow()
    h = 1.0 / 32
    x, v, Cm, F, aux = S.perturbed_blob(3, mat, n_grid=24, h=h, ppc=4, radius_cells=5, seed=9,
                                        center=np.full(3, 12 * h))
    g = _groups_for(mat, h, 4, 3)
    a = ocpu.OracleSim(3, (24,) * 3, h, 1e-4, [g], x, v, Cm, F, aux)
    b = ocpu.OracleSim(3, (24,) * 3, h, 1e-4, [g], x, v, Cm, F, aux)
    assert a.step(3, threads=1) == 0
    assert b.step(3, threads=4) == 0
    for k in ("x", "v", "C", "F", "aux"):
        assert np.allclose(a.state()[k], b.state()[k], rtol=1e-9, atol=1e-12)


# ------------------------------------------------ pin against the reference

import glob as _glob
import os as _os

from helpers import TOL_REF_MEDIAN, check_snow_f_percentile, golden_tolerance  # noqa: E402

_GOLDEN = sorted(_glob.glob(_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "golden", "ref3d_*.npz")))


@pytest.mark.parametrize("path", _GOLDEN, ids=lambda p: _os.path.basename(p))
def test_oracle_matches_reference_build_golden(path):
    """The FP64 oracle reproduces the reference's own CUDA substep
    (MPMSimulator::step(), MPMCUDA.cu:793-925, run on a B200 by
    tests/golden/make_golden.py) after 1 and 10 substeps.  The reference
    computes the stress and SVD in FP32, hence FP32-level tolerances."""
    z = np.load(path)
    h, dt, n = float(z["h"]), float(z["dt"]), int(z["n_grid"])
    groups, xs, vs, Cs, Fs, auxs, grp = [], [], [], [], [], [], []
    for gi in range(int(z["n_groups"])):
        p = f"g{gi}_"
        t = int(z[p + "type"])
        E, nu = float(z[p + "E"]), float(z[p + "nu"])
        mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
        groups.append(ocpu.OGroup(t, mu, lam, float(z[p + "p_mass"]), float(z[p + "p_vol"]), xi=10.0,
                                  theta_c=8e-2, theta_s=2e-2, bulk_k=2.51, gamma=7.0))
        for lst, k in ((xs, "in_x"), (vs, "in_v"), (Cs, "in_C"), (Fs, "in_F"), (auxs, "in_aux")):
            lst.append(np.float64(z[p + k]))
        grp.append(np.full(len(z[p + "in_x"]), gi, np.int32))
    cat = lambda a: np.concatenate(a)
    sim = ocpu.OracleSim(3, (n, n, n), h, dt, groups, cat(xs), cat(vs), cat(Cs), cat(Fs), cat(auxs),
                         group=cat(grp), gravity=(0, -9.8, 0), bc_type=ocpu.BC_SLIP, ref_band=10.0)
    done = 0
    for k in (1, 10):
        assert sim.step(k - done) == 0
        done = k
        st = sim.state()
        off = 0
        for gi in range(int(z["n_groups"])):
            m = len(z[f"g{gi}_in_x"])
            gtype = int(z[f"g{gi}_type"])
            for f in ("x", "v", "C", "F", "aux"):
                ref = z[f"g{gi}_s{k}_{f}"]
                got = st[f][off:off + m]
                tol = golden_tolerance(gtype, k)[f]
                if f == "F" and gtype == ocpu.SNOW:
                    check_snow_f_percentile(got, ref, k)
                if f == "x":
                    err = np.abs(got - ref).max()
                else:
                    err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)
                assert err < tol, (f, k, err)
                # most particles agree to FP32 round-off; the max is set by a few
                # particles with near-equal singular values (FP32 SVD conditioning)
                med = np.median(np.abs(got - ref)) / max(np.abs(ref).max(), 1e-30)
                assert med < TOL_REF_MEDIAN[k], (f, k, med)
            off += m


def test_c0_stated_stiffness_violates_the_cfl_bound():
    """The 2D jello workload at E = 1e4 (rho = 1, dx = 1/128, dt = 1e-4) has an
    elastic CFL number of 1.28 and diverges in the FP64 oracle; the script's
    own E = 1e3 (MPMJello.py:12) stays bounded.  The c0 workload uses 1e3."""
    from mpm_cuda_b200 import scenes as S
    from helpers import oracle_for
    stiff = oracle_for(S.c0_jello2d(E=1e4))
    assert any(stiff.step(1) != 0 for _ in range(120))
    soft = oracle_for(S.c0_jello2d())
    assert all(soft.step(1) == 0 for _ in range(300))
    assert float(np.abs(soft.state()["v"]).max()) < 5.0


def _reference_band(n, h, band=10.0, origin=0.0):
    """Nodes the reference's VelUpdate marks as walls (MPMCUDA.cu:462-469 with
    the bounds of :845-850), restated in FP64: (lower count, upper count)."""
    import math
    lower = origin + band * h
    upper = (origin + h * n) - band * h
    pos = [math.fma(i, h, origin) if hasattr(math, "fma") else origin + i * h for i in range(n)]
    return sum(p <= lower for p in pos), sum(p >= upper for p in pos)


def test_reference_band_rounds_node_n_minus_10_out_for_h_1_48():
    # the reference's position test is not an integer count: for n = 48,
    # h = 1/48 the FP64 rounding leaves node 38 outside the upper band
    assert _reference_band(48, 1.0 / 48) == (11, 9)
    assert _reference_band(48, 1.0 / 64) == (11, 10)
    assert _reference_band(256, 1.0 / 256) == (11, 10)


@pytest.mark.parametrize("n,h", [(48, 1.0 / 48), (48, 1.0 / 64), (40, 1.0 / 30), (57, 1.0 / 57)])
def test_oracle_grid_update_applies_the_reference_band(n, h):
    """With ref_band = 10, the oracle's grid update zeroes the wall-normal
    velocity exactly at the nodes the reference's FP64 test marks."""
    lo, hi = _reference_band(n, h)
    g = ocpu.OGroup(ocpu.JELLO, 1.0, 1.0, 1.0, 1.0)
    x = np.array([[0.5, 0.5, 0.5]])
    sim = ocpu.OracleSim(3, (n, n, n), h, 1e-4, [g], x, np.zeros((1, 3)), np.zeros((1, 3, 3)),
                         np.tile(np.eye(3), (1, 1, 1)), np.ones(1), gravity=(0, 0, 0), bc_type=ocpu.BC_SLIP,
                         ref_band=10.0)
    G = n ** 3
    mass = np.ones(G)
    mom = np.ones((G, 3))
    vel = sim.grid_update(mass, mom)
    ix = np.arange(G) % n
    wall = (ix < lo) | (ix >= n - hi)
    assert np.all(vel[wall, 0] == 0.0) and np.all(vel[~wall, 0] == 1.0)
