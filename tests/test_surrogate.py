"""Learned stress surrogate: the FP64 CPU oracle (oracle/mlp.py), the GPU
training kernels' gradients against it, the trained network's stress error
against the SVD path, and the fused substep with the network against the
plain substep."""
import os

import ctypes as C

import numpy as np
import pytest

from oracle import mlp as M


def random_F(rng, n, spread=0.15, rotate=True):
    def rot(k):
        q = rng.normal(size=(k, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        w, x, y, z = q.T
        return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                         2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                         2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1).reshape(k, 3, 3)
    s = np.clip(1 + spread * rng.normal(size=(n, 3)), 0.3, None)
    if not rotate:
        return np.einsum("ni,ij->nij", s, np.eye(3))
    U, V = rot(n), rot(n)
    return (U * s[:, None, :]) @ V.transpose(0, 2, 1)


def agg_rel(a, b):
    """Aggregate relative error sqrt(sum |a - b|^2 / sum |b|^2)."""
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


# ----------------------------------------------------------- CPU: oracle --

def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = np.zeros(M.N_PARAMS)
    w = {"W1": rng.normal(0, 0.3, (64, 10)), "W2": rng.normal(0, 0.12, (64, 64)), "W3": rng.normal(0, 0.12, (9, 64)),
         "b1": rng.normal(0, 0.1, 64), "b2": rng.normal(0, 0.1, 64), "b3": rng.normal(0, 0.1, 9)}
    p = M.pack(w)
    x = rng.normal(size=(32, 10))
    y = rng.normal(size=(32, 9))
    _, g = M.forward_backward(p, x, y)
    real = np.flatnonzero(M.pack({k: np.ones_like(v) for k, v in w.items()}))
    for idx in rng.choice(real, 40, replace=False):
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[idx] += e
        pm[idx] -= e
        fd = (M.forward_backward(pp, x, y)[0] - M.forward_backward(pm, x, y)[0]) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, g[idx])
    # padding entries get no gradient
    assert np.all(g[np.setdiff1d(np.arange(M.N_PARAMS), real)] == 0)


def test_exact_residual_reproduces_fixed_corotated_stress():
    rng = np.random.default_rng(1)
    F = random_F(rng, 2000, spread=0.3)
    for lam in (0.0, 1.5, 4.0):
        t = M.tau_from_residual(F, M.residual_target(F), 1.0, lam)
        assert agg_rel(t, M.fcr_tau(F, 1.0, lam)) < 1e-12


def test_residual_is_third_order_and_rotation_free():
    rng = np.random.default_rng(2)
    A = rng.normal(size=(100, 3, 3))
    A = 0.5 * (A + A.transpose(0, 2, 1))
    for eps in (1e-2, 1e-3):
        r = M.residual_target(np.eye(3) + eps * A)
        assert np.max(np.abs(r)) < 0.2 * eps ** 3 * np.max(np.abs(A)) ** 3 * 27
    # a rigid rotation has X = 0 and zero residual
    R = random_F(rng, 50, spread=0.0)
    assert np.max(np.abs(M.strain_b(R))) < 1e-12
    assert np.max(np.abs(M.residual_target(R))) < 1e-12


def test_bf16_rounding_is_nearest_even():
    assert M.bf16(np.float32(1 + 2 ** -9))[()] == 1.0          # tie -> even
    assert M.bf16(np.float32(1 + 3 * 2 ** -9))[()] == 1 + 2 ** -7  # tie -> even (up)
    assert M.bf16(np.float32(1 + 2 ** -8 + 2 ** -12))[()] == 1 + 2 ** -7


# ------------------------------------------------------------- GPU parts --

@pytest.fixture(scope="module")
def surrogate_cls(gpu):
    from mpm_cuda_b200.surrogate import StressSurrogate
    return StressSurrogate


def fall_scene(n_grid=64, edge=0.3, seed=5):
    from mpm_cuda_b200 import scenes as S
    return S.c1_jello3d(seed=seed, n_grid=n_grid, edge=edge)


@pytest.fixture(scope="module")
def harvested(gpu):
    """Deformation gradients of a falling, bouncing jello cube (64^3, 0.3
    edge, ~56k particles) from plain substeps: training snapshots after the
    impact, a held-out snapshot later, and the state just before impact."""
    from mpm_cuda_b200.sim import Simulation
    snaps, before = [], None
    with Simulation([fall_scene()]) as sim:
        sim.step(1400)
        before = sim.get_state(0)
        for _ in range(8):
            sim.step(200)
            snaps.append(sim.get_state(0)["F"])
        sim.step(350)
        held = sim.get_state(0)["F"]
    return np.concatenate(snaps), held, before


@pytest.fixture(scope="module")
def trained(surrogate_cls, harvested):
    sur = surrogate_cls(seed=11)
    loss = sur.train(harvested[0])
    yield sur, loss
    sur.close()


@pytest.mark.gpu
def test_gpu_gradients_match_cpu_oracle(surrogate_cls):
    rng = np.random.default_rng(3)
    sur = surrogate_cls(seed=7)
    p, _ = sur.params()
    x = rng.normal(size=(1024, 10)).astype(np.float32)
    y = (0.5 * rng.normal(size=(1024, 9))).astype(np.float32)
    g_gpu, loss_gpu = sur.gradients(x, y)
    loss_bf, g_bf = M.forward_backward(p, x, y, bf16_ops=True)
    loss_64, g_64 = M.forward_backward(p, x, y, bf16_ops=False)
    sur.close()
    blocks = {"W1": (M.OFF_W1, M.OFF_W2), "W2": (M.OFF_W2, M.OFF_W3), "W3": (M.OFF_W3, M.OFF_B1),
              "b1": (M.OFF_B1, M.OFF_B2), "b2": (M.OFF_B2, M.OFF_B3), "b3": (M.OFF_B3, M.N_PARAMS)}
    assert abs(loss_gpu - loss_bf) <= 2e-3 * loss_bf
    assert abs(loss_gpu - loss_64) <= 2e-2 * loss_64
    for name, (a, b) in blocks.items():
        # same BF16 operand rounding as the kernels, FP64 accumulation
        assert agg_rel(g_gpu[a:b], g_bf[a:b]) < 5e-3, name
        # plain FP64 MLP: the BF16 rounding of operands is the whole difference
        assert agg_rel(g_gpu[a:b], g_64[a:b]) < 5e-2, name


@pytest.mark.gpu
def test_trained_network_stress_error(trained, harvested):
    """On held-out deformation gradients of the run, the stress from the
    network is within 1 % (aggregate) of the SVD path's, nearly every particle
    is accepted, and the network is far more accurate than the same formula
    without it (the second-order series of sqrt(B) alone)."""
    sur, loss = trained
    held = harvested[1].reshape(-1, 3, 3)
    nu = 0.3
    lam_mu = 2 * nu / (1 - 2 * nu)
    tp, tr, ok = sur.eval(held, lam_mu)
    assert ok.mean() > 0.97, ok.mean()
    err_net = agg_rel(tp[ok], tr[ok])
    t_series = M.tau_from_residual(held[ok], np.zeros_like(held[ok]), 1.0, lam_mu)
    err_series = agg_rel(t_series, M.fcr_tau(held[ok], 1.0, lam_mu))
    print(f"loss {loss:.3e} accepted {ok.mean():.4f} stress error: network {err_net:.4%} series only {err_series:.4%}")
    assert err_net <= 0.01
    assert err_net < 0.5 * err_series
    # the SVD path itself agrees with the FP64 oracle
    assert agg_rel(tr[ok], M.fcr_tau(held[ok], 1.0, lam_mu)) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("config", [1, 9], ids=["one-round", "two-round"])
def test_untrained_network_always_falls_back(surrogate_cls, gpu, config):
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200.sim import Simulation
    from helpers import TOL_STEP, compare
    from mpm_cuda_b200 import scenes as S
    from mpm_cuda_b200.sim import Scene
    from helpers import group_from_arrays
    sur = surrogate_cls(seed=1)
    # a blob with perturbed v, C, F so that every state field carries signal
    mat, h = S.jello(), 1.0 / 32
    x, v, C_, F, aux = S.perturbed_blob(3, mat, n_grid=32, h=h, ppc=2, radius_cells=5.0, seed=3,
                                        center=np.full(3, 0.5))
    sc = Scene(dim=3, n=(32,) * 3, h=h, dt=1e-4, groups=[group_from_arrays(mat, h, 2, x, v, C_, F, aux)],
               bc_type=L.BC_SLIP, bc_lo=3, bc_hi=3, gravity=(0.0, -9.8, 0.0))
    rounds = C.c_int()
    assert L.load().mpm_kernel_config_info(config, None, None, C.byref(rounds)) == L.OK
    assert rounds.value == (1 if config == 1 else 2)
    with Simulation([sc], kernel_config=config) as plain, Simulation([sc], kernel_config=config) as sim:
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        plain.step(3)
        sim.step(3)
        n, fb = sim.stress_stats()
        assert n == 0 and fb == 3 * sim.num_particles()
        compare(sim.get_state(0), plain.get_state(0), TOL_STEP)
    sur.close()


@pytest.mark.gpu
def test_fused_surrogate_drift_vs_plain(trained, harvested, gpu):
    """1000 substeps through the impact: mean position drift of the network
    stress against the plain SVD stress <= 0.5 % of the cube edge."""
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200.sim import Simulation
    sur, _ = trained
    st = harvested[2]
    sc = fall_scene()
    with Simulation([sc]) as plain, Simulation([sc]) as sim:
        for s in (plain, sim):
            s.set_state(0, st["x"], st["v"], st["C"], st["F"], st["aux"])
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        plain.step(1000)
        sim.step(1000)
        n_net, n_fb = sim.stress_stats()
        xp, xs = plain.get_state(0)["x"], sim.get_state(0)["x"]
    drift = float(np.mean(np.linalg.norm(xs - xp, axis=1))) / 0.3
    share = n_net / (n_net + n_fb)
    print(f"network share {share:.4f} mean drift {drift:.3e} of the edge")
    assert share > 0.95
    assert drift <= 5e-3


@pytest.mark.gpu
def test_c3_scene_stress_error_and_drift(surrogate_cls, gpu):
    """The 256^3 jello scene (0.245 cube, ~2.0M particles, v = (0, -2, 0)):
    trained on deformation gradients harvested after the impact (substeps
    1600-3000 of a plain run), the network's held-out stress error is <= 1 %
    and, from the state at substep 1400, 1000 substeps through the impact
    drift <= 0.5 % of the cube edge (mean position distance) from the plain
    path."""
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200 import scenes as S
    from mpm_cuda_b200.sim import Simulation
    from mpm_cuda_b200.train_surrogate import stress_error
    edge = 0.245
    snaps = []
    with Simulation([S.c3_jello3d(edge=edge)]) as sim:
        sim.step(1400)
        before = sim.get_state(0)
        for _ in range(8):
            sim.step(200)
            snaps.append(sim.get_state(0)["F"])
        sim.step(350)
        held = sim.get_state(0)["F"]
    rng = np.random.default_rng(0)
    train = np.concatenate(snaps)
    train = train[rng.choice(len(train), 2_000_000, replace=False)]
    sur = surrogate_cls(seed=11)
    sur.train(train)
    err, accepted = stress_error(sur, held[rng.choice(len(held), 500_000, replace=False)], 0.3)
    assert err <= 1e-2 and accepted > 0.95, (err, accepted)
    sc = S.c3_jello3d(edge=edge)
    with Simulation([sc]) as plain, Simulation([sc]) as sim:
        for s in (plain, sim):
            s.set_state(0, before["x"], before["v"], before["C"], before["F"], before["aux"])
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        plain.step(1000)
        sim.step(1000)
        assert sim.device_errors() == 0
        n_net, n_fb = sim.stress_stats()
        xp, xs = plain.get_state(0)["x"], sim.get_state(0)["x"]
    sur.close()
    drift = float(np.mean(np.linalg.norm(xs.astype(np.float64) - xp, axis=1))) / edge
    share = n_net / (n_net + n_fb)
    print(f"c3: held-out stress error {err:.4f}, network share {share:.4f}, mean drift {drift:.3e} of the edge")
    assert share > 0.95
    assert drift <= 5e-3


@pytest.mark.gpu
def test_snow_keeps_the_plain_stress(trained, gpu):
    # snow's exact stress reuses its plasticity decomposition, so surrogate
    # mode leaves it on the plain kernel: no particle goes through the network
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200 import scenes as S
    from mpm_cuda_b200.sim import Simulation
    sur, _ = trained
    sc = S.c2_snow3d(n_grid=64)
    with Simulation([sc]) as plain, Simulation([sc]) as sim:
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        plain.step(800)
        sim.step(800)
        assert sim.device_errors() == 0
        n_net, n_fb = sim.stress_stats()
        xp, xs = plain.get_state(0)["x"], sim.get_state(0)["x"]
    assert n_net == 0 and n_fb == 0
    assert float(np.mean(np.linalg.norm(xs - xp, axis=1))) / 0.24 <= 5e-3


@pytest.mark.gpu
def test_save_load_roundtrip(trained, surrogate_cls, tmp_path):
    sur, _ = trained
    path = os.path.join(tmp_path, "net.mpmsur")
    sur.save(path)
    other = surrogate_cls.load(path)
    p0, m0 = sur.params()
    p1, m1 = other.params()
    assert np.array_equal(p0, p1) and m0 == m1
    F = random_F(np.random.default_rng(4), 512, spread=0.05)
    a = sur.eval(F, 1.5)
    b = other.eval(F, 1.5)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    other.close()


@pytest.mark.gpu
def test_stress_mode_errors(surrogate_cls, gpu):
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200.sim import Simulation
    sur = surrogate_cls(seed=2)
    sc = fall_scene(n_grid=32)
    with Simulation([sc], p2g_mode=L.P2G_DIRECT) as sim:
        with pytest.raises(L.MPMError) as e:
            sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        assert e.value.code == L.ERR_UNSUPPORTED
    with Simulation([sc]) as sim:
        with pytest.raises(L.MPMError) as e:
            sim.set_stress_mode(L.STRESS_SURROGATE, None)
        assert e.value.code == L.ERR_INVALID
        sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        with pytest.raises(L.MPMError) as e:
            sim.set_p2g_mode(L.P2G_DIRECT)
        assert e.value.code == L.ERR_UNSUPPORTED
        sim.set_stress_mode(L.STRESS_PLAIN)
        sim.set_p2g_mode(L.P2G_DIRECT)
        sim.step(2)
    with pytest.raises(L.MPMError):
        sur.train(np.eye(3, dtype=np.float32)[None], n_samples=10)
    sur.close()
