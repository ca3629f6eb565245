"""Python host layer over the C ABI: scene descriptors and a simulation handle.

``Simulation`` wraps one ``mpm_handle``: it owns the device state of one or
more scenes and advances them with the CUDA-graph substep.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L


@dataclass
class MaterialParams:
    """Material of a particle group (Elasiticity.cuh:19-45 plus the constants
    the reference hard-codes in its kernels).  Defaults reproduce the
    reference: xi = 10 (MPMCUDA.cu:344), clamp 8e-2 / 2e-2 (:658-660), water
    2.51 (J^-7 - 1) (:353)."""
    type: int
    E: float
    nu: float
    rho: float
    xi: float = 10.0
    theta_c: float = 8e-2
    theta_s: float = 2e-2
    bulk_k: float = 2.51
    gamma: float = 7.0

    @property
    def mu(self) -> float:
        return self.E / (2.0 * (1.0 + self.nu))

    @property
    def lam(self) -> float:
        return self.E * self.nu / ((1.0 + self.nu) * (1.0 - 2.0 * self.nu))


@dataclass
class Group:
    material: MaterialParams
    p_mass: float
    p_vol: float
    x: np.ndarray                       # (n, dim) float32
    v: Optional[np.ndarray] = None      # (n, dim)
    init_v: Sequence[float] = (0.0, 0.0, 0.0)
    F: Optional[np.ndarray] = None      # (n, dim, dim)
    C: Optional[np.ndarray] = None
    aux: Optional[np.ndarray] = None    # (n,) Jp / J

    @property
    def n(self) -> int:
        return int(self.x.shape[0])


@dataclass
class Scene:
    dim: int
    n: Sequence[int]
    h: float
    dt: float
    groups: List[Group] = field(default_factory=list)
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    gravity: Sequence[float] = (0.0, -9.8, 0.0)
    bc_type: int = L.BC_SLIP
    bc_lo: int = 3
    bc_hi: int = 3
    mass_eps: float = 2.220446049250313e-16
    name: str = ""
    # > 0: walls from the reference's FP64 position test with this band in
    # cells (bc_lo / bc_hi ignored); see mpm_scene_desc.ref_band
    ref_band: float = 0.0

    @property
    def n_particles(self) -> int:
        return sum(g.n for g in self.groups)


def _f32(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


def scene_descs(scenes: Sequence[Scene]):
    """C descriptors (mpm_scene_desc[]) of the scenes, plus the list of
    Python objects that must stay alive while the descriptors are used."""
    keep = []
    sdescs = (L.SceneDesc * len(scenes))()
    for si, s in enumerate(scenes):
        if True:
            gdescs = (L.GroupDesc * max(1, len(s.groups)))()
            keep.append(gdescs)
            for gi, g in enumerate(s.groups):
                d = s.dim
                x = _f32(g.x, (-1,))
                v = _f32(g.v, (-1,))
                F = _f32(g.F, (-1,))
                Cm = _f32(g.C, (-1,))
                aux = _f32(g.aux, (-1,))
                keep.extend([x, v, F, Cm, aux])
                m = g.material
                gd = gdescs[gi]
                gd.material = L.MaterialDesc(m.type, m.E, m.nu, m.rho, m.xi, m.theta_c, m.theta_s,
                                             m.bulk_k, m.gamma)
                gd.p_mass, gd.p_vol, gd.n = g.p_mass, g.p_vol, g.n
                gd.x, gd.v, gd.F, gd.C, gd.aux = (L.fptr(x), L.fptr(v), L.fptr(F), L.fptr(Cm),
                                                  L.fptr(aux))
                iv = list(g.init_v) + [0.0] * (3 - len(g.init_v))
                gd.init_v = (C.c_double * 3)(*iv[:3])
                assert x.size == g.n * d
            sd = sdescs[si]
            sd.dim = s.dim
            nn = list(s.n) + [1] * (3 - len(s.n))
            sd.n = (C.c_int * 3)(*nn[:3])
            sd.h, sd.dt = s.h, s.dt
            o = list(s.origin) + [0.0] * (3 - len(s.origin))
            gr = list(s.gravity) + [0.0] * (3 - len(s.gravity))
            sd.origin = (C.c_double * 3)(*o[:3])
            sd.gravity = (C.c_double * 3)(*gr[:3])
            sd.bc_type, sd.bc_lo, sd.bc_hi = s.bc_type, s.bc_lo, s.bc_hi
            sd.mass_eps = s.mass_eps
            sd.ref_band = s.ref_band
            sd.n_groups = len(s.groups)
            sd.groups = gdescs
    return sdescs, keep


class Simulation:
    """One C-ABI handle over a list of scenes (all of the same dimension)."""

    def __init__(self, scenes: Sequence[Scene], p2g_mode: int = L.P2G_ATOMIC,
                 stress_mode: int = L.STRESS_PLAIN, use_graph: bool = True, device: int = 0,
                 rebin_interval: int = 0, kernel_config: int = -1, adaptive_dt: bool = False,
                 cfl: float = 0.5, grid_pool_blocks: int = 0):
        lib = L.load()
        self.scenes = list(scenes)
        self.dim = self.scenes[0].dim
        self.device = device
        sdescs, keep = scene_descs(self.scenes)
        opt = L.Options()
        lib.mpm_default_options(C.byref(opt))
        opt.p2g_mode, opt.stress_mode, opt.use_graph, opt.device = p2g_mode, stress_mode, int(use_graph), device
        opt.rebin_interval = rebin_interval
        opt.kernel_config = kernel_config
        opt.adaptive_dt = int(adaptive_dt)
        opt.cfl = cfl
        opt.grid_pool_blocks = grid_pool_blocks
        h = C.c_void_p()
        L.check(lib.mpm_create(sdescs, len(self.scenes), C.byref(opt), C.byref(h)))
        self._h = h
        self._lib = lib

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.mpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, code):
        return L.check(code, self._h)

    # ------------------------------------------------------------- stepping
    def step(self, n: int = 1):
        self._check(self._lib.mpm_step(self._h, n))

    def step_async(self, n: int = 1):
        self._check(self._lib.mpm_step_async(self._h, n))

    def synchronize(self):
        self._check(self._lib.mpm_synchronize(self._h))

    def step_status(self, n: int = 1) -> int:
        """Like step() but returns the status code instead of raising."""
        return self._lib.mpm_step(self._h, n)

    def device_errors(self) -> int:
        bits = C.c_uint32()
        self._check(self._lib.mpm_get_device_errors(self._h, C.byref(bits)))
        return int(bits.value)

    def clear_device_errors(self):
        self._check(self._lib.mpm_clear_device_errors(self._h))

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._check(self._lib.mpm_get_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def set_p2g_mode(self, mode: int):
        self._check(self._lib.mpm_set_p2g_mode(self._h, mode))

    def set_stress_mode(self, mode: int, surrogate=None):
        """MPM_STRESS_PLAIN, or MPM_STRESS_SURROGATE with a trained
        ``StressSurrogate`` (kept alive by this object while it is in use)."""
        self._surrogate = surrogate if mode == L.STRESS_SURROGATE else None
        self._check(self._lib.mpm_set_stress_mode(self._h, mode, surrogate.handle if surrogate else None))

    def stress_stats(self):
        """(stresses from the network, SVD fallbacks) since the mode was set."""
        a, b = C.c_int64(), C.c_int64()
        self._check(self._lib.mpm_get_stress_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def scene_time(self, scene: int = 0):
        """(simulated time, current dt) of one scene."""
        t, dt = C.c_double(), C.c_float()
        self._check(self._lib.mpm_get_scene_time(self._h, scene, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def time(self):
        t, f = C.c_double(), C.c_int64()
        self._check(self._lib.mpm_get_time(self._h, C.byref(t), C.byref(f)))
        return t.value, f.value

    # ----------------------------------------------------------------- state
    def num_particles(self, scene: int = -1) -> int:
        n = C.c_int64()
        self._check(self._lib.mpm_num_particles(self._h, scene, C.byref(n)))
        return n.value

    def positions(self, scene: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Positions in creation order.  `out` may be a preallocated (e.g.
        page-locked) float32 array of shape (n, dim)."""
        n = self.num_particles(scene)
        if out is None:
            out = np.empty((n, self.dim), np.float32)
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.size >= n * self.dim
        self._check(self._lib.mpm_get_positions(self._h, scene, L.fptr(out), out.size))
        return out

    def positions_async(self, out: np.ndarray, scene: int = 0) -> int:
        """Starts copying the positions after the substeps enqueued so far into
        `out` (float32 (n, dim), page-locked for overlap) and returns a ticket;
        `out` is valid after wait_positions(ticket)."""
        n = self.num_particles(scene)  # scene < 0: every scene
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.size >= n * self.dim
        t = C.c_int64()
        self._check(self._lib.mpm_get_positions_async(self._h, scene, L.fptr(out), out.size, C.byref(t)))
        return t.value

    def wait_positions(self, ticket: int):
        self._check(self._lib.mpm_wait_positions(self._h, ticket))

    def get_state(self, scene: int = 0) -> dict:
        n, d = self.num_particles(scene), self.dim
        st = {"x": np.empty((n, d), np.float32), "v": np.empty((n, d), np.float32),
              "C": np.empty((n, d, d), np.float32), "F": np.empty((n, d, d), np.float32),
              "aux": np.empty((n,), np.float32)}
        self._check(self._lib.mpm_get_state(self._h, scene, L.fptr(st["x"]), L.fptr(st["v"]),
                                            L.fptr(st["C"]), L.fptr(st["F"]), L.fptr(st["aux"])))
        return st

    def set_state(self, scene: int = 0, x=None, v=None, C_=None, F=None, aux=None):
        arrs = [_f32(a) for a in (x, v, C_, F, aux)]
        self._check(self._lib.mpm_set_state(self._h, scene, *[L.fptr(a) for a in arrs]))

    def get_grid(self, scene: int = 0):
        s = self.scenes[scene]
        nn = list(s.n)[: self.dim]
        G = int(np.prod(nn))
        mass = np.empty(G, np.float32)
        vel = np.empty(G * self.dim, np.float32)
        self._check(self._lib.mpm_get_grid(self._h, scene, L.fptr(mass), L.fptr(vel)))
        return mass, vel.reshape(G, self.dim)

    def count_active_nodes(self, scene: int = 0) -> int:
        n = C.c_int64()
        self._check(self._lib.mpm_count_active_nodes(self._h, scene, C.byref(n)))
        return n.value

    def kernel_config(self) -> int:
        c = C.c_int()
        self._check(self._lib.mpm_get_kernel_config(self._h, C.byref(c)))
        return c.value

    def set_kernel_config(self, config: int):
        self._check(self._lib.mpm_set_kernel_config(self._h, config))

    def autotune(self, n_substeps: int = 8):
        """(chosen configuration, ms per substep); does not advance the state."""
        c, ms = C.c_int(), C.c_float()
        self._check(self._lib.mpm_autotune(self._h, n_substeps, C.byref(c), C.byref(ms)))
        return c.value, ms.value

    def grid_pool(self):
        """(pool capacity, blocks in use) of the grid, in 64-node blocks."""
        cap, used = C.c_int64(), C.c_int64()
        self._check(self._lib.mpm_get_grid_pool(self._h, C.byref(cap), C.byref(used)))
        return cap.value, used.value

    def bin_stats(self):
        """(fallback gathers/scatters served from global memory, re-binnings)."""
        fb, rb = C.c_int64(), C.c_int64()
        self._check(self._lib.mpm_get_bin_stats(self._h, C.byref(fb), C.byref(rb)))
        return fb.value, rb.value

    def write_bgeo(self, path: str, scene: int = 0):
        self._check(self._lib.mpm_write_bgeo(self._h, scene, path.encode()))

    def profile_stages(self, n: int = 10):
        out = (C.c_float * 8)()
        nw = C.c_int()
        self._check(self._lib.mpm_profile_stages(self._h, n, out, 8, C.byref(nw)))
        return [out[i] for i in range(nw.value)]
