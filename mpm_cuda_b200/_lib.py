"""ctypes binding of ``libmpm_b200.so`` (the C ABI in ``include/mpm_b200.h``).

This module is what a Python caller of the C ABI binds: the structs mirror
the header field by field and every entry point gets its prototype here.
Loading fails loudly when the shared library is missing: there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpm_b200.so")

# enums (include/mpm_b200.h)
JELLO, SNOW, WATER, SAND = 0, 1, 2, 3
BC_STICKY, BC_SLIP, BC_SEPARATE = 0, 1, 2
P2G_ATOMIC, P2G_DETERMINISTIC, P2G_DIRECT = 0, 1, 2
STRESS_PLAIN, STRESS_SURROGATE = 0, 1
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_SIM, ERR_IO = 0, -1, -2, -3, -4, -5, -6
DEVERR_OUT_OF_GRID, DEVERR_NONFINITE, DEVERR_DET, DEVERR_BINNING, DEVERR_TIMEOUT, DEVERR_POOL = 1, 2, 4, 8, 16, 32

_FP = C.POINTER(C.c_float)


class MaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
                ("xi", C.c_double), ("theta_c", C.c_double), ("theta_s", C.c_double),
                ("bulk_k", C.c_double), ("gamma", C.c_double)]


class GroupDesc(C.Structure):
    _fields_ = [("material", MaterialDesc), ("p_mass", C.c_double), ("p_vol", C.c_double),
                ("n", C.c_int64), ("x", _FP), ("v", _FP), ("init_v", C.c_double * 3),
                ("F", _FP), ("C", _FP), ("aux", _FP)]


class SceneDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3), ("h", C.c_double), ("origin", C.c_double * 3),
                ("dt", C.c_double), ("gravity", C.c_double * 3), ("bc_type", C.c_int),
                ("bc_lo", C.c_int), ("bc_hi", C.c_int), ("mass_eps", C.c_double),
                ("n_groups", C.c_int), ("groups", C.POINTER(GroupDesc)), ("ref_band", C.c_double)]


class Options(C.Structure):
    _fields_ = [("p2g_mode", C.c_int), ("stress_mode", C.c_int), ("use_graph", C.c_int),
                ("block_threads", C.c_int), ("device", C.c_int), ("rebin_interval", C.c_int),
                ("kernel_config", C.c_int), ("adaptive_dt", C.c_int), ("cfl", C.c_float),
                ("grid_pool_blocks", C.c_int)]


SHAPE_CUBE, SHAPE_SPHERE, SHAPE_CYLINDER, SHAPE_MESH = 0, 1, 2, 3


class SeedObject(C.Structure):
    _fields_ = [("shape", C.c_int), ("rotation", C.c_double * 9), ("scale", C.c_double * 3),
                ("translation", C.c_double * 3), ("vertices", _FP), ("n_vertices", C.c_int64),
                ("triangles", C.POINTER(C.c_int32)), ("n_triangles", C.c_int64)]


class SurrogateTrainOptions(C.Structure):
    _fields_ = [("n_samples", C.c_int64), ("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float),
                ("lr_final", C.c_float), ("sigma", C.c_float), ("rotation_fraction", C.c_float),
                ("skew_tol", C.c_float), ("seed", C.c_uint64)]


_U8P = C.POINTER(C.c_uint8)

EXPORTS = {
    # name: (restype, argtypes)
    "mpm_default_options": (None, [C.POINTER(Options)]),
    "mpm_create": (C.c_int, [C.POINTER(SceneDesc), C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "mpm_destroy": (C.c_int, [C.c_void_p]),
    "mpm_step": (C.c_int, [C.c_void_p, C.c_int]),
    "mpm_step_async": (C.c_int, [C.c_void_p, C.c_int]),
    "mpm_synchronize": (C.c_int, [C.c_void_p]),
    "mpm_get_device_errors": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "mpm_clear_device_errors": (C.c_int, [C.c_void_p]),
    "mpm_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mpm_num_particles": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
    "mpm_get_positions": (C.c_int, [C.c_void_p, C.c_int, _FP, C.c_size_t]),
    "mpm_get_positions_async": (C.c_int, [C.c_void_p, C.c_int, _FP, C.c_size_t, C.POINTER(C.c_int64)]),
    "mpm_wait_positions": (C.c_int, [C.c_void_p, C.c_int64]),
    "mpm_get_state": (C.c_int, [C.c_void_p, C.c_int, _FP, _FP, _FP, _FP, _FP]),
    "mpm_set_state": (C.c_int, [C.c_void_p, C.c_int, _FP, _FP, _FP, _FP, _FP]),
    "mpm_get_grid": (C.c_int, [C.c_void_p, C.c_int, _FP, _FP]),
    "mpm_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "mpm_get_scene_time": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "mpm_write_bgeo": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
    "mpm_write_bgeo_positions": (C.c_int, [C.c_char_p, _FP, C.c_int64]),
    "mpm_set_p2g_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "mpm_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "mpm_profile_stages": (C.c_int, [C.c_void_p, C.c_int, _FP, C.c_int, C.POINTER(C.c_int)]),
    "mpm_count_active_nodes": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
    "mpm_get_bin_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mpm_get_grid_pool": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mpm_num_kernel_configs": (C.c_int, []),
    "mpm_kernel_config_info": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mpm_kernel_config_scatter": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mpm_get_kernel_config": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mpm_set_kernel_config": (C.c_int, [C.c_void_p, C.c_int]),
    "mpm_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "mpm_step_noalloc": (C.c_int, [C.POINTER(SceneDesc), C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_void_p]),
    "mpm_surrogate_default_train_options": (None, [C.POINTER(SurrogateTrainOptions)]),
    "mpm_surrogate_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "mpm_surrogate_destroy": (C.c_int, [C.c_void_p]),
    "mpm_surrogate_train": (C.c_int, [C.c_void_p, _FP, C.c_int64, C.POINTER(SurrogateTrainOptions),
                                      C.POINTER(C.c_float)]),
    "mpm_surrogate_eval": (C.c_int, [C.c_void_p, _FP, C.c_int64, C.c_float, _FP, _FP, _U8P]),
    "mpm_surrogate_gradients": (C.c_int, [C.c_void_p, _FP, _FP, C.c_int64, _FP, C.POINTER(C.c_float)]),
    "mpm_surrogate_num_params": (C.c_int, []),
    "mpm_surrogate_num_meta": (C.c_int, []),
    "mpm_surrogate_get_params": (C.c_int, [C.c_void_p, _FP, _FP]),
    "mpm_surrogate_set_params": (C.c_int, [C.c_void_p, _FP, _FP]),
    "mpm_surrogate_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mpm_surrogate_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mpm_set_stress_mode": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mpm_seed": (C.c_int, [C.POINTER(SeedObject), C.c_int, C.c_double, C.POINTER(C.c_double), C.c_int, C.c_uint64,
                           C.c_int, _FP, C.c_size_t, C.POINTER(C.c_int64)]),
    "mpm_get_stress_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree ``libmpm_b200.so``; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m mpm_cuda_b200.build` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def fptr(a):
    """float* of a C-contiguous float32 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], "expects contiguous float32"
    return a.ctypes.data_as(_FP)


class MPMError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(1024)
    load().mpm_last_error(handle, buf, 1024)
    return buf.value.decode(errors="replace")


def check(code: int, handle=None) -> int:
    if code != OK:
        raise MPMError(code, last_error(handle))
    return code
