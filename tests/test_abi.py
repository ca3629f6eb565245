"""CPU checks of the C ABI: the library loads, exports exactly what
include/mpm_b200.h declares, the ctypes structs match the header layout,
and mpm_create rejects bad descriptors with status codes (validation runs
before any CUDA call, so no GPU is needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mpm_cuda_b200 import _lib as L
from mpm_cuda_b200 import scenes as S
from mpm_cuda_b200.sim import Simulation

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in ("mpm_b200.h",):
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(?:int|void)\s+(mpm_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    decl = declared_functions()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(lib, name), name
    assert decl == set(L.EXPORTS), decl ^ set(L.EXPORTS)


def test_struct_sizes_match_header_layout():
    # natural alignment of the C structs in include/mpm_b200.h
    assert C.sizeof(L.MaterialDesc) == 8 + 8 * 8
    assert C.sizeof(L.GroupDesc) == 72 + 16 + 8 + 16 + 24 + 24
    assert C.sizeof(L.Options) == 40


def _mk(**kw):
    s = S.c0_jello2d()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


@pytest.mark.parametrize("bad,code", [
    (dict(h=0.0), L.ERR_INVALID),
    (dict(dt=-1.0), L.ERR_INVALID),
    (dict(n=(3, 128)), L.ERR_INVALID),
    (dict(bc_type=7), L.ERR_INVALID),
])
def test_create_rejects_bad_scene(bad, code):
    with pytest.raises(L.MPMError) as e:
        Simulation([_mk(**bad)])
    assert e.value.code == code


def test_paged_grid_options_are_checked_on_the_host():
    # a negative pool, or a pool with a path that needs a dense grid: refused
    # before any CUDA call
    for kw, code in ((dict(grid_pool_blocks=-1), L.ERR_INVALID),
                     (dict(grid_pool_blocks=64, p2g_mode=L.P2G_DIRECT), L.ERR_UNSUPPORTED),
                     (dict(grid_pool_blocks=64, p2g_mode=L.P2G_DETERMINISTIC), L.ERR_UNSUPPORTED)):
        with pytest.raises(L.MPMError) as e:
            Simulation([S.c0_jello2d()], **kw)
        assert e.value.code == code, kw


def test_create_rejects_sand_and_bad_material():
    s = S.c0_jello2d()
    s.groups[0].material.type = L.SAND
    with pytest.raises(L.MPMError) as e:
        Simulation([s])
    assert e.value.code == L.ERR_UNSUPPORTED and "SAND" in str(e.value)
    s = S.c0_jello2d()
    s.groups[0].material.nu = 0.6  # Elasiticity.cuh:38-41 range check
    with pytest.raises(L.MPMError) as e:
        Simulation([s])
    assert e.value.code == L.ERR_INVALID and "Poisson" in str(e.value)
    s = S.c0_jello2d()
    s.groups[0].material.E = -1.0
    with pytest.raises(L.MPMError):
        Simulation([s])


def test_create_rejects_mixed_dims():
    with pytest.raises(L.MPMError) as e:
        Simulation([S.c0_jello2d(), S.c1_jello3d(n_grid=32, edge=0.2)])
    assert "same dim" in str(e.value)


def test_kernel_config_table():
    lib = L.load()
    n = lib.mpm_num_kernel_configs()
    assert n >= 2
    seen = set()
    for i in range(n):
        ch, mb, rd = C.c_int(), C.c_int(), C.c_int()
        cm, sg = C.c_int(), C.c_int()
        assert lib.mpm_kernel_config_info(i, C.byref(ch), C.byref(mb), C.byref(rd)) == L.OK
        assert lib.mpm_kernel_config_scatter(i, C.byref(cm), C.byref(sg)) == L.OK
        assert ch.value in (64, 128, 256) and ch.value * mb.value <= 2048
        assert rd.value in (1, 2, 3, 4)
        assert cm.value in (0, 1) and sg.value in (0, 1)
        assert not (sg.value and not cm.value)  # the segmented scatter runs on cell-major chunks
        seen.add((ch.value, mb.value, rd.value, cm.value, sg.value))
    assert len(seen) == n  # no duplicate configuration
    assert any(c[2] == 2 for c in seen)
    assert {(c[3], c[4]) for c in seen} == {(0, 0), (1, 0), (1, 1)}
    assert lib.mpm_kernel_config_info(n, None, None, None) == L.ERR_INVALID
    assert lib.mpm_kernel_config_scatter(n, None, None) == L.ERR_INVALID


def test_null_handle_calls_fail_cleanly():
    lib = L.load()
    assert lib.mpm_step(None, 1) == L.ERR_INVALID
    assert lib.mpm_destroy(None) == L.OK
    n = C.c_int64()
    assert lib.mpm_num_particles(None, 0, C.byref(n)) == L.ERR_INVALID
