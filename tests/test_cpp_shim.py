"""The reference-style C++ interface (include/mpm_simulator.hpp): it compiles
with the reference's call pattern (CPU), and on a GPU it seeds, steps, reads
positions and writes a .bgeo frame; an .obj cube seeds exactly like the
built-in cube."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_demo.cpp")
LIBDIR = os.path.join(ROOT, "mpm_cuda_b200")


def build_demo(out_dir):
    exe = os.path.join(out_dir, "shim_demo")
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIBDIR, "-lmpm_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


CUBE_OBJ = """# unit cube [-0.5, 0.5]^3
v -0.5 -0.5 -0.5
v 0.5 -0.5 -0.5
v 0.5 0.5 -0.5
v -0.5 0.5 -0.5
v -0.5 -0.5 0.5
v 0.5 -0.5 0.5
v 0.5 0.5 0.5
v -0.5 0.5 0.5
f 1 4 3 2
f 5 6 7 8
f 1 2 6 5
f 2 3 7 6
f 3 4 8 7
f 4 1 5 8
"""


def test_shim_compiles_with_reference_call_pattern(tmp_path):
    build_demo(str(tmp_path))


@pytest.mark.gpu
def test_shim_runs_and_obj_cube_matches_builtin(gpu, tmp_path):
    from test_bgeo import read_bgeo
    exe = build_demo(str(tmp_path))
    obj = tmp_path / "cube.obj"
    obj.write_text(CUBE_OBJ)
    outs = {}
    for name, shape in (("builtin", "builtin:cube"), ("obj", str(obj))):
        frame = str(tmp_path / f"{name}.bgeo")
        r = subprocess.run([exe, shape, "20", frame], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[name] = (json.loads(r.stdout.strip().splitlines()[-1]), read_bgeo(frame))
    (jb, pb), (jo, po) = outs["builtin"], outs["obj"]
    assert jb["particles"] > 1000 and jb["frame"] == 20 and abs(jb["time"] - 20e-4) < 1e-9
    assert jb["particles"] == jo["particles"]
    assert np.allclose(pb, po, atol=1e-6)
    # the falling cube moved down, the resting water sphere stayed inside the grid
    assert np.all((pb > 0.0) & (pb < 1.0))
