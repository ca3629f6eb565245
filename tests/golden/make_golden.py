"""Generates the golden fixtures of the 3D substep from the reference itself.

Runs the reference's own MPMSimulator::step() (src/simulator/MPMCUDA.cu,
compiled unmodified into oracle/_ref/libmpm_ref.so by oracle/Makefile) on
small seeded scenes and stores inputs and outputs after 1 and 10 substeps:

    python tests/golden/make_golden.py --out tests/golden

Needs a GPU (the reference is CUDA code).  The first four scenes keep every
particle far from the reference's hard-coded 10h wall band: blobs of radius 4
cells centred in a 48^3 grid (h = 1/64).  The wall scenes put a blob across
the band (48^3 grid, h = 1/48, where the reference's FP64 band test leaves
node n - 10 outside the upper band, MPMCUDA.cu:462-469, 845-850), moving
into it.  Every particle stays at least 3 cells inside the grid, so the
reference's unchecked (NDEBUG) indexing stays in bounds; blobs move less than
a cell in 10 substeps.

Inputs are rounded to float32 so the FP32 CUDA path starts from exactly the
same state.  Snow starts from Fp = diag(Jp^(1/3)); water from J.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mpm_cuda_b200 import scenes as S  # noqa: E402
from oracle import ref as R  # noqa: E402

N_GRID, H, DT, PPC = 48, 1.0 / 64, 1e-4, 2
STEPS = (1, 10)
SNOW_REF = dict(E=1.4e5, nu=0.2, rho=400.0, theta_c=8e-2, theta_s=2e-2)

# (name, grid nodes per axis, h, [(material, center cells, seed, mean velocity)])
V0 = (0.3, -0.5, 0.2)
CASES = [
    ("jello", N_GRID, H, [(S.jello(), (24, 24, 24), 11, V0)]),
    ("snow", N_GRID, H, [(S.snow(**SNOW_REF), (24, 24, 24), 12, V0)]),
    ("water", N_GRID, H, [(S.water(K=2.51, rho=1000.0), (24, 24, 24), 13, V0)]),
    ("mixed", N_GRID, H, [(S.jello(), (20, 24, 24), 14, V0), (S.water(K=2.51, rho=1000.0), (28, 24, 24), 15, V0)]),
    # across the upper band (nodes n - 11 .. n - 9 of every axis), moving into it
    ("wall_upper", 48, 1.0 / 48, [(S.jello(), (38, 38, 38), 16, (1.0, 1.0, 1.0))]),
    # across the lower band (nodes 9 .. 11), snow moving into it
    ("wall_lower", 48, 1.0 / 48, [(S.snow(**SNOW_REF), (10, 10, 10), 17, (-1.0, -1.0, -1.0))]),
    # water across the upper x band and the lower y band
    ("wall_mixed", 48, 1.0 / 48, [(S.water(K=2.51, rho=1000.0), (38, 10, 24), 18, (1.0, -1.0, 0.0))]),
]


def build_inputs(mat, center_cells, seed, n_grid, h, v0):
    x, v, C, F, aux = S.perturbed_blob(3, mat, n_grid=n_grid, h=h, ppc=PPC, radius_cells=4.0, seed=seed,
                                       center=np.asarray(center_cells, float) * h, v0=v0)
    f32 = lambda a: np.asarray(a, np.float32)
    return f32(x), f32(v), f32(C), f32(F), f32(aux)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only", default="", help="comma-separated case names (default: all)")
    args = ap.parse_args()
    only = set(filter(None, args.only.split(",")))
    os.makedirs(args.out, exist_ok=True)
    for name, n_grid, h, groups in CASES:
        if only and name not in only:
            continue
        sim = R.RefSim(h, DT, (n_grid,) * 3)
        rec = {"h": h, "dt": DT, "n_grid": n_grid, "ppc": PPC, "n_groups": len(groups)}
        for gi, (mat, cc, seed, v0) in enumerate(groups):
            x, v, C, F, aux = build_inputs(mat, cc, seed, n_grid, h, v0)
            lo, hi = x.min(), x.max()
            assert lo >= 4 * h and hi <= (n_grid - 4) * h, "blob too close to the grid edge"
            vol = h ** 3 / PPC
            mass = mat.rho * vol
            Fp = J = None
            if mat.type == 1:
                Fp = np.zeros((len(x), 3, 3))
                s = aux.astype(np.float64) ** (1.0 / 3.0)
                for a in range(3):
                    Fp[:, a, a] = s
            if mat.type == 2:
                J = aux.astype(np.float64)
            E = mat.E if mat.type != 2 else 1e4
            nu = mat.nu if mat.type != 2 else 0.2
            sim.add_group(mat.type, E, nu, mat.rho, mass, vol, x, v, F, Fp=Fp, J=J, C_=C)
            pre = f"g{gi}_"
            rec.update({pre + "type": mat.type, pre + "E": E, pre + "nu": nu, pre + "rho": mat.rho,
                        pre + "p_mass": mass, pre + "p_vol": vol, pre + "in_x": x, pre + "in_v": v,
                        pre + "in_C": C, pre + "in_F": F, pre + "in_aux": aux})
        done = 0
        for k in STEPS:
            sim.step(k - done)
            done = k
            for gi in range(len(groups)):
                out = sim.get_group(gi)
                pre = f"g{gi}_s{k}_"
                for key in ("x", "v", "C", "F"):
                    rec[pre + key] = out[key]
                if "Fp" in out:
                    rec[pre + "aux"] = np.linalg.det(out["Fp"])
                elif "J" in out:
                    rec[pre + "aux"] = out["J"]
                else:
                    rec[pre + "aux"] = np.ones(len(out["x"]))
        sim.close()
        path = os.path.join(args.out, f"ref3d_{name}.npz")
        np.savez_compressed(path, **rec)
        print(path, {k: v.shape for k, v in rec.items() if hasattr(v, "shape") and v.ndim > 0}.get("g0_in_x"))


if __name__ == "__main__":
    main()
