"""Generates the golden fixtures of the 3D substep from the reference itself.

Runs the reference's own MPMSimulator::step() (src/simulator/MPMCUDA.cu,
compiled unmodified into oracle/_ref/libmpm_ref.so by oracle/Makefile) on
small seeded scenes and stores inputs and outputs after 1 and 10 substeps:

    python tests/golden/make_golden.py --out tests/golden

Needs a GPU (the reference is CUDA code).  Scenes keep every particle far
from the reference's hard-coded 10h wall band, so the reference's unchecked
(NDEBUG) indexing stays in bounds: blobs of radius 4 cells centred in a 48^3
grid (h = 1/64) move less than a cell in 10 substeps.

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

# (name, [(material, center cells, seed)])
CASES = [
    ("jello", [(S.jello(), (24, 24, 24), 11)]),
    ("snow", [(S.snow(E=1.4e5, nu=0.2, rho=400.0, theta_c=8e-2, theta_s=2e-2), (24, 24, 24), 12)]),
    ("water", [(S.water(K=2.51, rho=1000.0), (24, 24, 24), 13)]),
    ("mixed", [(S.jello(), (20, 24, 24), 14), (S.water(K=2.51, rho=1000.0), (28, 24, 24), 15)]),
]


def build_inputs(mat, center_cells, seed):
    x, v, C, F, aux = S.perturbed_blob(3, mat, n_grid=N_GRID, h=H, ppc=PPC, radius_cells=4.0, seed=seed,
                                       center=np.asarray(center_cells, float) * H)
    f32 = lambda a: np.asarray(a, np.float32)
    return f32(x), f32(v), f32(C), f32(F), f32(aux)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name, groups in CASES:
        sim = R.RefSim(H, DT, (N_GRID,) * 3)
        rec = {"h": H, "dt": DT, "n_grid": N_GRID, "ppc": PPC, "n_groups": len(groups)}
        for gi, (mat, cc, seed) in enumerate(groups):
            x, v, C, F, aux = build_inputs(mat, cc, seed)
            vol = H ** 3 / PPC
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
