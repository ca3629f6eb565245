"""Small driver for profiling one workload's substep (e.g. under ncu):

    python -m mpm_cuda_b200.profile --workload c1 --mode binned --warmup 3 --steps 3

Builds the seeded workload, runs `warmup` substeps, then `steps` more, and
prints per-stage CUDA-event times.  Under a profiler, select the kernel with
its name (k_g2p2g, k_grid_update_active, k_p2g_direct, ...) and skip the
warm-up launches.
"""
from __future__ import annotations

import argparse
import json

from . import _lib as L
from . import scenes as S
from .sim import Simulation

WORKLOADS = {
    "c0": lambda: [S.c0_jello2d()],
    "c1": lambda: [S.c1_jello3d()],
    "c1small": lambda: [S.c1_jello3d(n_grid=64, edge=0.3)],
    "c2": lambda: [S.c2_snow3d()],
    "c3": lambda: [S.c3_jello3d()],
    "c4": lambda: S.c4_batched(),
}
MODES = {"binned": L.P2G_ATOMIC, "direct": L.P2G_DIRECT, "deterministic": L.P2G_DETERMINISTIC}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", default="binned", choices=sorted(MODES))
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--rebin-interval", type=int, default=0)
    ap.add_argument("--kernel-config", type=int, default=-1, help="-1 = autotune")
    ap.add_argument("--surrogate", default=None, help="trained surrogate file: run with the network stress")
    args = ap.parse_args()
    scenes = WORKLOADS[args.workload]()
    sur = None
    with Simulation(scenes, p2g_mode=MODES[args.mode], rebin_interval=args.rebin_interval,
                    kernel_config=args.kernel_config) as sim:
        if args.surrogate:
            from .surrogate import StressSurrogate
            sur = StressSurrogate.load(args.surrogate)
            sim.set_stress_mode(L.STRESS_SURROGATE, sur)
        sim.step(args.warmup)
        sim.step(args.steps)
        stages = sim.profile_stages(max(1, args.steps))
        fb, rb = sim.bin_stats()
        print(json.dumps({"workload": args.workload, "mode": args.mode, "kernel_config": sim.kernel_config(),
                          "particles": sim.num_particles(),
                          "stage_ms": [round(s, 5) for s in stages], "tile_fallbacks": fb, "rebins": rb,
                          "stress": "surrogate" if sur else "plain",
                          "network_fallback": list(sim.stress_stats()) if sur else None}))
    if sur:
        sur.close()


if __name__ == "__main__":
    main()
