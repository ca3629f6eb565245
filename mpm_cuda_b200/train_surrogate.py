"""Harvests deformation gradients from plain substeps of a workload, trains
the learned stress surrogate on the GPU and reports its stress error on a
held-out snapshot against the SVD path:

    python -m mpm_cuda_b200.train_surrogate --workload c1 --out net.mpmsur

The plain run starts from the workload's initial state; snapshots are taken
every `--every` substeps after `--start`, and one more `--held` substeps
after the last as the held-out set.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib as L
from .profile import WORKLOADS
from .sim import Simulation
from .surrogate import StressSurrogate


def harvest(scenes, start: int, every: int, count: int, held: int):
    """(training F (n, 3, 3), held-out F, lambda / mu of the held-out groups)."""
    snaps = []
    with Simulation(scenes) as sim:
        sim.step(start)
        for _ in range(count):
            sim.step(every)
            snaps.append(np.concatenate([sim.get_state(s)["F"] for s in range(len(scenes))]))
        sim.step(held)
        held_F = np.concatenate([sim.get_state(s)["F"] for s in range(len(scenes))])
    return np.concatenate(snaps), held_F


def stress_error(sur: StressSurrogate, F: np.ndarray, nu: float):
    """(aggregate relative stress error of accepted particles, accepted share)."""
    lam_mu = 2 * nu / (1 - 2 * nu)
    tp, tr, ok = sur.eval(F, lam_mu)
    if not ok.any():
        return float("nan"), 0.0
    d = (tp[ok] - tr[ok]).astype(np.float64)
    return float(np.sqrt(np.sum(d * d) / np.sum(tr[ok].astype(np.float64) ** 2))), float(ok.mean())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--out", required=True)
    ap.add_argument("--start", type=int, default=1400)
    ap.add_argument("--every", type=int, default=200)
    ap.add_argument("--count", type=int, default=8)
    ap.add_argument("--held", type=int, default=350)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--samples", type=int, default=1 << 21)
    ap.add_argument("--seed", type=int, default=11)
    args = ap.parse_args()
    scenes = WORKLOADS[args.workload]()
    nu = next(g.material.nu for s in scenes for g in s.groups if g.material.type in (L.JELLO, L.SNOW))
    t0 = time.perf_counter()
    train_F, held_F = harvest(scenes, args.start, args.every, args.count, args.held)
    t1 = time.perf_counter()
    sur = StressSurrogate(seed=args.seed)
    loss = sur.train(train_F, n_samples=args.samples, epochs=args.epochs)
    t2 = time.perf_counter()
    err, acc = stress_error(sur, held_F, nu)
    sur.save(args.out)
    print(json.dumps({"workload": args.workload, "train_samples_seed": int(train_F.shape[0]), "loss": loss,
                      "harvest_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3),
                      "held_out_stress_error": err, "accepted": acc, "meta": sur.params()[1]}))
    sur.close()


if __name__ == "__main__":
    main()
