"""Benchmark of the MPM substep: particle-substeps/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3]
                    [--impl ours|reference]

A step is one explicit MPM substep (P2G with stress, grid update, G2P with
the F update and advection) over every particle of the workload, state
resident in HBM.  The default workload is the 256^3 3D jello scene on which
the learned-stress comparison and the comparison with the reference build are
stated: 256^3 grid, dx = 1/256, a 0.245 cube centred at (0.5, 0.6, 0.5) at 8
particles/cell (~1.97M particles), v = (0, -2, 0), E = 5e4, nu = 0.3,
rho = 1000, dt = 1e-4, slip walls 3 cells wide; synthetic seeded particles
(no dataset exists for this scene).  --workload c1 runs the 128^3 jello scene
(0.3 cube, ~453k particles), c2 the 256^3 snow scene, c4 the 64 batched scenes.

Multi-GPU (torchrun, one process per GPU): every rank simulates its own
replica of the workload (c1, c2, c3) or its share of the 64 batched scenes (c4); the
path has no exchange step, so there is no data-path collective ("weak"
scaling).  Timing: CUDA events on the simulation's stream, max over ranks;
a workload whose particle state is larger than L2 (c2, c3, c3big, c4) runs
its K substeps back to back in one call, a smaller one (c0, c1) is timed
substep by substep with L2 flushed (256 MB write) between substeps outside
the events.

--impl reference runs the reference's own substep (MPMSimulator::step() of
MPMCUDA.cu, built unmodified into oracle/_ref/libmpm_ref.so) on the same
scene through its own code path (FP64 state, host syncs and a device-to-host
position copy every substep).  Its time varies between runs on a shared box,
so it is timed three times on the same simulation and the median is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-substeps/sec @1 B200, surrogate vs plain at stated stress/position error; HBM GB/s"
UNIT = "particle-substeps/s"
L2_FLUSH_BYTES = 256 << 20
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# plain-run substeps at which the surrogate's training set is harvested:
# start, interval, snapshots, held-out offset after the last.  The batched
# scenes are harvested within their stated 500 substeps: past ~1,500 substeps
# at the fixed dt = 1e-4, hardening makes some snow scenes break the CFL bound.
SURROGATE_HARVEST = (1400, 200, 8, 350)
SURROGATE_HARVEST_BY_WORKLOAD = {"c4": (100, 50, 6, 100)}
# timings of the reference arm (median reported)
REF_REPEATS = 3


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ helpers

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path:
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_workload(name: str, rank: int, world: int):
    from mpm_cuda_b200 import scenes as S
    from mpm_cuda_b200.ranks import replica_seed, shard
    seed = replica_seed(1234, rank)
    if name == "c4":
        return shard(S.c4_batched(), rank, world), "c4 64 batched scenes (jello/snow/water)"
    if name == "c0":
        return [S.c0_jello2d(seed=seed)], "c0 2D jello 128^2, 9000 particles, E=1e3 (MPMJello.py:12; E=1e4 breaks the CFL bound)"
    if name == "c2":
        return [S.c2_snow3d(seed=seed)], "c2 3D snow 256^3, two spheres r=0.12, 8 ppc"
    if name == "c3":
        return [S.c3_jello3d(seed=seed)], "c3 3D jello 256^3, 0.245 cube, 8 ppc"
    if name == "c3big":
        return [S.c3_jello3d(seed=seed, edge=0.45)], "c3 3D jello 256^3, 0.45 cube, 8 ppc"
    return [S.c1_jello3d(seed=seed)], "c1 3D jello 128^3, 0.3 cube, 8 ppc"


def measured_traffic(workload: str, kernel: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summaries (profiles/dram_traffic.txt), or None without a capture."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == workload and f[1] == kernel:
            return int(f[2])
    return None


def measured_counter(workload: str, kernel: str, metric: str):
    """A per-particle counter of `kernel` on `workload` from the committed ncu
    summaries (profiles/fused_counters.txt), or None without a capture."""
    path = os.path.join(ROOT, "profiles", "fused_counters.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 4 and not line.startswith("#") and f[:3] == [workload, kernel, metric]:
            return float(f[3])
    return None


def state_bytes_per_particle(scenes):
    """Algorithmic bytes of one particle's state, FP32: x v C F for solids
    (+ det Fp for snow), x v C J for water."""
    from mpm_cuda_b200 import _lib as L
    tot, n = 0, 0
    for s in scenes:
        d = s.dim
        for g in s.groups:
            base = 4 * (2 * d + d * d)
            per = base + 4 * d * d if g.material.type != L.WATER else base + 4
            if g.material.type == L.SNOW:
                per += 4
            tot += per * g.n
            n += g.n
    return tot / max(n, 1)


def cpu_baseline(scene, budget_s: float = 12.0):
    """The FP64 oracle (OpenMP, all host cores) on the same scene."""
    from oracle import cpu as ocpu
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_for
    orc = oracle_for(scene)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    steps = 0
    while True:
        orc.step(1, threads=cores)
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 50:
            break
    dt = time.perf_counter() - t0
    return {"value": scene.n_particles * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} substeps of the full {scene.name} scene ({scene.n_particles} particles), "
                      f"FP64 C oracle, OpenMP {cores} threads, {dt:.1f} s"}


def reference_errors(scene, kernel_config: int, steps: int = 200):
    """Checker leg: the divergence of this path from the reference build's
    step() on the workload's scene (reference constants where they differ),
    after `steps` substeps from the same initial state (tests/helpers.py)."""
    from oracle import ref as R
    if scene.dim != 3:
        return {"unavailable": "the reference build is 3D only"}
    if not R.available():
        return {"unavailable": "oracle/_ref/libmpm_ref.so was not built (needs the reference tree)"}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import reference_build_errors
    e = reference_build_errors(scene, steps, kernel_config=kernel_config)
    e["vs"] = ("reference MPMSimulator::step() built unmodified (FP64 state, FP32 stress), same float32 initial "
               "state, reference constants (10h slip band, its snow clamp / water EOS)")
    return e


# ----------------------------------------------------------------- our arm

def time_substeps(sim, stream, flush, steps: int) -> float:
    """Device time (ms) of `steps` substeps on the simulation's stream.  With
    a flush buffer: CUDA events around each substep, L2 flushed between
    substeps outside them.  Without (flush None, for workloads whose particle
    state alone is larger than L2): one mpm_step_async call of `steps`
    substeps between two events, as a simulation loop runs them."""
    import torch
    if flush is None:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            a.record(stream)
            sim.step_async(steps)
            b.record(stream)
        sim.synchronize()
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(steps):
            starts[k].record(stream)
            sim.step_async(1)
            ends[k].record(stream)
            flush.zero_()
    sim.synchronize()
    torch.cuda.synchronize()
    return sum(s.elapsed_time(e) for s, e in zip(starts, ends))


def surrogate_leg(args, sim, scenes, stream, flush, plain_ms_per_step: float):
    """The learned-stress path on the same workload: deformation gradients
    harvested from a separate plain run of it (snapshots after the impact),
    network trained on the GPU, held-out stress error against the SVD path,
    then the same timed loop with the network stress."""
    from mpm_cuda_b200 import _lib as L
    from mpm_cuda_b200.surrogate import StressSurrogate
    from mpm_cuda_b200.train_surrogate import harvest, stress_error
    solids = [g for s in scenes for g in s.groups if g.material.type == L.JELLO]
    if scenes[0].dim != 3 or not solids:
        return {"unavailable": "no 3D jello group in this workload (snow's exact stress reuses the "
                               "decomposition of its plasticity clamp, so it keeps the plain path)"}
    fresh, _ = build_workload(args.workload, 0, 1)
    hv = SURROGATE_HARVEST_BY_WORKLOAD.get(args.workload, SURROGATE_HARVEST)
    t0 = time.perf_counter()
    try:
        train_F, held_F = harvest(fresh, start=hv[0], every=hv[1], count=hv[2], held=hv[3])
    except L.MPMError as e:
        return {"unavailable": f"the plain run that harvests the training set failed: {e}"}
    rng = np.random.default_rng(0)
    if train_F.shape[0] > 2_000_000:
        train_F = train_F[rng.choice(train_F.shape[0], 2_000_000, replace=False)]
    if held_F.shape[0] > 500_000:
        held_F = held_F[rng.choice(held_F.shape[0], 500_000, replace=False)]
    t1 = time.perf_counter()
    sur = StressSurrogate(device=sim.device)
    loss = sur.train(train_F)
    t2 = time.perf_counter()
    err, accepted = stress_error(sur, held_F, solids[0].material.nu)
    # timed on a fresh copy of the workload over the same substeps as the
    # plain line (W warm-up, then K timed from the start of the run)
    import torch
    from mpm_cuda_b200.sim import Simulation
    timed, _ = build_workload(args.workload, 0, 1)
    try:
        with Simulation(timed, device=sim.device, kernel_config=sim.kernel_config()) as s2:
            s2.set_stress_mode(L.STRESS_SURROGATE, sur)
            if args.kernel_config < 0:
                s2.autotune()  # the launch configuration for the network kernel
            s2.step(args.warmup)
            s2.synchronize()
            t_ms = time_substeps(s2, torch.cuda.ExternalStream(s2.stream_ptr(), device=sim.device), flush,
                                 args.steps)
            n_net, n_fb = s2.stress_stats()
    except L.MPMError as e:
        return {"unavailable": f"the timed run with the learned stress failed: {e}"}
    finally:
        sur.close()
    n_part = sum(s.n_particles for s in scenes)
    ms = t_ms / args.steps
    return {"value": n_part * args.steps / (t_ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "speedup_vs_plain": plain_ms_per_step / ms,
            "held_out_stress_error": err, "held_out_accepted": accepted,
            "network_share_timed": n_net / max(1, n_net + n_fb), "train_loss": loss,
            "harvest_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 3),
            "how": "BF16 MLP 10-64-64-9 (SiLU) trained on the GPU from F harvested at substeps "
                   f"{hv[0]}+{hv[1]}k (k=1..{hv[2]}) of a plain run; "
                   "error = aggregate relative Kirchhoff stress error vs the SVD path on a later held-out "
                   "snapshot; timed like the plain line (same K, W and L2 treatment)"}


def run_ours(args, rank, world, local_rank, dist):
    import ctypes as C

    import torch
    from mpm_cuda_b200.sim import Simulation

    from mpm_cuda_b200.ranks import reduce_max, reduce_max_sum
    torch.cuda.set_device(local_rank)
    scenes, desc = build_workload(args.workload, rank, world)
    n_part = sum(s.n_particles for s in scenes)
    from mpm_cuda_b200 import _lib as L
    mode = {"binned": L.P2G_ATOMIC, "direct": L.P2G_DIRECT}[args.mode]
    sim = Simulation(scenes, device=local_rank, p2g_mode=mode, kernel_config=args.kernel_config,
                     grid_pool_blocks=args.grid_pool_blocks)
    kcfg = sim.kernel_config()
    chunk, min_ctas, rounds = C.c_int(), C.c_int(), C.c_int()
    L.load().mpm_kernel_config_info(kcfg, C.byref(chunk), C.byref(min_ctas), C.byref(rounds))
    stream = torch.cuda.ExternalStream(sim.stream_ptr(), device=local_rank)
    # L2 between timed substeps: a workload whose particle state (read and
    # written by every substep) is larger than L2 runs back to back; a smaller
    # one gets L2 flushed between substeps
    l2 = torch.cuda.get_device_properties(local_rank).L2_cache_size
    state_mb = state_bytes_per_particle(scenes) * n_part / 1e6
    if state_bytes_per_particle(scenes) * n_part > l2:
        flush = None
        l2_desc = (f"not flushed: every substep reads and writes the {state_mb:.0f} MB particle state, larger than "
                   f"the {l2 / 1e6:.0f} MB L2; the K substeps run back to back in one mpm_step_async call")
    else:
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")
        l2_desc = (f"flushed between substeps (256 MB write, outside the timed events): the {state_mb:.0f} MB "
                   f"particle state fits in the {l2 / 1e6:.0f} MB L2")

    sim.step(args.warmup)
    sim.synchronize()
    _, rebins_before = sim.bin_stats()
    if dist is not None:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        t_ms = time_substeps(sim, stream, flush, args.steps)
    if dist is not None:
        dist.barrier()
    t_max_ms, total_particles = reduce_max_sum(dist, t_ms, n_part, device=f"cuda:{local_rank}")
    t_max_s = t_max_ms / 1e3
    value = total_particles * args.steps / t_max_s
    clocks = clk.summary()

    # per-kernel device time (separate launches, CUDA events on the same stream)
    fallbacks, rebins = sim.bin_stats()
    pool_cap, pool_used = sim.grid_pool()
    grid_desc = ("dense" if args.grid_pool_blocks == 0 else
                 f"paged: {pool_used} of {pool_cap} pool blocks in use")
    stages = sim.profile_stages(20)
    active_nodes = sum(sim.count_active_nodes(i) for i in range(len(scenes)))
    sp = state_bytes_per_particle(scenes)
    # algorithmic bytes (each particle's state read once and written once, each
    # touched node's float4 written by P2G, read and written by the grid
    # update, read by G2P)
    sub_bytes = n_part * 2 * sp + active_nodes * 64
    if args.mode == "binned":
        stage_names = ["rebin", "grid_update", "g2p2g"]
        alg = {"rebin": n_part * 2 * sp, "grid_update": active_nodes * 32,
               "g2p2g": n_part * 2 * sp + active_nodes * 32}
        # grid update + one fused kernel per material present
        launches_per_step = 1 + len({g.material.type for sc in scenes for g in sc.groups})
    else:
        stage_names = ["p2g", "grid_update", "g2p"]
        alg = {"p2g": n_part * sp + active_nodes * 16, "grid_update": active_nodes * 32,
               "g2p": n_part * sp + active_nodes * 16}
        launches_per_step = 3
    timed = {k: v for k, v in zip(stage_names, stages) if k != "rebin"}
    dom_name = max(timed, key=timed.get)
    dom_ms = timed[dom_name]
    peak, peak_kind = hbm_peak()
    achieved = alg[dom_name] / (dom_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": measured_traffic(args.workload, dom_name) if args.mode == "binned" else None,
                "traffic_source": "profiles/dram_traffic.txt (ncu dram__bytes read + write per launch)",
                "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)", "algorithmic_bytes": int(alg[dom_name]),
                "stage_ms": {n: round(s, 4) for n, s in zip(stage_names, stages)},
                "substep_algorithmic_bytes": int(sub_bytes),
                "substep_achieved": round(sub_bytes / (t_max_s / args.steps) / 1e9, 1),
                "substep_frac": round(sub_bytes / (t_max_s / args.steps) / 1e9 / peak, 4)}
    if args.mode == "binned":
        # the two other ceilings of the fused kernel, beside HBM: its FP32 rate
        # against the SMs' non-tensor FP32 peak at the sampled clock, and its
        # node reductions (27 per particle in 3D, 9 in 2D)
        fused_s = stages[stage_names.index("g2p2g")] * 1e-3
        props = torch.cuda.get_device_properties(local_rank)
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 0.0
        flops = measured_counter(args.workload, "g2p2g", "fp32_flops_per_particle")
        if flops is not None and mhz:
            fp32_peak = props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
            achieved_tf = flops * n_part / fused_s / 1e12
            roofline["fp32"] = {"flops_per_particle": flops, "achieved": round(achieved_tf, 2),
                                "peak": round(fp32_peak, 1), "unit": "TFLOP/s",
                                "frac": round(achieved_tf / fp32_peak, 4),
                                "source": "profiles/fused_counters.txt (ncu FFMA x2 + FMUL + FADD + FFMA2 x4 "
                                          "+ FMUL2 x2 + FADD2 x2 per particle); "
                                          "peak = SMs x 128 FP32 lanes x 2 x median SM clock"}
        per = 27 if scenes[0].dim == 3 else 9
        roofline["reductions"] = {"per_particle": per, "achieved": round(per * n_part / fused_s / 1e9, 1),
                                  "unit": "G node reductions/s (red.global.add.v4.f32)",
                                  "l2_requests_per_particle": measured_counter(args.workload, "g2p2g",
                                                                               "l2_red_requests_per_particle")}

    # end to end through the public API: every substep's positions reach host
    # memory inside the timed region.  Pipelined: two substeps are in flight
    # (mpm_get_positions_async), so each copy overlaps the following substeps;
    # the host reads every substep's result.  Run on a fresh copy of the
    # workload (W warm-up substeps, then K timed from the start of the run,
    # like the device line), so the length of the earlier runs does not matter.
    e2e_steps = args.steps
    d = scenes[0].dim
    host = [torch.empty((n_part, d), dtype=torch.float32, pin_memory=True).numpy() for _ in range(3)]
    e2e_scenes, _ = build_workload(args.workload, rank, world)
    s3 = Simulation(e2e_scenes, device=local_rank, p2g_mode=mode, kernel_config=kcfg,
                    grid_pool_blocks=args.grid_pool_blocks)

    def e2e_pass(n):
        """n substeps, each followed by its positions' copy to the host;
        returns the wall time of every iteration (ms)."""
        tickets, checksum, iters = [], 0.0, []
        for k in range(n):
            t_it = time.perf_counter()
            s3.step_async(1)
            tickets.append(s3.positions_async(host[k % 3], scene=-1))
            if k >= 2:  # two substeps in flight: the host reads substep k - 2
                s3.wait_positions(tickets[k - 2])
                checksum += float(host[(k - 2) % 3][-1, 0])
            iters.append((time.perf_counter() - t_it) * 1e3)
        for k in range(max(0, n - 2), n):
            s3.wait_positions(tickets[k])
            checksum += float(host[k % 3][-1, 0])
        return iters

    # warm-up through the same loop: the staging buffers, the copy stream and
    # the substep graphs of both buffer parities (with and without a
    # re-binning) exist before the timed region
    e2e_pass(max(args.warmup, 2 * 16 + 2))
    s3.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_iters = e2e_pass(e2e_steps)
    s3.synchronize()
    e2e_t = reduce_max(dist, time.perf_counter() - t0, device=f"cuda:{local_rank}")
    s3.close()
    sur = None
    if world == 1 and not args.no_surrogate:
        sur = surrogate_leg(args, sim, scenes, stream, flush, t_max_s * 1e3 / args.steps)
    e2e = {"value": total_particles * e2e_steps / e2e_t, "unit": UNIT,
           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(n_part * d * 4),
           "iteration_ms": {"median": round(statistics.median(e2e_iters), 4), "max": round(max(e2e_iters), 4)},
           "how": "every substep: mpm_step_async(h, 1), mpm_get_positions_async of all positions into "
                  "page-locked host memory, then mpm_wait_positions for the copy of two substeps earlier and a "
                  "host read of it (two substeps in flight); K substeps on a fresh copy of the workload after a "
                  "warm-up of the same loop (at least W substeps and two re-binning intervals); wall clock (the reference's loop copies positions to the host every substep); "
                  "state stays resident in HBM between substeps as in the reference"}
    sim.close()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": desc, "particles_per_gpu": n_part, "particles_total": int(total_particles),
                       "active_nodes": active_nodes, "stress": "plain (SVD)", "path": args.mode,
                       "tile_fallbacks": fallbacks, "rebins": rebins,
                       "grid": grid_desc,
                       "kernel_config": {"index": kcfg, "chunk": chunk.value, "min_ctas_per_sm": min_ctas.value,
                                         "particles_per_thread": rounds.value,
                                         "chosen_by": "autotuner" if args.kernel_config < 0 else "flag"},
                       "l2": l2_desc,
                       "parallelism": f"replicas x{world}" if args.workload != "c4" else f"scenes split over {world}"},
            "roofline": roofline, "e2e": e2e, "surrogate": sur,
            # 7 kernels per re-binning: count, scan (2), place, chunk lists, reset, counter
            "gpu_launches": launches_per_step * args.steps + 7 * (rebins - rebins_before),
            "clocks": clocks}
    return line, scenes


# ----------------------------------------------------------- reference arm

def _ref_sim(sc):
    """The reference simulator holding one scene's particles (its constants)."""
    from oracle import ref as R
    sim = R.RefSim(sc.h, sc.dt, sc.n)
    for g in sc.groups:
        m = g.material
        n = g.n
        x = np.float64(g.x)
        v = np.tile(np.float64(g.init_v[:3]), (n, 1))
        F = np.tile(np.eye(3), (n, 1, 1))
        Fp = np.tile(np.eye(3), (n, 1, 1)) if m.type == 1 else None
        J = np.ones(n) if m.type == 2 else None
        sim.add_group(m.type, m.E if m.type != 2 else 1e4, m.nu if m.type != 2 else 0.2, m.rho, g.p_mass,
                      g.p_vol, x, v, F, Fp=Fp, J=J, C_=np.zeros((n, 3, 3)))
    return sim


def run_reference(args):
    """The reference's own implementation of the substep on the workload: its
    CUDA step() (oracle/_ref) for the 3D scenes -- the 64 batched scenes as 64
    reference simulators stepped one after the other, as the reference runs one
    scene per simulator -- and, for the 2D scene, whose reference is a Taichi
    script that is not installed on either machine, the CPU port on all host
    cores."""
    from oracle import ref as R
    scenes, desc = build_workload(args.workload, 0, 1)
    steps = min(args.steps, 200)
    warm = min(args.warmup, 20)
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded)"}
    if scenes[0].dim == 2:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from helpers import oracle_for
        sc = scenes[0]
        orc = oracle_for(sc)
        cores = os.cpu_count() or 1
        orc.step(warm, threads=cores)
        t0 = time.perf_counter()
        orc.step(steps, threads=cores)
        dt = time.perf_counter() - t0
        value = sc.n_particles * steps / dt
        sample = (f"{steps} substeps of {desc} after {warm} warm-up; the reference's 2D path is the Taichi script "
                  "MPMJello.py (not installed here or on the GPU box), so its C restatement (FP64, OpenMP) runs")
        return {**base, "value": value, "steps": steps, "warmup": warm, "ms_per_step": dt * 1e3 / steps,
                "dtype": "f64", "config": {"workload": desc, "particles_per_gpu": sc.n_particles},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libmpm_ref.so was not built (needs the reference tree)"}
    n = sum(sc.n_particles for sc in scenes)
    if len(scenes) == 1:
        sim = _ref_sim(scenes[0])
        sim.step(warm)
        repeats = [sim.time_steps(steps) for _ in range(REF_REPEATS)]
        sim.close()
        how = f"median of {REF_REPEATS} timings of {steps} consecutive substeps"
    else:
        # one reference simulator per scene; each repeat times `steps` substeps
        # of every scene, scene after scene
        sims = [_ref_sim(sc) for sc in scenes]
        for sim in sims:
            sim.step(warm)
        repeats = [sum(sim.time_steps(steps) for sim in sims) for _ in range(REF_REPEATS)]
        for sim in sims:
            sim.close()
        how = (f"{len(scenes)} reference simulators, one per scene; median of {REF_REPEATS} timings of {steps} "
               "substeps of every scene")
    ms = statistics.median(repeats)
    value = n * steps / (ms * 1e-3)
    return {**base, "value": value, "steps": steps, "warmup": warm, "ms_per_step": ms / steps, "dtype": "f64",
            "config": {"workload": desc, "particles_per_gpu": n,
                       "repeats_ms_per_step": [round(r / steps, 4) for r in repeats],
                       "note": "reference MPMSimulator::step() (MPMCUDA.cu:793-925) built unmodified for sm_100a; "
                               "its stock path: FP64 state, 3 device syncs and a D2H position copy per substep; "
                               f"its hard-coded 10h walls and constants; {how}"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{steps} substeps of {desc}; the reference implementation of this path "
                                       "is CUDA, so it runs on the B200 driven by one host thread"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default="c3", choices=["c0", "c1", "c2", "c3", "c3big", "c4"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="binned", choices=["binned", "direct"])
    ap.add_argument("--kernel-config", type=int, default=-1, help="fused-kernel configuration; -1 = autotune")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-stress comparison")
    ap.add_argument("--grid-pool-blocks", type=int, default=0,
                    help="paged grid with a pool of this many 64-node blocks (0 = dense grid)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0

    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device(f"cuda:{local_rank}"))
        dist = tdist
    line, scenes = run_ours(args, rank, world, local_rank, dist)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            # the checker legs: the CPU oracle's throughput and the divergence
            # from the reference build
            line["cpu_baseline"] = cpu_baseline(scenes[0])
            if len(scenes) == 1:
                fresh, _ = build_workload(args.workload, 0, 1)
                line["errors"] = reference_errors(fresh[0], line["config"]["kernel_config"]["index"])
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
