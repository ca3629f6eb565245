"""Host-side pieces of bench.py (no GPU): the workloads it builds, the
algorithmic bytes per particle, the traffic table and peak it reports, and the
learned-stress harvest schedule staying inside each workload's run."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_workload_sizes_and_per_rank_seeds():
    c0, _ = bench.build_workload("c0", 0, 1)
    assert sum(s.n_particles for s in c0) == 9000 and c0[0].dim == 2
    c1, desc = bench.build_workload("c1", 0, 1)
    assert sum(s.n_particles for s in c1) == 452949 and "128^3" in desc
    c1b, _ = bench.build_workload("c1", 1, 2)  # replica on rank 1: another seed, ~ the same size
    assert abs(sum(s.n_particles for s in c1b) - 452949) < 500  # jitter kept inside the cube
    assert not np.array_equal(c1[0].groups[0].x[:100], c1b[0].groups[0].x[:100])


def test_state_bytes_per_particle_follow_the_materials():
    c1, _ = bench.build_workload("c1", 0, 1)
    assert bench.state_bytes_per_particle(c1) == 96.0       # x v C F
    c2, _ = bench.build_workload("c2", 0, 1)
    assert bench.state_bytes_per_particle(c2) == 100.0      # + det Fp
    from mpm_cuda_b200 import scenes as S
    from mpm_cuda_b200.sim import Scene
    h = 1.0 / 32
    x = S.jitter_fill([0.3] * 3, [0.5] * 3, h, 2, S.box([0.3] * 3, [0.5] * 3), np.random.default_rng(0))
    water = Scene(dim=3, n=(32,) * 3, h=h, dt=1e-4, groups=[S.make_group(S.water(), x, h, 2, (0, 0, 0))])
    assert bench.state_bytes_per_particle([water]) == 64.0  # x v C J


def test_traffic_table_and_peak():
    for w in ("c1", "c2", "c3"):
        t = bench.measured_traffic(w, "g2p2g")
        assert isinstance(t, int) and 1e6 < t < 1e9
    assert bench.measured_traffic("c4", "g2p2g") is None
    assert bench.measured_traffic("c1", "grid_update") is None
    peak, kind = bench.hbm_peak()
    assert peak > 1000.0 and kind in ("measured", "fallback")


def test_harvest_schedules_stay_inside_the_runs():
    start, every, count, held = bench.SURROGATE_HARVEST_BY_WORKLOAD["c4"]
    assert start + every * count + held <= 500  # the 64-scene workload's stated length
    start, every, count, held = bench.SURROGATE_HARVEST
    assert start + every * count + held <= 4000
