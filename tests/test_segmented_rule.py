"""The run masks of the segmented P2G scatter (scatter_segmented in
mpm_kernels_binned.cuh), restated on the host: lanes that take part and share
a stencil base with the previous lane continue its run; a run ends where the
next lane does not continue it.  Summing each row over the runs and emitting
at the run ends must give the same grid as every lane scattering directly."""
import numpy as np

FULL = 0xFFFFFFFF


def masks(keys, part):
    """part: 32 bools; keys: 32 ints (ignored where part is False)."""
    heads = 0
    pm = 0
    for lane in range(32):
        if part[lane]:
            pm |= 1 << lane
            prev = keys[lane - 1] if lane > 0 and part[lane - 1] else -1
            if lane == 0 or prev != keys[lane]:
                heads |= 1 << lane
    ends = pm & ~(((pm & ~heads) & FULL) >> 1) & FULL
    return pm, heads, ends


def walk(values, keys, part):
    """Lane `row` walks the columns: the per-run sums emitted at run ends."""
    pm, heads, ends = masks(keys, part)
    out = {}
    acc = None
    for m in range(32):
        if not (pm >> m) & 1:
            continue
        acc = values[m].copy() if (heads >> m) & 1 else acc + values[m]
        if (ends >> m) & 1:
            out.setdefault(keys[m], []).append(acc.copy())
    return out


def test_run_sums_equal_direct_scatter():
    rng = np.random.default_rng(11)
    for trial in range(400):
        # cell-major runs of random length, some drifted lanes with other keys,
        # some lanes not taking part
        keys = np.repeat(rng.integers(0, 300, 12), rng.integers(1, 9, 12))[:32]
        keys = np.concatenate([keys, rng.integers(0, 300, 32)])[:32]
        drift = rng.random(32) < 0.1
        keys = np.where(drift, rng.integers(0, 300, 32), keys)
        part = rng.random(32) < (0.9 if trial % 3 else 1.0)
        values = rng.standard_normal((32, 27, 4))
        got = {}
        for k, sums in walk(values, keys, part).items():
            got[k] = np.sum(sums, axis=0)
        want = {}
        for lane in range(32):
            if part[lane]:
                want[keys[lane]] = want.get(keys[lane], 0) + values[lane]
        assert set(got) == set(want)
        for k in want:
            np.testing.assert_allclose(got[k], want[k], rtol=1e-12, atol=1e-12)


def test_every_participating_lane_is_in_exactly_one_run():
    rng = np.random.default_rng(12)
    for _ in range(200):
        keys = rng.integers(0, 4, 32)
        part = rng.random(32) < 0.8
        pm, heads, ends = masks(keys, part)
        assert heads & ~pm == 0 and ends & ~pm == 0
        assert bin(heads).count("1") == bin(ends).count("1")
        # walking the lanes, heads and ends alternate
        open_run = False
        for m in range(32):
            if (heads >> m) & 1:
                assert not open_run
                open_run = True
            if (pm >> m) & 1:
                assert open_run
            if (ends >> m) & 1:
                open_run = False
        assert not open_run
