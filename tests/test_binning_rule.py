"""The counting placement of the re-binning (k_bin_place), restated on the
host: for a segment with cell counts n_c, the particle of rank r in cell c goes
to slot sum_c' min(n_c', r) + #{c' < c : n_c' > r}.  The slots must be a
permutation of the segment, ordered rank-major and by cell within a rank (the
order a radix sort of (rank, cell) keys would give)."""
import numpy as np


def slots(counts: np.ndarray) -> dict:
    out = {}
    for c, nc in enumerate(counts):
        for r in range(nc):
            lower = int(np.minimum(counts, r).sum())
            before = int(np.count_nonzero(counts[:c] > r))
            out[(r, c)] = lower + before
    return out


def test_slots_are_the_rank_major_permutation():
    rng = np.random.default_rng(5)
    cases = [np.full(64, 8), np.zeros(64, int), rng.integers(0, 12, 64),
             np.where(rng.random(64) < 0.3, rng.integers(0, 40, 64), 0)]
    cases[1][17] = 1  # a single particle
    for counts in cases:
        s = slots(counts)
        total = int(counts.sum())
        assert sorted(s.values()) == list(range(total))
        ordered = sorted(s, key=lambda rc: (rc[0], rc[1]))  # what a (rank, cell) sort gives
        assert [s[k] for k in ordered] == list(range(total))


def cell_major_slots(counts: np.ndarray) -> dict:
    """k_bin_place's cell-major slot: sum_{c' < c} n_c' + r."""
    out = {}
    for c, nc in enumerate(counts):
        for r in range(nc):
            out[(r, c)] = int(counts[:c].sum()) + r
    return out


def test_cell_major_slots_keep_a_cells_particles_together():
    rng = np.random.default_rng(6)
    for counts in [np.full(64, 8), rng.integers(0, 12, 64), np.where(rng.random(64) < 0.3, rng.integers(0, 40, 64), 0)]:
        s = cell_major_slots(counts)
        total = int(counts.sum())
        assert sorted(s.values()) == list(range(total))
        ordered = sorted(s, key=lambda rc: (rc[1], rc[0]))  # what a (cell, rank) sort gives
        assert [s[k] for k in ordered] == list(range(total))
