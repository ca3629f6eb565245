"""Host logic of multi-GPU runs: one process per GPU, no data-path exchange.

Independent scenes are the path's unit of parallelism (the reference runs one
scene per process, MPMSimulator.cpp:178-285): a batch of scenes is dealt out
round-robin to the ranks, or every rank runs its own replica of a single
scene with a rank-dependent seed.  The only collectives are the reductions
of the measurements: the slowest rank's device time and the total particle
count.  Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of `items` for `rank` out of `world` ranks."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return [s for i, s in enumerate(items) if i % world == rank]


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's own replica of a single-scene workload."""
    return base + rank


def reduce_max_sum(dist, t_ms: float, count: float, device="cpu") -> Tuple[float, float]:
    """(max over ranks of t_ms, sum over ranks of count); identity when dist
    is None (one process)."""
    import torch
    t = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    n = torch.tensor([float(count)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


def reduce_max(dist, value: float, device="cpu") -> float:
    return reduce_max_sum(dist, value, 0.0, device)[0]
