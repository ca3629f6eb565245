"""Multi-rank host logic (mpm_cuda_b200/ranks.py) with two gloo ranks on CPU:
the scene shards of the batched workload partition the batch, and the
measurement reductions give the slowest rank's time and the total count."""
import socket

import pytest
import torch.multiprocessing as mp

from mpm_cuda_b200.ranks import reduce_max_sum, replica_seed, shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard(list(range(64)), rank, world)
        # device time of this rank and its particle count
        t_ms, n = 10.0 + 5.0 * rank, float(sum(mine))
        out[rank] = (mine, reduce_max_sum(dist, t_ms, n), replica_seed(1234, rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_partitions_the_batch():
    for world in (1, 2, 3, 8):
        parts = [shard(list(range(64)), r, world) for r in range(world)]
        assert sorted(x for p in parts for x in p) == list(range(64))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        shard([1, 2], 2, 2)


def test_reductions_without_process_group():
    assert reduce_max_sum(None, 3.0, 7.0) == (3.0, 7.0)


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    shards = [res[r][0] for r in range(world)]
    assert sorted(shards[0] + shards[1]) == list(range(64)) and not set(shards[0]) & set(shards[1])
    for r in range(world):
        t_max, n_total = res[r][1]
        assert t_max == 15.0                      # the slower rank's time on every rank
        assert n_total == float(sum(range(64)))   # every rank's count
    assert res[0][2] != res[1][2]                 # replicas differ by seed
