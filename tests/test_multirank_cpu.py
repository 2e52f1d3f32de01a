"""CPU, world size 2 over gloo: the multi-GPU host logic of the benchmark
(max over ranks, whole-job rate, per-rank batches) and the cost-balanced
partition of a batch across GPUs.  No GPU and no collective in the data path:
batched work shards with nothing exchanged but the final timing maximum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from blockedbunchkaufmanldlt_b200 import sharding
        # the slowest rank's time decides the job rate
        my_ms = 10.0 * (rank + 1)
        mx = bench.reduce_max_over_ranks(my_ms, world, torch.device("cpu"))
        rate = bench.job_throughput(4096, world, mx)
        # per-rank batches differ
        sizes = bench.batched_sizes(64, bench.batch_seed(7, rank))
        gathered = [None] * world
        dist.all_gather_object(gathered, sizes)
        # every rank derives the same partition of one global batch
        glob = bench.batched_sizes(1000, 11)
        mine = sharding.shard_for_rank(glob, rank, world)
        shards = [None] * world
        dist.all_gather_object(shards, mine.tolist())
        out[rank] = {"max": mx, "rate": rate, "batches": gathered, "shards": shards, "glob": glob}
    finally:
        dist.destroy_process_group()


def test_two_rank_host_logic():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        codes = [p.exitcode for p in procs]
        res = dict(out)
    assert codes == [0, 0], codes
    for r in range(world):
        assert res[r]["max"] == 20.0
        assert res[r]["rate"] == pytest.approx(2 * 4096 / 0.020)
    b0, b1 = res[0]["batches"]
    assert b0 != b1  # own batch per rank (weak scaling)
    s0, s1 = res[0]["shards"]
    assert res[1]["shards"] == [s0, s1]  # same partition on every rank
    glob = res[0]["glob"]
    assert sorted(s0 + s1) == list(range(len(glob)))
    c0 = sum(glob[k] ** 3 for k in s0)
    c1 = sum(glob[k] ** 3 for k in s1)
    assert abs(c0 - c1) / max(c0, c1) < 0.01  # balanced work


def test_partition_by_cost_properties():
    from blockedbunchkaufmanldlt_b200 import sharding
    rng = np.random.default_rng(3)
    sizes = rng.integers(16, 513, size=4096)
    for parts in (1, 2, 4, 8):
        bins = sharding.partition_by_cost(sizes, parts)
        allidx = np.sort(np.concatenate(bins))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        costs = [sharding.cost(sizes[b]) for b in bins]
        assert max(costs) / min(costs) < 1.01
    with pytest.raises(ValueError):
        sharding.partition_by_cost(sizes, 0)
