"""The multi-rank path on CPU: two gloo ranks on 127.0.0.1, no GPU.

Covers what bench.py does under torchrun: every rank computes the same
shard assignment of the batched workload without communicating (checked by
gathering the assignments), the shards are disjoint, complete and balanced,
and the timing reduction (max over ranks) and barrier work on the gloo
backend. The plain single-cloud path runs replicas (no collective on the
data path); its only collectives are this barrier and this reduction.
"""

import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from dbscan_torch.shard import shard_clouds, shard_loads
        from dbscan_torch.synthetic import batch_layout
        sizes, _, _ = batch_layout(4096, seed=0)
        shards = shard_clouds(sizes, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, shards[rank])
        m = bench.max_over_ranks(float(rank + 1) * 1.5, world)
        bench.barrier(world)
        q.put((rank, gathered, shards, m, shard_loads(sizes, shards)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    from dbscan_torch.synthetic import batch_layout
    sizes, _, _ = batch_layout(4096, seed=0)
    for rank, gathered, shards, m, loads in results:
        assert m == 3.0                      # max over ranks of 1.5, 3.0
        assert gathered == shards            # every rank computed the same assignment
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(4096))     # disjoint and complete
        assert max(loads) - min(loads) <= int(np.max(sizes))


def test_shard_clouds_rules():
    from dbscan_torch.shard import shard_clouds, shard_loads
    assert shard_clouds([5, 1, 1], 1) == [[0, 1, 2]]
    assert shard_clouds([], 3) == [[], [], []]
    assert shard_clouds([10, 9, 8, 1], 2) == [[0, 3], [1, 2]]
    sh = shard_clouds([7, 7, 7, 7], 4)
    assert sorted(len(s) for s in sh) == [1, 1, 1, 1]
    with pytest.raises(ValueError):
        shard_clouds([1, 2], 0)
    rng = np.random.default_rng(3)
    sizes = rng.integers(0, 10_000, size=500)
    sh = shard_clouds(sizes, 7)
    loads = shard_loads(sizes, sh)
    assert max(loads) <= sum(loads) / 7 + sizes.max()
