"""World-size-2 gloo test of the multi-GPU bench logic (replicas only: the
only collective is the max-over-ranks reduction of the timed interval)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        ms = 100.0 + 50.0 * rank          # rank 1 is the slowest
        value, slow = bench.aggregate(ms, steps=20, world=world)
        q.put((rank, value, slow))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_takes_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=5) for _ in range(2))
    for rank, value, slow in out:
        assert slow == pytest.approx(150.0)
        assert value == pytest.approx(2 * 20 / 0.150)


def _shard_worker(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from ysim_b200 import generators as G
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        full = G.config_c4(instances=40, lo=8, hi=48, level=1)
        mine = G.shard_instances(full, rank, world)
        groups = sorted({m.group for m in mine.meshes})
        everyone = [None] * world
        dist.all_gather_object(everyone, (groups, mine.nV))
        q.put((rank, everyone, full.nV, len({m.group for m in full.meshes})))
    finally:
        dist.destroy_process_group()


def test_batched_instances_shard_over_ranks():
    """Every instance runs on exactly one rank, and the ranks' vertex counts
    are balanced (the largest instance bounds the difference)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = [q.get(timeout=5) for _ in range(2)]
    _, everyone, total_v, n_groups = out[0]
    assert everyone == out[1][1]
    all_groups = [g for groups, _ in everyone for g in groups]
    assert sorted(all_groups) == list(range(n_groups))
    assert sum(v for _, v in everyone) == total_v
    largest = (48 * 48) + 42  # largest cloth + its level-1 icosphere
    assert abs(everyone[0][1] - everyone[1][1]) <= largest
