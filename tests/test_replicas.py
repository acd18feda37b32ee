"""Replica sharding across ranks (world size 2, gloo, CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from beep3_b200.replicas import ReplicaError, run_replicated, shard


def test_shard_round_robin():
    items = list("abcdefg")
    a = shard(items, 0, 2)
    b = shard(items, 1, 2)
    assert [i for i, _ in a] == [0, 2, 4, 6] and [i for i, _ in b] == [1, 3, 5]
    assert sorted(a + b) == list(enumerate(items))
    with pytest.raises(ValueError):
        shard(items, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = run_replicated(list(range(10)), lambda v: (v * v, rank), dist)
        if rank == 0:
            q.put(res)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_run_replicated_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [v for v, _ in res] == [i * i for i in range(10)]
    # items alternate between the two ranks
    assert [r for _, r in res] == [i % 2 for i in range(10)]


def test_single_process_path():
    assert run_replicated([1, 2, 3], lambda v: v + 1, None) == [2, 3, 4]


def _failing(v):
    if v == 3:
        raise ValueError("pose 3 has no solution")
    return v + 100


def _worker_fail(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        try:
            res = run_replicated(list(range(6)), _failing, dist)
            q.put(("ok", rank, res))
        except ReplicaError as e:
            q.put(("error", rank, e.failures))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_failing_item_reported_on_rank0_without_hang():
    """Item 3 (rank 1) raises; both ranks finish the gather and rank 0 gets
    a ReplicaError naming it, while rank 1 returns normally."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_fail, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    by_rank = {r: (kind, v) for kind, r, v in got}
    assert by_rank[0][0] == "error" and set(by_rank[0][1]) == {3}
    assert by_rank[0][1][3][0] == 1 and "no solution" in by_rank[0][1][3][1]
    assert by_rank[1] == ("ok", None)
