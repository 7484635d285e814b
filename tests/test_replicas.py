"""Replica plumbing on CPU: two gloo ranks (the multi-GPU path without GPUs).

Each rank combines timings by max and counts by sum, routes gauge fields with
owner()/shard(), and checks that every unit lands on exactly one rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    from hila_b200.replicas import ReplicaGroup, owner, shard
    g = ReplicaGroup("gloo", timeout_s=60)
    try:
        g.barrier()
        # device times differ per rank; the job time is the slowest rank's
        t = g.max(1.0 + rank)
        n = g.sum(10 * (rank + 1))
        mine = shard(list(range(17)), g.rank, g.world)
        counts = g.sum(len(mine))
        gauges = [owner(k, g.world) for k in range(8)]
        out.put((rank, g.world, t, n, mine, counts, gauges))
    finally:
        g.close()


@pytest.mark.timeout(180)
def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[0] for r in res] == [0, 1]
    for rank, w, t, n, mine, counts, gauges in res:
        assert w == 2 and t == 2.0 and n == 30 and counts == 17
        assert gauges == [0, 1, 0, 1, 0, 1, 0, 1]
    assert sorted(res[0][4] + res[1][4]) == list(range(17))
    assert not set(res[0][4]) & set(res[1][4])


def test_single_process_identity():
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    from hila_b200.replicas import ReplicaGroup, owner, shard
    g = ReplicaGroup("gloo")
    assert (g.world, g.rank, g.pg) == (1, 0, False)
    assert g.max(3.5) == 3.5 and g.sum(2) == 2.0
    g.barrier()
    g.close()
    assert shard([5, 6, 7], 0, 1) == [5, 6, 7]
    with pytest.raises(ValueError):
        owner(3, 0)
