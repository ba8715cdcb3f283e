"""Replica plumbing on CPU with two gloo ranks (the multi-GPU path shards
snapshots across ranks and only reduces the timing)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "forceconstants.jl_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from fcb200 import replicas
    dist = replicas.init("gloo", timeout_s=60)
    mine = list(replicas.shard(48, rank, world))
    replicas.barrier(dist)
    t = replicas.max_over_ranks(1.5 + rank, dist)
    q.put((rank, mine, t))
    replicas.finalize(dist)


def test_two_rank_shard_and_max():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] + res[1][1] == list(range(48))        # every snapshot exactly once
    assert res[0][2] == res[1][2] == pytest.approx(2.5)     # job time = slowest rank


def test_shard_edge_cases():
    sys.path.insert(0, os.path.join(ROOT, "forceconstants.jl_b200"))
    from fcb200.replicas import shard
    for n in (0, 1, 7, 48):
        for w in (1, 2, 3, 8):
            got = [i for r in range(w) for i in shard(n, r, w)]
            assert got == list(range(n))
