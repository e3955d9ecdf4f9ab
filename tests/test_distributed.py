"""The multi-process plumbing of the benchmark (poker_trainer_b200.dist) on
CPU with the gloo backend and two ranks: sharding covers every unit once,
the barrier completes, and the job time is the maximum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from poker_trainer_b200.dist import Group, shard


def test_shard_partitions_units():
    items = list(range(513))
    for world in (1, 2, 3, 8):
        parts = [shard(items, r, world) for r in range(world)]
        assert sum(parts, []) == items
        assert max(map(len, parts)) - min(map(len, parts)) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    g = Group(backend="gloo", timeout_s=30)
    mine = shard(list(range(10)), g.rank, g.world)
    g.barrier()
    t = g.reduce(float(rank + 1) * 1.5, "max")
    total = g.reduce(float(len(mine)), "sum")
    g.barrier()
    out.put((rank, mine, t, total))
    g.close()


def test_two_ranks_with_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] + res[1][1] == list(range(10))
    assert res[0][2] == res[1][2] == 3.0
    assert res[0][3] == res[1][3] == 10.0
