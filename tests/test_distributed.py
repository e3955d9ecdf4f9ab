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


class _OracleNet:
    """A CPU stand-in for LeafNet in the data-parallel training loop
    (poker_trainer_b200.train_leaf.train): gradients and Adam from the FP64
    oracle of the network (oracle/mlp_fp64.py, pinned by finite
    differences), the gradient buffer a CPU tensor for gloo."""

    def __init__(self, dims, seed):
        import numpy as np
        import torch
        rng = np.random.default_rng(seed)
        self.layers = [(rng.normal(0, 1.0 / np.sqrt(k), (n, k)), rng.normal(0, 0.1, n))
                       for k, n in zip(dims[:-1], dims[1:])]
        self.size = sum(w.size + b.size for w, b in self.layers)
        self.g = torch.zeros(self.size, dtype=torch.float64)
        self.m = np.zeros(self.size)
        self.v = np.zeros(self.size)
        self.step = 0

    def flat(self):
        import numpy as np
        return np.concatenate([np.concatenate([w.ravel(), b]) for w, b in self.layers])

    def _set(self, flat):
        off = 0
        for i, (w, b) in enumerate(self.layers):
            w2 = flat[off:off + w.size].reshape(w.shape)
            off += w.size
            b2 = flat[off:off + b.size]
            off += b.size
            self.layers[i] = (w2, b2)

    def backward(self, x, t, mask):
        import numpy as np
        import torch
        from oracle import mlp_fp64
        loss, grads = mlp_fp64.loss_and_gradients(self.layers, x.numpy(), t.numpy(), mask.numpy())
        self.g.copy_(torch.from_numpy(np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])))
        return loss

    def grad_tensor(self):
        return self.g

    def adam_step(self, lr, grad_scale=1.0):
        from oracle import mlp_fp64
        self.step += 1
        w, self.m, self.v = mlp_fp64.adam_step(self.flat(), self.g.numpy() * grad_scale, self.m, self.v, self.step, lr)
        self._set(w)

    def train_step(self, x, t, mask, lr):
        loss = self.backward(x, t, mask)
        self.adam_step(lr, 1.0)
        return loss


def _dp_data():
    import numpy as np
    rng = np.random.default_rng(3)
    X = rng.normal(size=(16, 5))
    Y = rng.normal(size=(16, 3))
    M = np.ones((16, 3))
    return X, Y, M


def _dp_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from poker_trainer_b200.train_leaf import train
    g = Group(backend="gloo", timeout_s=30)
    X, Y, M = _dp_data()
    net = _OracleNet([5, 6, 3], seed=1)
    train(X, Y, M, steps=4, batch=8, lr=1e-2, seed=0, group=g, net=net, device="cpu")
    out.put((rank, net.flat()))
    g.close()


def test_data_parallel_training_with_gloo():
    """Two ranks, each on its half of 16 samples with minibatches of its 8:
    the all-reduced, averaged gradient is the full batch's, so both ranks'
    weights stay identical and equal one process training on all 16."""
    import numpy as np
    from poker_trainer_b200.train_leaf import train

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((r, w) for r, w in (out.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(res[0][1], res[1][1])
    X, Y, M = _dp_data()
    single = _OracleNet([5, 6, 3], seed=1)
    train(X, Y, M, steps=4, batch=16, lr=1e-2, seed=0, net=single, device="cpu")
    assert np.allclose(res[0][1], single.flat(), rtol=1e-10, atol=1e-12)


def _spots():
    from poker_trainer_b200 import workloads
    return workloads.batched_river_spots(count=5, seed=3000)


def _batch_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from oracle_api import OracleSolver
    g = Group(backend="gloo", timeout_s=60)
    mine = shard(list(range(5)), g.rank, g.world)
    spots = _spots()
    expl = []
    for i in mine:
        o = OracleSolver(spots[i])
        o.iterate(3)
        expl.append((i, o.exploitability()))
    got = g.gather_concat(expl)
    out.put((rank, got))
    g.close()


def test_batch_spots_partitioned_and_gathered_with_gloo():
    """The batched workload's multi-rank form (bench.py --workload batch):
    the spots are partitioned across two ranks, each rank solves its own
    (here with the CPU oracle), and rank 0 gathers every spot's
    exploitability in spot order; each spot is solved exactly once and the
    gathered values equal one process solving them all."""
    from oracle_api import OracleSolver

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] == []
    assert [i for i, _ in res[0]] == list(range(5))
    for i, cfg in enumerate(_spots()):
        o = OracleSolver(cfg)
        o.iterate(3)
        assert res[0][i][1] == o.exploitability()
