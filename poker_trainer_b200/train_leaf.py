"""Trains the leaf-value network on turn subgames solved by the GPU solver.

    python -m poker_trainer_b200.train_leaf [--samples N] [--hidden 1024]
        [--layers 4] [--steps S] [--out weights.npz]
    torchrun --nproc-per-node R -m poker_trainer_b200.train_leaf ...

Under torchrun every rank solves its share of the subgames and training is
data-parallel (train: an NCCL all-reduce of the gradients each step); rank 0
reports.

Generation (leafdata.make_dataset) and training both run on the GPU: the
subgames through libdcfr's solver, the network through libdcfr's BF16
tcgen05 kernels (dcfr_mlp_train_step). Prints one JSON line with the
held-out loss of the network beside two estimators without it: the per-hand
mean of the training targets, and showdown equity (the same state with no
chips behind).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import leafdata
from .mlp import LeafNet


def masked_mse(pred: np.ndarray, y: np.ndarray, m: np.ndarray) -> float:
    return float((m * (pred - y) ** 2).sum() / max(m.sum(), 1.0))


def train(X, Y, M, hidden=1024, layers=4, steps=2000, batch=256, lr=1e-3, seed=0, log=None, group=None, net=None,
          device="cuda", local=False):
    """Adam on minibatches of `batch` samples. With a process group of R
    ranks (poker_trainer_b200.dist.Group over NCCL) training is data-parallel:
    every rank holds the same initial weights, draws its minibatch from its
    own shard of the samples, and the ranks' gradients are summed by an
    all-reduce on the library's device gradient buffer and averaged in the
    Adam step, so the weights stay identical on every rank. `net` (default:
    a new LeafNet) is anything with LeafNet's train_step, backward,
    grad_tensor and adam_step on tensors of `device`. local: X, Y, M are
    already this rank's shard."""
    import torch
    world = group.world if group is not None else 1
    rank = group.rank if group is not None else 0
    n = X.shape[0]
    if net is None:
        net = LeafNet(leafdata.IN_DIM, hidden, layers, leafdata.OUT_DIM, max_batch=batch, seed=seed)
    shard = np.arange(n) if local else np.arange(rank, n, world)
    Xd = torch.tensor(X[shard], device=device)
    Yd = torch.tensor(Y[shard], device=device)
    Md = torch.tensor(M[shard], device=device)
    ns = len(shard)
    rng = np.random.default_rng(seed + 7919 * rank)
    grads = net.grad_tensor() if world > 1 else None
    losses = []
    for s in range(steps):
        idx = torch.tensor(rng.choice(ns, min(batch, ns), replace=False), device=device)
        xb, yb, mb = Xd[idx].contiguous(), Yd[idx].contiguous(), Md[idx].contiguous()
        if world > 1:
            loss = net.backward(xb, yb, mb)
            group.all_reduce_(grads)
            net.adam_step(lr, 1.0 / world)
        else:
            loss = net.train_step(xb, yb, mb, lr=lr)
        losses.append(loss)
        if log and (s % max(1, steps // 10) == 0 or s == steps - 1):
            log(s, loss)
    return net, losses


def predict(net: LeafNet, X: np.ndarray) -> np.ndarray:
    import torch
    out = []
    for i in range(0, X.shape[0], net.max_batch):
        out.append(net.forward(torch.tensor(X[i:i + net.max_batch], device="cuda")).cpu().numpy())
    return np.concatenate(out)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--samples", type=int, default=1024)
    ap.add_argument("--heldout", type=int, default=128)
    ap.add_argument("--hidden", type=int, default=1024)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--target-pct", type=float, default=0.3)
    ap.add_argument("--max-iterations", type=int, default=400)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import torch
    from .dist import Group
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    group = Group("nccl", torch.device("cuda", local_rank))
    t0 = time.perf_counter()
    X, Y, M, _, iters = leafdata.make_dataset(args.samples, seed=4000, target_pct=args.target_pct,
                                              max_iterations=args.max_iterations, part=(group.rank, group.world))
    if group.rank == 0:
        Xh, Yh, Mh, Eh, _ = leafdata.make_dataset(args.heldout, seed=5000, target_pct=args.target_pct,
                                                  max_iterations=args.max_iterations, with_equity=True)
    t_data = group.reduce(time.perf_counter() - t0, "max")
    t0 = time.perf_counter()
    net, losses = train(X, Y, M, args.hidden, args.layers, args.steps, args.batch, args.lr, group=group, local=True)
    t_train = group.reduce(time.perf_counter() - t0, "max")
    group.close()
    if group.rank != 0:
        return
    pred = predict(net, Xh)
    mean = (Y * M).sum(0) / np.maximum(M.sum(0), 1.0)
    line = {
        "samples": args.samples, "heldout": args.heldout, "ranks": group.world,
        "solve_iterations_mean": float(np.mean(iters)),
        "data_seconds": t_data, "train_seconds": t_train, "steps": args.steps,
        "network": {"hidden": args.hidden, "layers": args.layers, "params": net.num_params},
        "train_loss_first": losses[0], "train_loss_last": float(np.mean(losses[-20:])),
        "heldout_mse": {"network": masked_mse(pred, Yh, Mh), "per_hand_mean": masked_mse(mean[None, :], Yh, Mh),
                        "showdown_equity": masked_mse(Eh, Yh, Mh)},
    }
    print(json.dumps(line), flush=True)
    if args.out:
        np.savez_compressed(args.out, params=net.params().astype(np.float16), hidden=args.hidden, layers=args.layers)


if __name__ == "__main__":
    main()
