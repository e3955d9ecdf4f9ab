"""One process per GPU for the multi-GPU runs.

The solves shard by spot (independent units): every rank solves its own
spots with no collective on the data path; torch.distributed is used there
only for the plumbing around the timed region (a barrier on entry and exit,
and the maximum of the ranks' device times). The leaf network's
data-parallel training sums gradients with an all-reduce (all_reduce_).
"""
from __future__ import annotations

import datetime as dt
import os


class Group:
    """The process group of a run (world size 1: no group at all)."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": dt.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def reduce(self, x: float, op: str = "max") -> float:
        """x reduced over ranks (max or sum)."""
        if self.dist is None:
            return x
        import torch
        dev = self.device if (self.backend == "nccl" and self.device is not None) else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def all_reduce_(self, t):
        """Sum of the tensor t over ranks, in place (NCCL for CUDA tensors,
        gloo for CPU ones); waits for the result."""
        if self.dist is None:
            return t
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        if t.is_cuda:
            import torch
            torch.cuda.synchronize(t.device)
        return t

    def gather_concat(self, items: list) -> list:
        """Every rank's list, concatenated in rank order, on rank 0 (other
        ranks get []); the lists may differ in length."""
        if self.dist is None:
            return list(items)
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object(list(items), out, dst=0)
        return [x for part in out for x in part] if self.rank == 0 else []

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def shard(items, rank: int, world: int):
    """The items rank `rank` of `world` owns: a contiguous block, sizes
    differing by at most one."""
    n = len(items)
    lo = rank * n // world
    hi = (rank + 1) * n // world
    return items[lo:hi]
