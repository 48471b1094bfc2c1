"""Replica plumbing for running independent simulations on several GPUs of one node.

A single k-space simulation does not shard (its global FFTs would need all-to-all transposes),
so multi-GPU work is replicas: one process per GPU, launched by torchrun, each running its own
simulations with no collective on the data path. What the processes share is host-side
bookkeeping: a rendezvous, barriers around a timed region, the slowest rank's time and, for a set
of independent simulations (batch members, scan lines, finite-difference directions), which rank
runs which. These helpers do that over torch.distributed: NCCL on GPUs, gloo on CPU (tests).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional


@dataclass
class Replicas:
    world: int
    rank: int
    local: int
    dist: Optional[object]   # torch.distributed when world > 1

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, value: float, device: str = "cpu") -> float:
        """The largest `value` over all ranks (the slowest rank's time)."""
        if self.dist is None:
            return float(value)
        import torch
        t = torch.tensor([float(value)], device=device, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, value: float, device: str = "cpu") -> float:
        if self.dist is None:
            return float(value)
        import torch
        t = torch.tensor([float(value)], device=device, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def my_items(self, n: int) -> list[int]:
        """Indices of `n` independent items this rank runs: contiguous, balanced to within one."""
        return own_range(n, self.world, self.rank)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def own_range(n: int, world: int, rank: int) -> list[int]:
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return list(range(lo, lo + base + (1 if rank < extra else 0)))


def init(backend: str = "nccl", timeout_s: int = 300) -> Replicas:
    """Join the job torchrun started (WORLD_SIZE / RANK / LOCAL_RANK / MASTER_* from the
    environment); a single process needs no process group."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return Replicas(world, rank, local, dist)
