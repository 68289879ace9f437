"""Replicas: one process per GPU, hydro events shared out with no data-path
collective.

Events are independent (the reference evolves one event per process), so N
GPUs run N replicas of the single-GPU path on disjoint sets of events.  The
only collectives are the barrier that brackets a timed region and the
reductions of per-rank results (max of durations, sum of counts); a
throughput is the units all ranks processed divided by the slowest rank's
time.  Works with NCCL (one GPU per rank) and with gloo (CPU tests).
"""
from __future__ import annotations

import os
from datetime import timedelta

import torch
import torch.distributed as dist


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self.device = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        if self.backend == "nccl":
            torch.cuda.set_device(self.local)
        if self.world > 1 and not dist.is_initialized():
            kw = {"device_id": self.device} if self.backend == "nccl" else {}
            dist.init_process_group(self.backend, timeout=timedelta(seconds=timeout_s), **kw)

    def barrier(self) -> None:
        if self.world > 1:
            dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return self._reduce(x, dist.ReduceOp.SUM)

    def shard(self, n: int) -> range:
        """The contiguous block of [0, n) this rank owns (sizes differ by at most 1)."""
        q, r = divmod(n, self.world)
        lo = self.rank * q + min(self.rank, r)
        return range(lo, lo + q + (1 if self.rank < r else 0))

    def close(self) -> None:
        if self.world > 1 and dist.is_initialized():
            dist.destroy_process_group()
