"""Replicas across GPUs: one independent lattice per rank, no data exchange.

A single TCLB case is not sharded here (one GPU per case), so a run on N GPUs
is N replicas (or N shares of independent batched cases). The only
cross-rank steps are host coordination: a barrier around the timed region and
reductions of the per-rank device times and work counts. The whole-job rate
is the work all ranks did divided by the slowest rank's time.

The backend is "nccl" with CUDA tensors on GPUs and "gloo" with CPU tensors
(the tests run two gloo ranks on CPU). Rendezvous uses the usual torchrun
environment (MASTER_ADDR, MASTER_PORT, RANK, WORLD_SIZE).
"""
from __future__ import annotations

import datetime
import os
from typing import Optional


def env() -> tuple:
    """(rank, world size, local rank) from the launcher's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        import torch

        self.rank, self.world, self.local = env()
        self.device = "cuda" if backend == "nccl" else "cpu"
        self._torch = torch
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist

            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def barrier(self) -> None:
        """All ranks reach this point (then the local device is drained)."""
        torch = self._torch
        if self._dist is not None:
            t = torch.ones(1, device=self.device)
            self._dist.all_reduce(t)
        if self.device == "cuda":
            torch.cuda.synchronize()

    def _reduce(self, v: float, op) -> float:
        if self._dist is None:
            return float(v)
        t = self._torch.tensor([float(v)], device=self.device, dtype=self._torch.float64)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def reduce_max(self, v: float) -> float:
        return self._reduce(v, None if self._dist is None else self._dist.ReduceOp.MAX)

    def reduce_sum(self, v: float) -> float:
        return self._reduce(v, None if self._dist is None else self._dist.ReduceOp.SUM)

    def whole_job_rate(self, units: float, seconds: float) -> tuple:
        """(units of all ranks / slowest rank's seconds, slowest seconds)."""
        t_max = self.reduce_max(seconds)
        total = self.reduce_sum(units)
        return (total / t_max if t_max > 0 else 0.0), t_max

    def close(self, graphs: Optional[list] = None) -> None:
        if self._dist is not None and self._dist.is_initialized():
            self._dist.destroy_process_group()
        self._dist = None
