"""Replicas across GPUs: one independent lattice per rank, no data exchange.

A single TCLB case is not sharded here (one GPU per case), so a run on N GPUs
is N replicas, or N shares of independent batched cases (partition_cases,
every case on exactly one rank). The only cross-rank steps are host
coordination: a barrier around the timed region, reductions of the per-rank
times and work counts, and a gather of per-case results. The whole-job rate
is the work all ranks did divided by the slowest rank's time.

The backend is "nccl" with CUDA tensors on GPUs and "gloo" with CPU tensors
(the tests run two gloo ranks on CPU). Rendezvous uses the usual torchrun
environment (MASTER_ADDR, MASTER_PORT, RANK, WORLD_SIZE).
"""
from __future__ import annotations

import datetime
import os
from typing import Optional


def partition_cases(weights, world: int) -> list:
    """Indices of the cases for each of `world` ranks: largest first, each to
    the rank with the least work so far (ties to the lower rank), so the
    ranks' shares of the total work differ by at most the largest case.
    Deterministic: every rank computes the same partition."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda i: (-weights[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += weights[i]
    return [sorted(p) for p in parts]


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

    def gather(self, obj) -> list:
        """Every rank's obj (a picklable host value), in rank order."""
        if self._dist is None:
            return [obj]
        out = [None] * self.world
        self._dist.all_gather_object(out, obj)
        return out

    def whole_job_rate(self, units: float, seconds: float) -> tuple:
        """(units of all ranks / slowest rank's seconds, slowest seconds)."""
        t_max = self.reduce_max(seconds)
        total = self.reduce_sum(units)
        return (total / t_max if t_max > 0 else 0.0), t_max

    def close(self, graphs: Optional[list] = None) -> None:
        if self._dist is not None and self._dist.is_initialized():
            self._dist.destroy_process_group()
        self._dist = None
