"""Continuous-batching request loop over tclb_batch.

Requests (a case of some model: node types, settings, iterations) arrive over
time. The loop admits queued requests in arrival order while their device
footprint fits the memory budget and keeps admitted lattices resident. Each
model has one batch on its own stream; the batches run independently: as soon
as a batch's graph replay has finished (a non-blocking query), its finished
cases are retired (Globals and, on request, a quantity are read back), waiting
requests are admitted into it, and its next replay is enqueued -- so the
models' work overlaps on the GPU and no batch waits for another. Time to
solution = completion time - arrival time.

No counterpart in the reference (TCLB runs one case per process).
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional, Tuple

import numpy as np

from . import models as M
from .batch import AdmissionRefused, Batch, CaseSpec, case_bytes


@dataclass
class Request:
    rid: int
    model: str
    spec: CaseSpec
    arrival: float  # seconds since the server clock started
    want_quantity: Optional[str] = None
    # filled in by the server
    admitted: float = -1.0
    finished: float = -1.0
    globals: Optional[np.ndarray] = None
    quantity: Optional[np.ndarray] = None

    @property
    def nodes(self) -> int:
        return int(np.prod(self.spec.shape))

    @property
    def updates(self) -> int:
        return self.nodes * self.spec.niter


class Server:
    def __init__(self, models=("d2q9", "d3q19"), precision="fp32", storage="same", budget_bytes: int = 150 << 30,
                 launch: Optional[Dict[str, Tuple[int, int, int]]] = None, max_cases: int = 4096,
                 high_priority: Tuple[str, ...] = ("d2q9",)):
        self.precision, self.storage = precision, storage
        self.budget = int(budget_bytes)
        self.batches: Dict[str, Batch] = {}
        for m in models:
            # each batch may use the whole budget; the server enforces the sum
            b = Batch(m, precision, storage, budget_bytes=self.budget, max_cases=max_cases)
            b.set_paths(globals_at_end=True)  # a result's Globals are read when it is done
            if launch and m in launch:
                b.set_launch(*launch[m])
            if m in high_priority:  # small cases: their blocks go first
                b.set_priority(True)
            self.batches[m] = b
        self.queue: Deque[Request] = deque()
        self.resident: Dict[Tuple[str, int], Request] = {}
        self.used = 0
        self.done: List[Request] = []
        self.t0 = time.perf_counter()
        self.rounds = 0
        self.busy = 0.0  # seconds with GPU work in flight (step to sync)

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def footprint(self, r: Request) -> int:
        nz, ny, nx = r.spec.shape
        return case_bytes(r.model, nx, ny, nz, self.precision, self.storage)

    def submit(self, r: Request):
        if self.footprint(r) > self.budget:
            raise AdmissionRefused(f"request {r.rid} needs more than the whole budget")
        self.queue.append(r)

    def _admit(self, idle):
        """Admit waiting requests in arrival order into idle batches while the
        budget allows (first come, first served: the head of the queue waits
        for memory, or for its batch's replay in flight)."""
        now = self.now()
        while self.queue and self.queue[0].arrival <= now:
            r = self.queue[0]
            fp = self.footprint(r)
            if self.used + fp > self.budget or not idle[r.model]:
                break
            cid = self.batches[r.model].add_case(r.spec)
            self.queue.popleft()
            self.used += fp
            r.admitted = self.now()
            self.resident[(r.model, cid)] = r

    def _retire(self, model):
        b = self.batches[model]
        for (m, cid), r in list(self.resident.items()):
            if m != model:
                continue
            _done, rem = b.poll(cid)
            if rem > 0:
                continue
            r.globals = b.globals(cid)
            if r.want_quantity:
                r.quantity = b.quantity(cid, r.want_quantity)
            b.remove_case(cid)
            self.used -= self.footprint(r)
            r.finished = self.now()
            del self.resident[(m, cid)]
            self.done.append(r)

    def run(self, requests: List[Request], timeout_s: float = 600.0) -> dict:
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        self.t0 = time.perf_counter()
        inflight = {m: False for m in self.batches}
        t_prev = time.perf_counter()
        while (self.queue or self.resident) and self.now() < timeout_s:
            progressed = False
            for m, b in self.batches.items():
                if inflight[m]:
                    if not b.done():
                        continue
                    b.sync()  # returns at once: updates the case status
                    inflight[m] = False
                    self._retire(m)
                    progressed = True
            idle = {m: not f for m, f in inflight.items()}
            self._admit(idle)
            for m, b in self.batches.items():
                if not inflight[m] and b.pending_updates() > 0:
                    b.step()
                    inflight[m] = True
                    self.rounds += 1
                    progressed = True
            t = time.perf_counter()
            if any(inflight.values()):
                self.busy += t - t_prev  # GPU work was in flight during this interval
            t_prev = t
            if not progressed:
                if not any(inflight.values()) and self.queue:
                    dt = self.queue[0].arrival - self.now()
                    if dt > 0:
                        time.sleep(min(dt, 0.005))
                        t_prev = time.perf_counter()
                else:
                    time.sleep(20e-6)
        wall = self.now()
        return self.report(wall)

    def report(self, wall: float) -> dict:
        tts = np.array([r.finished - r.arrival for r in self.done]) if self.done else np.zeros(1)
        upd = sum(r.updates for r in self.done)
        return {"requests": len(self.done), "wall_s": wall, "cases_per_s": len(self.done) / wall if wall else 0,
                "mlups": upd / wall / 1e6 if wall else 0, "busy_s": self.busy,
                "busy_mlups": upd / self.busy / 1e6 if self.busy else 0, "p50_s": float(np.percentile(tts, 50)),
                "p99_s": float(np.percentile(tts, 99)), "rounds": self.rounds, "pending": len(self.queue) +
                len(self.resident)}

    def close(self):
        for b in self.batches.values():
            b.close()
