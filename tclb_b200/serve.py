"""Continuous-batching request loop over tclb_batch.

Requests (a case of some model: node types, settings, iterations) arrive over
time. Admission (`Admission`, host logic only) keeps one FIFO queue per model
under one device-memory budget: a request is admitted when it has arrived and
its footprint fits; one that waits for memory does not hold up the other
models' requests unless it has waited longer than a bound, after which
nothing younger goes ahead of it. An admitted request is reserved at once; it
joins its model's batch at the batch's next replay boundary (a pending list),
so admission never waits for a replay in flight. Admitted lattices stay
resident. Each model has one batch on its own stream and the batches run
independently: when a batch's graph replay has finished (a non-blocking
query), its finished and cancelled cases are retired (Globals and, on
request, a quantity are read back for finished ones), its pending cases join,
and its next replay is enqueued -- so the models' work overlaps on the GPU.
A request can be cancelled while it waits, while it is pending, or while it
runs (it leaves at its batch's next boundary). Time to solution = completion
time - arrival time.

Optionally (`solo_nodes`), a request of at least that many nodes runs as a
lattice of its own instead of joining its model's batch: one of the largest
cases fills the GPU alone, and the one-lattice kernels carry none of the
batch's per-tile case descriptors, so they run faster on it. It starts as soon
as it is admitted, on its own stream, in chunks of `solo_iters` iterations
whose completion is queried without blocking; its last iteration computes
its Globals. Admission, the budget, cancellation and results are the same.

No counterpart in the reference (TCLB runs one case per process).
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import models as M
from .batch import AdmissionRefused, Batch, CaseSpec, case_bytes


@dataclass
class _Solo:
    """A request running as a lattice of its own."""

    request: "Request"
    lattice: object
    stream: object
    remaining: int
    event: object = None  # completion of the chunk in flight
    chunk: int = 0
    cancel: bool = False


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
    cancelled: bool = False
    globals: Optional[np.ndarray] = None
    quantity: Optional[np.ndarray] = None

    @property
    def nodes(self) -> int:
        return int(np.prod(self.spec.shape))

    @property
    def updates(self) -> int:
        return self.nodes * self.spec.niter


class Admission:
    """Admission under one device-memory budget, one FIFO queue per model.

    `admit(now)` takes the queue heads that have arrived, oldest first, and
    admits each whose footprint fits what is left of the budget. A head that
    does not fit leaves the other queues free to go on -- unless it has been
    waiting for memory for `max_bypass_s` or longer: then nothing else is
    admitted until it fits (no request starves behind a stream of smaller
    ones). `release` returns a finished or cancelled request's memory.
    """

    def __init__(self, budget_bytes: int, footprint: Callable[[Request], int], models=(), max_bypass_s: float = 5.0):
        self.budget = int(budget_bytes)
        self.footprint = footprint
        self.max_bypass_s = float(max_bypass_s)
        self.queues: Dict[str, Deque[Request]] = {m: deque() for m in models}
        self.used = 0
        self._blocked: Dict[int, float] = {}  # rid -> when it first did not fit

    def submit(self, r: Request):
        if self.footprint(r) > self.budget:
            raise AdmissionRefused(f"request {r.rid} needs more than the whole budget")
        self.queues.setdefault(r.model, deque()).append(r)

    def cancel(self, rid: int) -> Optional[Request]:
        """Remove a waiting request; None if no queue holds it."""
        for q in self.queues.values():
            for r in q:
                if r.rid == rid:
                    q.remove(r)
                    self._blocked.pop(rid, None)
                    return r
        return None

    def admit(self, now: float) -> List[Request]:
        out: List[Request] = []
        while True:
            heads = sorted((q[0] for q in self.queues.values() if q and q[0].arrival <= now),
                           key=lambda r: r.arrival)
            took = False
            for r in heads:
                fp = self.footprint(r)
                if self.used + fp <= self.budget:
                    self.queues[r.model].popleft()
                    self._blocked.pop(r.rid, None)
                    self.used += fp
                    out.append(r)
                    took = True
                    break  # the heads change: look again, oldest first
                if now - self._blocked.setdefault(r.rid, now) >= self.max_bypass_s:
                    return out  # it has waited long enough: nothing younger goes ahead of it
            if not took:
                return out

    def release(self, r: Request):
        self.used -= self.footprint(r)

    def waiting(self) -> int:
        return sum(len(q) for q in self.queues.values())


class Server:
    def __init__(self, models=("d2q9", "d3q19"), precision="fp32", storage="same", budget_bytes: int = 150 << 30,
                 launch: Optional[Dict[str, Tuple[int, int, int]]] = None, max_cases: int = 4096,
                 high_priority: Tuple[str, ...] = ("d2q9",), max_bypass_s: float = 5.0,
                 reserve: Optional[Dict[str, int]] = None, solo_nodes: Optional[int] = None,
                 solo_iters: int = 64):
        """reserve: device bytes to set aside per model at start-up (Batch.reserve), so that the
        first admissions take memory from the pools like those of a server that has been running;
        the sum must stay within the budget. The reserve does not count against the budget, and a
        request run as a lattice of its own (solo_nodes) allocates its memory outside the pools
        (its footprint does count), so budget + reserve must fit the device."""
        if reserve and sum(reserve.values()) > budget_bytes:
            raise ValueError("reserve exceeds the budget")
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
            if reserve and reserve.get(m):
                b.reserve(reserve[m])
            self.batches[m] = b
        self.adm = Admission(self.budget, self.footprint, models, max_bypass_s)
        self.pending: Dict[str, List[Request]] = {m: [] for m in models}  # admitted, joining at the next boundary
        self.resident: Dict[Tuple[str, int], Request] = {}
        self.done: List[Request] = []
        self.cancelled: List[Request] = []
        self._cancel_resident: set = set()
        self.solo_nodes, self.solo_iters = solo_nodes, int(solo_iters)
        self.solo: Dict[int, _Solo] = {}  # rid -> a request running as its own lattice
        self.t0 = time.perf_counter()
        self.rounds = 0
        self.busy = 0.0  # seconds with GPU work in flight (step to sync)
        self.busy_by_model: Dict[str, float] = {m: 0.0 for m in models}  # seconds each model's batch was in flight
        self.busy_all = 0.0  # seconds every model's batch was in flight at once

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def footprint(self, r: Request) -> int:
        nz, ny, nx = r.spec.shape
        return case_bytes(r.model, nx, ny, nz, self.precision, self.storage)

    @property
    def used(self) -> int:
        return self.adm.used

    def submit(self, r: Request):
        self.adm.submit(r)

    def cancel(self, rid: int) -> bool:
        """Cancel a request: a waiting or pending one leaves at once, a running one at its batch's next
        boundary. False if the request is unknown, finished or already cancelled."""
        r = self.adm.cancel(rid)
        if r is not None:
            self._mark_cancelled(r, release=False)
            return True
        for m, lst in self.pending.items():
            for r in lst:
                if r.rid == rid:
                    lst.remove(r)
                    self._mark_cancelled(r)
                    return True
        for (m, cid), r in self.resident.items():
            if r.rid == rid and not r.cancelled:
                self._cancel_resident.add((m, cid))
                return True
        if rid in self.solo and not self.solo[rid].cancel:
            self.solo[rid].cancel = True  # leaves when its chunk in flight has finished
            return True
        return False

    def _mark_cancelled(self, r: Request, release: bool = True):
        if release:
            self.adm.release(r)
        r.cancelled = True
        r.finished = self.now()
        self.cancelled.append(r)

    def _admit(self):
        """Admit what has arrived and fits (per-model queues, see Admission); admitted requests wait in their
        model's pending list for the batch's next replay boundary."""
        for r in self.adm.admit(self.now()):
            r.admitted = self.now()
            if self.solo_nodes is not None and r.nodes >= self.solo_nodes:
                self._start_solo(r)
            else:
                self.pending[r.model].append(r)

    def _start_solo(self, r: Request):
        import torch

        from .lattice import Lattice

        nz, ny, nx = r.spec.shape
        lat = Lattice(r.model, nx, ny, nz, precision=self.precision, storage=self.storage)
        fl = r.spec.flags if r.spec.flags.ndim == 3 else r.spec.flags[None]
        lat.set_flags(np.ascontiguousarray(fl, np.uint16))
        for k, v in r.spec.settings.items():
            lat.SetSetting(k, v)
        for z, d in r.spec.zone_settings.items():
            for k, v in d.items():
                lat.set_zone_setting(k, v, z)
        lat.Init()  # BaseInit equilibrium, as a batch case starts
        self.solo[r.rid] = _Solo(r, lat, torch.cuda.Stream(), int(r.spec.niter))

    def _step_solo(self, sl: _Solo) -> bool:
        """Advance one request running as its own lattice; True if anything happened."""
        r = sl.request
        if sl.event is not None:
            if not sl.event.query():
                return False
            sl.event = None
            sl.remaining -= sl.chunk
        if sl.cancel:
            sl.lattice.close()
            del self.solo[r.rid]
            self._mark_cancelled(r)
            return True
        if sl.remaining <= 1:
            if sl.remaining == 1:  # the last iteration integrates the Globals (returns when done)
                sl.lattice.Iterate(1, M.ITER_NORM | M.ITER_LASTGLOB, stream=sl.stream.cuda_stream)
            r.globals = sl.lattice.globals
            if r.want_quantity:
                r.quantity = sl.lattice.GetQuantity(r.want_quantity)
            sl.lattice.close()
            del self.solo[r.rid]
            self.adm.release(r)
            r.finished = self.now()
            self.done.append(r)
            return True
        import torch

        sl.chunk = min(sl.remaining - 1, self.solo_iters)
        sl.lattice.Iterate(sl.chunk, M.ITER_NORM, stream=sl.stream.cuda_stream)
        sl.event = torch.cuda.Event()
        sl.event.record(sl.stream)
        return True

    def _join(self, model):
        """At a replay boundary of the model's batch: its pending cases join."""
        b = self.batches[model]
        for r in self.pending[model]:
            cid = b.add_case(r.spec)
            self.resident[(model, cid)] = r
        self.pending[model] = []

    def _retire(self, model):
        b = self.batches[model]
        for (m, cid), r in list(self.resident.items()):
            if m != model:
                continue
            if (m, cid) in self._cancel_resident:
                self._cancel_resident.discard((m, cid))
                b.remove_case(cid)
                del self.resident[(m, cid)]
                self._mark_cancelled(r)
                continue
            _done, rem = b.poll(cid)
            if rem > 0:
                continue
            r.globals = b.globals(cid)
            if r.want_quantity:
                r.quantity = b.quantity(cid, r.want_quantity)
            b.remove_case(cid)
            self.adm.release(r)
            r.finished = self.now()
            del self.resident[(m, cid)]
            self.done.append(r)

    def run(self, requests: List[Request], timeout_s: float = 600.0,
            cancels: Sequence[Tuple[float, int]] = ()) -> dict:
        """Serve `requests` (arrival times relative to the start); `cancels` are (time, request id) events."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        cancel_events = sorted(cancels)
        self.t0 = time.perf_counter()
        inflight = {m: False for m in self.batches}
        t_prev = time.perf_counter()
        while (self.adm.waiting() or any(self.pending.values()) or self.resident or self.solo) and \
                self.now() < timeout_s:
            progressed = False
            while cancel_events and cancel_events[0][0] <= self.now():
                self.cancel(cancel_events.pop(0)[1])
            self._admit()
            for m, b in self.batches.items():
                if inflight[m]:
                    if not b.done():
                        continue
                    b.sync()  # returns at once: updates the case status
                    inflight[m] = False
                    self._retire(m)
                    progressed = True
                if self.pending[m] or self._cancel_resident:
                    self._retire(m)  # cancelled cases leave before new ones join
                    self._join(m)
                if b.pending_updates() > 0:
                    b.step()
                    inflight[m] = True
                    self.rounds += 1
                    progressed = True
            # a model with a lattice of its own in flight during this interval, including one whose
            # chunk completes now and whose last (Globals) iteration runs in _step_solo, counts as busy
            solo_busy = {sl.request.model for sl in self.solo.values() if sl.event is not None}
            for sl in list(self.solo.values()):
                solo_busy |= {sl.request.model} if sl.remaining <= 1 or sl.event is not None else set()
                progressed = self._step_solo(sl) or progressed
            solo_busy |= {sl.request.model for sl in self.solo.values() if sl.event is not None}
            t = time.perf_counter()
            busy = {m: f or m in solo_busy for m, f in inflight.items()}
            if any(busy.values()):
                self.busy += t - t_prev  # GPU work was in flight during this interval
                for m, f in busy.items():
                    if f:
                        self.busy_by_model[m] += t - t_prev
                if all(busy.values()):
                    self.busy_all += t - t_prev
            t_prev = t
            if not progressed:
                if not any(inflight.values()) and not any(sl.event is not None for sl in self.solo.values()):
                    nxt = [q[0].arrival for q in self.adm.queues.values() if q]
                    dt = (min(nxt) - self.now()) if nxt else 0.0
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
                "p99_s": float(np.percentile(tts, 99)), "rounds": self.rounds, "cancelled": len(self.cancelled),
                "busy_by_model_s": dict(self.busy_by_model), "busy_all_models_s": self.busy_all,
                "updates_by_model": {m: sum(r.updates for r in self.done if r.model == m) for m in self.batches},
                "pending": self.adm.waiting() + sum(len(v) for v in self.pending.values()) + len(self.resident) +
                len(self.solo)}

    def close(self):
        for sl in self.solo.values():
            sl.lattice.close()
        self.solo.clear()
        for b in self.batches.values():
            b.close()
