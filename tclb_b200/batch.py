"""Batches of independent cases over the C ABI (tclb_batch_*), and the
autotuner that picks their launch shape.

A batch holds cases of one model/precision/storage; each ``step()`` enqueues
one CUDA-graph replay that advances every active case by up to K iterations,
one launch per iteration for all cases (one thread block per tile by
default). No counterpart in the reference (TCLB runs one lattice per
process).
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import models as M
from .lattice import PRECISION, STORAGE, TCLBError, load_library

_bound = False


def _lib():
    global _bound
    L = load_library()
    if not _bound:
        h, i, d, vp, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
        ip = ctypes.POINTER(ctypes.c_int)
        dp = ctypes.POINTER(ctypes.c_double)
        L.tclb_batch_last_error.restype = ctypes.c_char_p
        L.tclb_batch_case_bytes.argtypes = [i, i, i, i, i, i]
        L.tclb_batch_case_bytes.restype = sz
        L.tclb_batch_create.argtypes = [ctypes.POINTER(h), i, i, i, sz, i]
        L.tclb_batch_destroy.argtypes = [h]
        L.tclb_batch_reserve.argtypes = [h, sz]
        L.tclb_batch_add_case.argtypes = [h, i, i, i, ctypes.POINTER(ctypes.c_uint16), dp, dp, i, i, ip]
        L.tclb_batch_remove_case.argtypes = [h, i]
        L.tclb_batch_set_launch.argtypes = [h, i, i, i, i]
        L.tclb_batch_get_launch.argtypes = [h, ip, ip, ip]
        L.tclb_batch_step.argtypes = [h]
        L.tclb_batch_sync.argtypes = [h]
        L.tclb_batch_done.argtypes = [h]
        L.tclb_batch_set_priority.argtypes = [h, i]
        L.tclb_batch_set_paths.argtypes = [h, i]
        L.tclb_batch_get_paths.argtypes = [h, ip]
        L.tclb_batch_poll.argtypes = [h, i, ctypes.POINTER(ctypes.c_longlong), ip]
        L.tclb_batch_get_globals.argtypes = [h, i, dp]
        L.tclb_batch_get_quantity.argtypes = [h, i, i, vp, d]
        L.tclb_batch_info.argtypes = [h, ip, ip, ctypes.POINTER(sz), ctypes.POINTER(sz)]
        L.tclb_batch_pending_updates.argtypes = [h]
        L.tclb_batch_pending_updates.restype = ctypes.c_longlong
        _bound = True
    return L


def _check(rc: int):
    if rc != 0:
        raise TCLBError(_lib().tclb_batch_last_error().decode() or f"error {rc}")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class AdmissionRefused(TCLBError):
    pass


@dataclass
class CaseSpec:
    """One case: node types, settings by name, zonal settings by zone, iterations."""

    flags: np.ndarray  # (nz, ny, nx) uint16
    settings: Dict[str, float]
    zone_settings: Dict[int, Dict[str, float]]
    niter: int

    @property
    def shape(self) -> Tuple[int, int, int]:
        f = self.flags if self.flags.ndim == 3 else self.flags[None]
        return f.shape


def case_bytes(model, nx, ny, nz=1, precision="fp32", storage="same") -> int:
    m = M.get(model)
    return int(_lib().tclb_batch_case_bytes(m.mid, PRECISION[precision], STORAGE[storage], nx, ny, nz))


class Batch:
    def __init__(self, model, precision="fp32", storage="same", budget_bytes: int = 8 << 30, max_cases: int = 4096):
        self.lib = _lib()
        self.model = M.get(model)
        self.precision, self.storage = precision, storage
        self.real = np.float64 if precision == "fp64" else np.float32
        h = ctypes.c_void_p()
        _check(self.lib.tclb_batch_create(ctypes.byref(h), self.model.mid, PRECISION[precision], STORAGE[storage],
                                          int(budget_bytes), int(max_cases)))
        self._h = h
        self.shapes: Dict[int, Tuple[int, int, int]] = {}

    def close(self):
        if getattr(self, "_h", None):
            self.lib.tclb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, nbytes: int):
        """Grow the device memory pool to hold nbytes for future cases (at most the budget), so that
        admissions within it do not map new device memory (tclb_batch_reserve)."""
        rc = self.lib.tclb_batch_reserve(self._h, int(nbytes))
        if rc == -3:
            raise AdmissionRefused(self.lib.tclb_batch_last_error().decode())
        _check(rc)

    # -- cases -----------------------------------------------------------------
    def settings_vector(self, settings: Dict[str, float]) -> np.ndarray:
        vals = self.model.default_settings()
        for k, v in settings.items():
            self.model.apply_setting(vals, k, float(v))
        return np.array(vals, np.float64)

    def zone_table(self, zone_settings: Dict[int, Dict[str, float]]) -> Tuple[np.ndarray, int]:
        nzs = len(self.model.zone_settings)
        rows = (max(zone_settings) + 1) if zone_settings else 0
        t = np.zeros((max(rows, 1), nzs))
        for z in range(rows):
            t[z] = [s.default for s in self.model.zone_settings]
        for z, d in zone_settings.items():
            for k, v in d.items():
                t[z, self.model.zone_setting_index(k)] = v
        return t, rows

    def add_case(self, spec: CaseSpec) -> int:
        fl = np.ascontiguousarray(spec.flags, np.uint16)
        if fl.ndim == 2:
            fl = fl[None]
        nz, ny, nx = fl.shape
        s = self.settings_vector(spec.settings)
        zt, rows = self.zone_table(spec.zone_settings)
        cid = ctypes.c_int()
        rc = self.lib.tclb_batch_add_case(self._h, nx, ny, nz, fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                          _dp(s), _dp(zt), rows, int(spec.niter), ctypes.byref(cid))
        if rc == -3:
            raise AdmissionRefused(self.lib.tclb_batch_last_error().decode())
        _check(rc)
        self.shapes[cid.value] = (nz, ny, nx)
        return cid.value

    def remove_case(self, cid: int):
        _check(self.lib.tclb_batch_remove_case(self._h, cid))
        self.shapes.pop(cid, None)

    # -- running ---------------------------------------------------------------
    def set_launch(self, bx: int, by: int, iters_per_launch: int, grid_blocks: int = 0):
        _check(self.lib.tclb_batch_set_launch(self._h, bx, by, iters_per_launch, grid_blocks))

    def get_launch(self) -> Tuple[int, int, int]:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.lib.tclb_batch_get_launch(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def set_paths(self, use_pairs: bool = True, adaptive: bool = True, use_tma: bool = True,
                  globals_at_end: bool = False):
        """use_pairs: 16-bit storage lets plain launches update two nodes per
        thread when the tile shape allows it. use_tma: 16-bit cases whose rows
        fit one TMA box take the tile-staged kernel. adaptive: lower the tile
        height, and leave the tile-staged kernel out, while the live cases give
        too few tiles to fill the GPU. These three are on by default.
        globals_at_end (off by default): a case's Globals are computed only in
        the replay where it finishes (globals() holds them once it is done)."""
        flags = (2 if use_pairs else 0) | (4 if use_tma else 0) | (8 if adaptive else 0) | \
            (16 if globals_at_end else 0)
        _check(self.lib.tclb_batch_set_paths(self._h, flags))

    def _paths(self) -> int:
        f = ctypes.c_int()
        _check(self.lib.tclb_batch_get_paths(self._h, ctypes.byref(f)))
        return f.value

    def uses_pairs(self) -> bool:
        """True when the plain launches of the current shape take the
        two-nodes-per-thread kernel (for the cases not tile-staged)."""
        return bool(self._paths() & 2)

    def uses_tma(self) -> bool:
        """True when at least one live case takes the tile-staged kernel."""
        return bool(self._paths() & 4)

    def step(self):
        _check(self.lib.tclb_batch_step(self._h))

    def sync(self):
        _check(self.lib.tclb_batch_sync(self._h))

    def set_priority(self, high: bool):
        """Schedule this batch's blocks ahead of normal-priority batches."""
        _check(self.lib.tclb_batch_set_priority(self._h, 1 if high else 0))

    def done(self) -> bool:
        """True when the enqueued replays have finished (never blocks)."""
        rc = self.lib.tclb_batch_done(self._h)
        if rc < 0:
            _check(rc)
        return rc == 1

    def poll(self, cid: int) -> Tuple[int, int]:
        done, rem = ctypes.c_longlong(), ctypes.c_int()
        _check(self.lib.tclb_batch_poll(self._h, cid, ctypes.byref(done), ctypes.byref(rem)))
        return done.value, rem.value

    def pending_updates(self) -> int:
        return int(self.lib.tclb_batch_pending_updates(self._h))

    def run_to_completion(self, max_steps: int = 1 << 30) -> int:
        steps = 0
        while self.pending_updates() > 0 and steps < max_steps:
            self.step()
            self.sync()
            steps += 1
        return steps

    # -- results ---------------------------------------------------------------
    def globals(self, cid: int) -> np.ndarray:
        out = np.zeros(len(self.model.globals))
        _check(self.lib.tclb_batch_get_globals(self._h, cid, _dp(out)))
        return out

    def quantity(self, cid: int, name, scale: float = 1.0) -> np.ndarray:
        q = name if isinstance(name, int) else self.model.quantity_index(name)
        vec = self.model.quantities[q][1]
        shp = self.shapes[cid] + ((3,) if vec else ())
        out = np.zeros(shp, self.real)
        _check(self.lib.tclb_batch_get_quantity(self._h, cid, q, ctypes.c_void_p(out.ctypes.data), float(scale)))
        return out

    def info(self) -> dict:
        n, t = ctypes.c_int(), ctypes.c_int()
        u, b = ctypes.c_size_t(), ctypes.c_size_t()
        _check(self.lib.tclb_batch_info(self._h, ctypes.byref(n), ctypes.byref(t), ctypes.byref(u), ctypes.byref(b)))
        return {"cases": n.value, "tiles": t.value, "used_bytes": u.value, "budget_bytes": b.value}


# ---------------------------------------------------------------------------
# Autotuner
# ---------------------------------------------------------------------------
# tiles bx x by nodes; a block has at most 256 threads and walks taller tiles
TILE_CANDIDATES = [(32, 8), (32, 32), (32, 64), (64, 16), (64, 64), (128, 16), (256, 8)]
K_CANDIDATES = [1, 4, 16, 64]


def autotune(model, specs: Sequence[CaseSpec], precision="fp32", storage="same", tiles=TILE_CANDIDATES,
             ks=K_CANDIDATES, trial_iters: int = 64, budget_bytes: int = 16 << 30, globals_at_end=False) -> dict:
    """Pick the tile shape and iterations per launch that maximise node updates
    per second on a scratch batch holding the given cases (the caller's cases
    are not advanced), with the Globals mode the caller will use. Returns
    {"bx","by","K","mlups","table"}."""
    b = Batch(model, precision, storage, budget_bytes=budget_bytes, max_cases=max(1, len(specs)))
    b.set_paths(globals_at_end=globals_at_end)
    big = 1 << 30
    try:
        for s in specs:
            b.add_case(CaseSpec(s.flags, s.settings, s.zone_settings, big))
        nodes = sum(int(np.prod(s.shape)) for s in specs)
        table = []
        for (bx, by) in tiles:
            for K in ks:
                b.set_launch(bx, by, K)
                reps = max(1, trial_iters // K)
                b.step()  # capture + warm
                b.sync()
                t0 = time.perf_counter()
                for _ in range(reps):
                    b.step()
                b.sync()
                dt = time.perf_counter() - t0
                table.append({"bx": bx, "by": by, "K": K, "mlups": nodes * K * reps / dt / 1e6})
        best = max(table, key=lambda r: r["mlups"])
        return {"bx": best["bx"], "by": best["by"], "K": best["K"], "mlups": best["mlups"], "table": table}
    finally:
        b.close()
