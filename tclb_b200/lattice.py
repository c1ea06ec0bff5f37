"""Host-side mirror of TCLB's ``Lattice`` (src/Lattice.h.Rt:39-191) over the C ABI.

Method names follow the reference (``FlagOverwrite``, ``SetSetting``, ``Init``,
``Iterate``, ``globals``, ``GetQuantity``, ``save``/``load``); arguments keep
their meaning. Errors raise ``TCLBError`` carrying the library's message, where
TCLB would print and exit (src/cross.cu:24-32).

The shared library is required: there is no CPU fallback. Importing works on a
machine without a GPU, but creating a lattice there fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import models as M

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtclb_b200.so")

FP32, FP64 = 0, 1
STORAGE = {"same": 0, "fp16": 1, "fp16s": 2, "bf16": 3, "bf16s": 4}
PRECISION = {"fp32": FP32, "fp64": FP64}

_lib = None


class TCLBError(RuntimeError):
    pass


def load_library(path: Optional[str] = None):
    """Load libtclb_b200.so (built in-tree by tclb_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise TCLBError(f"CUDA library missing: {p} (build it with `python -m tclb_b200.build`)")
    L = ctypes.CDLL(p)
    h, i, d, vp, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    L.tclb_last_error.restype = ctypes.c_char_p
    L.tclb_model_info.argtypes = [i, ip, ip, ip, ip, ip, ip]
    L.tclb_model_item.argtypes = [i, i, i, ctypes.POINTER(ctypes.c_char_p), ip, ip]
    L.tclb_create.argtypes = [ctypes.POINTER(h), i, i, i, i, i, i]
    L.tclb_destroy.argtypes = [h]
    L.tclb_get_size.argtypes = [h, ip, ip, ip]
    L.tclb_set_flags.argtypes = [h, ctypes.POINTER(ctypes.c_uint16), i, i, i, i, i, i]
    L.tclb_get_flags.argtypes = [h, ctypes.POINTER(ctypes.c_uint16)]
    L.tclb_set_setting.argtypes = [h, i, d]
    L.tclb_get_setting.argtypes = [h, i, dp]
    L.tclb_set_zone_setting.argtypes = [h, i, i, d]
    L.tclb_init.argtypes = [h]
    L.tclb_iterate.argtypes = [h, i, i, vp]
    L.tclb_init_equilibrium.argtypes = [h, vp, vp, vp]
    L.tclb_get_globals.argtypes = [h, dp]
    L.tclb_clear_globals.argtypes = [h]
    L.tclb_get_quantity.argtypes = [h, i, ip, vp, d, vp]
    L.tclb_get_quantity_noalloc.argtypes = [h, i, ip, vp, d, vp]
    L.tclb_get_densities.argtypes = [h, dp]
    L.tclb_set_densities.argtypes = [h, dp]
    L.tclb_snapshot_bytes.argtypes = [h]
    L.tclb_snapshot_bytes.restype = sz
    L.tclb_save.argtypes = [h, vp, sz, vp]
    L.tclb_load.argtypes = [h, vp, sz, vp]
    L.tclb_get_iteration.argtypes = [h, ctypes.POINTER(ctypes.c_longlong)]
    L.tclb_bytes_per_update.argtypes = [h]
    L.tclb_bytes_per_update.restype = d
    L.tclb_sync.argtypes = [h]
    L.tclb_set_launch.argtypes = [h, i, i, i]
    L.tclb_pri_bytes.argtypes = [h]
    L.tclb_pri_bytes.restype = sz
    L.tclb_save_pri.argtypes = [h, vp, sz]
    L.tclb_load_pri.argtypes = [h, vp, sz]
    L.tclb_color.argtypes = [h, vp, i, i, vp]
    L.tclb_get_launch.argtypes = [h, ip, ip, ip]
    L.tclb_set_fault_injection.argtypes = [h, i, ctypes.c_longlong]
    L.tclb_energy_enstrophy.argtypes = [h, dp, vp]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise TCLBError(load_library().tclb_last_error().decode() or f"error {rc}")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Lattice:
    """One lattice of a TCLB model on the current CUDA device."""

    def __init__(self, model, nx: int, ny: int, nz: int = 1, precision: str = "fp32", storage: str = "same"):
        self.lib = load_library()
        self.model = M.get(model)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.shape = (nz, ny, nx)
        self.precision = precision
        self.storage = storage
        self.real = np.float64 if precision == "fp64" else np.float32
        h = ctypes.c_void_p()
        _check(self.lib.tclb_create(ctypes.byref(h), self.model.mid, nx, ny, nz, PRECISION[precision],
                                    STORAGE[storage]))
        self._h = h

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self.lib.tclb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- geometry / settings ---------------------------------------------------
    def FlagOverwrite(self, flags: np.ndarray, offset: Sequence[int] = (0, 0, 0)):
        """Copy a (nz, ny, nx) box of node types at offset (dx, dy, dz)."""
        fl = np.ascontiguousarray(flags, dtype=np.uint16)
        if fl.ndim == 2:
            fl = fl[None]
        bz, by, bx = fl.shape
        dx, dy, dz = offset
        _check(self.lib.tclb_set_flags(self._h, fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), dx, dy, dz, bx,
                                       by, bz))

    set_flags = FlagOverwrite

    def get_flags(self) -> np.ndarray:
        out = np.zeros(self.shape, np.uint16)
        _check(self.lib.tclb_get_flags(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))))
        return out

    def SetSetting(self, name, value: float):
        i = name if isinstance(name, int) else self.model.setting_index(name)
        _check(self.lib.tclb_set_setting(self._h, i, float(value)))

    set_setting = SetSetting

    def get_setting(self, name) -> float:
        i = name if isinstance(name, int) else self.model.setting_index(name)
        v = ctypes.c_double()
        _check(self.lib.tclb_get_setting(self._h, i, ctypes.byref(v)))
        return v.value

    def set_zone_setting(self, name, value: float, zone: int = -1):
        i = name if isinstance(name, int) else self.model.zone_setting_index(name)
        _check(self.lib.tclb_set_zone_setting(self._h, i, zone, float(value)))

    # -- run -------------------------------------------------------------------
    def Init(self):
        _check(self.lib.tclb_init(self._h))

    def init_equilibrium(self, rho: np.ndarray, u: np.ndarray, stream: int = 0):
        """Equilibrium at density rho (N) and velocity u (N x 3), x fastest."""
        r = np.ascontiguousarray(rho, dtype=self.real).reshape(-1)
        v = np.ascontiguousarray(u, dtype=self.real).reshape(-1)
        assert r.size == self.N and v.size == 3 * self.N
        _check(self.lib.tclb_init_equilibrium(self._h, ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(v.ctypes.data),
                                              ctypes.c_void_p(stream or None)))

    def Iterate(self, niter: int, iter_type: int = M.ITER_NORM, stream: int = 0):
        _check(self.lib.tclb_iterate(self._h, int(niter), int(iter_type), ctypes.c_void_p(stream or None)))

    iterate = Iterate

    @property
    def globals(self) -> np.ndarray:
        out = np.zeros(len(self.model.globals))
        _check(self.lib.tclb_get_globals(self._h, _dp(out)))
        return out

    def globals_dict(self) -> dict:
        return dict(zip([g[0] for g in self.model.globals], self.globals))

    def clearGlobals(self):
        _check(self.lib.tclb_clear_globals(self._h))

    def GetQuantity(self, name, region: Optional[Sequence[int]] = None, scale: float = 1.0, out=None,
                    stream: int = 0) -> np.ndarray:
        q = name if isinstance(name, int) else self.model.quantity_index(name)
        vec = self.model.quantities[q][1]
        r = list(region) if region is not None else [0, 0, 0, self.nx, self.ny, self.nz]
        shp = (r[5], r[4], r[3]) + ((3,) if vec else ())
        if out is None:
            out = np.zeros(shp, self.real)
        reg = (ctypes.c_int * 6)(*r)
        _check(self.lib.tclb_get_quantity(self._h, q, reg, ctypes.c_void_p(out.ctypes.data), float(scale),
                                          ctypes.c_void_p(stream or None)))
        return out

    quantity = GetQuantity

    def GetQuantityNoAlloc(self, name, region: Optional[Sequence[int]] = None, scale: float = 1.0, out=None,
                           stream: int = 0) -> np.ndarray:
        """GetQuantity through tclb_get_quantity_noalloc: no device allocation, the quantity staged in the
        library's fixed 8 MiB device array (larger regions raise TCLBError; overlapping calls race)."""
        q = name if isinstance(name, int) else self.model.quantity_index(name)
        vec = self.model.quantities[q][1]
        r = list(region) if region is not None else [0, 0, 0, self.nx, self.ny, self.nz]
        shp = (r[5], r[4], r[3]) + ((3,) if vec else ())
        if out is None:
            out = np.zeros(shp, self.real)
        reg = (ctypes.c_int * 6)(*r)
        _check(self.lib.tclb_get_quantity_noalloc(self._h, q, reg, ctypes.c_void_p(out.ctypes.data), float(scale),
                                                  ctypes.c_void_p(stream or None)))
        return out

    def densities(self) -> np.ndarray:
        out = np.zeros((self.model.Q,) + self.shape)
        _check(self.lib.tclb_get_densities(self._h, _dp(out)))
        return out

    def set_densities(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64)
        assert a.size == self.model.Q * self.N
        _check(self.lib.tclb_set_densities(self._h, _dp(a)))

    def snapshot_bytes(self) -> int:
        return int(self.lib.tclb_snapshot_bytes(self._h))

    def save(self, buf=None, stream: int = 0):
        n = self.snapshot_bytes()
        if buf is None:
            buf = np.empty(n, np.uint8)
        _check(self.lib.tclb_save(self._h, ctypes.c_void_p(buf.ctypes.data if hasattr(buf, "ctypes") else buf), n,
                                  ctypes.c_void_p(stream or None)))
        return buf

    def load(self, buf, stream: int = 0):
        n = self.snapshot_bytes()
        ptr = buf.ctypes.data if hasattr(buf, "ctypes") else buf
        _check(self.lib.tclb_load(self._h, ctypes.c_void_p(ptr), n, ctypes.c_void_p(stream or None)))

    def Color(self, z: int = -1, device_ptr: Optional[int] = None, stream: int = 0) -> Optional[np.ndarray]:
        """Lattice::Color, headless: RGBA bytes (ny, nx, 4) of plane z (default
        nz/2). With device_ptr the bytes go to that device buffer on `stream`
        and nothing is returned."""
        if device_ptr is not None:
            _check(self.lib.tclb_color(self._h, ctypes.c_void_p(device_ptr), int(z), 0,
                                       ctypes.c_void_p(stream or None)))
            return None
        out = np.zeros((self.ny, self.nx, 4), np.uint8)
        _check(self.lib.tclb_color(self._h, ctypes.c_void_p(out.ctypes.data), int(z), 1,
                                   ctypes.c_void_p(stream or None)))
        return out

    color = Color

    def save_pri(self) -> np.ndarray:
        """TCLB's .pri layout of the current snapshot (margin blocks concatenated)."""
        buf = np.empty(int(self.lib.tclb_pri_bytes(self._h)), np.uint8)
        _check(self.lib.tclb_save_pri(self._h, ctypes.c_void_p(buf.ctypes.data), buf.size))
        return buf

    def load_pri(self, buf: np.ndarray):
        b = np.ascontiguousarray(buf, np.uint8)
        _check(self.lib.tclb_load_pri(self._h, ctypes.c_void_p(b.ctypes.data), b.size))

    @property
    def iteration(self) -> int:
        v = ctypes.c_longlong()
        _check(self.lib.tclb_get_iteration(self._h, ctypes.byref(v)))
        return v.value

    @property
    def bytes_per_update(self) -> float:
        return float(self.lib.tclb_bytes_per_update(self._h))

    def sync(self):
        _check(self.lib.tclb_sync(self._h))

    def energy_enstrophy(self, stream: int = 0) -> tuple:
        """(kinetic energy 1/2 sum |U|^2, enstrophy 1/2 sum |curl U|^2), FP64, lattice units."""
        out = np.zeros(2)
        _check(self.lib.tclb_energy_enstrophy(self._h, _dp(out), ctypes.c_void_p(stream or None)))
        return float(out[0]), float(out[1])

    def launch_path(self) -> dict:
        """The paths plain iterations take: graphs, pairs, tma (enabled and applicable)."""
        bx, by, fl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.lib.tclb_get_launch(self._h, ctypes.byref(bx), ctypes.byref(by), ctypes.byref(fl)))
        return {"bx": bx.value, "by": by.value, "graphs": bool(fl.value & 1), "pairs": bool(fl.value & 2),
                "tma": bool(fl.value & 4)}

    def set_fault_injection(self, tile: int = -1, wait_cycles: int = 0):
        """Failure-path test of the tile-staged kernel: skip the copies of one tile and bound every staging
        wait by wait_cycles clock cycles; the next sync() raises TCLBError. tile=-1, wait_cycles=0: off."""
        _check(self.lib.tclb_set_fault_injection(self._h, int(tile), int(wait_cycles)))

    def set_launch(self, bx: int, by: int, use_graphs: bool = True, use_pairs: bool = True, use_tma: bool = True,
                   tma_always: bool = False):
        flags = (1 if use_graphs else 0) | (2 if use_pairs else 0) | (4 if use_tma else 0) | (8 if tma_always else 0)
        _check(self.lib.tclb_set_launch(self._h, int(bx), int(by), flags))
