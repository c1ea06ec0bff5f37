"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle restates TCLB's per-node pull-stream + collide iteration for the
d2q9, d3q19 and d3q27_cumulant models on the CPU (see tclb_oracle.cpp). Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
checker; the product library never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtclb_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "tclb_oracle.cpp")
    ):
        subprocess.check_call(["make", "-s", "-C", _HERE, "CXX=g++"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i, i, i, i, i]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [i]
        L.orc_set_storage.argtypes = [vp, i, ctypes.c_uint, d]
        L.orc_set_flags.argtypes = [vp, ctypes.POINTER(ctypes.c_uint16)]
        L.orc_set_setting.argtypes = [vp, i, d]
        L.orc_get_setting.argtypes = [vp, i, dp]
        L.orc_set_zone_setting.argtypes = [vp, i, i, d]
        L.orc_init.argtypes = [vp]
        L.orc_iterate.argtypes = [vp, i, i]
        L.orc_get_globals.argtypes = [vp, dp]
        L.orc_get_globals_scale.argtypes = [vp, dp]
        L.orc_get_quantity.argtypes = [vp, i, dp]
        L.orc_get_densities.argtypes = [vp, dp]
        L.orc_set_densities.argtypes = [vp, dp]
        L.orc_feq.argtypes = [i, d, dp, dp]
        L.orc_d2q9_basis.argtypes = [dp, ctypes.POINTER(ctypes.c_int)]
        L.orc_node_type_value.argtypes = [i, ctypes.c_char_p]
        L.orc_node_update.argtypes = [vp, dp, ctypes.c_uint16, dp]
        L.orc_color.argtypes = [vp, i, vp]
        L.orc_color_map.argtypes = [vp, vp, i, vp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int) -> int:
    return lib().orc_set_threads(n)


class OracleLattice:
    """CPU restatement of TCLB's Lattice for one model (FP64 or FP32)."""

    def __init__(self, model, nx: int, ny: int, nz: int = 1, precision: str = "fp64"):
        from tclb_b200 import models as M

        self.model = M.get(model)
        self.shape = (nz, ny, nx)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.N = nx * ny * nz
        self.precision = precision
        self._h = lib().orc_create(self.model.mid, nx, ny, nz, 1 if precision == "fp64" else 0)
        if not self._h:
            raise RuntimeError("oracle: create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    STORAGE_EMULATION = {"same": 0, "fp16s": 1, "fp16s_sr": 2, "bf16s": 3, "bf16s_sr": 4, "mant": 5, "fixed": 6, "exm": 7}

    def set_storage(self, storage: str, seed: int = 0, param: float = 0.0):
        """Emulate a shifted storage format on every store (FP32 oracle): f is kept as
        decode(encode(float(f - w_i))) + w_i. "_sr" rounds stochastically; "mant" keeps
        `param` mantissa bits; "fixed" stores (f - w_i) as a 16-bit count of w_i * param / 32768."""
        if lib().orc_set_storage(self._h, self.STORAGE_EMULATION[storage], seed, float(param)) != 0:
            raise ValueError(storage)

    def set_flags(self, flags: np.ndarray):
        fl = np.ascontiguousarray(flags, dtype=np.uint16).reshape(-1)
        assert fl.size == self.N
        lib().orc_set_flags(self._h, fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))

    def set_setting(self, name, v: float):
        i = name if isinstance(name, int) else self.model.setting_index(name)
        lib().orc_set_setting(self._h, i, float(v))

    def get_setting(self, name) -> float:
        i = name if isinstance(name, int) else self.model.setting_index(name)
        out = ctypes.c_double()
        lib().orc_get_setting(self._h, i, ctypes.byref(out))
        return out.value

    def set_zone_setting(self, name, v: float, zone: int = -1):
        i = name if isinstance(name, int) else self.model.zone_setting_index(name)
        lib().orc_set_zone_setting(self._h, i, zone, float(v))

    def init(self):
        lib().orc_init(self._h)

    def iterate(self, niter: int, iter_type: int = 0x001):
        lib().orc_iterate(self._h, niter, iter_type)

    def globals(self) -> np.ndarray:
        out = np.zeros(len(self.model.globals))
        lib().orc_get_globals(self._h, _dp(out))
        return out

    def globals_scale(self) -> np.ndarray:
        """Sum of |contribution| per Global: the scale for comparing sums."""
        out = np.zeros(len(self.model.globals))
        lib().orc_get_globals_scale(self._h, _dp(out))
        return out

    def quantity(self, name) -> np.ndarray:
        q = name if isinstance(name, int) else self.model.quantity_index(name)
        vec = self.model.quantities[q][1]
        out = np.zeros(self.N * (3 if vec else 1))
        lib().orc_get_quantity(self._h, q, _dp(out))
        return out.reshape(self.shape + ((3,) if vec else ()))

    def densities(self) -> np.ndarray:
        out = np.zeros(self.model.Q * self.N)
        lib().orc_get_densities(self._h, _dp(out))
        return out.reshape((self.model.Q,) + self.shape)

    def set_densities(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        assert a.size == self.model.Q * self.N
        lib().orc_set_densities(self._h, _dp(a))

    def color(self, z: int = -1) -> np.ndarray:
        """Headless ColorKernel of plane z (default nz/2): (ny, nx, 4) RGBA."""
        out = np.zeros((self.ny, self.nx, 4), np.uint8)
        lib().orc_color(self._h, self.nz // 2 if z < 0 else z, out.ctypes.data)
        return out

    def node_update(self, fin, flag: int) -> np.ndarray:
        a = np.ascontiguousarray(fin, dtype=np.float64)
        out = np.zeros(self.model.Q)
        lib().orc_node_update(self._h, _dp(a), flag, _dp(out))
        return out


def color_map(l, w) -> np.ndarray:
    """ColorKernel's colour map of float l = |U| and weight w: (n, 4) RGBA."""
    la = np.asarray(l, np.float32)
    lv = np.ascontiguousarray(la).ravel()
    wv = np.ascontiguousarray(np.broadcast_to(np.asarray(w, np.float32), la.shape)).ravel()
    out = np.zeros((lv.size, 4), np.uint8)
    lib().orc_color_map(lv.ctypes.data, wv.ctypes.data, lv.size, out.ctypes.data)
    return out


def feq(model, rho: float, J) -> np.ndarray:
    from tclb_b200 import models as M

    m = M.get(model)
    j = np.zeros(3)
    j[: len(J)] = J
    out = np.zeros(27)
    q = lib().orc_feq(m.mid, float(rho), _dp(j), _dp(out))
    return out[:q]


def d2q9_basis():
    B = np.zeros(81)
    order = (ctypes.c_int * 9)()
    lib().orc_d2q9_basis(_dp(B), order)
    return B.reshape(9, 9), list(order)


def node_type_value(model, name: str) -> int:
    from tclb_b200 import models as M

    return lib().orc_node_type_value(M.get(model).mid, name.encode())
