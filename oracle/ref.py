"""ctypes wrapper of oracle/_ref/libtclb_ref.so: TCLB's own per-node model code on the CPU.

TEST INFRASTRUCTURE ONLY. `oracle/make_ref.py` builds the library from TCLB's
sources (the literal-C regions of models/flow/d3q27_cumulant/Dynamics.c.Rt,
models/flow/d3q19/Dynamics.c.Rt and models/flow/d2q9_SRT/Dynamics.c). It is a
checker for the restated oracle and for the golden fixtures under
tests/golden/; the product library never loads it.

Every function takes populations as float64 arrays of shape (n, Q) in TCLB's
density order and a `precision` of "fp64" (real_t = double) or "fp32"
(real_t = float, TCLB's single-precision build).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import make_ref

_lib = None

D3Q19_KINDS = {"WVelocity": 0, "WPressure": 1, "WPressureL": 2, "EPressure": 3}
D2Q9_OPS = {"BGK": 0, "BounceBack": 1, "EVelocity": 2, "WPressure": 3, "WVelocity": 4, "EPressure": 5,
            "feq": 6, "rho_u": 7}
D3Q27C_SETTINGS = ("nu", "nubuffer", "GalileanCorrection", "ForceX", "ForceY", "ForceZ", "Omega")
D3Q27C_GLOBALS = ("Density", "Flux", "Mass", "XMomentum", "YMomentum", "ZMomentum")


def available() -> bool:
    """True when the library exists or can be built from a TCLB tree on this machine."""
    return os.path.exists(make_ref.LIB) or os.path.isdir(make_ref.DEFAULT_REF)


def lib():
    global _lib
    if _lib is None:
        if os.path.isdir(make_ref.DEFAULT_REF):
            make_ref.build()
        if not os.path.exists(make_ref.LIB):
            raise FileNotFoundError("oracle/_ref/libtclb_ref.so is not built and no TCLB tree is present")
        L = ctypes.CDLL(make_ref.LIB)
        i, vp = ctypes.c_int, ctypes.c_void_p
        L.ref_d3q27c_collide.argtypes = [i, i, vp, vp, vp, vp]
        L.ref_d3q27c_rho_u.argtypes = [i, i, vp, vp, vp]
        L.ref_d3q19_boundary.argtypes = [i, i, i, vp, vp]
        L.ref_d2q9srt.argtypes = [i, i, i, vp, vp]
        L.ref_threads.argtypes = [i]
        L.ref_d3q27c_iterate.argtypes = [i, i, i, i, vp, vp, vp]
        _lib = L
    return _lib


def _fp64(precision: str) -> int:
    if precision not in ("fp64", "fp32"):
        raise ValueError(precision)
    return 1 if precision == "fp64" else 0


def _rows(f, q):
    a = np.array(f, dtype=np.float64, order="C", copy=True)
    if a.ndim != 2 or a.shape[1] != q:
        raise ValueError(f"populations must have shape (n, {q})")
    return a


def d3q27c_collide(f, settings: dict, boundary, precision="fp64"):
    """CollisionMRT of d3q27_cumulant (Dynamics.c.Rt:309-519) on each row of f.

    boundary[k] true marks a BOUNDARY-flagged node (relaxes with nubuffer).
    Returns (f_after, globals) with globals (n, 6) in D3Q27C_GLOBALS order.
    """
    a = _rows(f, 27)
    s = np.array([float(settings.get(k, d)) for k, d in zip(D3Q27C_SETTINGS, (1 / 6, 0.01, 1.0, 0, 0, 0, 1.0))])
    b = np.ascontiguousarray(np.asarray(boundary, dtype=np.int32).reshape(-1))
    if b.size != a.shape[0]:
        raise ValueError("boundary must have one entry per row")
    g = np.zeros((a.shape[0], 6))
    lib().ref_d3q27c_collide(_fp64(precision), a.shape[0], a.ctypes.data, s.ctypes.data, b.ctypes.data, g.ctypes.data)
    return a, g


def d3q27c_rho_u(f, settings: dict, precision="fp64"):
    """getRho and getU_ of d3q27_cumulant (Dynamics.c.Rt:23-45) for non-wall nodes: (n, 4) rho, ux, uy, uz."""
    a = _rows(f, 27)
    s = np.array([float(settings.get(k, 0.0)) for k in D3Q27C_SETTINGS])
    out = np.zeros((a.shape[0], 4))
    lib().ref_d3q27c_rho_u(_fp64(precision), a.shape[0], a.ctypes.data, s.ctypes.data, out.ctypes.data)
    return out


def d3q19_boundary(kind: str, f, inlet_velocity: float, inlet_density: float, precision="fp64"):
    """One of d3q19's Zou-He closures (Dynamics.c.Rt:110-179) on each row of f."""
    a = _rows(f, 19)
    s = np.array([inlet_velocity, inlet_density], np.float64)
    lib().ref_d3q19_boundary(_fp64(precision), D3Q19_KINDS[kind], a.shape[0], a.ctypes.data, s.ctypes.data)
    return a


def d2q9srt(op: str, f, omega=1.0, velocity_x=0.0, velocity_y=0.0, density=1.0, grav_x=0.0, grav_y=0.0,
            precision="fp64"):
    """An operation of d2q9_SRT (Dynamics.c:34-176) on each row of f.

    op "feq" reads (rho, ux, uy) from columns 0-2 and returns the equilibrium;
    op "rho_u" returns (rho, ux, uy) in columns 0-2.
    """
    a = _rows(f, 9)
    s = np.array([omega, velocity_x, velocity_y, density, grav_x, grav_y], np.float64)
    lib().ref_d2q9srt(_fp64(precision), D2Q9_OPS[op], a.shape[0], a.ctypes.data, s.ctypes.data)
    return a


def threads(n: int = 0) -> int:
    """Set (n > 0) and return the OpenMP threads of the lattice loop."""
    return lib().ref_threads(int(n))


def d3q27c_iterate(src, dst, settings: dict):
    """One iteration of a periodic all-MRT d3q27_cumulant lattice (Q, nz, ny, nx), float64 or float32:
    pull-stream in this harness's loop, then TCLB's CollisionMRT at every node. Writes dst."""
    if src.dtype != dst.dtype or src.shape != dst.shape or src.shape[0] != 27 or src.dtype not in (np.float64,
                                                                                                     np.float32):
        raise ValueError("src and dst: (27, nz, ny, nx) arrays of one float type")
    if not (src.flags.c_contiguous and dst.flags.c_contiguous):
        raise ValueError("contiguous arrays needed")
    s = np.array([float(settings.get(k, d)) for k, d in zip(D3Q27C_SETTINGS, (1 / 6, 0.01, 1.0, 0, 0, 0, 1.0))])
    _, nz, ny, nx = src.shape
    lib().ref_d3q27c_iterate(1 if src.dtype == np.float64 else 0, nx, ny, nz, src.ctypes.data, dst.ctypes.data,
                             s.ctypes.data)
