"""Node-type rasteriser and the synthetic cases of the benchmark configurations.

``Geometry`` follows TCLB's XML geometry semantics (src/Geometry.cpp.Rt):
``set_flag`` picks the foreground node type and its group mask (setFlag,
:141-152), ``name=`` assigns a zone (setZone, :192-206), ``mask=`` overrides
the mask, and every drawn node becomes ``(geom & ~mask) | fg`` (Dot,
:307-319). Shapes: ``box`` with TCLB's dx/nx/fx region arithmetic
(getRegion, :216-304) and ``sphere`` (inSphere over the region, :782-792);
the default zones Inlet/Outlet/Channel/Tunnel of src/def.cpp.Rt:10-33.

All cases are seeded synthetic inputs standing in for the configurations the
reference is measured on; none is a public dataset.
"""
from __future__ import annotations

import math
from typing import Dict, Optional, Tuple

import numpy as np

from . import models as M


class Geometry:
    def __init__(self, model, nx: int, ny: int, nz: int = 1):
        self.model = M.get(model)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.geom = np.zeros((nz, ny, nx), np.uint16)
        self.zones: Dict[str, int] = {"DefaultZone": 0}
        self.fg = 0
        self.mask = 0
        self.mode = "overwrite"

    # --- foreground ----------------------------------------------------------
    def set_flag(self, name: str, zone: Optional[str] = None, mask: Optional[str] = None, mode: str = "overwrite"):
        if name == "None":
            self.fg, self.mask = 0, 0
        else:
            v, m, _grp = self.model.node_types[name]
            self.fg, self.mask = v, m
        if zone is not None:
            z = self.zones.setdefault(zone, len(self.zones))
            zs = self.model.zone_shift
            self.fg = (self.fg & ~(0xFFFF << zs & 0xFFFF)) | (z << zs)
            self.mask |= (0xFFFF << zs) & 0xFFFF
        if mask is not None:
            self.mask = 0xFFFF if mask == "ALL" else (0 if mask == "NONE" else self.model.groups[mask][0])
        self.mode = mode
        return self

    # --- regions (getRegion arithmetic) -------------------------------------
    def region(self, dx=None, dy=None, dz=None, nx=None, ny=None, nz=None, fx=None, fy=None, fz=None,
               parent=None) -> Tuple[int, int, int, int, int, int]:
        r = list(parent) if parent is not None else [0, 0, 0, self.nx, self.ny, self.nz]
        for ax, d in enumerate((dx, dy, dz)):
            if d is not None:
                r[ax] += d if d >= 0 else r[3 + ax] + d
                r[3 + ax] -= d if d >= 0 else r[3 + ax] + d
        for ax, f in enumerate((fx, fy, fz)):
            if f is not None:
                w = f if f >= 0 else r[3 + ax] + f + r[ax]
                r[3 + ax] = w - r[ax] + 1
        for ax, n in enumerate((nx, ny, nz)):
            if n is not None:
                r[3 + ax] = n
        return tuple(r)

    def _dot(self, sel: Tuple[slice, slice, slice], inside: Optional[np.ndarray] = None):
        g = self.geom[sel]
        m = np.ones(g.shape, bool) if inside is None else inside
        if self.mode == "fill":
            m &= (g & self.mask) == 0
        elif self.mode == "change":
            m &= (g & self.mask) != 0
        g[m] = (g[m] & (~self.mask & 0xFFFF)) | self.fg

    def box(self, **kw):
        dx, dy, dz, nx, ny, nz = self.region(**kw)
        x0, x1 = max(dx, 0), min(dx + nx, self.nx)
        y0, y1 = max(dy, 0), min(dy + ny, self.ny)
        z0, z1 = max(dz, 0), min(dz + nz, self.nz)
        if x1 > x0 and y1 > y0 and z1 > z0:
            self._dot((slice(z0, z1), slice(y0, y1), slice(x0, x1)))
        return self

    def sphere(self, **kw):
        dx, dy, dz, nx, ny, nz = self.region(**kw)
        x = np.arange(dx, dx + nx)
        y = np.arange(dy, dy + ny)
        z = np.arange(dz, dz + nz)
        X = 2 * ((0.5 + x - dx) / nx) - 1
        Y = 2 * ((0.5 + y - dy) / ny) - 1
        Z = 2 * ((0.5 + z - dz) / nz) - 1
        ins = (Z[:, None, None] ** 2 + Y[None, :, None] ** 2 + X[None, None, :] ** 2) < 1
        okx = (x >= 0) & (x < self.nx)
        oky = (y >= 0) & (y < self.ny)
        okz = (z >= 0) & (z < self.nz)
        ins = ins[np.ix_(okz, oky, okx)]
        xs, ys, zs = x[okx], y[oky], z[okz]
        if xs.size and ys.size and zs.size:
            self._dot((slice(zs[0], zs[-1] + 1), slice(ys[0], ys[-1] + 1), slice(xs[0], xs[-1] + 1)), ins)
        return self

    # default zones (src/def.cpp.Rt:10-33)
    def inlet(self):
        return self.box(dx=0, dy=0, dz=0, fx=0, fy=-1, fz=-1)

    def outlet(self):
        return self.box(dx=-1, dy=0, dz=0, fx=-1, fy=-1, fz=-1)

    def channel(self):
        self.box(dx=0, dy=0, dz=0, fx=-1, fy=0, fz=-1)
        return self.box(dx=0, dy=-1, dz=0, fx=-1, fy=-1, fz=-1)

    def tunnel(self):
        self.channel()
        self.box(dx=0, dy=0, dz=0, fx=-1, fy=-1, fz=0)
        return self.box(dx=0, dy=0, dz=-1, fx=-1, fy=-1, fz=-1)


def pad_nx(nx: int, xsdim: int = 32) -> int:
    """TCLB pads nx to a multiple of the x block (src/Solver.cpp.Rt:273)."""
    return nx + xsdim - 1 - ((nx - 1) % xsdim)


# ---------------------------------------------------------------------------
# Configuration 1: d2q9 channel with a disc (karman.xml-style geometry)
# ---------------------------------------------------------------------------
def channel_disc_d2q9(nx=1024, ny=256, r=16, cx=256, cy=128, objective_offset=5) -> np.ndarray:
    g = Geometry("d2q9", nx, ny)
    g.set_flag("MRT").box()
    g.set_flag("WVelocity", zone="Inlet").inlet()
    g.set_flag("EPressure", zone="Outlet").outlet()
    g.set_flag("Inlet").box(nx=1, dx=objective_offset)
    g.set_flag("Outlet").box(nx=1, dx=-objective_offset)
    g.set_flag("Wall", mask="ALL").channel()
    g.sphere(dx=cx - r, nx=2 * r, dy=cy - r, ny=2 * r)
    return g.geom


def channel_disc_settings(ux=0.01, nu=0.02, bgk=True):
    """<Param> list for configuration 1: VelocityX, Viscosity and, for BGK, S3=S4=1-omega."""
    omega = 1.0 / (3 * nu + 0.5)
    p = [("zone", "VelocityX", ux), ("setting", "Viscosity", nu)]
    if bgk:
        p += [("setting", "S3", 1 - omega), ("setting", "S4", 1 - omega)]
    return p


# ---------------------------------------------------------------------------
# Configuration 2: triply periodic Taylor-Green vortex (d3q27_cumulant)
# ---------------------------------------------------------------------------
def tgv_fields(n=256, u0=0.05, rho0=1.0, nz=None, dtype=np.float32):
    """rho (N) and u (N x 3) at node centres of [0, 2pi)^3, x fastest.

    u = u0 (sin x cos y cos z, -cos x sin y cos z, 0); the matching pressure
    p = rho0 u0^2/16 (cos 2x + cos 2y)(cos 2z + 2) enters as rho = rho0 + 3p.
    """
    nz = nz or n
    t = 2 * np.pi * (np.arange(n) + 0.5) / n
    tz = 2 * np.pi * (np.arange(nz) + 0.5) / nz
    sx, cx = np.sin(t), np.cos(t)
    sz, cz = np.sin(tz), np.cos(tz)
    u = np.empty((nz, n, n, 3), dtype)
    u[..., 0] = u0 * (cz[:, None, None] * cx[None, :, None] * sx[None, None, :])
    u[..., 1] = -u0 * (cz[:, None, None] * sx[None, :, None] * cx[None, None, :])
    u[..., 2] = 0
    p = rho0 * u0 * u0 / 16.0 * (np.cos(2 * t)[None, None, :] + np.cos(2 * t)[None, :, None]) * (
        np.cos(2 * tz)[:, None, None] + 2)
    rho = (rho0 + 3 * p).astype(dtype)
    return rho, u


def tgv_flags(model, n=256, nz=None) -> np.ndarray:
    m = M.get(model)
    return np.full((nz or n, n, n), m.flag("MRT"), np.uint16)


# ---------------------------------------------------------------------------
# Configuration 3: d3q19 body-force channel with random porous obstacles
# ---------------------------------------------------------------------------
def porous_channel_d3q19(nx=384, ny=192, nz=192, p=0.08, band=4, seed=0) -> np.ndarray:
    g = Geometry("d3q19", nx, ny, nz)
    g.set_flag("MRT").box()
    rng = np.random.default_rng(seed)
    solid = rng.random((nz, ny, nx)) < p
    solid[:, :band, :] = False
    solid[:, ny - band:, :] = False
    solid[:band, :, :] = False
    solid[nz - band:, :, :] = False
    wall = m_flag("d3q19", "Wall")
    g.geom[solid] = wall  # <Wall mask="ALL"> on the obstacle nodes
    g.set_flag("Wall", mask="ALL").channel()
    g.box(dx=0, dy=0, dz=0, fx=-1, fy=-1, fz=0)
    g.box(dx=0, dy=0, dz=-1, fx=-1, fy=-1, fz=-1)
    return g.geom


def m_flag(model, *names, zone=0) -> int:
    return M.get(model).flag(*names, zone=zone)


# ---------------------------------------------------------------------------
# Configuration 4: batched d2q9 obstacle channels
# ---------------------------------------------------------------------------
def batch_cases_d2q9(n_cases=512, seed=0, w_min=64, w_max=2048, ux=0.02, re_range=(20.0, 200.0)):
    """Seeded case list: W log-uniform in [w_min, w_max] (rounded to 32), H=W/4
    (>= 32), one disc of radius U[H/16, H/6] centred in the first third."""
    rng = np.random.default_rng(seed)
    out = []
    clamps = 0
    for _ in range(n_cases):
        W = int(round(math.exp(rng.uniform(math.log(w_min), math.log(w_max)))))
        W = max(32, pad_nx(W))
        H = max(32, W // 4)
        r = rng.uniform(H / 16, H / 6)
        cx = rng.uniform(r + 1, max(r + 2, W / 3))
        cy = rng.uniform(r + 1, H - r - 2)
        re = rng.uniform(*re_range)
        nu = ux * 2 * r / re
        omega = 1.0 / (3 * nu + 0.5)
        if omega > 1.99:
            clamps += 1
            nu = (1 / 1.99 - 0.5) / 3
        out.append(dict(W=W, H=H, r=r, cx=cx, cy=cy, nu=nu, ux=ux))
    return out, clamps


def sphere_channel_d3q27(nx=192, ny=64, nz=64, r=8, cx=48) -> Tuple[np.ndarray, Dict[str, int]]:
    """d3q27_cumulant flow past a sphere in a square duct: velocity inlet
    (zone Inlet) at x = 0, pressure outlet (zone Outlet) at x = nx-1, walls on
    the y and z faces, and a sphere of radius r at (cx, ny/2, nz/2) of Wall
    nodes flagged Body, on which the model accumulates Drag, Lift and Lateral.
    Returns the node types and the zone indices."""
    g = Geometry("d3q27_cumulant", nx, ny, nz)
    g.set_flag("MRT").box()
    g.set_flag("WVelocity", zone="Inlet").inlet()
    g.set_flag("EPressure", zone="Outlet").outlet()
    g.set_flag("Wall", mask="ALL").tunnel()
    cy, cz = ny // 2, nz // 2
    g.sphere(dx=cx - r, nx=2 * r, dy=cy - r, ny=2 * r, dz=cz - r, nz=2 * r)
    g.set_flag("Body").sphere(dx=cx - r, nx=2 * r, dy=cy - r, ny=2 * r, dz=cz - r, nz=2 * r)
    return g.geom, dict(g.zones)


def disc_channel_flags(W, H, r, cx, cy) -> np.ndarray:
    g = Geometry("d2q9", W, H)
    g.set_flag("MRT").box()
    g.set_flag("WVelocity", zone="Inlet").inlet()
    g.set_flag("EPressure", zone="Outlet").outlet()
    g.set_flag("Wall", mask="ALL").channel()
    ri = int(round(r))
    g.sphere(dx=int(round(cx)) - ri, nx=2 * ri, dy=int(round(cy)) - ri, ny=2 * ri)
    return g.geom
