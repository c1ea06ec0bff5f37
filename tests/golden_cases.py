"""The fixture cases pinned to TCLB's own model code (tests/golden/ref_pin.npz).

Each case is one iteration of a small periodic lattice: pull-stream (node x
takes f_i from x - e_i), then the node's boundary closure and collision, in
the order TCLB's Run() applies them. Expected values come from
oracle/_ref/libtclb_ref.so, TCLB's literal per-node code compiled on the CPU
by oracle/make_ref.py:

* d3q27c (16x4x4): CollisionMRT of d3q27_cumulant
  (models/flow/d3q27_cumulant/Dynamics.c.Rt:309-519) at MRT nodes and at
  MRT|Buffer nodes (a BOUNDARY type with no closure, which relaxes with
  nubuffer, :321-322), in TCLB's double and float builds, with the Globals
  Density, Flux, Mass and X/Y/ZMomentum summed over the nodes.
* d3q19 (16x4x4): the Zou-He closures WVelocity, WPressure,
  WPressureLimited and EPressure (models/flow/d3q19/Dynamics.c.Rt:110-179) on
  nodes without the MRT bit; untyped nodes only stream.
* d2q9 (32x8): the closures, bounce-back and BGK collision of
  models/flow/d2q9_SRT/Dynamics.c:34-176 at d2q9's node types, with d2q9's MRT
  rates all 1 - omega (BGK) and no gravity; a node with a closure and the MRT
  bit runs the closure, then the collision (d2q9/Dynamics.c.Rt:108-142).
* d2q9_init: SetEquilibrium (d2q9_SRT/Dynamics.c:145-155) at
  rho = 1 + 3 Pressure, u = (VelocityX, VelocityY), the values d2q9's Init
  computes (d2q9/Dynamics.c.Rt:91-106).

`generate()` recomputes the fixture (it needs oracle/_ref); `setup()` prepares
a GPU or oracle lattice for a case, so the CPU and GPU tests check the same
thing.
"""
from __future__ import annotations

import os

import numpy as np

from tclb_b200 import models as M

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_pin.npz")

D3Q27C_SET = dict(nu=0.02, nubuffer=0.1, GalileanCorrection=1.0, ForceX=1e-5, ForceY=-2e-5, ForceZ=3e-5, Omega=0.8)
D3Q19_SET = dict(InletVelocity=0.03, InletDensity=1.006)
D2Q9_NU, D2Q9_VX, D2Q9_P = 0.05, 0.02, 0.01
D2Q9_INIT = (0.03, -0.01, 0.02)  # VelocityX, VelocityY, Pressure

# case -> (model, (nz, ny, nx))
CASES = {"d3q27c": ("d3q27_cumulant", (4, 4, 16)), "d3q19": ("d3q19", (4, 4, 16)), "d2q9": ("d2q9", (1, 8, 32))}
D3Q27C_GLOBAL_NAMES = ("Density", "Flux", "Mass", "XMomentum", "YMomentum", "ZMomentum")


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def load():
    return np.load(FIXTURE)


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
def feq_poly(model, rho, u):
    """Second-order polynomial equilibrium w_i rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2): only to draw inputs."""
    m = M.get(model)
    e = np.array(m.velocities, np.float64)[:, : m.dim]
    w = np.array(m.weights, np.float64)
    eu = u @ e.T
    uu = np.sum(u * u, axis=-1, keepdims=True)
    return w * rho[..., None] * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * uu)


def near_equilibrium(model, shape, seed, umax, noise=1e-2):
    """Seeded populations (Q, *shape): equilibrium of random rho, u, times (1 + noise * N(0,1))."""
    m = M.get(model)
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    rho = 1 + 0.05 * rng.uniform(-1, 1, n)
    u = rng.uniform(-umax, umax, (n, m.dim))
    f = feq_poly(model, rho, u) * (1 + noise * rng.standard_normal((n, m.Q)))
    return np.ascontiguousarray(f.T.reshape((m.Q,) + tuple(shape)))


def pulled(model, f):
    """Node x takes f_i from x - e_i on the periodic lattice; returns rows (n, Q)."""
    m = M.get(model)
    out = np.empty_like(f)
    for i, (ex, ey, ez) in enumerate(m.velocities):
        out[i] = np.roll(f[i], shift=(ez, ey, ex), axis=(0, 1, 2))
    return out.reshape(m.Q, -1).T.copy()


def to_lattice(model, rows, shape):
    return np.ascontiguousarray(rows.T.reshape((M.get(model).Q,) + tuple(shape)))


def d2q9_omega() -> float:
    return 1.0 / (3 * D2Q9_NU + 0.5)


def d2q9_srt_args() -> dict:
    """d2q9_SRT's settings matching d2q9_params()."""
    return dict(omega=d2q9_omega(), velocity_x=D2Q9_VX, density=1 + 3 * D2Q9_P)


def _set(lat, name, v):
    (lat.SetSetting if hasattr(lat, "SetSetting") else lat.set_setting)(name, v)


def d2q9_params(lat):
    """d2q9 as BGK: Viscosity (-> RelaxationRate, S2), S3 = S4 = 1 - omega; zone VelocityX and Pressure."""
    _set(lat, "Viscosity", D2Q9_NU)
    _set(lat, "S3", 1 - d2q9_omega())
    _set(lat, "S4", 1 - d2q9_omega())
    lat.set_zone_setting("VelocityX", D2Q9_VX)
    lat.set_zone_setting("Pressure", D2Q9_P)


def d2q9_init_params(lat):
    vx, vy, p = D2Q9_INIT
    lat.set_zone_setting("VelocityX", vx)
    lat.set_zone_setting("VelocityY", vy)
    lat.set_zone_setting("Pressure", p)


def setup(lat, case, fx):
    """Flags, settings and the input populations of a fixture case on a GPU or oracle lattice."""
    flags = fx[f"{case}_flags"]
    if hasattr(lat, "FlagOverwrite"):
        lat.FlagOverwrite(flags)
    else:
        lat.set_flags(flags)
    if case == "d3q27c":
        for k, v in D3Q27C_SET.items():
            _set(lat, k, v)
    elif case == "d3q19":
        for k, v in D3Q19_SET.items():
            _set(lat, k, v)
    else:
        d2q9_params(lat)
    lat.set_densities(fx[f"{case}_in"])


def d3q27c_globals(g) -> np.ndarray:
    """The six fixture Globals out of a d3q27_cumulant Globals vector."""
    m = M.get("d3q27_cumulant")
    return np.array([g[m.global_index(n)] for n in D3Q27C_GLOBAL_NAMES])


# ---------------------------------------------------------------------------
# expected values from oracle/_ref
# ---------------------------------------------------------------------------
def _case_d3q27c(out, ref):
    model, shape = CASES["d3q27c"]
    m = M.get(model)
    rng = np.random.default_rng(11)
    f = near_equilibrium(model, shape, 1, 0.1)
    buffer = rng.random(shape) < 0.3
    mrt, buf = m.node_types["MRT"][0], m.node_types["Buffer"][0]
    out["d3q27c_in"] = f
    out["d3q27c_flags"] = np.where(buffer, mrt | buf, mrt).astype(np.uint16)
    for prec, dt in (("fp64", np.float64), ("fp32", np.float32)):
        rows = pulled(model, f.astype(dt).astype(np.float64))
        res, g = ref.d3q27c_collide(rows, D3Q27C_SET, buffer.reshape(-1), prec)
        out[f"d3q27c_out_{prec}"] = to_lattice(model, res, shape)
        out[f"d3q27c_glob_{prec}"] = g.sum(axis=0)
        out[f"d3q27c_globabs_{prec}"] = np.abs(g).sum(axis=0)


def _case_d3q19(out, ref):
    model, shape = CASES["d3q19"]
    m = M.get(model)
    rng = np.random.default_rng(12)
    f = near_equilibrium(model, shape, 2, 0.06)
    kinds = ["WVelocity", "WPressure", "WPressureL", "EPressure", None]
    pick = rng.integers(0, len(kinds), shape)
    flags = np.zeros(shape, np.uint16)
    for k, name in enumerate(kinds):
        if name:
            flags[pick == k] = m.node_types[name][0]
    out["d3q19_in"] = f
    out["d3q19_flags"] = flags
    for prec, dt in (("fp64", np.float64), ("fp32", np.float32)):
        rows = pulled(model, f.astype(dt).astype(np.float64))
        res = rows.copy()
        pk = pick.reshape(-1)
        for k, name in enumerate(kinds):
            sel = pk == k
            if name and sel.any():
                res[sel] = ref.d3q19_boundary(name, rows[sel], D3Q19_SET["InletVelocity"], D3Q19_SET["InletDensity"],
                                              prec)
        out[f"d3q19_out_{prec}"] = to_lattice(model, res, shape)


def _case_d2q9(out, ref):
    model, shape = CASES["d2q9"]
    m = M.get(model)
    rng = np.random.default_rng(13)
    f = near_equilibrium(model, shape, 3, 0.06)
    kinds = ["WVelocity", "EVelocity", "WPressure", "EPressure", "Wall", None]
    pick = rng.integers(0, len(kinds), shape)
    mrt = (rng.random(shape) < 0.6) & (pick != kinds.index("Wall"))
    flags = np.zeros(shape, np.uint16)
    for k, name in enumerate(kinds):
        if name:
            flags[pick == k] = m.node_types[name][0]
    flags[mrt] |= m.node_types["MRT"][0]
    out["d2q9_in"] = f
    out["d2q9_flags"] = flags
    for prec, dt in (("fp64", np.float64), ("fp32", np.float32)):
        rows = pulled(model, f.astype(dt).astype(np.float64))
        res = rows.copy()
        pk, mk = pick.reshape(-1), mrt.reshape(-1)
        for k, name in enumerate(kinds):
            sel = pk == k
            if name and sel.any():
                op = "BounceBack" if name == "Wall" else name
                res[sel] = ref.d2q9srt(op, res[sel], precision=prec, **d2q9_srt_args())
        res[mk] = ref.d2q9srt("BGK", res[mk], precision=prec, **d2q9_srt_args())
        out[f"d2q9_out_{prec}"] = to_lattice(model, res, shape)
    vx, vy, p = D2Q9_INIT
    for prec in ("fp64", "fp32"):
        arg = np.zeros((1, 9))
        arg[0, :3] = (1 + 3 * p, vx, vy)
        out[f"d2q9_init_{prec}"] = ref.d2q9srt("feq", arg, precision=prec)[0]


def generate() -> dict:
    """The fixture's arrays, computed by oracle/_ref."""
    from oracle import ref

    out = {}
    _case_d3q27c(out, ref)
    _case_d3q19(out, ref)
    _case_d2q9(out, ref)
    return out
