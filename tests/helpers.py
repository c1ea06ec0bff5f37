"""Shared helpers of the parity tests: build the same case on the CUDA
library and on the CPU oracle, run both, compare."""
from __future__ import annotations

import numpy as np

import oracle
from tclb_b200 import models as M


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)


def apply_params(lat, params):
    """params: list of (kind, name, value[, zone]) with kind 'setting' or 'zone'."""
    for p in params:
        kind, name, v = p[0], p[1], p[2]
        zone = p[3] if len(p) > 3 else -1
        if kind == "setting":
            if hasattr(lat, "SetSetting"):
                lat.SetSetting(name, v)
            else:
                lat.set_setting(name, v)
        else:
            lat.set_zone_setting(name, v, zone)


def random_flags(model, shape, types, zones=1, seed=0, p_type=0.3, mrt=True, extra_groups=()):
    """Random node types drawn from `types` (BOUNDARY-group names) on a
    fraction p_type of nodes, MRT elsewhere (and on boundary nodes too when
    mrt=True), random zone index < zones, and random values of the extra
    groups (e.g. ADDITIONALS, BODY, OBJECTIVE)."""
    m = M.get(model)
    rng = np.random.default_rng(seed)
    fl = np.zeros(shape, np.uint16)
    if mrt:
        fl |= m.node_types["MRT"][0]
    pick = rng.random(shape) < p_type
    idx = rng.integers(0, len(types), shape)
    vals = np.array([m.node_types[t][0] for t in types], np.uint16)
    fl[pick] |= vals[idx[pick]]
    for grp in extra_groups:
        names = [n for n, v in m.node_types.items() if v[2] == grp]
        sel = rng.random(shape) < 0.2
        gi = rng.integers(0, len(names), shape)
        gv = np.array([m.node_types[n][0] for n in names], np.uint16)
        fl[sel] |= gv[gi[sel]]
    if zones > 1:
        z = rng.integers(0, zones, shape).astype(np.uint16)
        fl |= (z << m.zone_shift).astype(np.uint16)
    return fl


def perturbed_equilibrium(model, shape, seed=0, amp=1e-3, u=0.02):
    m = M.get(model)
    rng = np.random.default_rng(seed)
    N = int(np.prod(shape))
    base = oracle.feq(model, 1.0, [u, -u / 2, u / 3][: (2 if m.dim == 2 else 3)])
    f = np.repeat(base[:, None], N, axis=1)
    f *= 1 + amp * rng.standard_normal(f.shape)
    return f.reshape((m.Q,) + tuple(shape))
