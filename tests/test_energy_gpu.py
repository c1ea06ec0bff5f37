"""Kinetic energy and enstrophy diagnostics (tclb_energy_enstrophy) against
closed forms for the Taylor-Green field and against numpy on the exported U
field of the library and of the FP64 oracle."""
import numpy as np
import pytest

import oracle
from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice


def numpy_energy_enstrophy(u):
    """u: (nz, ny, nx, 3) -> (1/2 sum |u|^2, 1/2 sum |curl u|^2), periodic central differences."""
    u = np.asarray(u, np.float64)

    def d(c, axis):  # axis 0 z, 1 y, 2 x
        if u.shape[axis] == 1:
            return np.zeros(u.shape[:3])
        return 0.5 * (np.roll(u[..., c], -1, axis=axis) - np.roll(u[..., c], 1, axis=axis))

    wx = d(2, 1) - d(1, 0)
    wy = d(0, 0) - d(2, 2)
    wz = d(1, 2) - d(0, 1)
    return 0.5 * float((u * u).sum()), 0.5 * float((wx * wx + wy * wy + wz * wz).sum())


@pytest.mark.parametrize("n", [16, 32])
def test_reduction_closed_forms_on_the_taylor_green_field(n):
    """The reduction itself, on the analytic field (no GPU): the sum of sin^2
    over a full period of n >= 3 points is n/2, so E = N u0^2 / 8; the central
    difference of sin(kx) is sin(k) cos(kx), so Omega = 3 u0^2 sin(k)^2 N / 8."""
    u0 = 0.05
    _, u = cases.tgv_fields(n, u0=u0, dtype=np.float64)
    e, w = numpy_energy_enstrophy(u)
    N = n ** 3
    assert e == pytest.approx(N * u0 ** 2 / 8, rel=1e-12)
    assert w == pytest.approx(3 * u0 ** 2 * np.sin(2 * np.pi / n) ** 2 * N / 8, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_taylor_green_lattice_matches_numpy(precision):
    """On the lattice the velocity is that of the pulled populations (TCLB's
    quantity semantics), so the check is against numpy on the exported U."""
    n = 32
    lat = Lattice("d3q27_cumulant", n, n, n, precision=precision)
    lat.set_flags(cases.tgv_flags("d3q27_cumulant", n))
    lat.SetSetting("nu", 1e-3)
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=lat.real)
    lat.init_equilibrium(rho, u)
    for _ in range(2):
        e, w = lat.energy_enstrophy()
        e_np, w_np = numpy_energy_enstrophy(lat.GetQuantity("U"))
        tol = 1e-12 if precision == "fp64" else 1e-6
        assert e == pytest.approx(e_np, rel=tol) and w == pytest.approx(w_np, rel=tol)
        lat.Iterate(10)
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model,shape", [("d3q27_cumulant", (12, 16, 32)), ("d3q19", (10, 12, 32)),
                                         ("d2q9", (1, 24, 64))])
def test_matches_numpy_and_oracle(model, shape):
    m = M.get(model)
    nz, ny, nx = shape
    rng = np.random.default_rng(3)
    w = np.array(m.weights)[:, None, None, None]
    f0 = w * (1.0 + 0.05 * rng.standard_normal((m.Q,) + shape))
    fl = np.full(shape, m.flag("MRT"), np.uint16)
    g = Lattice(model, nx, ny, nz, precision="fp64")
    o = oracle.OracleLattice(model, nx, ny, nz, precision="fp64")
    for lat in (g, o):
        lat.set_flags(fl)
        lat.set_densities(f0)
    g.SetSetting("nu" if model != "d2q9" else "Viscosity", 0.05)
    o.set_setting("nu" if model != "d2q9" else "Viscosity", 0.05)
    g.Iterate(3)
    o.iterate(3)
    e, w2 = g.energy_enstrophy()
    e_np, w_np = numpy_energy_enstrophy(g.GetQuantity("U"))
    assert e == pytest.approx(e_np, rel=1e-12) and w2 == pytest.approx(w_np, rel=1e-12)
    e_o, w_o = numpy_energy_enstrophy(o.quantity("U").reshape(shape + (3,)))
    assert e == pytest.approx(e_o, rel=1e-9) and w2 == pytest.approx(w_o, rel=1e-9)
    g.close()
