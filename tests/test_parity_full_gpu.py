"""Parity at the benchmark configurations' sizes and full iteration counts.

* Configuration 1, full size: d2q9 BGK channel 1024x256, solid disc r = 16 at
  (256, 128), Zou-He velocity inlet (Ux = 0.01) and pressure outlet, walls at
  y = 0 and 255, nu = 0.02; 10,000 iterations with Globals every 100.
* Configuration 2 at 64^3 (the workload is 256^3): d3q27_cumulant
  Taylor-Green vortex, u0 = 0.05, nu = 1e-3; 2,000 iterations, Globals every 50.
* Configuration 3 at 96x48x48 (the workload is 384x192x192): d3q19 porous
  channel, Bernoulli(0.08) solids outside a 4-node wall band, ForceX = 1e-6,
  nu = 0.01; 5,000 iterations, Globals every 500.

Bars, written here and used below:
* FP64 (against the FP64 oracle; TCLB's double-build bar): densities relative
  L2 <= 1e-12. The velocity is a momentum, a small difference of populations,
  divided by rho; it is held to the same bar on the state, 1e-12 x
  ||f|| / ||J|| (about 5e-11 for the channel, whose ||J|| is 2% of ||f||).
  Globals at every log point within 1e-10 of the sum of |per-node
  contributions|. d2q9's PressureLoss adds s (Jx/rho^2)((rho - 1)/3 + ...),
  whose (rho - 1) is itself a cancellation; its scale is the sum of
  |Jx/rho^2|/3, the size of the terms before it (the flux Globals' scales / 3).
* FP32 (against the FP32 oracle; TCLB's float-build bar): velocity and
  densities relative L2 <= 1e-5, unless FP32 rounding itself moves the result
  further than that over the run. Then the GPU may differ from the FP32 oracle
  by at most twice what FP32 costs the oracle against FP64 at the same
  iteration count: e(gpu32, orc32) <= max(1e-5, 2 e(orc32, orc64)). The GPU
  FP32 result must also be as accurate as the oracle's:
  e(gpu32, orc64) <= max(1e-5, 2 e(orc32, orc64)). Globals use the same rule
  per Global, with errors relative to the sum of |per-node contributions| and
  taken as the largest over the log points.
The measured spreads are printed (pytest -s shows them).
"""
import numpy as np
import pytest

import oracle
from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice

from helpers import apply_params, rel_l2

pytestmark = pytest.mark.gpu

FP32_BAR = 1e-5


def _tgv_densities(n):
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=np.float64)
    m = M.get("d3q27_cumulant")
    w = np.array(m.weights)
    e = np.array(m.velocities, np.float64)
    J = rho[..., None] * u
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    j2 = (J ** 2).sum(-1)
    return w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * j2 / rho)


def _config(name):
    """(model, (nz, ny, nx), setup(lattice), iterations, log interval)."""
    if name == "config1":
        fl = cases.channel_disc_d2q9(1024, 256, r=16, cx=256, cy=128)

        def setup(lat):
            lat.set_flags(fl)
            apply_params(lat, cases.channel_disc_settings(ux=0.01, nu=0.02, bgk=True))
            lat.Init() if hasattr(lat, "Init") else lat.init()

        return "d2q9", (1, 256, 1024), setup, 10000, 100
    if name == "config2":
        n = 64
        f0 = _tgv_densities(n)

        def setup(lat):
            lat.set_flags(cases.tgv_flags("d3q27_cumulant", n))
            lat.set_setting("nu", 1e-3)
            lat.set_densities(f0)

        return "d3q27_cumulant", (n, n, n), setup, 2000, 50
    fl = cases.porous_channel_d3q19(96, 48, 48, p=0.08, band=4, seed=3)

    def setup(lat):
        lat.set_flags(fl)
        apply_params(lat, [("setting", "nu", 0.01), ("setting", "ForceX", 1e-6)])
        lat.Init() if hasattr(lat, "Init") else lat.init()

    return "d3q19", (48, 48, 96), setup, 5000, 500


_ORACLE = {}


def _oracle_run(name, precision):
    """Oracle result (densities, U, Globals per log point, Globals scale per log point), cached per module."""
    key = (name, precision)
    if key not in _ORACLE:
        model, (nz, ny, nx), setup, niter, every = _config(name)
        o = oracle.OracleLattice(model, nx, ny, nz, precision=precision)
        setup(o)
        gl, sc = [], []
        for _ in range(niter // every):
            o.iterate(every, M.ITER_NORM | M.ITER_LASTGLOB)
            gl.append(o.globals())
            sc.append(o.globals_scale())
        _ORACLE[key] = (o.densities(), o.quantity("U"), np.array(gl), np.array(sc))
    return _ORACLE[key]


def _gpu_run(name, precision):
    model, (nz, ny, nx), setup, niter, every = _config(name)
    with Lattice(model, nx, ny, nz, precision=precision) as g:
        setup(g)
        gl = []
        for _ in range(niter // every):
            g.Iterate(every, M.ITER_NORM | M.ITER_LASTGLOB)
            gl.append(g.globals)
        return g.densities(), g.GetQuantity("U"), np.array(gl)


def _globals_scale(name, scale):
    """Per-node contribution scale; for d2q9 PressureLoss the terms before the (rho - 1) cancellation."""
    scale = np.array(scale, np.float64)
    if name == "config1":
        m = M.get("d2q9")
        pl, fo, fi = (m.global_index(g) for g in ("PressureLoss", "OutletFlux", "InletFlux"))
        scale[..., pl] = np.maximum(scale[..., pl], (scale[..., fo] + scale[..., fi]) / 3)
    return scale


def _globals_err(a, b, scale):
    return np.where(scale > 0, np.abs(a - b) / np.where(scale > 0, scale, 1), np.abs(a - b))


def _momentum_ratio(name, f):
    """||f|| / ||J|| of a state: the factor from the densities' bar to the velocity's."""
    m = M.get(_config(name)[0])
    e = np.array(m.velocities, np.float64)
    J = np.einsum("qd,q...->d...", e, f.reshape((m.Q, -1)))
    return float(np.linalg.norm(f) / np.linalg.norm(J))


@pytest.mark.parametrize("name", ["config1", "config2", "config3"])
def test_full_count_fp64(name):
    f_o, u_o, g_o, s_o = _oracle_run(name, "fp64")
    f_g, u_g, g_g = _gpu_run(name, "fp64")
    ef, eu = rel_l2(f_g, f_o), rel_l2(u_g, u_o)
    bar_u = 1e-12 * _momentum_ratio(name, f_o)
    ge = _globals_err(g_g, g_o, _globals_scale(name, s_o)).max(axis=0)
    print(f"{name} fp64: densities {ef:.2e} velocity {eu:.2e} (bar {bar_u:.1e}) globals {np.array2string(ge, precision=1)}")
    assert ef < 1e-12 and eu < bar_u, (ef, eu)
    assert np.all(ge < 1e-10), ge


@pytest.mark.parametrize("name", ["config1", "config2", "config3"])
def test_full_count_fp32(name):
    f64, u64, g64, s64 = _oracle_run(name, "fp64")
    f32, u32, g32, _ = _oracle_run(name, "fp32")
    f_g, u_g, g_g = _gpu_run(name, "fp32")
    spread_f, spread_u = rel_l2(f32, f64), rel_l2(u32, u64)
    ef, eu = rel_l2(f_g, f32), rel_l2(u_g, u32)
    af, au = rel_l2(f_g, f64), rel_l2(u_g, u64)
    print(f"{name} fp32: gpu-vs-orc32 densities {ef:.2e} velocity {eu:.2e}; orc32-vs-orc64 densities {spread_f:.2e} "
          f"velocity {spread_u:.2e}; gpu32-vs-orc64 densities {af:.2e} velocity {au:.2e}")
    assert ef <= max(FP32_BAR, 2 * spread_f), (ef, spread_f)
    assert eu <= max(FP32_BAR, 2 * spread_u), (eu, spread_u)
    assert af <= max(FP32_BAR, 2 * spread_f), (af, spread_f)
    assert au <= max(FP32_BAR, 2 * spread_u), (au, spread_u)
    sc = _globals_scale(name, s64)
    eg = _globals_err(g_g, g32, sc)
    sg = _globals_err(g32, g64, sc)
    print(f"{name} fp32 globals: gpu-vs-orc32 {np.array2string(eg.max(axis=0), precision=1)}, "
          f"orc32-vs-orc64 {np.array2string(sg.max(axis=0), precision=1)}")
    # per Global, over all log points
    assert np.all(eg.max(axis=0) <= np.maximum(FP32_BAR, 2 * sg.max(axis=0))), (eg.max(axis=0), sg.max(axis=0))
