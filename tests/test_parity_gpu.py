"""Parity of the CUDA library (through its C ABI) against the CPU oracle.

Tolerances (written here, used below):
* FP64 path: densities relative L2 <= 1e-12 (the bar against TCLB's double
  build); velocity, a derived quantity that divides small momentum differences
  by rho, <= 1e-11.
* FP32 path: densities and velocity relative L2 <= 1e-5 (the bar against
  TCLB's float build) for flows of speed >= 0.01; in the porous-media flow,
  still accelerating after 200 iterations (|u| ~ 0.01), the FP32 noise floor
  eps32*rho/|u| times the random walk over the iterations sets a 1e-4 bar.
* Globals: |difference| <= tol * sum_i |x_i| (sum of absolute per-node
  contributions, from the oracle) -- the scale that bounds summation and
  rounding differences; tol = 1e-10 for FP64, 3e-3 for FP32 (per-node FP32
  values such as d2q9's (rho-1)/3 with rho-1 ~ 1e-3 lose about three digits to
  cancellation, so FP32 state differences of ~1e-6 show up at ~1e-3 there).
"""
import numpy as np
import pytest

import oracle
from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice, TCLBError

from helpers import apply_params, perturbed_equilibrium, random_flags, rel_l2

pytestmark = pytest.mark.gpu

TOL_F = {"fp64": 1e-12, "fp32": 1e-5}
TOL_U = {"fp64": 1e-11, "fp32": 1e-5}
TOL_G = {"fp64": 1e-10, "fp32": 3e-3}

BOUNDARY_TYPES = {
    "d2q9": ["EPressure", "WPressure", "NVelocity", "SVelocity", "WVelocity", "EVelocity", "NSymmetry", "SSymmetry",
             "Solid", "Wall"],
    "d3q19": ["EPressure", "Solid", "Wall", "WPressure", "WPressureL", "WVelocity"],
    "d3q27_cumulant": ["Buffer", "WVelocityTurbulent", "NVelocity", "SVelocity", "NPressure", "SPressure",
                       "EPressure", "EVelocity", "Solid", "Wall", "WPressure", "WVelocity"],
}
EXTRA_GROUPS = {"d2q9": ["OBJECTIVE"], "d3q19": ["ADDITIONALS"], "d3q27_cumulant": ["ADDITIONALS", "BODY"]}

PARAMS = {
    "d2q9": [("setting", "Viscosity", 0.05), ("setting", "S3", 0.3), ("setting", "S4", -0.2),
             ("setting", "GravitationX", 1e-5), ("setting", "GravitationY", -2e-6),
             ("zone", "VelocityX", 0.02, 0), ("zone", "VelocityX", 0.03, 1), ("zone", "VelocityY", 0.005, 2),
             ("zone", "Pressure", 0.01, 1), ("zone", "Pressure", -0.005, 2),
             ("zone", "OutletFluxInObj", 0.5, 1), ("zone", "PressureLossInObj", 2.0, 2)],
    "d3q19": [("setting", "nu", 0.05), ("setting", "InletVelocity", 0.02), ("setting", "InletPressure", 0.01),
              ("setting", "ForceX", 1e-5), ("setting", "ForceZ", -3e-6), ("zone", "VOLvxInObj", 1.5, 1)],
    "d3q27_cumulant": [("setting", "nu", 0.02), ("setting", "nubuffer", 0.05), ("setting", "ForceX", 1e-5),
                       ("setting", "ForceY", 2e-6), ("setting", "Omega", 0.8),
                       ("zone", "Velocity", 0.02, 0), ("zone", "Velocity", 0.03, 1), ("zone", "Pressure", 0.01, 2),
                       ("zone", "DragInObj", 0.7, 1)],
}


def make_pair(model, shape, precision, storage="same"):
    nz, ny, nx = shape
    g = Lattice(model, nx, ny, nz, precision=precision, storage=storage)
    o = oracle.OracleLattice(model, nx, ny, nz, precision="fp64" if precision == "fp64" else "fp32")
    return g, o


def run_both(g, o, niter, iter_type):
    g.Iterate(niter, iter_type)
    o.iterate(niter, iter_type)


def compare_globals(g, o, precision):
    """max over Globals of |gpu - oracle| / sum|contributions|."""
    gg, og, sc = g.globals, o.globals(), o.globals_scale()
    err = np.where(sc > 0, np.abs(gg - og) / np.where(sc > 0, sc, 1), np.abs(gg - og))
    return float(err.max()), gg, og


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_all_node_types(model, precision):
    """Every boundary type, zone and extra group on random nodes; a few
    iterations from a perturbed equilibrium; Globals on the last one."""
    m = M.get(model)
    shape = (1, 24, 64) if m.dim == 2 else (12, 10, 32)
    fl = random_flags(model, shape, BOUNDARY_TYPES[model], zones=3, seed=1, p_type=0.35,
                      extra_groups=EXTRA_GROUPS[model])
    f0 = perturbed_equilibrium(model, shape, seed=2)
    g, o = make_pair(model, shape, precision)
    for lat in (g, o):
        lat.set_flags(fl)
        apply_params(lat, PARAMS[model])
        lat.set_densities(f0)
    run_both(g, o, 6, M.ITER_NORM | M.ITER_LASTGLOB)
    e = rel_l2(g.densities(), o.densities())
    assert e < TOL_F[precision], f"densities rel L2 {e:.3e}"
    ge, gg, og = compare_globals(g, o, precision)
    assert ge < TOL_G[precision], f"globals rel err {ge:.3e}\n{gg}\n{og}"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_init_and_quantities(model, precision):
    m = M.get(model)
    shape = (1, 16, 64) if m.dim == 2 else (8, 8, 32)
    fl = random_flags(model, shape, BOUNDARY_TYPES[model], zones=3, seed=5, p_type=0.3,
                      extra_groups=EXTRA_GROUPS[model])
    g, o = make_pair(model, shape, precision)
    for lat in (g, o):
        lat.set_flags(fl)
        apply_params(lat, PARAMS[model])
        lat.Init() if hasattr(lat, "Init") else lat.init()
    tol = TOL_F[precision]
    assert rel_l2(g.densities(), o.densities()) < tol
    run_both(g, o, 3, M.ITER_NORM)
    for qi, (qn, vec) in enumerate(m.quantities):
        a = g.GetQuantity(qn)
        b = o.quantity(qn)
        if np.linalg.norm(b) == 0:
            assert np.abs(a).max() < tol
        else:
            assert rel_l2(a, b) < 10 * tol, f"quantity {qn}"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_channel_disc_d2q9(precision):
    """Configuration 1 at reduced size: 256x64 channel, disc r=8, 500 iterations,
    Globals every 100 (ITER_LASTGLOB)."""
    nx, ny = 256, 64
    fl = cases.channel_disc_d2q9(nx, ny, r=8, cx=64, cy=32)
    g, o = make_pair("d2q9", (1, ny, nx), precision)
    for lat in (g, o):
        lat.set_flags(fl)
        apply_params(lat, cases.channel_disc_settings(ux=0.01, nu=0.02, bgk=True))
        lat.Init() if hasattr(lat, "Init") else lat.init()
    for _ in range(5):
        run_both(g, o, 100, M.ITER_NORM | M.ITER_LASTGLOB)
        ge, gg, og = compare_globals(g, o, precision)
        assert ge < TOL_G[precision], f"globals {gg} vs {og}"
    u_g, u_o = g.GetQuantity("U"), o.quantity("U")
    ef, eu = rel_l2(g.densities(), o.densities()), rel_l2(u_g, u_o)
    if precision == "fp64":
        assert ef < TOL_F[precision] and eu < TOL_U[precision], f"densities {ef:.3e} velocity {eu:.3e}"
        return
    # FP32: two FP32 implementations that round in a different order drift
    # apart by about eps32*|f|/|u| per iteration (|u| = 0.01 here), a random
    # walk of ~1e-4 after 500 iterations with acoustic waves from the Zou-He
    # ends -- TCLB's float build shows the same spread against any other FP32
    # build. The densities meet 1e-5; the velocity is held to that noise floor
    # and, more usefully, to the accuracy of the FP32 oracle against FP64.
    assert ef < TOL_F[precision], f"densities {ef:.3e}"
    assert eu < 2e-4, f"velocity {eu:.3e}"
    o64 = oracle.OracleLattice("d2q9", nx, ny, 1, precision="fp64")
    o64.set_flags(fl)
    apply_params(o64, cases.channel_disc_settings(ux=0.01, nu=0.02, bgk=True))
    o64.init()
    o64.iterate(500)
    u64 = o64.quantity("U")
    e_gpu, e_orc = rel_l2(u_g, u64), rel_l2(u_o, u64)
    assert e_gpu < 2 * e_orc + 1e-6, f"GPU FP32 vs FP64 {e_gpu:.3e}, oracle FP32 vs FP64 {e_orc:.3e}"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tgv_d3q27(precision):
    """Configuration 2 at 32^3: Taylor-Green vortex, 100 iterations."""
    n = 32
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=np.float64)
    # equilibrium populations from (rho, rho*u) on the host
    w = np.array(M.get("d3q27_cumulant").weights)
    e = np.array(M.get("d3q27_cumulant").velocities, np.float64)
    J = rho[..., None] * u
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    j2 = (J ** 2).sum(-1)
    f = w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * j2 / rho)
    g, o = make_pair("d3q27_cumulant", (n, n, n), precision)
    for lat in (g, o):
        lat.set_flags(cases.tgv_flags("d3q27_cumulant", n))
        lat.set_setting("nu", 1e-3)
        lat.set_densities(f)
    for _ in range(2):
        run_both(g, o, 50, M.ITER_NORM | M.ITER_LASTGLOB)
        ge, gg, og = compare_globals(g, o, precision)
        assert ge < TOL_G[precision], f"{gg} vs {og}"
    ef, eu = rel_l2(g.densities(), o.densities()), rel_l2(g.GetQuantity("U"), o.quantity("U"))
    assert ef < TOL_F[precision] and eu < TOL_U[precision], f"densities {ef:.3e} velocity {eu:.3e}"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_porous_d3q19(precision):
    """Configuration 3 at 64x32x32: porous channel with body force, 200 iterations."""
    nx, ny, nz = 64, 32, 32
    fl = cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=3)
    g, o = make_pair("d3q19", (nz, ny, nx), precision)
    for lat in (g, o):
        lat.set_flags(fl)
        apply_params(lat, [("setting", "nu", 0.01), ("setting", "ForceX", 1e-4)])
        lat.Init() if hasattr(lat, "Init") else lat.init()
    run_both(g, o, 200, M.ITER_NORM | M.ITER_LASTGLOB)
    ef, eu = rel_l2(g.densities(), o.densities()), rel_l2(g.GetQuantity("U"), o.quantity("U"))
    tol_u = {"fp64": 1e-11, "fp32": 1e-4}[precision]
    assert ef < TOL_F[precision] and eu < tol_u, f"densities {ef:.3e} velocity {eu:.3e}"
    ge, gg, og = compare_globals(g, o, precision)
    assert ge < TOL_G[precision], f"{gg} vs {og}"


@pytest.mark.parametrize("storage", ["fp16s", "bf16s", "fp16", "bf16"])
def test_reduced_storage_d3q19(storage):
    """Reduced-precision storage against the FP64 oracle: velocity error bound."""
    nx, ny, nz = 64, 32, 32
    fl = cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=3)
    g = Lattice("d3q19", nx, ny, nz, precision="fp32", storage=storage)
    o = oracle.OracleLattice("d3q19", nx, ny, nz, precision="fp64")
    for lat in (g, o):
        lat.set_flags(fl)
        apply_params(lat, [("setting", "nu", 0.01), ("setting", "ForceX", 1e-4)])
        lat.Init() if hasattr(lat, "Init") else lat.init()
    run_both(g, o, 200, M.ITER_NORM)
    err = rel_l2(g.GetQuantity("U"), o.quantity("U"))
    print(f"{storage}: velocity rel L2 against the FP64 oracle {err:.3e}")
    # Measured on B200: fp16s 2.9e-4, bf16s 3.0e-3, fp16 1.9e-2, bf16 1.0. The
    # shifted FP16 format meets the 1e-3 bar on this flow; the bars below are
    # about 3x the measured errors. Unshifted 16-bit storage cannot hold the
    # ~1e-3 velocity signal on top of f ~ w_i (BF16 loses it entirely: its
    # spacing at w_i is above the per-step increments); the shifted formats
    # store f - w_i.
    bound = {"fp16s": 1e-3, "bf16s": 1e-2, "fp16": 6e-2, "bf16": 2.0}[storage]
    assert err < bound, f"{storage}: velocity rel L2 {err:.3e}"


def test_globals_cadence():
    """ITER_LASTGLOB replaces the host Globals with the last iteration's;
    ITER_INTEG integrates every iteration and accumulates across calls
    (src/Lattice.cu.Rt:900-989)."""
    shape = (8, 8, 32)
    g, o = make_pair("d3q27_cumulant", shape, "fp64")
    for lat in (g, o):
        lat.set_flags(cases.tgv_flags("d3q27_cumulant", 32, nz=8)[:, :8, :])
        lat.set_densities(perturbed_equilibrium("d3q27_cumulant", shape, seed=9))
    for it in (M.ITER_NORM | M.ITER_LASTGLOB, M.ITER_INTEG, M.ITER_INTEG, M.ITER_NORM, M.ITER_NORM | M.ITER_LASTGLOB):
        run_both(g, o, 3, it)
        ge, gg, og = compare_globals(g, o, "fp64")
        assert ge < 1e-10, (it, gg, og)


def test_save_load_roundtrip():
    g = Lattice("d3q19", 32, 8, 8, precision="fp32", storage="fp16s")
    g.set_flags(np.full((8, 8, 32), M.get("d3q19").flag("MRT"), np.uint16))
    g.Init()
    g.Iterate(3)
    snap = g.save()
    d0 = g.densities()
    g.Iterate(2)
    g.load(snap)
    assert np.array_equal(g.densities(), d0)
    assert snap.nbytes == 19 * 32 * 8 * 8 * 2


def test_flag_subbox():
    m = M.get("d2q9")
    g = Lattice("d2q9", 64, 16)
    full = np.full((1, 16, 64), m.flag("MRT"), np.uint16)
    g.FlagOverwrite(full)
    box = np.full((1, 4, 8), m.flag("Wall"), np.uint16)
    g.FlagOverwrite(box, offset=(10, 3, 0))
    full[:, 3:7, 10:18] = m.flag("Wall")
    assert np.array_equal(g.get_flags(), full)


def test_errors_are_status_codes():
    with pytest.raises(TCLBError):
        Lattice("d2q9", 64, 16, 2)  # 2D model with nz > 1
    with pytest.raises(TCLBError):
        Lattice("d3q19", 16, 16, 16, precision="fp64", storage="fp16s")
    g = Lattice("d2q9", 64, 16)
    with pytest.raises(TCLBError):
        g.GetQuantity("U", region=[60, 0, 0, 8, 16, 1])
    with pytest.raises(TCLBError):
        g.FlagOverwrite(np.zeros((1, 4, 8), np.uint16), offset=(60, 0, 0))


@pytest.mark.parametrize("shape", [(32, 8), (128, 2), (256, 1)])
def test_graph_replay_and_block_shape_do_not_change_results(shape):
    """CUDA-graph replays of plain iterations and any block shape give the
    same result as direct launches (the node arithmetic is identical)."""
    fl = cases.channel_disc_d2q9(256, 64, r=8, cx=64, cy=32)
    out = []
    for graphs, (bx, by) in ((False, (128, 2)), (True, shape)):
        g = Lattice("d2q9", 256, 64, precision="fp64")
        g.set_launch(bx, by, graphs)
        g.set_flags(fl)
        apply_params(g, cases.channel_disc_settings(ux=0.01, nu=0.02, bgk=True))
        g.Init()
        g.Iterate(150, M.ITER_NORM | M.ITER_LASTGLOB)
        out.append((g.densities(), g.globals))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.allclose(out[0][1], out[1][1], rtol=1e-12, atol=1e-18)


@pytest.mark.parametrize("storage", ["fp16s", "bf16s"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_two_nodes_per_thread_path(model, storage):
    """16-bit storage with nx % 64 == 0 updates two nodes per thread with
    32-bit accesses and shuffles for the x shifts; it must agree with the
    one-node path (a float rounding difference may flip a 16-bit rounding, so
    the bar is 1e-3 relative L2 after a few iterations) and be as accurate
    against the FP64 oracle."""
    m = M.get(model)
    shape = (1, 24, 128) if m.dim == 2 else (6, 10, 64)
    fl = random_flags(model, shape, BOUNDARY_TYPES[model], zones=3, seed=7, p_type=0.2,
                      extra_groups=EXTRA_GROUPS[model])
    f0 = perturbed_equilibrium(model, shape, seed=8)
    outs = []
    for pairs in (False, True):
        g = Lattice(model, shape[2], shape[1], shape[0], precision="fp32", storage=storage)
        g.set_launch(32, 8, use_graphs=True, use_pairs=pairs)
        g.set_flags(fl)
        apply_params(g, PARAMS[model])
        g.set_densities(f0)
        g.Iterate(4, M.ITER_NORM | M.ITER_LASTGLOB)
        outs.append((g.densities(), g.globals))
        g.close()
    o = oracle.OracleLattice(model, shape[2], shape[1], shape[0], precision="fp64")
    o.set_flags(fl)
    apply_params(o, PARAMS[model])
    o.set_densities(f0)
    o.iterate(4, M.ITER_NORM | M.ITER_LASTGLOB)
    ref = o.densities()
    assert np.isfinite(outs[1][0]).all()
    assert rel_l2(outs[1][0], outs[0][0]) < 1e-3
    e_single, e_pair = rel_l2(outs[0][0], ref), rel_l2(outs[1][0], ref)
    assert e_pair < 1.5 * e_single + 1e-6, (e_single, e_pair)


DEGENERATE = {2: [(1, 1, 1), (1, 1, 5), (1, 3, 1), (1, 7, 33)],
              3: [(1, 1, 1), (1, 1, 7), (3, 1, 5), (1, 4, 1), (2, 2, 33), (5, 3, 1)]}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp16s"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_degenerate_shapes(model, precision):
    """Lattices of one node, and with one or two nodes along an axis (the periodic
    pull then reads the node itself or its one neighbour from both sides), and a
    width that is not a multiple of 32: every boundary type on random nodes, four
    iterations, Globals on the last, against the oracle. 16-bit storage against the
    FP64 oracle within the storage bar."""
    m = M.get(model)
    for k, shape in enumerate(DEGENERATE[m.dim]):
        fl = random_flags(model, shape, BOUNDARY_TYPES[model], zones=3, seed=40 + k, p_type=0.3,
                          extra_groups=EXTRA_GROUPS[model])
        f0 = perturbed_equilibrium(model, shape, seed=50 + k)
        nz, ny, nx = shape
        prec = "fp32" if precision == "fp16s" else precision
        g = Lattice(model, nx, ny, nz, precision=prec, storage="fp16s" if precision == "fp16s" else "same")
        o = oracle.OracleLattice(model, nx, ny, nz, precision="fp64" if precision != "fp32" else "fp32")
        for lat in (g, o):
            lat.set_flags(fl)
            apply_params(lat, PARAMS[model])
            lat.set_densities(f0)
        run_both(g, o, 4, M.ITER_NORM | M.ITER_LASTGLOB)
        f_g, f_o = g.densities(), o.densities()
        assert np.isfinite(f_g).all(), shape
        bar = {"fp64": TOL_F["fp64"], "fp32": TOL_F["fp32"], "fp16s": 2e-3}[precision]
        assert rel_l2(f_g, f_o) < bar, (shape, rel_l2(f_g, f_o))
        if precision != "fp16s":
            ge, gg, og = compare_globals(g, o, precision)
            assert ge < TOL_G[precision], (shape, gg, og)
        g.close()
