"""Batched cases (tclb_batch_*): every case's result must be the same as the
same case run alone -- through a single lattice (tclb_iterate) and alone in a
batch. Tolerances: FP64 velocity relative L2 1e-12; FP32 1e-5 between the
batched and the single-lattice kernel (the same node code compiled into two
kernels may contract multiply-adds differently) and 1e-6 between two runs of
the batched kernel; Globals within 1e-9 relative (FP64 sums in another order)."""
import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.batch import AdmissionRefused, Batch, CaseSpec, autotune, case_bytes
from tclb_b200.lattice import Lattice

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL_U = {"fp64": 1e-12, "fp32": 1e-5}


def d2q9_specs():
    out = []
    for (W, H, r, nu, n) in [(64, 32, 4.0, 0.05, 23), (96, 32, 5.0, 0.03, 40), (128, 64, 9.0, 0.02, 57)]:
        fl = cases.disc_channel_flags(W, H, r, W / 4, H / 2)
        out.append(CaseSpec(fl, {"Viscosity": nu, "S3": 0.1, "S4": -0.1},
                            {0: {"VelocityX": 0.02}, 1: {"VelocityX": 0.03}, 2: {"Pressure": 0.001}}, n))
    return out


def run_single(model, spec, precision, storage="same"):
    nz, ny, nx = spec.shape
    lat = Lattice(model, nx, ny, nz, precision=precision, storage=storage)
    lat.set_flags(spec.flags)
    for k, v in spec.settings.items():
        lat.SetSetting(k, v)
    for z, d in spec.zone_settings.items():
        for k, v in d.items():
            lat.set_zone_setting(k, v, z)
    lat.Init()
    lat.Iterate(spec.niter, M.ITER_NORM | M.ITER_LASTGLOB)
    u, g = lat.GetQuantity("U"), lat.globals
    lat.close()
    return u, g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_equals_single_lattice(precision):
    specs = d2q9_specs()
    b = Batch("d2q9", precision, budget_bytes=1 << 30)
    b.set_launch(64, 4, 8)  # K does not divide the iteration counts
    ids = [b.add_case(s) for s in specs]
    steps = b.run_to_completion()
    assert steps == int(np.ceil(max(s.niter for s in specs) / 8))
    for cid, s in zip(ids, specs):
        assert b.poll(cid) == (s.niter, 0)
        u_s, g_s = run_single("d2q9", s, precision)
        u_b, g_b = b.quantity(cid, "U"), b.globals(cid)
        assert rel_l2(u_b, u_s) <= TOL_U[precision]
        assert np.allclose(g_b, g_s, rtol=1e-9, atol=1e-15), (g_b, g_s)
    b.close()


def test_result_same_alone_and_in_the_mix():
    specs = d2q9_specs()
    alone = Batch("d2q9", "fp32", storage="fp16s")
    alone.set_launch(128, 2, 16)
    a = alone.add_case(specs[1])
    alone.run_to_completion()
    u_alone = alone.quantity(a, "U")
    mix = Batch("d2q9", "fp32", storage="fp16s")
    mix.set_launch(32, 8, 5)
    ids = [mix.add_case(s) for s in specs]
    mix.run_to_completion()
    u_mix = mix.quantity(ids[1], "U")
    assert rel_l2(u_mix, u_alone) <= 1e-6
    alone.close()
    mix.close()


def test_d3q19_cases_and_late_admission():
    """d3q19 porous boxes; a case admitted while others are mid-run still
    matches its single-lattice result."""
    specs = []
    for i, (n, p) in enumerate([(32, 0.05), (48, 0.1)]):
        fl = cases.porous_channel_d3q19(n, n, n, p=p, band=2, seed=i)
        specs.append(CaseSpec(fl, {"nu": 0.02, "ForceX": 1e-5}, {}, 30 + 10 * i))
    b = Batch("d3q19", "fp64")  # FP64: the weak early flow (|u| ~ 3e-4) is below the FP32 noise floor
    b.set_launch(32, 4, 7)
    c0 = b.add_case(specs[0])
    b.step()
    b.sync()
    c1 = b.add_case(specs[1])  # joins after the first replay
    b.run_to_completion()
    for cid, s in ((c0, specs[0]), (c1, specs[1])):
        u_s, _ = run_single("d3q19", s, "fp64")
        assert rel_l2(b.quantity(cid, "U"), u_s) <= TOL_U["fp64"]
    b.close()


def test_admission_by_footprint():
    fl = cases.disc_channel_flags(128, 32, 4, 30, 16)
    per = case_bytes("d2q9", 128, 32)
    b = Batch("d2q9", "fp32", budget_bytes=2 * per + per // 2, max_cases=8)
    spec = CaseSpec(fl, {"Viscosity": 0.05}, {0: {"VelocityX": 0.02}}, 10)
    c0 = b.add_case(spec)
    b.add_case(spec)
    with pytest.raises(AdmissionRefused):
        b.add_case(spec)
    b.remove_case(c0)
    c2 = b.add_case(spec)  # memory of the retired case is reused
    assert b.info()["cases"] == 2 and b.info()["used_bytes"] <= 2 * per + per // 2
    b.run_to_completion()
    assert b.poll(c2) == (10, 0)
    b.close()


def test_autotune_picks_a_valid_shape():
    specs = d2q9_specs()
    r = autotune("d2q9", specs, tiles=[(32, 8), (128, 2)], ks=[1, 8], trial_iters=16)
    assert (r["bx"], r["by"]) in [(32, 8), (128, 2)] and r["K"] in (1, 8)
    assert r["mlups"] > 0 and len(r["table"]) == 4
