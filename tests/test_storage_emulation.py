"""What limits the accuracy of 16-bit storage: the oracle's storage emulation.

The oracle can round every stored population through a storage format
(OracleLattice.set_storage: decode(encode(f - w_i)) + w_i, the collision in
FP64). With it the error of a format against the plain FP64 run can be
measured on the CPU and compared across formats that differ in one respect.
These tests pin the findings on the accuracy of 16-bit storage, on a small
Taylor-Green vortex (d3q27_cumulant, 20^3, u0 = 0.05, nu = 1e-3, 400
iterations):

* FP16-shift storage errs as IEEE half's spacing predicts: rounding the same
  deviations to 10 explicit mantissa bits without half's exponent limit gives
  at most the FP16 error (half loses a little more in its subnormal range);
* extra mantissa bits lower the error in proportion to the spacing (two more
  bits: about 4x), so the error is the storage spacing accumulated over the
  run;
* stochastic rounding does not lower it (the errors are not a bias that
  persists from step to step), and BF16 (7 bits) is about 8x worse.

Run as a script for the full table at a larger size:
    python tests/test_storage_emulation.py [n] [iterations]
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tclb_b200 import cases  # noqa: E402
from tclb_b200 import models as M  # noqa: E402


def _tgv(n):
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=np.float64)
    m = M.get("d3q27_cumulant")
    w = np.array(m.weights)
    e = np.array(m.velocities, np.float64)
    J = rho[..., None] * u
    eu = np.einsum("qd,zyxd->qzyx", e, J)
    return w[:, None, None, None] * (rho + 3 * eu + 4.5 * eu ** 2 / rho - 1.5 * (J ** 2).sum(-1) / rho)


def velocity_error(storage: str, n: int, iters: int, param: float = 0.0, ref=None):
    """Relative L2 velocity error of the FP64 run with `storage` emulated, against the plain FP64 run."""
    f0 = _tgv(n)

    def run(st, p):
        o = oracle.OracleLattice("d3q27_cumulant", n, n, n, precision="fp64")
        o.set_flags(cases.tgv_flags("d3q27_cumulant", n))
        o.set_setting("nu", 1e-3)
        if st != "same":
            o.set_storage(st, 1, p)
        o.set_densities(f0)
        o.iterate(iters)
        return o.quantity("U")

    if ref is None:
        ref = run("same", 0.0)
    u = run(storage, param)
    return float(np.linalg.norm(u - ref) / np.linalg.norm(ref)), ref


@pytest.fixture(scope="module")
def errors():
    n, it = 20, 400
    out, ref = {}, None
    for name, st, p in [("fp16s", "fp16s", 0), ("m10", "mant", 10), ("m11", "mant", 11), ("m12", "mant", 12),
                        ("fp16s_sr", "fp16s_sr", 0), ("bf16s", "bf16s", 0)]:
        out[name], ref = velocity_error(st, n, it, p, ref)
    return out


def test_fp16_error_is_its_mantissa_spacing(errors):
    assert 1e-5 < errors["fp16s"] < 1e-2
    assert errors["m10"] <= errors["fp16s"] * 1.05


def test_error_follows_the_mantissa_spacing(errors):
    assert errors["m10"] > errors["m11"] > errors["m12"]
    assert 2.5 < errors["m10"] / errors["m12"] < 6.0


def test_stochastic_rounding_does_not_help_and_bf16_is_coarser(errors):
    assert errors["fp16s_sr"] > 0.8 * errors["fp16s"]
    assert errors["bf16s"] > 4 * errors["fp16s"]


if __name__ == "__main__":
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 32
    it = int(sys.argv[2]) if len(sys.argv) > 2 else 1000
    ref = None
    rows = [("FP16-shift (IEEE half)", "fp16s", 0), ("FP16-shift, stochastic rounding", "fp16s_sr", 0),
            ("BF16-shift", "bf16s", 0), ("BF16-shift, stochastic rounding", "bf16s_sr", 0)]
    rows += [(f"{k} mantissa bits, FP32 exponent range", "mant", k) for k in (10, 11, 12, 13, 14)]
    rows += [(f"16-bit fixed point of (f-w)/w, range +-{s:g}", "fixed", s) for s in (1.0, 0.5, 0.25)]
    rows += [(f"{E} exponent / {15 - E} mantissa bits of (f-w)/w below {2.0 ** -L:g}", "exm", E * 16 + L)
             for E in (2, 3, 4) for L in (0, 1)]
    print(f"d3q27_cumulant Taylor-Green {n}^3, u0 = 0.05, nu = 1e-3, {it} iterations, collision in FP64")
    for label, st, p in rows:
        err, ref = velocity_error(st, n, it, p, ref)
        print(f"{label:58s} velocity rel L2 {err:.3e}", flush=True)
