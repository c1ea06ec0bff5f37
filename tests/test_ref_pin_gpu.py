"""The CUDA path against TCLB's own model code (the committed fixture).

tests/golden/ref_pin.npz holds one iteration of three small lattices whose
expected populations were computed by TCLB's literal per-node code
(oracle/_ref, built from the reference tree by oracle/make_ref.py; the cases
are described in tests/golden_cases.py): the d3q27_cumulant collision, the
d3q19 Zou-He closures, and the d2q9_SRT closures, bounce-back and BGK at
d2q9's node types.

Bars (relative L2 over the lattice): FP64 1e-12 against TCLB's double build,
FP32 1e-6 against its float build. Globals (d3q27_cumulant): |difference| <=
tol x sum of |per-node contributions|, tol 1e-12 (FP64) / 1e-6 (FP32). The
check runs for a Globals iteration (one-node kernel with the reduction) and
a plain one (the kernel the hot loop uses).
"""
import numpy as np
import pytest

from tclb_b200 import models as M
from tclb_b200.lattice import Lattice

import golden_cases as G

pytestmark = pytest.mark.gpu

BAR = {"fp64": 1e-12, "fp32": 1e-6}
GBAR = {"fp64": 1e-12, "fp32": 1e-6}


@pytest.mark.parametrize("glob", [True, False])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["d3q27c", "d3q19", "d2q9"])
def test_gpu_vs_tclb_source(case, prec, glob):
    fx = G.load()
    model, (nz, ny, nx) = G.CASES[case]
    with Lattice(model, nx, ny, nz, precision=prec) as g:
        G.setup(g, case, fx)
        g.Iterate(1, M.ITER_NORM | (M.ITER_LASTGLOB if glob else 0))
        f = g.densities()
        exp = fx[f"{case}_out_{prec}"]
        assert G.rel_l2(f, exp) < BAR[prec]
        node = np.abs(f - exp).reshape(exp.shape[0], -1).max(axis=0) / np.abs(exp).reshape(exp.shape[0], -1).max(axis=0)
        assert node.max() < 10 * BAR[prec]
        if case == "d3q27c" and glob:
            gv, gx, gs = G.d3q27c_globals(g.globals), fx[f"d3q27c_glob_{prec}"], fx[f"d3q27c_globabs_{prec}"]
            assert np.all(np.abs(gv - gx) <= GBAR[prec] * gs), (gv, gx)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_gpu_d2q9_init_vs_tclb_source(prec):
    fx = G.load()
    with Lattice("d2q9", 32, 8, 1, precision=prec) as g:
        g.FlagOverwrite(np.full((1, 8, 32), M.get("d2q9").flag("MRT"), np.uint16))
        G.d2q9_init_params(g)
        g.Init()
        f = g.densities().reshape(9, -1)
        exp = fx[f"d2q9_init_{prec}"]
        assert np.max(np.abs(f - exp[:, None])) < BAR[prec] * np.max(np.abs(exp))
