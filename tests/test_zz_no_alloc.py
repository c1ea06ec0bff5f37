"""tclb_get_quantity_noalloc: the quantity read-out for callers that cannot
allocate device memory (their GPU memory belongs to their own pool or budget,
or cudaMalloc/cudaFree would stall a latency-critical loop).

Checked through the C ABI against tclb_get_quantity, on two calls in a row
(the second call reuses the shared fixed array), within the FP32 tolerance of
the parity tests (relative L2 <= 1e-5). This file is collected last so that a
run stopping at its first failure has already run every other test; it also
passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200.lattice import Lattice, load_library

pytestmark = pytest.mark.gpu

TOL = 1e-5
LIMIT_BYTES = 8 << 20


def _noalloc(lib, lat, q, region, out):
    fn = lib.tclb_get_quantity_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_double,
                   ctypes.c_void_p]
    reg = (ctypes.c_int * 6)(*region)
    return fn(lat.handle, q, reg, ctypes.c_void_p(out.ctypes.data), 1.0, None)


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def test_noalloc_quantity_matches_allocating_path_twice():
    lib = load_library()
    nx, ny, nz = 64, 32, 32
    lat = Lattice("d3q19", nx, ny, nz, precision="fp32")
    lat.set_flags(cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=3))
    lat.SetSetting("nu", 0.01)
    lat.SetSetting("ForceX", 1e-4)
    lat.Init()
    lat.Iterate(40)
    q_u = lat.model.quantity_index("U")
    full = [0, 0, 0, nx, ny, nz]
    ref = lat.GetQuantity("U", region=full)
    for _call in range(2):  # two calls in a row on the shared array
        out = np.full_like(ref, np.nan)
        assert _noalloc(lib, lat, q_u, full, out) == 0, lib.tclb_last_error().decode()
        assert np.isfinite(out).all()
        assert _rel(out, ref) <= TOL
    # a sub-box of another quantity right after, against the allocating path
    box = [3, 5, 2, 40, 17, 9]
    q_p = lat.model.quantity_index("P")
    ref_p = lat.GetQuantity("P", region=box)
    out_p = np.full_like(ref_p, np.nan)
    assert _noalloc(lib, lat, q_p, box, out_p) == 0, lib.tclb_last_error().decode()
    assert _rel(out_p, ref_p) <= TOL
    lat.close()


def test_noalloc_rejects_regions_above_the_limit():
    lib = load_library()
    n = 96  # U of 96^3 FP32 nodes needs 10.6 MB > 8 MiB
    lat = Lattice("d3q27_cumulant", n, n, n, precision="fp32")
    lat.set_flags(cases.tgv_flags("d3q27_cumulant", n))
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=np.float32)
    lat.init_equilibrium(rho, u)
    lat.Iterate(5)
    out = np.zeros((n, n, n, 3), np.float32)
    assert n ** 3 * 3 * 4 > LIMIT_BYTES
    rc = _noalloc(lib, lat, lat.model.quantity_index("U"), [0, 0, 0, n, n, n], out)
    assert rc != 0
    assert "no-allocation limit" in lib.tclb_last_error().decode()
    # a slab under the limit still works and matches
    slab = [0, 0, 10, n, n, 8]
    ref = lat.GetQuantity("U", region=slab)
    out2 = np.zeros_like(ref)
    assert _noalloc(lib, lat, lat.model.quantity_index("U"), slab, out2) == 0
    assert _rel(out2, ref) <= TOL
    lat.close()
