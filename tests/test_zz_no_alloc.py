"""tclb_get_quantity_noalloc: the quantity read-out for callers that cannot
allocate device memory (their GPU memory belongs to their own pool or budget,
or cudaMalloc/cudaFree would stall a latency-critical loop).

Checked through the C ABI (Lattice.GetQuantityNoAlloc) against
tclb_get_quantity within the parity tests' FP32 tolerance (relative L2 <=
1e-5): on two calls in a row (the second reuses the shared fixed array), for
FP32, FP64 and 16-bit storage, and for a region whose quantity needs exactly
the 8 MiB limit (accepted) or one node more (rejected). Around a call after
the first, the device's free memory must not change: the call allocates
nothing. This file is collected last so that a run stopping at its first
failure has already run every other test; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice, TCLBError

pytestmark = pytest.mark.gpu

TOL = 1e-5
LIMIT_BYTES = 8 << 20


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _porous(precision="fp32", storage="same"):
    nx, ny, nz = 64, 32, 32
    lat = Lattice("d3q19", nx, ny, nz, precision=precision, storage=storage)
    lat.set_flags(cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=3))
    lat.SetSetting("nu", 0.01)
    lat.SetSetting("ForceX", 1e-4)
    lat.Init()
    lat.Iterate(40)
    return lat


def test_noalloc_quantity_matches_allocating_path_twice():
    lat = _porous()
    full = [0, 0, 0, lat.nx, lat.ny, lat.nz]
    ref = lat.GetQuantity("U", region=full)
    for call in range(2):  # two calls in a row on the shared array
        out = np.full_like(ref, np.nan)
        free0 = _free_bytes()
        lat.GetQuantityNoAlloc("U", region=full, out=out)
        free1 = _free_bytes()
        if call == 1:  # the first call may load the library's code; later calls allocate nothing
            assert free1 == free0, (free0, free1)
        assert np.isfinite(out).all()
        assert _rel(out, ref) <= TOL
    # a sub-box of another quantity right after, against the allocating path
    box = [3, 5, 2, 40, 17, 9]
    ref_p = lat.GetQuantity("P", region=box)
    out_p = np.full_like(ref_p, np.nan)
    lat.GetQuantityNoAlloc("P", region=box, out=out_p)
    assert _rel(out_p, ref_p) <= TOL
    lat.close()


@pytest.mark.parametrize("precision,storage", [("fp64", "same"), ("fp32", "fp16s")])
def test_noalloc_fp64_and_16bit_storage(precision, storage):
    lat = _porous(precision, storage)
    for name in ("U", "P"):
        ref = lat.GetQuantity(name)
        for _call in range(2):
            out = np.full_like(ref, np.nan)
            lat.GetQuantityNoAlloc(name, out=out)
            assert out.dtype == ref.dtype
            assert _rel(out, ref) <= TOL
    lat.close()


def test_noalloc_limit_is_exact():
    # a d2q9 row of 2^21 + 1 nodes: its FP32 density needs 8 MiB + 4 bytes
    n = (LIMIT_BYTES // 4) + 1
    lat = Lattice("d2q9", n, 1, 1, precision="fp32")
    lat.set_flags(np.full((1, 1, n), M.get("d2q9").flag("MRT"), np.uint16))
    lat.set_zone_setting("Pressure", 0.01)
    lat.set_zone_setting("VelocityX", 0.02)
    lat.Init()
    lat.Iterate(3)
    at_limit = [0, 0, 0, n - 1, 1, 1]  # exactly 8 MiB: accepted
    ref = lat.GetQuantity("Rho", region=at_limit)
    assert ref.nbytes == LIMIT_BYTES
    out = np.full_like(ref, np.nan)
    lat.GetQuantityNoAlloc("Rho", region=at_limit, out=out)
    assert _rel(out, ref) <= TOL
    with pytest.raises(TCLBError, match="no-allocation limit"):  # one node more: rejected
        lat.GetQuantityNoAlloc("Rho", region=[0, 0, 0, n, 1, 1], out=np.zeros(n, np.float32))
    lat.close()


def test_noalloc_rejects_regions_above_the_limit():
    n = 96  # U of 96^3 FP32 nodes needs 10.6 MB > 8 MiB
    lat = Lattice("d3q27_cumulant", n, n, n, precision="fp32")
    lat.set_flags(cases.tgv_flags("d3q27_cumulant", n))
    rho, u = cases.tgv_fields(n, u0=0.05, dtype=np.float32)
    lat.init_equilibrium(rho, u)
    lat.Iterate(5)
    assert n ** 3 * 3 * 4 > LIMIT_BYTES
    with pytest.raises(TCLBError, match="no-allocation limit"):
        lat.GetQuantityNoAlloc("U", out=np.zeros((n, n, n, 3), np.float32))
    # a slab under the limit still works and matches
    slab = [0, 0, 10, n, n, 8]
    ref = lat.GetQuantity("U", region=slab)
    out = lat.GetQuantityNoAlloc("U", region=slab)
    assert _rel(out, ref) <= TOL
    lat.close()
