"""16-bit storage paths of a plain iteration: the tile-staged kernel (whole rows
copied into shared memory by TMA), the register two-node kernel and the
one-node kernel.

The tile-staged and register two-node kernels run the same update on the same
pulled values (packed FP32x2 collision for bulk pairs, the scalar node update
otherwise); only the route of the loads differs, so their snapshots must be
identical bit for bit where both apply (the register pair kernel needs nx a
multiple of 64, the tile-staged one a multiple of 32). The one-node kernel
contracts its arithmetic differently, so it is compared within a rounding bar,
and all three against the FP64 oracle."""
import numpy as np
import pytest

import oracle
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice

from helpers import apply_params, perturbed_equilibrium, random_flags, rel_l2

pytestmark = pytest.mark.gpu

TYPES = {
    "d2q9": ["Wall", "Solid", "WVelocity", "EPressure", "NSymmetry"],
    "d3q19": ["Wall", "Solid", "WVelocity", "EPressure", "WPressure"],
    "d3q27_cumulant": ["Wall", "Solid", "WVelocity", "EPressure", "NVelocity", "Buffer"],
}
PARAMS = {
    "d2q9": [("setting", "Viscosity", 0.05), ("zone", "VelocityX", 0.02, 1), ("zone", "Pressure", 0.01, 2)],
    "d3q19": [("setting", "nu", 0.05), ("setting", "InletVelocity", 0.02), ("setting", "ForceX", 1e-5)],
    "d3q27_cumulant": [("setting", "nu", 0.02), ("setting", "nubuffer", 0.05), ("setting", "ForceX", 1e-5),
                       ("zone", "Velocity", 0.02, 1), ("zone", "Pressure", 0.01, 2)],
}
# (nz, ny, nx): rows per tile = 512 / nx; ny a multiple of it. Small ny makes
# most tiles wrap at a y face (the one-row copies), larger ny has inner tiles.
# nx = 192 gives 2-row tiles of 384 nodes: fewer than the 512 of the stage
# layout, six consumer warps. Rows wider than 256 (288 ... 512) are one-row
# tiles copied with the split-x tensor maps (a (32, nx/32) box per row). nx a
# multiple of 32 but not of 64 (32, 96, 160, 288, 480) has warps that span two
# rows or end part-filled. The rows per tile are the largest count with at
# most 512 nodes that divides ny (96 x 6: 3 rows; 160 x 5: one row).
SHAPES = {
    "d2q9": [(1, 16, 128), (1, 8, 64), (1, 6, 256), (1, 8, 192), (1, 5, 384), (1, 3, 512), (1, 4, 448),
             (1, 10, 32), (1, 6, 96), (1, 5, 160), (1, 3, 288)],
    "d3q19": [(4, 8, 64), (3, 12, 128), (3, 6, 256), (3, 6, 192), (2, 3, 384), (2, 2, 512), (1, 4, 320),
              (2, 6, 96), (2, 5, 160), (1, 3, 480)],
    "d3q27_cumulant": [(4, 8, 64), (3, 12, 128), (2, 6, 256), (2, 8, 192), (2, 3, 384), (1, 2, 512),
                       (2, 6, 96), (2, 4, 224), (1, 3, 288)],
}


def run(model, shape, storage, fl, f0, tma, pairs, niter=5):
    m = M.get(model)
    g = Lattice(model, shape[2], shape[1], shape[0], precision="fp32", storage=storage)
    g.set_launch(32, 8, use_graphs=True, use_pairs=pairs, use_tma=tma, tma_always=tma)
    path = g.launch_path()
    g.set_flags(fl)
    apply_params(g, PARAMS[model])
    g.set_densities(f0)
    g.Iterate(niter, M.ITER_NORM | M.ITER_LASTGLOB)
    g.sync()
    out = (g.save().copy(), g.densities(), g.globals)
    g.close()
    return path, out


@pytest.mark.parametrize("storage", ["fp16s", "bf16s"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_tile_staged_matches_register_pairs_bit_for_bit(model, storage):
    m = M.get(model)
    for k, shape in enumerate(SHAPES[model]):
        extra = [g for g in ("ADDITIONALS", "BODY", "OBJECTIVE") if g in m.groups]
        fl = random_flags(model, shape, [t for t in TYPES[model] if t in m.node_types], zones=3, seed=20 + k,
                          p_type=0.15, extra_groups=extra[:1])
        f0 = perturbed_equilibrium(model, shape, seed=30 + k)
        p_tma, (raw_tma, f_tma, g_tma) = run(model, shape, storage, fl, f0, tma=True, pairs=True)
        p_one, (raw_one, f_one, g_one) = run(model, shape, storage, fl, f0, tma=False, pairs=False)
        assert p_tma["tma"] and not (p_one["tma"] or p_one["pairs"])
        assert np.isfinite(f_tma).all()
        if shape[2] % 64 == 0:  # the register pair kernel needs nx % 64 == 0
            p_pair, (raw_pair, f_pair, g_pair) = run(model, shape, storage, fl, f0, tma=False, pairs=True)
            assert not p_pair["tma"] and p_pair["pairs"]
            assert raw_tma.tobytes() == raw_pair.tobytes(), f"{shape}: tile-staged and register pairs differ"
            assert np.allclose(g_tma, g_pair, rtol=1e-12, atol=1e-12)  # FP64 atomics: order may differ
        assert rel_l2(f_tma, f_one) < 1e-3, shape
        o = oracle.OracleLattice(model, shape[2], shape[1], shape[0], precision="fp64")
        o.set_flags(fl)
        apply_params(o, PARAMS[model])
        o.set_densities(f0)
        o.iterate(5, M.ITER_NORM | M.ITER_LASTGLOB)
        ref = o.densities()
        e_one, e_tma = rel_l2(f_one, ref), rel_l2(f_tma, ref)
        assert e_tma < 1.5 * e_one + 1e-6, (shape, e_one, e_tma)


def test_tile_staged_only_where_it_applies():
    # FP32 storage, nx not a multiple of 32, nx above 512: no TMA
    for args in [("d3q19", 64, 8, 2, "same"), ("d3q19", 80, 8, 2, "fp16s"), ("d3q19", 576, 4, 2, "fp16s"),
                 ("d3q19", 48, 6, 2, "fp16s")]:
        model, nx, ny, nz, st = args
        g = Lattice(model, nx, ny, nz, precision="fp32", storage=st)
        assert not g.launch_path()["tma"], args
        g.close()
    for nx, ny in [(256, 4), (64, 8), (384, 3), (512, 2), (96, 7), (128, 6), (288, 5)]:
        g = Lattice("d3q27_cumulant", nx, ny, 2, precision="fp32", storage="fp16s")
        assert g.launch_path()["tma"], nx
        g.close()


def test_tile_staged_long_run_stays_identical():
    """Many replays of the captured iteration graph (tiles refill every stage
    many times) still match the register pair path."""
    model, shape, storage = "d3q27_cumulant", (8, 16, 128), "fp16s"
    m = M.get(model)
    fl = np.full(shape, m.flag("MRT"), np.uint16)
    f0 = perturbed_equilibrium(model, shape, seed=5)
    _, (raw_tma, _, _) = run(model, shape, storage, fl, f0, tma=True, pairs=True, niter=130)
    _, (raw_pair, _, _) = run(model, shape, storage, fl, f0, tma=False, pairs=True, niter=130)
    assert raw_tma.tobytes() == raw_pair.tobytes()


def test_d3q19_path_choice():
    """d3q19 16-bit lattices with nx % 64 == 0 take the register pair kernel where
    whole-row tiles would be under-filled (fewer than 448 nodes), too few (fewer
    than four per resident block) or one row wider than 256; full tiles stay
    staged. TCLB_LAUNCH_TMA_ALWAYS stages them anyway."""
    def path(nx, ny, nz, always=False):
        g = Lattice("d3q19", nx, ny, nz, precision="fp32", storage="fp16s")
        if always:
            g.set_launch(128, 2, use_tma=True, tma_always=True)
        p = g.launch_path()
        g.close()
        return "tma" if p["tma"] else ("pairs" if p["pairs"] else "one")

    assert path(256, 256, 64) == "tma"      # 2-row tiles of 512 nodes, many of them
    assert path(192, 192, 64) == "pairs"    # 2-row tiles of 384 nodes
    assert path(384, 64, 64) == "pairs"     # one row wider than 256
    assert path(64, 64, 64) == "pairs"      # 512 tiles: fewer than four per resident block
    assert path(192, 192, 64, always=True) == "tma"
    assert path(160, 160, 32) == "tma"      # nx % 64 != 0: no pair kernel, staged
    g = Lattice("d3q27_cumulant", 192, 192, 16, precision="fp32", storage="fp16s")
    assert g.launch_path()["tma"]            # the rule is d3q19's
    g.close()
