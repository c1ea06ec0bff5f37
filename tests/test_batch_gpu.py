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
    """A case's result does not depend on the batch around it, the tile shape or the
    iterations per replay. Globals are computed at the end only: the Globals launch runs the
    one-node update, whose scalar arithmetic differs from the packed two-node update at FP32
    rounding (amplified by the 16-bit storage), so it must fall on the same iteration
    (the case's last) in both batches."""
    specs = d2q9_specs()
    alone = Batch("d2q9", "fp32", storage="fp16s")
    alone.set_paths(globals_at_end=True)
    alone.set_launch(128, 2, 16)
    a = alone.add_case(specs[1])
    alone.run_to_completion()
    u_alone = alone.quantity(a, "U")
    mix = Batch("d2q9", "fp32", storage="fp16s")
    mix.set_paths(globals_at_end=True)
    mix.set_launch(64, 4, 5)  # another tile shape and K, the same (two-nodes-per-thread) kernel form
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


def test_batch_pair_paths_apply():
    """16-bit storage takes the two-nodes-per-thread kernel on plain launches
    when the tile width is a multiple of 64 and the block fits; FP32 never."""
    b = Batch("d3q27_cumulant", "fp32", storage="fp16s", budget_bytes=1 << 28)
    for (bx, by), want in {(64, 4): True, (128, 2): True, (256, 1): True, (32, 8): False}.items():
        b.set_launch(bx, by, 4)
        assert b.uses_pairs() == want, (bx, by)
    b.set_launch(64, 4, 4)
    b.set_paths(use_pairs=False)
    assert not b.uses_pairs()
    b.close()
    b = Batch("d2q9", "fp32", budget_bytes=1 << 28)
    b.set_launch(128, 2, 4)
    assert not b.uses_pairs()
    b.close()


def _doubled(spec):
    """The case twice side by side in x: with periodic wrap every node of the
    doubled lattice sees the same neighbourhood as in the case itself."""
    return CaseSpec(np.concatenate([spec.flags, spec.flags], axis=-1), spec.settings, spec.zone_settings, spec.niter)


def _random_case(model, shape, seed, niter=6):
    """Random node types of every boundary class, three zones, the parity
    tests' settings: flow from the first iteration on."""
    from helpers import random_flags
    from test_parity_gpu import BOUNDARY_TYPES, EXTRA_GROUPS, PARAMS

    fl = random_flags(model, shape, BOUNDARY_TYPES[model], zones=3, seed=seed, p_type=0.15,
                      extra_groups=EXTRA_GROUPS[model])
    settings = {p[1]: p[2] for p in PARAMS[model] if p[0] == "setting"}
    zones = {}
    for p in PARAMS[model]:
        if p[0] == "zone":
            zones.setdefault(p[3], {})[p[1]] = p[2]
    return CaseSpec(fl, settings, zones, niter)


PAIR_SHAPES = {"d2q9": [(1, 24, 96), (1, 16, 64)], "d3q19": [(6, 8, 96)], "d3q27_cumulant": [(4, 8, 160)]}


@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
@pytest.mark.parametrize("storage", ["fp16s", "bf16"])
def test_batch_pair_kernel_partial_tiles(model, storage):
    """The batch's pair kernel on cases whose width is not a multiple of 64
    (the last tile of each row is half past the row: those lanes load the
    wrapped pair and store nothing) against the doubled case in the same
    batch (no partial tile): bit for bit. Then against the single-lattice
    pair kernel on the doubled case: the settings reach the two kernels by
    different roundings, so a 16-bit rounding may flip (1e-3 relative L2)."""
    specs = [_random_case(model, sh, seed=11 + i) for i, sh in enumerate(PAIR_SHAPES[model])]
    b = Batch(model, "fp32", storage=storage, budget_bytes=1 << 30)
    b.set_launch(64, 4, 4)
    assert b.uses_pairs()
    ids = [(b.add_case(s), b.add_case(_doubled(s))) for s in specs]
    b.run_to_completion()
    qs = (M.get(model).quantities[0][0], "U")
    for (cid, did), s in zip(ids, specs):
        half = s.shape[-1]
        for q in qs:
            got, dbl = b.quantity(cid, q), b.quantity(did, q)
            if q == "U":
                dbl = np.moveaxis(dbl, -1, 0)
                got = np.moveaxis(got, -1, 0)
            assert np.array_equal(got, dbl[..., :half]) and np.array_equal(got, dbl[..., half:]), q
        d = _doubled(s)
        nz, ny, nx = d.shape
        lat = Lattice(model, nx, ny, nz, precision="fp32", storage=storage)
        lat.set_launch(32, 8, use_tma=False)
        assert lat.launch_path()["pairs"]
        lat.set_flags(d.flags)
        for k, v in d.settings.items():
            lat.SetSetting(k, v)
        for z, dd in d.zone_settings.items():
            for k, v in dd.items():
                lat.set_zone_setting(k, v, z)
        lat.Init()
        lat.Iterate(d.niter, M.ITER_NORM | M.ITER_LASTGLOB)
        for q in qs:
            assert rel_l2(b.quantity(did, q), lat.GetQuantity(q)) <= 1e-3, q
        lat.close()
    b.close()


def test_batch_pair_kernel_odd_width_takes_one_node_update():
    """A case with odd nx has no node pairs: in the pair form its tiles run the
    one-node update; the result matches the batch's one-node form."""
    fl = cases.disc_channel_flags(97, 32, 5.0, 24, 16)
    spec = CaseSpec(fl, {"Viscosity": 0.03}, {0: {"VelocityX": 0.02}}, 12)
    out = []
    for bx, by in ((64, 4), (32, 8)):
        b = Batch("d2q9", "fp32", storage="fp16s", budget_bytes=1 << 28)
        b.set_launch(bx, by, 4)
        c = b.add_case(spec)
        b.run_to_completion()
        out.append(b.quantity(c, "U"))
        b.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("storage,short,tall", [("same", (32, 8), (32, 48)), ("fp16s", (64, 4), (64, 24))])
def test_tall_tiles_walk_rows(storage, short, tall):
    """Tiles taller than the block (each thread walks several rows, the last
    pass partly past the tile) give the same fields as short tiles, and the
    same Globals up to summation order (a thread sums its rows in FP32
    before the FP64 block reduction)."""
    specs = [_random_case("d3q19", (5, 40, 64), seed=21, niter=7), _random_case("d3q19", (3, 13, 96), seed=22, niter=7)]
    out = []
    for bx, by in (short, tall):
        b = Batch("d3q19", "fp32", storage=storage, budget_bytes=1 << 30)
        b.set_launch(bx, by, 3)
        b.set_paths(adaptive=False)  # these few small cases would get short tiles
        ids = [b.add_case(s) for s in specs]
        b.step()
        want = sum(s.shape[0] * -(-s.shape[1] // by) * -(-s.shape[2] // bx) for s in specs)
        assert b.info()["tiles"] == want
        b.run_to_completion()
        out.append([(b.quantity(c, "U"), b.globals(c)) for c in ids])
        b.close()
    for (u0, g0), (u1, g1) in zip(*out):
        assert np.array_equal(u0, u1)
        assert np.allclose(g0, g1, rtol=1e-6, atol=1e-12)


def test_short_tiles_when_few():
    """With few live tiles the table lowers the tile height (more, shorter
    tiles); the fields stay the same."""
    spec = _random_case("d2q9", (1, 64, 128), seed=31, niter=5)
    res = []
    for short in (True, False):
        b = Batch("d2q9", "fp32", budget_bytes=1 << 28)
        b.set_launch(64, 64, 5)
        b.set_paths(adaptive=short)
        c = b.add_case(spec)
        b.step()
        res.append((b.info()["tiles"], b.quantity(c, "U")))
        b.close()
    assert res[1][0] == 2 and res[0][0] == 2 * 64 // 4  # short: 4-row tiles (the block's thread rows)
    assert np.array_equal(res[0][1], res[1][1])


TMA_SHAPES = {
    "d2q9": [(1, 16, 64), (1, 8, 128), (1, 6, 192), (1, 10, 96)],
    "d3q19": [(4, 16, 64), (3, 12, 128), (2, 10, 192), (2, 6, 256), (3, 8, 96)],
    "d3q27_cumulant": [(3, 16, 64), (2, 8, 128), (2, 4, 192), (3, 8, 96)],
}


@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
@pytest.mark.parametrize("storage", ["fp16s", "bf16"])
def test_batch_tile_staged_matches_pairs_bit_for_bit(model, storage):
    """Cases whose rows fit the tile-staged kernel (nx a multiple of 32 up to
    512: here 64, 96, 128, 192, 256; for d3q19 only those whose tiles hold at
    least 448 nodes) take the tile-staged batch kernel, a case
    with other settings the pair kernel, in one batch; every field and Globals
    vector must equal that of the same batch with staging off (the same pair
    update on the same values; nx = 96 runs its last tile of each row
    half-filled in the pair form)."""
    specs = [_random_case(model, sh, seed=41 + i, niter=9) for i, sh in enumerate(TMA_SHAPES[model])]
    # a case that fits the staged kernel but has other settings: for the
    # packed-collision models it leaves the staged group and takes the pairs
    odd = _random_case(model, TMA_SHAPES[model][0], seed=49, niter=9)
    odd.settings[next(iter(odd.settings))] *= 1.25
    specs.append(odd)
    out = []
    for tma in (True, False):
        b = Batch(model, "fp32", storage=storage, budget_bytes=1 << 30)
        b.set_launch(64, 4, 4)  # K does not divide the iteration count
        b.set_paths(use_tma=tma, adaptive=False)  # stage these small cases too
        ids = [b.add_case(s) for s in specs]
        assert b.uses_tma() == tma and b.uses_pairs()
        b.run_to_completion()
        out.append([(b.quantity(c, "U"), b.quantity(c, M.get(model).quantities[0][0]), b.globals(c)) for c in ids])
        b.close()
    for (u0, p0, g0), (u1, p1, g1) in zip(*out):
        assert np.isfinite(u0).all()
        assert np.array_equal(u0, u1) and np.array_equal(p0, p1)
        assert np.array_equal(g0, g1)


def test_batch_tile_staged_late_admission_and_retire():
    """Staged and unstaged d3q19 cases joining and leaving between replays
    (the staged tile table is rebuilt, the graph's grids resized): each result
    equals that of the case alone in a batch with staging off."""
    specs = [_random_case("d3q19", sh, seed=51 + i, niter=n)
             for i, (sh, n) in enumerate([((4, 16, 64), 13), ((3, 8, 96), 6), ((2, 12, 128), 20)])]
    b = Batch("d3q19", "fp32", storage="fp16s", budget_bytes=1 << 30)
    b.set_launch(64, 8, 5)
    b.set_paths(adaptive=False)  # stage these small cases too
    c0 = b.add_case(specs[0])
    c1 = b.add_case(specs[1])
    b.step()
    b.sync()
    c2 = b.add_case(specs[2])
    b.run_to_completion()
    got = [b.quantity(c, "U") for c in (c0, c1, c2)]
    b.close()
    for s, u in zip(specs, got):
        a = Batch("d3q19", "fp32", storage="fp16s", budget_bytes=1 << 30)
        a.set_launch(64, 8, 5)
        a.set_paths(use_tma=False)
        c = a.add_case(s)
        a.run_to_completion()
        assert np.array_equal(a.quantity(c, "U"), u)
        a.close()


@pytest.mark.parametrize("model,storage,shapes", [
    ("d3q19", "fp16s", [(4, 16, 64), (3, 8, 96), (2, 12, 128)]),
    ("d2q9", "same", [(1, 24, 64), (1, 16, 96)]),
])
def test_globals_at_end(model, storage, shapes):
    """With Globals only in each case's finishing replay, the last launch of
    the other replays takes the plain kernels. In FP32 that is the same node
    update: fields and final Globals equal those of the default mode. With
    16-bit storage the plain kernels are the two-node ones, whose float
    rounding may flip a 16-bit value (the 1e-3 bar of the two-node path).
    Before a case finishes its Globals are zero."""
    specs = [_random_case(model, sh, seed=61 + i, niter=n) for i, (sh, n) in enumerate(zip(shapes, (17, 9, 30)))]
    out = []
    for at_end in (False, True):
        b = Batch(model, "fp32", storage=storage, budget_bytes=1 << 30)
        b.set_launch(64, 8, 4)
        b.set_paths(globals_at_end=at_end)
        ids = [b.add_case(s) for s in specs]
        b.step()
        b.sync()
        mid = b.globals(ids[-1])  # 30 iterations: not finished after one replay
        b.run_to_completion()
        out.append((mid, [(b.quantity(c, "U"), b.globals(c)) for c in ids]))
        b.close()
    (mid0, r0), (mid1, r1) = out
    assert np.any(mid0 != 0) and not np.any(mid1 != 0)
    for (u0, g0), (u1, g1) in zip(r0, r1):
        if storage == "same":
            assert np.array_equal(u0, u1) and np.array_equal(g0, g1)
        else:
            assert rel_l2(u1, u0) < 1e-3
            assert np.allclose(g1, g0, rtol=1e-2, atol=1e-3 * np.abs(g0).max())


def test_staging_needs_enough_tiles():
    """Adaptive: a small stageable case alone runs the register kernels (too
    few tiles for the persistent staged kernel); a large one is staged."""
    def uses_tma(n):
        b = Batch("d3q19", "fp32", storage="fp16s", budget_bytes=4 << 30)
        b.set_launch(64, 16, 4)
        b.add_case(CaseSpec(cases.porous_channel_d3q19(n, n, n, p=0.05, band=2, seed=3), {"nu": 0.02}, {}, 4))
        r = b.uses_tma()
        b.close()
        return r
    assert not uses_tma(64) and uses_tma(128)


def test_reserve_grows_the_pool_and_changes_nothing_else():
    """tclb_batch_reserve: more than the budget is refused; a reserve within it
    leaves admission (budget accounting) and results unchanged."""
    from tclb_b200.lattice import TCLBError

    spec = CaseSpec(cases.porous_channel_d3q19(128, 64, 32, p=0.08, band=2, seed=9), {"nu": 0.02, "ForceX": 1e-5}, {}, 12)
    out = []
    for reserve in (0, 256 << 20):
        b = Batch("d3q19", "fp32", storage="fp16s", budget_bytes=512 << 20)
        with pytest.raises(TCLBError):
            b.reserve(1 << 30)
        if reserve:
            b.reserve(reserve)
        assert b.info()["used_bytes"] == 0
        c = b.add_case(spec)
        assert b.info()["used_bytes"] == case_bytes("d3q19", 128, 64, 32, "fp32", "fp16s")
        b.run_to_completion()
        out.append(b.quantity(c, "U"))
        b.close()
    assert np.array_equal(out[0], out[1])


def test_d3q19_cases_with_underfilled_tiles_take_the_pair_kernel():
    """In a batch, a d3q19 case whose staged tiles would hold fewer than 448 nodes
    (edge 192: 2 rows of 192) takes the register pair kernel; a 256-edge case is
    staged. Both give the single-lattice result."""
    def uses(n):
        b = Batch("d3q19", "fp32", storage="fp16s", budget_bytes=8 << 30)
        b.set_paths(adaptive=False)
        b.set_launch(64, 64, 4)
        b.add_case(CaseSpec(cases.porous_channel_d3q19(n, n, 16, p=0.05, band=2, seed=3), {"nu": 0.02}, {}, 4))
        r = (b.uses_tma(), b.uses_pairs())
        b.close()
        return r
    assert uses(192) == (False, True)
    assert uses(256)[0]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_degenerate_cases_in_a_batch(model, precision):
    """Cases of one node, with axes of one or two nodes, and widths that are not a
    multiple of 32, batched together with a regular case: each case's velocity and
    Globals equal its single-lattice run."""
    m = M.get(model)
    shapes = [(1, 1, 1), (1, 1, 5), (1, 3, 1), (1, 7, 33), (1, 16, 64)] if m.dim == 2 else \
        [(1, 1, 1), (1, 1, 7), (3, 1, 5), (1, 4, 1), (2, 2, 33), (4, 8, 32)]
    specs = [_random_case(model, sh, seed=80 + i, niter=7) for i, sh in enumerate(shapes)]
    b = Batch(model, precision, budget_bytes=1 << 30)
    b.set_launch(32, 4, 3)
    ids = [b.add_case(s) for s in specs]
    b.run_to_completion()
    for cid, s in zip(ids, specs):
        u_s, g_s = run_single(model, s, precision)
        u_b, g_b = b.quantity(cid, "U"), b.globals(cid)
        assert np.isfinite(u_b).all()
        if np.abs(u_s).max() > 0:
            assert rel_l2(u_b, u_s) <= TOL_U[precision], (s.shape, rel_l2(u_b, u_s))
        else:
            assert np.abs(u_b).max() <= 1e-12, s.shape
        assert np.allclose(g_b, g_s, rtol=1e-9 if precision == "fp64" else 1e-4, atol=1e-12), (s.shape, g_b, g_s)
    b.close()
