"""Headless ColorKernel (Lattice::Color -> LatticeContainer::Color,
src/LatticeContainer.inc.cpp.Rt:350-423): the oracle's colour map against
values worked out by hand from the reference's formula (CPU), and the CUDA
kernel against the oracle (GPU)."""
import numpy as np
import pytest

import oracle
from tclb_b200 import models as M

from helpers import random_flags

# (l, w) -> RGB, from src/LatticeContainer.inc.cpp.Rt:378-401 with l scaled by 111
KNOWN = [
    (0.0, 1, (0, 0, 0)),            # [0,1): r = 255 l
    (0.005, 1, (141, 0, 0)),        # 0.555 -> 141.5
    (0.05, 1, (255, 116, 0)),       # 5.55: g = 255 (l-1)/10 = 116.0
    (0.5, 1, (255, 255, 113)),      # 55.5: b = 255 (l-11)/100 = 113.5
    (2.0, 1, (255, 255, 255)),      # >= 111
    (-0.005, 1, (0, 0, 141)),       # [-1,0): b = 255 (-l)
    (-0.05, 1, (0, 116, 255)),      # [-11,-1): g = 255 (-l-1)/10
    (-0.5, 1, (113, 255, 255)),     # [-111,-11): r = 255 (-l-11)/100
    (-2.0, 1, (255, 255, 255)),     # < -111
    (0.05, 0, (0, 255, 0)),         # w = 0: green
    (float("nan"), 1, (255, 0, 255)),  # not finite: magenta
    (float("inf"), 0, (255, 0, 255)),
]


def test_color_map_known_values():
    l = np.array([k[0] for k in KNOWN], np.float32)
    w = np.array([k[1] for k in KNOWN], np.float32)
    got = oracle.color_map(l, w)
    for (lv, wv, rgb), row in zip(KNOWN, got):
        assert tuple(row[:3]) == rgb, (lv, wv, row)
        assert row[3] == 255


def speed32(u: np.ndarray, dim: int) -> np.ndarray:
    """|U| in float32 without contraction: (ux^2 + uy^2) [+ uz^2], sqrt."""
    u = u.astype(np.float32)
    s = u[..., 0] * u[..., 0] + u[..., 1] * u[..., 1]
    if dim == 3:
        s = s + u[..., 2] * u[..., 2]
    return np.sqrt(s)


BLANK = {"d2q9": ("Solid",), "d3q19": ("Wall",), "d3q27_cumulant": ("Solid",)}
TYPES = {"d2q9": ["Wall", "Solid", "WVelocity", "EPressure"], "d3q19": ["Wall", "Solid", "WVelocity", "EPressure"],
         "d3q27_cumulant": ["Wall", "Solid", "WVelocity", "EPressure", "NSymmetry"]}


def color_case(model, precision, seed):
    """Random node types (some nodes exactly Solid, with no other bit) and
    random densities spanning every colour band, plus one non-finite node."""
    from tclb_b200.lattice import Lattice

    m = M.get(model)
    shape = (1, 20, 64) if m.dim == 2 else (6, 10, 32)
    fl = random_flags(model, shape, [t for t in TYPES[model] if t in m.node_types], zones=1, seed=seed,
                      p_type=0.3)
    rng = np.random.default_rng(seed)
    fl[rng.random(shape) < 0.05] = m.flag("Solid")
    w = np.array(m.weights)[:, None, None, None]
    scale = rng.choice([0.001, 0.01, 0.1, 1.0], size=shape)[None]
    f = w * (1.0 + scale * rng.standard_normal((m.Q,) + shape))
    f[3, shape[0] // 2, 5, 7] = np.nan
    g = Lattice(model, shape[2], shape[1], shape[0], precision=precision)
    o = oracle.OracleLattice(model, shape[2], shape[1], shape[0], precision=precision)
    for lat in (g, o):
        lat.set_flags(fl)
        lat.set_densities(f)
    return g, o, shape


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_color_fp64_matches_oracle(model):
    g, o, shape = color_case(model, "fp64", seed=11)
    for z in sorted({-1, 0, shape[0] - 1}):
        a = g.Color(z)
        b = o.color(z)
        assert a.shape == (shape[1], shape[2], 4)
        assert np.array_equal(a, b), f"z={z}: {np.argwhere((a != b).any(-1))[:5]}"
    # every band and the special colours occur
    a = g.Color()
    assert (a[..., :3] == (255, 0, 255)).all(-1).any()
    assert (a[..., :3] == (0, 255, 0)).all(-1).any()
    assert len(np.unique(a.reshape(-1, 4), axis=0)) > 50
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_color_fp32_is_the_map_of_its_own_velocity(model):
    """FP32: the kernel's bytes equal the colour map of the FP32 |U| the
    library exports (same rounding), with the weight of each node's flag."""
    m = M.get(model)
    g, o, shape = color_case(model, "fp32", seed=12)
    g.Iterate(2)
    z = shape[0] // 2
    u = g.GetQuantity("U")[z]
    fl = g.get_flags()[z]
    if model == "d3q19":
        wgt = np.where((fl & m.groups["BOUNDARY"][0]) == m.flag("Wall"), 0, 1)
    else:
        wgt = np.where(fl == m.flag("Solid"), 0, 1)
    want = oracle.color_map(speed32(u, m.dim), wgt.astype(np.float32)).reshape(shape[1], shape[2], 4)
    assert np.array_equal(g.Color(), want)
    g.close()


@pytest.mark.gpu
def test_color_device_buffer_and_errors():
    import torch

    from tclb_b200.lattice import TCLBError

    g, o, shape = color_case("d3q19", "fp32", seed=13)
    buf = torch.zeros(shape[1] * shape[2] * 4, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g.Color(1, device_ptr=buf.data_ptr(), stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(buf.cpu().numpy().reshape(shape[1], shape[2], 4), g.Color(1))
    with pytest.raises(TCLBError):
        g.Color(shape[0])
    g.close()
