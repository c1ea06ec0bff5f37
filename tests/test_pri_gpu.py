"""TCLB's .pri snapshot (Lattice::save / load, src/Lattice.cu.Rt:642-769) and
the case runner's <SaveCheckpoint> / <LoadBinary> restart.

The expected bytes are built here in numpy from TCLB's layout rules, stated
independently of the library:
  * blocks d = (dx,dy,dz) in order k = 0..26, d = (k%3-1, (k//3)%3-1, k//9-1)
    (src/conf.R:771-778); density i with velocity e is a field spanning
    offsets -e (src/conf.R:89-91), so it has a box in block d iff every axis
    has d_a == 0 or d_a == -e_a; empty blocks are not written (listTabs,
    src/Lattice.cu.Rt:642-661);
  * a block holds its fields in density order, each an x-fastest box of
    extent n_a (d_a == 0) or 1 (src/conf.R:905-998, default GPU layout);
  * the put (src/conf.R:978-983): node n writes density i into the margin
    d_a = -e_a when it sits on the outgoing edge of axis a, else in place;
    d3q27_cumulant also writes the edge node in place
    (models/flow/d3q27_cumulant/Dynamics.R:51); slots never written are zero.
"""
import os
import subprocess

import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice, TCLBError

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INTERIOR_COPY = {"d2q9": False, "d3q19": False, "d3q27_cumulant": True}
ELEM = {("fp64", "same"): np.float64, ("fp32", "same"): np.float32, ("fp32", "fp16s"): np.float16}


def expected_pri(model: str, raw: np.ndarray) -> bytes:
    """raw: (Q, nz, ny, nx) array of storage words (any 1/2/4/8-byte dtype)."""
    m = M.get(model)
    Q, nz, ny, nx = raw.shape
    dims = (nx, ny, nz)
    out = []
    for k in range(27):
        d = (k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1)
        fields = [i for i, e in enumerate(m.velocities) if all(d[a] == 0 or e[a] == -d[a] for a in range(3))]
        for i in fields:
            e = m.velocities[i]
            sl = []
            for a in (2, 1, 0):  # z, y, x slicing of (nz, ny, nx)
                sl.append(slice(dims[a] - 1, dims[a]) if d[a] < 0 else slice(0, 1) if d[a] > 0 else slice(None))
            box = raw[i][tuple(sl)].copy()
            if not INTERIOR_COPY[model]:
                for a in range(3):
                    if d[a] != 0 or e[a] == 0:
                        continue
                    edge = dims[a] - 1 if e[a] > 0 else 0
                    idx = [slice(None)] * 3
                    idx[2 - a] = edge
                    box[tuple(idx)] = 0  # the edge node wrote into the margin only
            out.append(box.tobytes())
    return b"".join(out)


def random_lattice(model, nx, ny, nz, precision, storage, seed):
    m = M.get(model)
    lat = Lattice(model, nx, ny, nz, precision=precision, storage=storage)
    lat.set_flags(np.full((nz, ny, nx), m.flag("MRT"), np.uint16))
    rng = np.random.default_rng(seed)
    w = np.array(m.weights)[:, None, None, None]
    f = w * (1.0 + 0.05 * rng.standard_normal((m.Q, nz, ny, nx)))
    lat.set_densities(f)
    return lat


@pytest.mark.parametrize("model,shape", [("d2q9", (32, 12, 1)), ("d3q19", (32, 6, 5)),
                                         ("d3q27_cumulant", (32, 5, 4))])
@pytest.mark.parametrize("precision,storage", [("fp64", "same"), ("fp32", "same"), ("fp32", "fp16s")])
def test_pri_bytes_follow_tclb_layout(model, shape, precision, storage):
    m = M.get(model)
    nx, ny, nz = shape
    lat = random_lattice(model, nx, ny, nz, precision, storage, seed=1)
    lat.Iterate(3)
    dt = ELEM[(precision, storage)]
    raw = lat.save().view(dt).reshape(m.Q, nz, ny, nx)
    pri = lat.save_pri()
    want = expected_pri(model, raw)
    assert pri.size == len(want)
    assert pri.tobytes() == want
    lat.close()


@pytest.mark.parametrize("model,shape", [("d2q9", (32, 12, 1)), ("d3q19", (32, 6, 5)),
                                         ("d3q27_cumulant", (32, 5, 4))])
def test_pri_load_restores_state_and_run(model, shape):
    """save_pri -> load_pri into a fresh lattice gives the same snapshot, and
    both lattices then iterate to identical states."""
    m = M.get(model)
    nx, ny, nz = shape
    a = random_lattice(model, nx, ny, nz, "fp32", "same", seed=2)
    a.Iterate(5)
    pri = a.save_pri()
    b = Lattice(model, nx, ny, nz, precision="fp32")
    b.set_flags(np.full((nz, ny, nx), m.flag("MRT"), np.uint16))
    b.load_pri(pri)
    assert a.save().tobytes() == b.save().tobytes()
    a.Iterate(7)
    b.Iterate(7)
    assert a.save().tobytes() == b.save().tobytes()
    a.close()
    b.close()


def test_pri_load_reads_margins_not_stale_interior():
    """d2q9: the interior slots of an edge node's outgoing densities are never
    written by TCLB; whatever they hold, the loader takes the margin copy."""
    nx, ny = 32, 8
    a = random_lattice("d2q9", nx, ny, 1, "fp64", "same", seed=3)
    pri = a.save_pri().view(np.float64).copy()
    ref = a.save().tobytes()
    # walk the blocks to the interior one (k = 13)
    m = M.get("d2q9")
    off = 0
    for k in range(27):
        d = (k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1)
        nf = sum(all(d[a_] == 0 or e[a_] == -d[a_] for a_ in range(3)) for e in m.velocities)
        size = nf * (nx if d[0] == 0 else 1) * (ny if d[1] == 0 else 1) * (1 if d[2] == 0 else 1)
        if d == (0, 0, 0):
            box = pri[off:off + size].reshape(9, ny, nx)
            assert box[1, :, nx - 1].tolist() == [0.0] * ny  # never written by TCLB
            box[1, :, nx - 1] = 123.0  # garbage in the stale slots
            box[5, ny - 1, :] = -7.0
        off += size
    assert off == pri.size
    b = Lattice("d2q9", nx, ny, 1, precision="fp64")
    b.load_pri(pri.view(np.uint8))
    assert b.save().tobytes() == ref
    a.close()
    b.close()


def test_pri_size_mismatch_is_an_error():
    lat = random_lattice("d2q9", 32, 8, 1, "fp32", "same", seed=4)
    pri = lat.save_pri()
    with pytest.raises(TCLBError):
        lat.load_pri(pri[:-4])
    lat.close()


CHECKPOINT_CASE = """<?xml version="1.0"?>
<CLBConfig version="2.0" output="{out}">
\t<Geometry nx="128" ny="32">
\t\t<MRT><Box/></MRT>
\t\t<WVelocity name="Inlet"><Box nx="1"/></WVelocity>
\t\t<EPressure name="Outlet"><Box dx="-1"/></EPressure>
\t\t<Wall mask="ALL">
\t\t\t<Channel/>
\t\t\t<Sphere dx="24" nx="8" dy="12" ny="8"/>
\t\t</Wall>
\t</Geometry>
\t<Model>
\t\t<Param name="VelocityX" value="0.02"/>
\t\t<Param name="Viscosity" value="0.05"/>
\t</Model>
\t<Solve Iterations="100">
\t\t<SaveCheckpoint Iterations="50" keep="all"/>
\t\t<BIN Iterations="100"/>
\t</Solve>
</CLBConfig>
"""


def test_checkpoint_restart_resumes_bit_exactly(tmp_path):
    """<SaveCheckpoint> writes <out>_checkpoint_<it>_0.pri and a restart case
    with <LoadBinary> before <Solve>; running the restart from iteration 50
    for 100 iterations gives the state of an uninterrupted 150-iteration run
    (TCLB does not store the iteration counter in the .pri)."""
    runner = os.path.join(ROOT, "tclb_b200", "tclb_run")
    out = str(tmp_path) + "/"
    case = tmp_path / "ck.xml"
    case.write_text(CHECKPOINT_CASE.format(out=out))
    r = subprocess.run([runner, "d2q9", str(case), "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for it in (50, 100):
        assert os.path.exists(f"{out}ck_checkpoint_{it:08d}_0.pri")
        assert os.path.exists(f"{out}ck_restart_{it:08d}.xml")
    restart = f"{out}ck_restart_00000050.xml"
    text = open(restart).read()
    assert "<LoadBinary" in text and text.index("<LoadBinary") < text.index("<Solve")
    # the restart writes into a fresh folder so its BIN does not overwrite
    out2 = tmp_path / "again"
    out2.mkdir()
    r = subprocess.run([runner, "d2q9", restart, "--output", str(out2) + "/", "--quiet"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    u_restart = np.fromfile(str(out2) + "/ck_restart_00000050_BIN_P00_00000100.U.bin", np.float32)
    # uninterrupted run through the API: same geometry and settings, 150 iterations
    g = cases.Geometry("d2q9", 128, 32)
    g.set_flag("MRT").box()
    g.set_flag("WVelocity", zone="Inlet").box(nx=1)
    g.set_flag("EPressure", zone="Outlet").box(dx=-1)
    g.set_flag("Wall", mask="ALL").channel()
    g.set_flag("Wall", mask="ALL").sphere(dx=24, nx=8, dy=12, ny=8)
    lat = Lattice("d2q9", 128, 32)
    lat.set_flags(g.geom)
    lat.set_zone_setting("VelocityX", 0.02)
    lat.SetSetting("Viscosity", 0.05)
    lat.Init()
    lat.Iterate(150)
    assert np.array_equal(u_restart, lat.GetQuantity("U").ravel())
    # and the 100-iteration checkpoint equals the API state at 100
    lat2 = Lattice("d2q9", 128, 32)
    lat2.set_flags(g.geom)
    lat2.set_zone_setting("VelocityX", 0.02)
    lat2.SetSetting("Viscosity", 0.05)
    lat2.Init()
    lat2.Iterate(100)
    pri = np.fromfile(f"{out}ck_checkpoint_00000100_0.pri", np.uint8)
    assert pri.tobytes() == lat2.save_pri().tobytes()
    lat.close()
    lat2.close()


@pytest.mark.gpu
def test_save_binary(tmp_path):
    """<SaveBinary>: the .pri snapshot to <out>_<file>_0.pri (the name fixed when
    the element is read, so each call overwrites it), or without file= to
    <out>_Save_P00_<iteration>_0.pri; both equal the checkpoint at the same
    iteration. comp= names a parameter density, which these models lack, so
    nothing is written."""
    runner = os.path.join(ROOT, "tclb_b200", "tclb_run")
    out = str(tmp_path) + "/"
    text = CHECKPOINT_CASE.format(out=out).replace(
        '<BIN Iterations="100"/>', '<SaveBinary Iterations="50" file="snap"/><SaveBinary Iterations="50" comp="Rho"/>')
    text = text.replace("</Solve>", "</Solve>\n\t<SaveBinary/><SaveMemoryDump file=\"dump\"/>")
    case = tmp_path / "ck.xml"
    case.write_text(text)
    r = subprocess.run([runner, "d2q9", str(case), "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ck = open(f"{out}ck_checkpoint_00000100_0.pri", "rb").read()
    assert open(f"{out}ck_snap_0.pri", "rb").read() == ck
    assert open(f"{out}ck_Save_P00_00000100_0.pri", "rb").read() == ck
    assert open(f"{out}ck_checkpoint_00000050_0.pri", "rb").read() != ck
    assert not [f for f in os.listdir(tmp_path) if "Rho" in f]
    assert open(f"{out}ck_dump_0.pri", "rb").read() == ck
    # <LoadMemoryDump> reads it back: saved again right away, the bytes are the same
    load = CHECKPOINT_CASE.format(out=out + "re_")
    start, end = load.index("<Solve"), load.index("</CLBConfig>")
    load = load[:start] + f'<LoadMemoryDump file="{out}ck_dump"/><SaveBinary file="again"/>\n' + load[end:]
    case2 = tmp_path / "re.xml"
    case2.write_text(load)
    r = subprocess.run([runner, "d2q9", str(case2), "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert open(f"{out}re_re_again_0.pri", "rb").read() == ck
