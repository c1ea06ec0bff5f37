"""XML case front-end (tclb_case_geometry / tclb_case_run): the native C++
rasteriser against the Python one and hand-computed shapes (CPU), and a case
file run end to end against the API (GPU)."""
import ctypes
import glob
import os

import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import load_library

HERE = os.path.dirname(os.path.abspath(__file__))


def case_geometry(xml: str, model: str) -> np.ndarray:
    lib = load_library()
    lib.tclb_case_geometry.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_uint16), ctypes.c_size_t]
    lib.tclb_case_last_error.restype = ctypes.c_char_p
    dims = (ctypes.c_int * 3)()
    mid = M.get(model).mid
    assert lib.tclb_case_geometry(xml.encode(), mid, dims, None, 0) == 0, lib.tclb_case_last_error()
    nx, ny, nz = dims
    out = np.zeros((nz, ny, nx), np.uint16)
    rc = lib.tclb_case_geometry(xml.encode(), mid, dims, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size)
    assert rc == 0, lib.tclb_case_last_error()
    return out


def test_channel_disc_matches_python_rasteriser():
    xml = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    fl = case_geometry(xml, "d2q9")
    assert fl.shape == (1, 64, 256)  # nx padded 250 -> 256 (src/Solver.cpp.Rt:273)
    ref = cases.channel_disc_d2q9(256, 64, r=8, cx=64, cy=32)
    assert np.array_equal(fl, ref)


def test_tunnel_text_and_modes_d3q19(tmp_path):
    m = M.get("d3q19")
    rng = np.random.default_rng(0)
    pts = (rng.random((4, 8, 6)) < 0.3).astype(int)  # x outer, y, z inner
    f = tmp_path / "solid.txt"
    f.write_text(" ".join(str(v) for v in pts.ravel()))
    xml = f"""<CLBConfig><Geometry nx="32" ny="12" nz="10">
      <MRT><Box/></MRT>
      <Wall mask="ALL"><Tunnel/></Wall>
      <Solid mode="fill"><Text file="{f}" dx="4" nx="4" dy="2" ny="8" dz="2" nz="6"/></Solid>
      <WVelocity name="in" mode="change"><Box nx="1"/></WVelocity>
    </Geometry></CLBConfig>"""
    fl = case_geometry(xml, "d3q19")
    g = cases.Geometry("d3q19", 32, 12, 10)
    g.set_flag("MRT").box()
    g.set_flag("Wall", mask="ALL").tunnel()
    g.set_flag("Solid", mode="fill")
    sel = np.zeros((10, 12, 32), bool)
    for x in range(4):
        for y in range(8):
            for z in range(6):
                if pts[x, y, z]:
                    sel[2 + z, 2 + y, 4 + x] = True
    cur = g.geom[sel]
    keep = (cur & g.mask) != 0
    cur[~keep] = (cur[~keep] & (~g.mask & 0xFFFF)) | g.fg
    g.geom[sel] = cur
    g.set_flag("WVelocity", zone="in", mode="change").box(nx=1)
    assert np.array_equal(fl, g.geom)
    assert (fl[:, :, 0] >> m.zone_shift).max() == 1


def test_wedge_and_units():
    xml = """<CLBConfig><Geometry nx="32" ny="8">
      <Wall><Wedge dx="2" nx="5" dy="1" ny="5" direction="LowerRight"/></Wall>
      <Solid><Box dx="20mm" nx="1m" dy="0" ny="1"/></Solid>
    </Geometry></CLBConfig>"""
    fl = case_geometry(xml, "d2q9")
    wall = M.get("d2q9").flag("Wall")
    got = {(x, y) for y in range(8) for x in range(32) if fl[0, y, x] == wall}
    # inWedge LowerRight: (1-x) - (1-y) < 1e-10 on the 5x5 box at (2,1)
    want = {(2 + i, 1 + j) for i in range(5) for j in range(5) if (1 - i / 4) - (1 - j / 4) < 1e-10}
    assert got == want
    assert fl[0, 0, 0] == M.get("d2q9").flag("Solid")  # 20mm -> 0.02 -> column 0, 1m -> nx=1


def test_pipes():
    """<Pipe>, <PipeY>, <PipeZ>: every node of the box (grown by one layer across
    the axis, clipped to the lattice) outside the inscribed circle of the cross
    section, (2u-1)^2 + (2v-1)^2 >= 1 with u, v the node centres over the box."""
    wall = M.get("d3q19").flag("Wall")
    box = dict(dx=3, nx=10, dy=2, ny=8, dz=1, nz=6)
    for name, axis in (("Pipe", 0), ("PipeY", 1), ("PipeZ", 2)):
        attrs = " ".join(f'{k}="{v}"' for k, v in box.items())
        fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="12" nz="10"><Wall><{name} {attrs}/></Wall>'
                           '</Geometry></CLBConfig>', "d3q19")
        want = np.zeros_like(fl)
        d = (box["dx"], box["dy"], box["dz"])
        n = (box["nx"], box["ny"], box["nz"])
        for z in range(10):
            for y in range(12):
                for x in range(32):
                    c = (x, y, z)
                    grow = [0 if a == axis else 1 for a in range(3)]
                    if not all(d[a] - grow[a] <= c[a] < d[a] + n[a] + grow[a] for a in range(3)):
                        continue
                    u = [(0.5 + c[a] - d[a]) / n[a] for a in range(3) if a != axis]
                    if (2 * u[0] - 1) ** 2 + (2 * u[1] - 1) ** 2 >= 1:
                        want[z, y, x] = wall
        assert np.array_equal(fl, want), name
        assert (fl != 0).any() and (fl == 0).any(), name


def test_offgrid_pipes():
    """<OffgridPipe>/<ZPipe> (axis z), <XPipe>, <YPipe> and <XAnnulus>: nodes whose
    centres lie inside the ellipse about the off-grid centre, over a box of the
    radii + 5 nodes across the axis. YPipe and ZPipe take the x offset from y
    (TCLB's .5 + x - y0), so their x centre is y."""
    wall = M.get("d3q19").flag("Wall")
    X, Y, Z = 64, 24, 20  # nx a multiple of 32 (no padding)

    def want(axis, c, R, Ri=None, ca=None):
        a, b = [k for k in range(3) if k != axis]
        out = np.zeros((Z, Y, X), np.uint16)
        lo = [int(c[k] - R[k] - 5) if k != axis else 0 for k in range(3)]
        hi = [lo[k] + int(2 * R[k] + 10) if k != axis else (X, Y, Z)[k] for k in range(3)]
        ca = c[a] if ca is None else ca
        for z in range(max(lo[2], 0), min(hi[2], Z)):
            for y in range(max(lo[1], 0), min(hi[1], Y)):
                for x in range(max(lo[0], 0), min(hi[0], X)):
                    p = (x, y, z)
                    pa, pb = 0.5 + p[a] - ca, 0.5 + p[b] - c[b]
                    inside = pa * pa / R[a] ** 2 + pb * pb / R[b] ** 2 < 1
                    if Ri is not None:
                        inside = inside and pa * pa / Ri[a] ** 2 + pb * pb / Ri[b] ** 2 > 1
                    if inside:
                        out[z, y, x] = wall
        return out

    c = (17.3, 9.6, 8.2)
    shapes = [
        ('<OffgridPipe x="17.3" y="9.6" z="8.2" Rx="6.5" Ry="4.2"/>', want(2, c, (6.5, 4.2, 0))),
        ('<ZPipe x="17.3" y="9.6" z="8.2" R="5.5"/>', want(2, c, (5.5, 5.5, 0), ca=9.6)),
        ('<XPipe x="17.3" y="9.6" z="8.2" Ry="6.1" Rz="3.7"/>', want(0, c, (0, 6.1, 3.7))),
        ('<YPipe x="17.3" y="9.6" z="8.2" Rx="4.4" Rz="5.2"/>', want(1, c, (4.4, 0, 5.2), ca=9.6)),
        ('<XAnnulus x="17.3" y="9.6" z="8.2" Ro="7.5" Ri="4"/>', want(0, c, (0, 7.5, 7.5), Ri=(0, 4, 4))),
    ]
    for elem, ref in shapes:
        fl = case_geometry(f'<CLBConfig><Geometry nx="{X}" ny="{Y}" nz="{Z}"><Wall>{elem}</Wall></Geometry></CLBConfig>',
                           "d3q19")
        assert fl.shape == ref.shape and np.array_equal(fl, ref), elem
        assert (fl != 0).any(), elem


def write_stl_box(path, lo, hi, header=b"box"):
    """A closed axis-aligned box as 12 triangles of a binary STL file."""
    corners = np.array([[(lo, hi)[(i >> k) & 1][k] for k in range(3)] for i in range(8)], np.float32)
    quads = [(0, 2, 6, 4), (1, 3, 7, 5), (0, 1, 5, 4), (2, 3, 7, 6), (0, 1, 3, 2), (4, 5, 7, 6)]
    rec = np.zeros(12, dtype=[("n", "<f4", 3), ("p", "<f4", (3, 3)), ("a", "<u2")])
    for i, (a, b, c, d) in enumerate(quads):
        rec["p"][2 * i] = corners[[a, b, c]]
        rec["p"][2 * i + 1] = corners[[a, c, d]]
    with open(path, "wb") as f:
        f.write(header.ljust(80, b" "))
        f.write(np.uint32(12).tobytes())
        f.write(rec.tobytes())


STL_SHIFT = np.array([0.1403e-4, 0.1687e-4, 0.1987e-4]) - 0.5  # node i sits at STL coordinate i + 0.5


def stl_inside(shape, lo, hi):
    """Nodes strictly inside the box [lo, hi] given in STL coordinates."""
    z, y, x = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    lo, hi = np.asarray(lo) + STL_SHIFT, np.asarray(hi) + STL_SHIFT
    return ((x > lo[0]) & (x < hi[0]) & (y > lo[1]) & (y < hi[1]) & (z > lo[2]) & (z < hi[2]))


def test_stl_inside_outside(tmp_path):
    """<STL> side in / out by ray parity along each ray axis, and the rotate /
    move transform: the nodes of an STL box, and of the same box turned by
    90 degrees about z and moved in x."""
    wall = M.get("d3q19").flag("Wall")
    lo, hi = (3.3, 2.45, 1.65), (11.8, 9.6, 7.15)
    f = tmp_path / "box.stl"
    write_stl_box(f, lo, hi)
    shape = (12, 16, 32)
    inside = stl_inside(shape, lo, hi)
    assert inside.sum() == 9 * 8 * 5
    for extra in ('', ' ray_axis="x"', ' ray_axis="z"'):
        fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="16" nz="12"><Wall><STL file="{f}"{extra}/></Wall>'
                           '</Geometry></CLBConfig>', "d3q19")
        assert np.array_equal(fl == wall, inside), extra
    fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="16" nz="12"><Wall><STL file="{f}" side="out"/></Wall>'
                       '</Geometry></CLBConfig>', "d3q19")
    assert np.array_equal(fl == wall, ~inside)
    # Zrot turns (x, y) into (-y, x); then x moves by 20
    fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="16" nz="12"><Wall><STL file="{f}" Zrot="1.5707963267948966" '
                       'x="20"/></Wall></Geometry></CLBConfig>', "d3q19")
    turned = stl_inside(shape, (20 - hi[1], lo[0], lo[2]), (20 - lo[1], hi[0], hi[2]))
    assert turned.sum() == 8 * 9 * 5
    assert np.array_equal(fl == wall, turned)


def test_stl_surface(tmp_path):
    """<STL side="surface">: the nodes whose link to one of the 26 neighbours
    crosses the surface of the box (a segment-box slab test)."""
    wall = M.get("d3q19").flag("Wall")
    lo, hi = (3.3, 2.45, 1.65), (11.8, 9.6, 7.15)
    f = tmp_path / "box.stl"
    write_stl_box(f, lo, hi)
    fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="16" nz="12"><Wall><STL file="{f}" side="surface"/></Wall>'
                       '</Geometry></CLBConfig>', "d3q19")
    blo, bhi = np.asarray(lo) + STL_SHIFT, np.asarray(hi) + STL_SHIFT
    want = np.zeros((12, 16, 32), bool)
    dirs = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dx or dy or dz]
    for z in range(12):
        for y in range(16):
            for x in range(32):
                X = np.array([x, y, z], float)
                inside0 = np.all((X > blo) & (X < bhi))
                for d in dirs:
                    d = np.array(d, float)
                    r0, r1 = 0.0, 1.0
                    for k in range(3):
                        if d[k] == 0:
                            if not blo[k] <= X[k] <= bhi[k]:
                                r0, r1 = 1.0, 0.0
                        else:
                            a, b = sorted(((blo[k] - X[k]) / d[k], (bhi[k] - X[k]) / d[k]))
                            r0, r1 = max(r0, a), min(r1, b)
                    if r0 <= r1 and not (inside0 and np.all((X + d > blo) & (X + d < bhi))):
                        want[z, y, x] = True
                        break
    assert want.sum() > 0
    assert np.array_equal(fl == wall, want)


def test_stl_errors(tmp_path):
    """An ASCII STL file and a bad side are errors with a message."""
    lib = load_library()
    lib.tclb_case_last_error.restype = ctypes.c_char_p
    f = tmp_path / "ascii.stl"
    write_stl_box(f, (1, 1, 1), (2, 2, 2), header=b"solid box")
    dims = (ctypes.c_int * 3)()
    out = np.zeros(32 * 8 * 8, np.uint16)
    for elem, msg in ((f'<STL file="{f}"/>', b"binary"), (f'<STL file="{f}" side="top"/>', b"side")):
        xml = f'<CLBConfig><Geometry nx="32" ny="8" nz="8"><Wall>{elem}</Wall></Geometry></CLBConfig>'
        rc = lib.tclb_case_geometry(xml.encode(), M.get("d3q19").mid, dims,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size)
        assert rc != 0 and msg in lib.tclb_case_last_error()


def test_sweep():
    """<Sweep>: balls of radius 2.5 moved along the straight segment from x = 5 to
    x = 25 at y = z = 8.5, as a linear B-spline of two points and as a quadratic
    one of three collinear points. The balls lie at most ~0.26 apart, so every
    node of the capsule around the segment is drawn and no other."""
    wall = M.get("d3q19").flag("Wall")
    z, y, x = np.meshgrid(np.arange(16), np.arange(16), np.arange(32), indexing="ij")
    nearest = np.clip(0.5 + x, 5, 25)
    want = (0.5 + x - nearest) ** 2 + (0.5 + y - 8.5) ** 2 + (0.5 + z - 8.5) ** 2 < 2.5 ** 2
    for points in (((5, 8.5, 8.5), (25, 8.5, 8.5)), ((5, 8.5, 8.5), (12, 8.5, 8.5), (25, 8.5, 8.5))):
        pts = "".join(f'<Point x="{a}" y="{b}" z="{c}"/>' for a, b, c in points)
        fl = case_geometry(f'<CLBConfig><Geometry nx="32" ny="16" nz="16"><Wall><Sweep order="{len(points) - 1}" '
                           f'r="2.5" step="0.001">{pts}</Sweep></Wall></Geometry></CLBConfig>', "d3q19")
        assert np.array_equal(fl == wall, want), len(points)


def test_zone_attribute_draws_the_zone():
    """A flag element's zone= attribute draws that <Zone> (here one of the case's
    own, and the default Inlet) before the element's own children."""
    wall = M.get("d2q9").flag("Wall")
    fl = case_geometry("""<CLBConfig><Geometry nx="32" ny="8">
      <Zone name="blk"><Box dx="2" nx="3" dy="1" ny="2"/></Zone>
      <Wall zone="blk"><Box dx="10" nx="1" dy="5" ny="1"/></Wall>
      <Solid zone="Inlet"/>
    </Geometry></CLBConfig>""", "d2q9")
    want = np.zeros((1, 8, 32), np.uint16)
    want[0, 1:3, 2:5] = wall
    want[0, 5, 10] = wall
    want[0, :, 0] = M.get("d2q9").flag("Solid")  # the default Inlet zone: the x = 0 column
    assert np.array_equal(fl, want)


def test_bad_case_is_an_error_not_an_exit():
    lib = load_library()
    lib.tclb_case_last_error.restype = ctypes.c_char_p
    dims = (ctypes.c_int * 3)()
    rc = lib.tclb_case_geometry(b"<CLBConfig><Geometry nx='8' ny='8'><Wal><Box/></Wal></Geometry></CLBConfig>",
                                0, dims, None, 0)
    assert rc == 0  # size query does not rasterise
    out = np.zeros(8 * 32, np.uint16)
    rc = lib.tclb_case_geometry(b"<CLBConfig><Geometry nx='8' ny='8'><Wal><Box/></Wal></Geometry></CLBConfig>",
                                0, dims, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size)
    assert rc != 0 and b"Wal" in lib.tclb_case_last_error()
    rc = lib.tclb_case_geometry(b"<CLBConfig><Geometry nx='8'>", 0, dims, None, 0)
    assert rc != 0 and b"XML" in lib.tclb_case_last_error()


def test_units_gauges_scale_the_geometry():
    """<Units> gauges (1 mm = 1 lattice length, 1e-6 m2/s = 0.02) make the
    SI version of the channel case rasterise exactly like the lattice one."""
    plain = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    si = open(os.path.join(HERE, "cases", "channel_disc_si.xml")).read()
    a, b = case_geometry(plain, "d2q9"), case_geometry(si, "d2q9")
    assert a.shape == b.shape and np.array_equal(a, b)


def test_units_errors():
    """Gauges that fix one base unit twice, and unknown unit symbols, are errors
    (status codes with a message), not silent zeros."""
    lib = load_library()
    dims = (ctypes.c_int * 3)()
    over = (b"<CLBConfig><Units><Param value='1m' gauge='10'/><Param value='2m' gauge='5'/></Units>"
            b"<Geometry nx='8' ny='8'/></CLBConfig>")
    assert lib.tclb_case_geometry(over, 0, dims, None, 0) != 0
    assert b"over-determine" in lib.tclb_case_last_error()
    unknown = b"<CLBConfig><Geometry nx='8qq' ny='8'/></CLBConfig>"
    assert lib.tclb_case_geometry(unknown, 0, dims, None, 0) != 0
    assert b"unknown unit" in lib.tclb_case_last_error()
    ok = b"<CLBConfig><Units><Param value='1cm' gauge='4'/></Units><Geometry nx='8cm' ny='2cm+1mm'/></CLBConfig>"
    assert lib.tclb_case_geometry(ok, 0, dims, None, 0) == 0
    assert list(dims) == [32, 8, 1]  # nx 32 (already a multiple of 32), ny round(8.4)


@pytest.mark.gpu
def test_case_file_run_with_units(tmp_path):
    """The SI version of the channel case through tclb_run: the same lattice
    values as the plain case (Log value columns), SI columns scaled by the
    gauges (1 s = 50 iterations, 1 mm = 1), Time_si the iteration in seconds."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    res = {}
    for name in ("channel_disc", "channel_disc_si"):
        out = str(tmp_path / name) + "/"
        r = subprocess.run([runner, "d2q9", os.path.join(HERE, "cases", name + ".xml"), "--output", out, "--quiet"],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        rows = open(glob.glob(out + name + "_Log_P00_00000000.csv")[0]).read().strip().splitlines()
        hdr = [h.strip('"') for h in rows[0].split(",")]
        res[name] = (hdr, np.array([[float(v) for v in row.split(",")] for row in rows[1:]]))
    (hp, dp), (hs, ds) = res["channel_disc"], res["channel_disc_si"]
    assert hp == hs and list(ds[:, 0]) == [50, 100, 150, 200]
    for col in ("Viscosity", "VelocityX-Inlet", "PressureLoss", "OutletFlux", "InletFlux"):
        i = hp.index(col)
        assert ds[:, i] == pytest.approx(dp[:, i], rel=1e-5, abs=1e-12), col
    assert ds[:, hs.index("Time_si")] == pytest.approx(ds[:, 0] / 50)
    assert ds[-1, hs.index("dx_si")] == pytest.approx(1e-3) and ds[-1, hs.index("dt_si")] == pytest.approx(0.02)
    assert ds[-1, hs.index("dm_si")] == pytest.approx(1.0)
    # PressureLoss is in mPa = kg/s2: one lattice unit of it is 1 / 50^2 of one, so SI = lattice * 2500
    i = hs.index("PressureLoss")
    assert ds[:, i + 1] == pytest.approx(ds[:, i] * 2500, rel=1e-9)
    # the plain case has no gauges: SI columns equal the lattice ones
    assert dp[:, i + 1] == pytest.approx(dp[:, i], rel=1e-12)


@pytest.mark.gpu
def test_stop_ends_the_solve(tmp_path):
    """<Stop> (cbStop): every criterion holding on Times consecutive checks
    ends the enclosing <Solve>; a Change criterion's first check never holds;
    a Stop without criteria is an error."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    plain = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    head = plain[:plain.index("<Log")]

    def run(solve):
        path = tmp_path / "case.xml"
        path.write_text(head + '<Log Iterations="50"/>' + solve + "</CLBConfig>")
        out = str(tmp_path / "out") + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        if r.returncode != 0:
            return None, r.stderr + r.stdout
        rows = open(out + "case_Log_P00_00000000.csv").read().strip().splitlines()[1:]
        return [int(row.split(",")[0]) for row in rows], ""

    its, err = run('<Solve Iterations="100000"><Stop InletFluxAbove="-1e30" Times="2" Iterations="50"/></Solve>')
    assert its == [50, 100], err
    its, err = run('<Solve Iterations="300"><Stop PressureLossChange="0" Iterations="50"/></Solve>')
    assert its == [50, 100, 150, 200, 250, 300], err
    its, err = run('<Solve Iterations="300"><Stop Times="2" Iterations="50"/></Solve>')
    assert its is None and "Stop" in err


def read_vti(path):
    """Cell arrays of a VTK XML ImageData file with inline base64 arrays (a
    4-byte length block, then the data block) -> {name: array}, spacing."""
    import base64
    import xml.etree.ElementTree as ET

    root = ET.parse(path).getroot()
    img = root.find("ImageData")
    spacing = [float(v) for v in img.get("Spacing").split()]
    types = {"Float32": np.float32, "Float64": np.float64, "UInt8": np.uint8, "UInt16": np.uint16}
    out = {}
    for da in img.iter("DataArray"):
        text = da.text.strip()
        n = np.frombuffer(base64.b64decode(text[:8]), np.int32)[0]
        data = np.frombuffer(base64.b64decode(text[8:]), types[da.get("type")])
        assert data.nbytes == n
        out[da.get("Name")] = data.reshape(-1, int(da.get("NumberOfComponents")))
    return out, spacing


@pytest.mark.gpu
def test_vtk_output(tmp_path):
    """<VTK> writes the quantities in SI units, the node-type groups and,
    when named, the raw node types; with no gauges SI is the lattice value."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    got = {}
    for name in ("channel_disc", "channel_disc_si"):
        text = open(os.path.join(HERE, "cases", name + ".xml")).read()
        text = text.replace("<BIN ", '<VTK Iterations="%s"/><VTK name="part" what="U,BOUNDARY,flag" dx="10" nx="20" '
                                     'Iterations="%s"/><BIN ' % (("200", "200") if name == "channel_disc" else ("4s", "4s")))
        path = tmp_path / (name + ".xml")
        path.write_text(text)
        out = str(tmp_path / name) + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert os.path.exists(out + name + "_VTK_P00_00000200.pvti")
        got[name] = (read_vti(out + name + "_VTK_P00_00000200.vti"), read_vti(out + name + "_part_P00_00000200.vti"),
                     np.fromfile(out + name + "_BIN_P00_00000200.U.bin", np.float32).reshape(-1, 3))
    (full, sp), (part, _), u_bin = got["channel_disc"]
    assert sp == [1.0, 1.0, 1.0]
    assert set(full) == {"BOUNDARY", "COLLISION", "OBJECTIVE", "SETTINGZONE", "Rho", "U"}
    assert np.array_equal(full["U"], u_bin)
    fl = case_geometry(open(os.path.join(HERE, "cases", "channel_disc.xml")).read(), "d2q9")
    assert np.array_equal(full["BOUNDARY"][:, 0], (fl & 0xF).ravel())
    assert set(part) == {"U", "BOUNDARY", "flag"}
    nz, ny, nx = fl.shape
    assert np.array_equal(part["flag"][:, 0], fl[:, :, 10:30].ravel())
    assert np.array_equal(part["U"], u_bin.reshape(ny, nx, 3)[:, 10:30].reshape(-1, 3))
    (full_si, sp_si), _, u_bin_si = got["channel_disc_si"]
    assert sp_si == pytest.approx([1e-3] * 3)
    # 1 lattice velocity = 1 mm per 1/50 s = 0.05 m/s
    assert full_si["U"][:, 0] == pytest.approx(u_bin_si[:, 0] * 0.05, rel=1e-5, abs=1e-12)


@pytest.mark.gpu
def test_sample_output(tmp_path):
    """<Sample>: after every iteration the chosen quantities at the <Point> nodes;
    each Iterations period appends its rows to <case>_Sampler_P00_<it>.csv. The
    row labelled 199 holds the state after the 200th iteration, the one the BIN
    files hold."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    text = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    text = text.replace("<BIN ", '<Sample Iterations="50" what="Rho,U"><Point dx="100" dy="32"/>'
                                 '<Point dx="30" dy="10"/><Point dx="900" dy="1"/></Sample><BIN ')
    path = tmp_path / "case.xml"
    path.write_text(text)
    out = str(tmp_path / "out") + "/"
    r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = open(out + "case_Sampler_P00_00000000.csv").read().strip().splitlines()
    assert lines[0] == "Iteration,X,Y,Z,Rho,U.x,U.y,U.z"
    rows = np.array([[float(v) for v in line.split(",")] for line in lines[1:]])
    assert rows.shape == (200 * 2, 8)  # the point outside the lattice is dropped
    assert np.array_equal(rows[::2, 0], np.arange(200)) and np.array_equal(rows[1::2, 0], np.arange(200))
    assert np.all(rows[::2, 1:4] == [100, 32, 0]) and np.all(rows[1::2, 1:4] == [30, 10, 0])
    rho = np.fromfile(out + "case_BIN_P00_00000200.Rho.bin", np.float32).reshape(64, 256)
    u = np.fromfile(out + "case_BIN_P00_00000200.U.bin", np.float32).reshape(64, 256, 3)
    for row, (x, y) in ((rows[-2], (100, 32)), (rows[-1], (30, 10))):
        assert np.allclose(row[4], rho[y, x], rtol=1e-5, atol=0)
        assert np.allclose(row[5:8], u[y, x], rtol=1e-5, atol=1e-12)
    assert abs(rows[-2, 5] - rows[0, 5]) > 0  # the flow develops


@pytest.mark.gpu
def test_repeat_and_container(tmp_path):
    """<Repeat Times> runs its children that many times; <Container> runs its
    children and then drops the callbacks they registered; <EvalIf> runs its
    children when a model option is present (opt_present) or absent
    (opt_missing), and the plain d2q9 has autosym off. Four 50-iteration Solves
    in a Repeat and one more in the opt_missing branch reach the state of one
    250-iteration Solve bit for bit; the Log inside the Container stops with it."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    base = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    start = base.index("<Log ")
    end = base.index("</CLBConfig>")
    plain = base[:start] + '<Solve Iterations="250"/><BIN/>' + base[end:]
    nested = (base[:start] + '<Container><Log Iterations="50"/><Repeat Times="4"><Solve Iterations="50"/>'
              '</Repeat></Container><EvalIf opt_present="autosym"><Solve Iterations="1000"/></EvalIf>'
              '<EvalIf opt_missing="autosym"><Solve Iterations="50"/></EvalIf><BIN/>' + base[end:])
    outs = []
    for name, text in (("plain", plain), ("nested", nested)):
        path = tmp_path / f"{name}.xml"
        path.write_text(text)
        out = str(tmp_path / name) + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        outs.append(out)
    for q in ("Rho", "U"):
        a = open(outs[0] + f"plain_BIN_P00_00000250.{q}.bin", "rb").read()
        b = open(outs[1] + f"nested_BIN_P00_00000250.{q}.bin", "rb").read()
        assert a == b, q
    log = open(outs[1] + "nested_Log_P00_00000000.csv").read().strip().splitlines()
    assert [int(float(line.split(",")[0])) for line in log[1:]] == [50, 100, 150, 200]


@pytest.mark.gpu
def test_pid_control(tmp_path):
    """<PID>: every 10 iterations the inlet velocity becomes
    base + scale * (e + integral / IntegrationTime + de/dt * DerivativeTime),
    e = target - InletFlux, the integral by the trapezoid rule. The Log (checked
    first, at the same iterations) holds each InletFlux and the velocity set at
    the check before, so the whole control sequence is replayed from it."""
    import csv
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    text = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    start, end = text.index("<Log "), text.index("</CLBConfig>")
    text = (text[:start] + '<Solve Iterations="200"><Log Iterations="10"/><PID Iterations="10" integral="InletFlux" '
            'target="1.0" control="VelocityX" zone="Inlet" IntegrationTime="200" DerivativeTime="2" '
            'scale="2e-4"/></Solve>' + text[end:])
    path = tmp_path / "case.xml"
    path.write_text(text)
    out = str(tmp_path / "out") + "/"
    r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with open(out + "case_Log_P00_00000000.csv") as f:
        rows = list(csv.reader(f, skipinitialspace=True))
    head = rows[0]
    flux = np.array([float(r_[head.index("InletFlux")]) for r_ in rows[1:]])
    vel = np.array([float(r_[head.index("VelocityX-Inlet")]) for r_ in rows[1:]])
    assert len(flux) == 20 and vel[0] == 0.01
    integral, old = 0.0, 0.0
    for k in range(19):
        err = 1.0 - flux[k]
        integral += (old + err) * 10 / 2
        control = err + integral / 200 + (err - old) / 10 * 2
        old = err
        assert vel[k + 1] == pytest.approx(0.01 + control * 2e-4, rel=1e-9, abs=1e-15), k
    assert vel[-1] != vel[0]


@pytest.mark.gpu
def test_keep(tmp_path):
    """<Keep What="InletFlux" Above=...>: at each check InletFluxInObj becomes
    (threshold - InletFlux) * Force in every zone when that is positive, else 0;
    the Log (checked first) shows the value set at the check before."""
    import csv
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    text = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    start, end = text.index("<Log "), text.index("</CLBConfig>")
    outs = {}
    for kind, thr in (("Above", "0.7"), ("Below", "0.7"), ("Equal", "0.5")):
        case = (text[:start] + f'<Solve Iterations="100"><Log Iterations="10"/><Keep Iterations="10" What="InletFlux" '
                f'{kind}="{thr}" Force="3"/></Solve>' + text[end:])
        path = tmp_path / f"{kind}.xml"
        path.write_text(case)
        out = str(tmp_path / kind) + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        with open(out + f"{kind}_Log_P00_00000000.csv") as f:
            rows = list(csv.reader(f, skipinitialspace=True))
        head = rows[0]
        flux = np.array([float(r_[head.index("InletFlux")]) for r_ in rows[1:]])
        for zone in ("Inlet", "Outlet"):
            w = np.array([float(r_[head.index(f"InletFluxInObj-{zone}")]) for r_ in rows[1:]])
            v = (float(thr) - flux[:-1]) * 3
            want = {"Above": np.where(v > 0, v, 0), "Below": np.where(v < 0, v, 0), "Equal": v}[kind]
            assert np.allclose(w[1:], want, rtol=1e-12, atol=1e-15), (kind, zone)
        outs[kind] = flux
    assert (outs["Equal"] != 0).all()


@pytest.mark.gpu
def test_param_inside_solve(tmp_path):
    """A <Param> among a <Solve>'s children takes effect when the Solve starts
    (acSolve runs its children like any container): the same state as the Param
    placed just before the Solve."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    base = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    start, end = base.index("<Log "), base.index("</CLBConfig>")
    param = '<Param name="VelocityX" value="0.02" zone="Inlet"/>'
    texts = {"before": base[:start] + param + '<Solve Iterations="100"><BIN Iterations="100"/></Solve>' + base[end:],
             "inside": base[:start] + '<Solve Iterations="100">' + param + '<BIN Iterations="100"/></Solve>' + base[end:],
             "none": base[:start] + '<Solve Iterations="100"><BIN Iterations="100"/></Solve>' + base[end:]}
    u = {}
    for name, text in texts.items():
        path = tmp_path / f"{name}.xml"
        path.write_text(text)
        out = str(tmp_path / name) + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        u[name] = open(out + f"{name}_BIN_P00_00000100.U.bin", "rb").read()
    assert u["inside"] == u["before"] and u["inside"] != u["none"]


@pytest.mark.gpu
def test_failcheck_stops_and_runs_final_actions(tmp_path):
    """<Failcheck> over the whole lattice (nx, ny given, as TCLB's examples do):
    a negative viscosity makes the run overflow to NaN (plain IEEE arithmetic);
    the check stops the Solve at its first failing call and runs its child
    <VTK> there first. A child with its own Iterations= is not registered as a
    periodic callback: it runs once, at the failing check, as TCLB's
    Handler::DoIt runs each child once. A Failcheck with a what= list naming no
    quantity checks nothing and never stops the run."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    base = open(os.path.join(HERE, "cases", "channel_disc.xml")).read().replace(
        '<Param name="Viscosity" value="0.02"/>', '<Param name="Viscosity" value="-0.2"/>')
    start, end = base.index("<Log "), base.index("</CLBConfig>")
    for name, fc, stops in (("whole", '<Failcheck Iterations="10" nx="256" ny="64"><VTK what="Rho"/></Failcheck>', True),
                            ("child_iters", '<Failcheck Iterations="10" nx="256" ny="64"><VTK Iterations="5" '
                                            'what="Rho"/></Failcheck>', True),
                            ("none", '<Failcheck Iterations="10" nx="256" ny="64" what="NoSuch"/>', False)):
        text = base[:start] + f'<Solve Iterations="300">{fc}<BIN Iterations="300"/></Solve>' + base[end:]
        path = tmp_path / f"{name}.xml"
        path.write_text(text)
        out = str(tmp_path / name) + "/"
        r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        files = os.listdir(out)
        bins = [f for f in files if "_BIN_" in f]
        vtis = [f for f in files if f.endswith(".vti")]
        if stops:
            assert not bins and len(vtis) == 1, files
            it = int(vtis[0].split("_P00_")[1][:8])
            assert it % 10 == 0 and 0 < it < 300
            rho = read_vti(out + vtis[0])[0]["Rho"]
            assert np.isnan(rho).any()
        else:
            assert bins and not vtis, files


@pytest.mark.gpu
def test_txt_output(tmp_path):
    """<TXT>: the info file and one text file per quantity (SI units; rows of
    nx nodes; vectors x y z per node), the same values as the BIN files."""
    import subprocess

    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    text = open(os.path.join(HERE, "cases", "channel_disc.xml")).read()
    text = text.replace("<BIN ", '<TXT Iterations="200"/><TXT Iterations="200" name="Z" what="Rho" gzip="true"/><BIN ')
    path = tmp_path / "case.xml"
    path.write_text(text)
    out = str(tmp_path / "out") + "/"
    r = subprocess.run([runner, "d2q9", str(path), "--output", out, "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    base = out + "case_TXT_P00_00000200"
    info = dict(line.split(": ") for line in open(base + "_info.txt").read().strip().splitlines())
    assert info["NX"] == "256" and info["NY"] == "64" and info["NZ"] == "1" and float(info["dx"]) == 1.0
    rho = np.loadtxt(base + "_Rho.txt")
    assert rho.shape == (64, 256)
    rho_bin = np.fromfile(out + "case_BIN_P00_00000200.Rho.bin", np.float32).reshape(64, 256)
    assert np.allclose(rho, rho_bin, rtol=1e-7, atol=0)
    u = np.loadtxt(base + "_U.txt")
    assert u.shape == (64, 256 * 3)
    u_bin = np.fromfile(out + "case_BIN_P00_00000200.U.bin", np.float32).reshape(64, 256 * 3)
    assert np.allclose(u, u_bin, rtol=1e-7, atol=1e-30)
    import gzip
    zbase = out + "case_Z_P00_00000200"
    with gzip.open(zbase + "_Rho.txt.gz", "rt") as f:
        assert np.array_equal(np.loadtxt(f), rho)
    assert not os.path.exists(zbase + "_U.txt.gz")


@pytest.mark.gpu
def test_case_file_run_matches_api(tmp_path):
    """tclb_run on the channel case: the Log CSV rows and the final BIN files
    equal what the Python API produces for the same flags and settings."""
    import subprocess

    from tclb_b200.lattice import Lattice

    xml = os.path.join(HERE, "cases", "channel_disc.xml")
    runner = os.path.join(os.path.dirname(HERE), "tclb_b200", "tclb_run")
    out = str(tmp_path) + "/"
    r = subprocess.run([runner, "d2q9", xml, "--output", out, "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    logs = glob.glob(out + "channel_disc_Log_P00_00000000.csv")
    assert logs, os.listdir(out)
    rows = open(logs[0]).read().strip().splitlines()
    hdr = [h.strip('"') for h in rows[0].split(",")]
    data = np.array([[float(v) for v in r.split(",")] for r in rows[1:]])
    assert list(data[:, 0]) == [50, 100, 150, 200]
    # the same through the API
    m = M.get("d2q9")
    lat = Lattice("d2q9", 256, 64)
    lat.set_flags(cases.channel_disc_d2q9(256, 64, r=8, cx=64, cy=32))
    lat.set_zone_setting("VelocityX", 0.01)
    lat.SetSetting("Viscosity", 0.02)
    lat.SetSetting("S3", -0.7857142857142858)
    lat.SetSetting("S4", -0.7857142857142858)
    lat.Init()
    for k in range(4):
        lat.Iterate(50, M.ITER_NORM | M.ITER_LASTGLOB)
        g = lat.globals
        for gi, (gname, _op) in enumerate(m.globals):
            assert data[k, hdr.index(gname)] == pytest.approx(g[gi], rel=1e-6, abs=1e-12)
    assert data[-1, hdr.index("S2")] == pytest.approx(1 - 1 / (3 * 0.02 + 0.5))
    assert data[-1, hdr.index("VelocityX-Inlet")] == pytest.approx(0.01)
    u = np.fromfile(out + "channel_disc_BIN_P00_00000200.U.bin", dtype=np.float32).reshape(1, 64, 256, 3)
    assert np.array_equal(u, lat.GetQuantity("U"))
    rho = np.fromfile(out + "channel_disc_BIN_P00_00000200.Rho.bin", dtype=np.float32)
    assert rho.size == 64 * 256
    lat.close()
