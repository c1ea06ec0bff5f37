"""The failure path of the tile-staged kernel, exercised without faulting anything.

tclb_set_fault_injection makes the producer warp arm one tile's stage without
issuing its copies, and bounds every staging wait by 2,000,000 SM clock cycles
(about 1 ms). The consumers of that tile give up, record the device error word
and return; the producer, whose next wait on the stage runs out as well,
drains (bounded) the copies it issued and returns. Every other block finishes
normally. The test checks that:

* tclb_sync reports TCLB_ERR_CUDA with the tile-pipeline message;
* the error word is cleared (the next sync is clean);
* with injection off and the state restored, the next clean iterations match
  the register pair kernel bit for bit.
"""
import numpy as np
import pytest

from tclb_b200 import cases
from tclb_b200 import models as M
from tclb_b200.lattice import Lattice, TCLBError

pytestmark = pytest.mark.gpu

SHAPE = (64, 64, 256)  # nz, ny, nx: 2-row tiles, 2048 tiles, several per block of the persistent grid


def _lattice(tma: bool):
    nz, ny, nx = SHAPE
    g = Lattice("d3q19", nx, ny, nz, precision="fp32", storage="fp16s")
    if not tma:
        g.set_launch(128, 2, use_graphs=True, use_pairs=True, use_tma=False)
    g.set_flags(cases.porous_channel_d3q19(nx, ny, nz, p=0.08, band=4, seed=5))
    g.SetSetting("nu", 0.02)
    g.SetSetting("ForceX", 1e-5)
    g.Init()
    return g


def test_staging_wait_runs_out_and_reports():
    g = _lattice(tma=True)
    assert g.launch_path()["tma"]
    g.Iterate(3)
    g.sync()
    snap = g.save()
    g.set_fault_injection(tile=700, wait_cycles=2_000_000)
    g.Iterate(1)
    with pytest.raises(TCLBError, match="tile pipeline"):
        g.sync()
    g.sync()  # the error word was cleared
    g.set_fault_injection(-1, 0)
    g.load(snap)
    g.Iterate(2)
    g.sync()
    p = _lattice(tma=False)
    assert not p.launch_path()["tma"] and p.launch_path()["pairs"]
    p.load(snap)
    p.Iterate(2)
    assert np.array_equal(g.densities(), p.densities())
    g.close()
    p.close()


def test_fault_injection_arguments():
    g = _lattice(tma=True)
    with pytest.raises(TCLBError):
        g.set_fault_injection(tile=-2)
    with pytest.raises(TCLBError):
        g.set_fault_injection(tile=0, wait_cycles=-1)
    g.set_fault_injection(-1, 0)
    g.Iterate(2)
    g.sync()
    g.close()
