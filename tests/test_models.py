"""Model tables: the packing/ordering rules of src/conf.R (restated in
tclb_b200/models.py) against the tables compiled into the CUDA library, the
oracle and the hand-derived values."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from tclb_b200 import models as M
from tclb_b200.lattice import load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def lib_items(lib, mid, kind, n):
    out = []
    for i in range(n):
        name = ctypes.c_char_p()
        v, m = ctypes.c_int(), ctypes.c_int()
        assert lib.tclb_model_item(mid, kind, i, ctypes.byref(name), ctypes.byref(v), ctypes.byref(m)) == 0
        out.append((name.value.decode(), v.value, m.value))
    return out


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_library_tables_match_rules(name):
    lib = load_library()
    m = M.get(name)
    Q, ns, nzs, ng, nq, zsh = (ctypes.c_int() for _ in range(6))
    assert lib.tclb_model_info(m.mid, *(ctypes.byref(x) for x in (Q, ns, nzs, ng, nq, zsh))) == 0
    assert Q.value == m.Q
    assert ns.value == len(m.settings)
    assert nzs.value == len(m.zone_settings)
    assert ng.value == len(m.globals)
    assert nq.value == len(m.quantities)
    assert zsh.value == m.zone_shift
    assert [x[0] for x in lib_items(lib, m.mid, 0, ns.value)] == [s.name for s in m.settings]
    assert [x[0] for x in lib_items(lib, m.mid, 1, nzs.value)] == [s.name for s in m.zone_settings]
    assert [x[0] for x in lib_items(lib, m.mid, 2, ng.value)] == [g[0] for g in m.globals]
    nts = {x[0]: (x[1], x[2]) for x in lib_items(lib, m.mid, 3, len(m.node_types))}
    assert nts == {k: (v[0], v[1]) for k, v in m.node_types.items()}
    assert [x[0] for x in lib_items(lib, m.mid, 4, nq.value)] == [q[0] for q in m.quantities]


def test_hand_derived_values():
    d2 = M.get("d2q9").node_types
    assert (d2["Wall"][0], d2["MRT"][0], d2["Inlet"][0], d2["Outlet"][0]) == (10, 0x10, 0x20, 0x40)
    assert M.get("d2q9").zone_shift == 7
    d19 = M.get("d3q19").node_types
    assert (d19["Wall"][0], d19["WVelocity"][0], d19["MRT"][0], d19["YZslice"][0]) == (0x0C, 0x18, 0x20, 3)
    assert M.get("d3q19").zone_shift == 6
    d27 = M.get("d3q27_cumulant").node_types
    assert (d27["Wall"][0], d27["Body"][0], d27["MRT"][0], d27["WVelocity"][0]) == (0x50, 4, 0x80, 0x60)
    assert M.get("d3q27_cumulant").zone_shift == 8
    assert [g[0] for g in M.get("d2q9").globals] == ["PressureLoss", "OutletFlux", "InletFlux", "Objective"]
    g19 = [g[0] for g in M.get("d3q19").globals]
    assert g19[0] == "Flux" and g19[-2:] == ["Objective", "MaxV"] and len(g19) == 26
    assert M.get("d2q9").in_obj_offset == 3 and M.get("d3q19").in_obj_offset == 0
    assert M.get("d3q27_cumulant").in_obj_offset == 3


@pytest.mark.parametrize("name", ["d2q9", "d3q19", "d3q27_cumulant"])
def test_oracle_node_types(name):
    for nt, (v, _m, _g) in M.get(name).node_types.items():
        assert oracle.node_type_value(name, nt) == v


def test_settings_defaults_and_derived_chain():
    m = M.get("d2q9")
    vals = m.default_settings()
    assert vals[m.setting_index("RelaxationRate")] == 0.0  # derives S2: no default applied
    assert vals[m.setting_index("Threshold")] == 0.5
    m.apply_setting(vals, "Viscosity", 0.02)
    w = 1 / (3 * 0.02 + 0.5)
    assert vals[m.setting_index("RelaxationRate")] == pytest.approx(w)
    assert vals[m.setting_index("S2")] == pytest.approx(1 - w)
    o = oracle.OracleLattice("d2q9", 32, 8)
    o.set_setting("Viscosity", 0.02)
    assert o.get_setting("S2") == pytest.approx(1 - w)


def test_library_exports_header_symbols():
    """The C-ABI library exports every function include/tclb_b200.h declares."""
    hdr = open(os.path.join(ROOT, "include", "tclb_b200.h")).read()
    names = set(re.findall(r"^\s*(?:const char\*|int|size_t|double)\s+(tclb_\w+)\s*\(", hdr, re.M))
    assert len(names) > 20
    lib = load_library()
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_batch_case_footprint():
    from tclb_b200.batch import case_bytes

    # d2q9 FP32 128x32: 2 snapshots of 9 planes (256-byte aligned) + flags + zone table + Globals
    n = 128 * 32
    expect = 2 * 9 * n * 4 + n * 2 + 512 * 6 * 4 + 256
    assert case_bytes("d2q9", 128, 32) == expect
    assert case_bytes("d3q19", 64, 64, 64, storage="fp16s") > 2 * 19 * 64 ** 3 * 2
