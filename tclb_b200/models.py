"""Model descriptors for the three supported TCLB models.

Each model is declared the way its ``Dynamics.R`` declares it (densities,
settings, zonal settings, globals, node types, quantities) and the derived
tables are computed by the same rules TCLB's code generator applies:

* node-type packing: ``src/conf.R:600-699`` -- groups sorted alphabetically,
  ``ceil(log2(n+1))`` bits per group, values ``1..n`` shifted into the group's
  field, zone index in the remaining high bits of a 16-bit ``flag_t``;
* Globals order: ``src/conf.R:740-751`` -- SUM globals in declared order, then
  ``Objective``, then MAX globals; one zonal ``<Global>InObj`` setting per SUM
  global (``src/conf.R:753-762``), then the ``Threshold`` setting;
* settings defaults are applied only to settings that derive no other setting
  (``src/Solver.cpp.Rt:276-281``); zonal defaults to every zone
  (``src/Solver.cpp.Rt:393``).

The C-ABI library carries the same tables in C++; ``tests/test_models.py``
checks that both agree.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

D2Q9, D3Q19, D3Q27C = 0, 1, 2
MODEL_IDS = {"d2q9": D2Q9, "d3q19": D3Q19, "d3q27_cumulant": D3Q27C}

ITER_NORM = 0x001
ITER_GLOBS = 0x010
ITER_INTEG = 0x070
ITER_LASTGLOB = 0x080


@dataclass
class Setting:
    name: str
    default: float = 0.0
    derives: Optional[Tuple[str, Callable[[float], float]]] = None
    zonal: bool = False


@dataclass
class Model:
    name: str
    mid: int
    velocities: List[Tuple[int, int, int]]
    settings_decl: List[Setting]
    globals_decl: List[Tuple[str, str]]  # (name, op)
    node_types_decl: List[Tuple[str, str]]  # (name, group)
    quantities: List[Tuple[str, bool]]  # (name, is_vector)
    shift: Optional[List[float]] = None  # storage shift per density (AddDensity shift=)
    # derived tables
    settings: List[Setting] = field(default_factory=list)
    zone_settings: List[Setting] = field(default_factory=list)
    globals: List[Tuple[str, str]] = field(default_factory=list)
    node_types: Dict[str, Tuple[int, int, str]] = field(default_factory=dict)  # name -> (value, mask, group)
    groups: Dict[str, Tuple[int, int]] = field(default_factory=dict)  # group -> (mask, shift)
    zone_shift: int = 0
    in_obj_offset: int = 0

    def __post_init__(self):
        # settings / zonal settings in declaration order, InObj + Threshold appended
        self.settings = [s for s in self.settings_decl if not s.zonal]
        self.zone_settings = [s for s in self.settings_decl if s.zonal]
        sums = [g for g in self.globals_decl if g[1] == "SUM"]
        maxs = [g for g in self.globals_decl if g[1] != "SUM"]
        self.globals = sums + [("Objective", "SUM")] + maxs
        for g in sums:
            self.zone_settings.append(Setting(g[0] + "InObj", 0.0, zonal=True))
        self.settings.append(Setting("Threshold", 0.5))
        # node-type packing (src/conf.R:600-699)
        groups: Dict[str, List[str]] = {}
        for name, grp in self.node_types_decl:
            groups.setdefault(grp, [])
            if name not in groups[grp]:
                groups[grp].append(name)
        shift_val, shift_num = 1, 0
        for grp in sorted(groups):
            names = groups[grp]
            n = len(names)
            bits = math.ceil(math.log2(n + 1))
            mask = shift_val * (2 ** bits - 1)
            self.groups[grp] = (mask, shift_num)
            for i, nm in enumerate(names):
                self.node_types[nm] = (shift_val * (i + 1), mask, grp)
            shift_val *= 2 ** bits
            shift_num += bits
        if shift_num > 14:
            raise ValueError("flag_t would need 32 bits")
        self.zone_shift = shift_num
        self.groups["SETTINGZONE"] = (((1 << (16 - shift_num)) - 1) << shift_num, shift_num)
        zs_names = [s.name for s in self.zone_settings]
        glob_names = [g[0] for g in self.globals]
        offs = {zs_names.index(g + "InObj") - glob_names.index(g) for g, _ in sums}
        self.in_obj_offset = offs.pop() if offs else 0

    # --- convenience -------------------------------------------------------
    @property
    def Q(self) -> int:
        return len(self.velocities)

    @property
    def dim(self) -> int:
        return 2 if all(v[2] == 0 for v in self.velocities) else 3

    @property
    def max_zones(self) -> int:
        return 1 << (16 - self.zone_shift)

    def setting_index(self, name: str) -> int:
        return [s.name for s in self.settings].index(name)

    def zone_setting_index(self, name: str) -> int:
        return [s.name for s in self.zone_settings].index(name)

    def global_index(self, name: str) -> int:
        return [g[0] for g in self.globals].index(name)

    def quantity_index(self, name: str) -> int:
        return [q[0] for q in self.quantities].index(name)

    def flag(self, *names: str, zone: int = 0) -> int:
        v = 0
        for nm in names:
            v |= self.node_types[nm][0]
        return v | (zone << self.zone_shift)

    def default_settings(self) -> List[float]:
        """Setting values right after lattice creation (non-deriving settings only)."""
        return [0.0 if s.derives else float(s.default) for s in self.settings]

    def apply_setting(self, values: List[float], name: str, v: float) -> None:
        """Lattice::SetSetting semantics: set and follow the derived chain."""
        i = self.setting_index(name)
        values[i] = v
        s = self.settings[i]
        if s.derives:
            tgt, fn = s.derives
            self.apply_setting(values, tgt, fn(v))

    @property
    def weights(self) -> List[float]:
        """Lattice weights w_i of the second-order equilibrium at rest."""
        out = []
        for v in self.velocities:
            k = sum(abs(c) for c in v)
            if self.Q == 9:
                out.append([4 / 9, 1 / 9, 1 / 36][k])
            elif self.Q == 19:
                out.append([1 / 3, 1 / 18, 1 / 36][k])
            else:
                out.append([8 / 27, 2 / 27, 1 / 54, 1 / 216][k])
        return out


def _visc_to_rate(nu: float) -> float:
    return 1.0 / (3 * nu + 0.5)


# models/flow/d2q9/Dynamics.R
_d2q9 = Model(
    name="d2q9",
    mid=D2Q9,
    velocities=[(0, 0, 0), (1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0), (1, 1, 0), (-1, 1, 0), (-1, -1, 0), (1, -1, 0)],
    settings_decl=[
        Setting("RelaxationRate", 0.0, ("S2", lambda r: 1 - r)),
        Setting("Viscosity", 0.16666666, ("RelaxationRate", _visc_to_rate)),
        Setting("VelocityX", 0.0, zonal=True),
        Setting("VelocityY", 0.0, zonal=True),
        Setting("Pressure", 0.0, zonal=True),
        Setting("GravitationX"),
        Setting("GravitationY"),
        Setting("S2"),
        Setting("S3"),
        Setting("S4"),
    ],
    globals_decl=[("PressureLoss", "SUM"), ("OutletFlux", "SUM"), ("InletFlux", "SUM")],
    node_types_decl=[
        ("EPressure", "BOUNDARY"), ("WPressure", "BOUNDARY"), ("NVelocity", "BOUNDARY"), ("SVelocity", "BOUNDARY"),
        ("WVelocity", "BOUNDARY"), ("EVelocity", "BOUNDARY"), ("NSymmetry", "BOUNDARY"), ("SSymmetry", "BOUNDARY"),
        ("Inlet", "OBJECTIVE"), ("Outlet", "OBJECTIVE"), ("Solid", "BOUNDARY"), ("Wall", "BOUNDARY"),
        ("MRT", "COLLISION"),
    ],
    quantities=[("Rho", False), ("U", True)],
    shift=[4 / 9] + [1 / 9] * 4 + [1 / 36] * 4,
)

_D3Q19_E = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, 1, 0),
            (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1), (0, -1, 1), (0, 1, -1),
            (0, -1, -1)]

# models/flow/d3q19/Dynamics.R
_d3q19 = Model(
    name="d3q19",
    mid=D3Q19,
    velocities=_D3Q19_E,
    settings_decl=[
        Setting("omega"),
        Setting("nu", 0.16666666, ("omega", _visc_to_rate)),
        Setting("InletVelocity", 0.0),
        Setting("InletPressure", 0.0, ("InletDensity", lambda p: 1.0 + p * 3)),
        Setting("InletDensity", 1.0),
        Setting("ForceX"),
        Setting("ForceY"),
        Setting("ForceZ"),
    ],
    globals_decl=[("Flux", "SUM")]
    + [(p + q, "SUM") for p in ("XY", "XZ", "YZ") for q in ("vx", "vy", "vz", "rho", "area")]
    + [(n, "SUM") for n in ("VOLvx", "VOLvy", "VOLvz", "VOLpx", "VOLpy", "VOLpz", "VOLrho", "VOLvolume")]
    + [("MaxV", "MAX")],
    node_types_decl=[
        ("XYslice", "ADDITIONALS"), ("XZslice", "ADDITIONALS"), ("YZslice", "ADDITIONALS"),
        ("EPressure", "BOUNDARY"), ("Solid", "BOUNDARY"), ("Wall", "BOUNDARY"), ("WPressure", "BOUNDARY"),
        ("WPressureL", "BOUNDARY"), ("WVelocity", "BOUNDARY"), ("MRT", "COLLISION"),
    ],
    quantities=[("P", False), ("U", True)],
)

_m = (0, 1, -1)
# models/flow/d3q27_cumulant/Dynamics.R (plain variant: SMAG, IB, AVG off)
_d3q27c = Model(
    name="d3q27_cumulant",
    mid=D3Q27C,
    velocities=[(_m[a], _m[b], _m[c]) for c in range(3) for b in range(3) for a in range(3)],
    settings_decl=[
        Setting("nu", 0.16666666),
        Setting("nubuffer", 0.01),
        Setting("Velocity", 0.0, zonal=True),
        Setting("Pressure", 0.0, zonal=True),
        Setting("Turbulence", 0.0, zonal=True),
        Setting("GalileanCorrection", 1.0),
        Setting("ForceX"),
        Setting("ForceY"),
        Setting("ForceZ"),
        Setting("Omega", 1.0),
    ],
    globals_decl=[(n, "SUM") for n in ("Density", "Flux", "Drag", "Lift", "Lateral", "Mass", "XMomentum",
                                        "YMomentum", "ZMomentum")],
    node_types_decl=[
        ("Buffer", "BOUNDARY"), ("WVelocityTurbulent", "BOUNDARY"), ("NVelocity", "BOUNDARY"),
        ("SVelocity", "BOUNDARY"), ("NPressure", "BOUNDARY"), ("SPressure", "BOUNDARY"),
        ("NSymmetry", "ADDITIONALS"), ("SSymmetry", "ADDITIONALS"), ("Body", "BODY"),
        ("EPressure", "BOUNDARY"), ("EVelocity", "BOUNDARY"), ("Solid", "BOUNDARY"), ("Wall", "BOUNDARY"),
        ("WPressure", "BOUNDARY"), ("WVelocity", "BOUNDARY"), ("MRT", "COLLISION"),
    ],
    quantities=[("P", False), ("U", True), ("Solid", False)],
)

MODELS: Dict[str, Model] = {"d2q9": _d2q9, "d3q19": _d3q19, "d3q27_cumulant": _d3q27c}
BY_ID: Dict[int, Model] = {m.mid: m for m in MODELS.values()}


def get(model) -> Model:
    if isinstance(model, Model):
        return model
    if isinstance(model, int):
        return BY_ID[model]
    return MODELS[model]
