// Per-model constants shared by host and device code.
//
// Node-type values follow TCLB's packing rule (src/conf.R:600-699): groups in
// alphabetical order, ceil(log2(n+1)) bits each, zone index in the high bits.
// Settings / zonal settings / Globals indices follow src/conf.R:740-769 and the
// declaration order of each model's Dynamics.R.
#pragma once
#include <cstdint>

namespace tclb {

typedef uint16_t flag_t;

enum Model { MODEL_D2Q9 = 0, MODEL_D3Q19 = 1, MODEL_D3Q27C = 2 };

struct ModelTable {
  const char* name;
  int Q, dim;
  int nsettings, nzonesettings, nglobals, nsum, objective, in_obj_offset, zone_shift;
  const char* const* setting_names;
  const double* setting_defaults;     // applied at creation (NaN = not applied)
  const int* setting_derives;         // index of derived target or -1
  const char* const* zone_setting_names;
  const double* zone_setting_defaults;
  const char* const* global_names;
  const char* const* node_type_names;
  const int* node_type_values;
  const int* node_type_masks;
  int n_node_types;
  const char* const* quantity_names;
  const int* quantity_vector;
  int nquantities;
  const char* const* group_names;  // node-type groups and their masks
  const int* group_masks;
  int ngroups;
};

// ---------------------------------------------------------------- d2q9
// models/flow/d2q9/Dynamics.R
namespace d2q9 {
enum { BOUNDARY = 0x000F, EPressure = 1, WPressure = 2, NVelocity = 3, SVelocity = 4, WVelocity = 5, EVelocity = 6,
       NSymmetry = 7, SSymmetry = 8, Solid = 9, Wall = 10, COLLISION = 0x10, MRT = 0x10, OBJECTIVE = 0x60,
       Inlet = 0x20, Outlet = 0x40, ZONE_SHIFT = 7 };
enum { S_RelaxationRate = 0, S_Viscosity, S_GravitationX, S_GravitationY, S_S2, S_S3, S_S4, S_Threshold, NSET };
enum { Z_VelocityX = 0, Z_VelocityY, Z_Pressure, Z_PressureLossInObj, Z_OutletFluxInObj, Z_InletFluxInObj, NZS };
enum { G_PressureLoss = 0, G_OutletFlux, G_InletFlux, G_Objective, NG };
enum { NSUM = 4, IN_OBJ_OFFSET = 3 };
}  // namespace d2q9

// ---------------------------------------------------------------- d3q19
// models/flow/d3q19/Dynamics.R
namespace d3q19 {
enum { ADDITIONALS = 0x3, XYslice = 1, XZslice = 2, YZslice = 3, BOUNDARY = 0x1C, EPressure = 0x04, Solid = 0x08,
       Wall = 0x0C, WPressure = 0x10, WPressureL = 0x14, WVelocity = 0x18, COLLISION = 0x20, MRT = 0x20,
       ZONE_SHIFT = 6 };
enum { S_omega = 0, S_nu, S_InletVelocity, S_InletPressure, S_InletDensity, S_ForceX, S_ForceY, S_ForceZ, S_Threshold,
       NSET };
enum { NZS = 24 };  // <Global>InObj for the 24 SUM globals other than Objective
enum { G_Flux = 0, G_XY = 1, G_XZ = 6, G_YZ = 11, G_VOLvx = 16, G_VOLvy, G_VOLvz, G_VOLpx, G_VOLpy, G_VOLpz,
       G_VOLrho, G_VOLvolume, G_Objective = 24, G_MaxV = 25, NG = 26 };
enum { NSUM = 25, IN_OBJ_OFFSET = 0 };
}  // namespace d3q19

// ---------------------------------------------------------------- d3q27_cumulant
// models/flow/d3q27_cumulant/Dynamics.R (plain variant)
namespace d3q27c {
enum { ADDITIONALS = 0x3, NSymmetry = 1, SSymmetry = 2, BODY = 0x4, Body = 0x4, BOUNDARY = 0x78, Buffer = 0x08,
       WVelocityTurbulent = 0x10, NVelocity = 0x18, SVelocity = 0x20, NPressure = 0x28, SPressure = 0x30,
       EPressure = 0x38, EVelocity = 0x40, Solid = 0x48, Wall = 0x50, WPressure = 0x58, WVelocity = 0x60,
       COLLISION = 0x80, MRT = 0x80, ZONE_SHIFT = 8 };
enum { S_nu = 0, S_nubuffer, S_GalileanCorrection, S_ForceX, S_ForceY, S_ForceZ, S_Omega, S_Threshold, NSET };
enum { Z_Velocity = 0, Z_Pressure, Z_Turbulence, NZS = 12 };
enum { G_Density = 0, G_Flux, G_Drag, G_Lift, G_Lateral, G_Mass, G_XMomentum, G_YMomentum, G_ZMomentum,
       G_Objective, NG };
enum { NSUM = 10, IN_OBJ_OFFSET = 3 };
}  // namespace d3q27c

const ModelTable* model_table(int model);

}  // namespace tclb
