// Host runtime and C ABI of the B200 lattice-Boltzmann engine.
//
// One handle = one lattice (TCLB's Lattice + LatticeContainer, src/Lattice.cu.Rt,
// src/LatticeContainer.h.Rt): a single pooled device allocation holds both
// snapshots, the node types, the zonal-settings table and the FP64 Globals
// (TCLB pools its buffers the same way, src/cross.cu:52-102). Settings travel
// as kernel parameters instead of __constant__ memory, so handles are
// independent and any number of lattices can share a GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <utility>

#include "../../include/tclb_b200.h"
#include "lbm_tma.cuh"

using namespace tclb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define TCLB_CK(call)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(TCLB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ model tables
const double NA = NAN;

const char* const d2q9_set[] = {"RelaxationRate", "Viscosity", "GravitationX", "GravitationY", "S2", "S3", "S4",
                                "Threshold"};
const double d2q9_set_def[] = {NA, NA, 0, 0, 0, 0, 0, 0.5};
const int d2q9_set_der[] = {d2q9::S_S2, d2q9::S_RelaxationRate, -1, -1, -1, -1, -1, -1};
const char* const d2q9_zs[] = {"VelocityX", "VelocityY", "Pressure", "PressureLossInObj", "OutletFluxInObj",
                               "InletFluxInObj"};
const double d2q9_zs_def[] = {0, 0, 0, 0, 0, 0};
const char* const d2q9_gl[] = {"PressureLoss", "OutletFlux", "InletFlux", "Objective"};
const char* const d2q9_nt[] = {"EPressure", "WPressure", "NVelocity", "SVelocity", "WVelocity", "EVelocity", "NSymmetry",
                               "SSymmetry", "Solid", "Wall", "MRT", "Inlet", "Outlet"};
const int d2q9_nt_v[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 0x10, 0x20, 0x40};
const int d2q9_nt_m[] = {0xF, 0xF, 0xF, 0xF, 0xF, 0xF, 0xF, 0xF, 0xF, 0xF, 0x10, 0x60, 0x60};
const char* const d2q9_q[] = {"Rho", "U"};
const int d2q9_qv[] = {0, 1};

const char* const d3q19_set[] = {"omega", "nu", "InletVelocity", "InletPressure", "InletDensity", "ForceX", "ForceY",
                                 "ForceZ", "Threshold"};
const double d3q19_set_def[] = {0, NA, 0, NA, 1, 0, 0, 0, 0.5};
const int d3q19_set_der[] = {-1, d3q19::S_omega, -1, d3q19::S_InletDensity, -1, -1, -1, -1, -1};
const char* const d3q19_gl[] = {"Flux",   "XYvx",   "XYvy",   "XYvz",   "XYrho",     "XYarea",    "XZvx",
                                "XZvy",   "XZvz",   "XZrho",  "XZarea", "YZvx",      "YZvy",      "YZvz",
                                "YZrho",  "YZarea", "VOLvx",  "VOLvy",  "VOLvz",     "VOLpx",     "VOLpy",
                                "VOLpz",  "VOLrho", "VOLvolume", "Objective", "MaxV"};
const char* const d3q19_zs[] = {"FluxInObj",   "XYvxInObj",   "XYvyInObj",  "XYvzInObj",   "XYrhoInObj",
                                "XYareaInObj", "XZvxInObj",   "XZvyInObj",  "XZvzInObj",   "XZrhoInObj",
                                "XZareaInObj", "YZvxInObj",   "YZvyInObj",  "YZvzInObj",   "YZrhoInObj",
                                "YZareaInObj", "VOLvxInObj",  "VOLvyInObj", "VOLvzInObj",  "VOLpxInObj",
                                "VOLpyInObj",  "VOLpzInObj",  "VOLrhoInObj", "VOLvolumeInObj"};
const double d3q19_zs_def[24] = {0};
const char* const d3q19_nt[] = {"XYslice", "XZslice", "YZslice", "EPressure", "Solid", "Wall", "WPressure",
                                "WPressureL", "WVelocity", "MRT"};
const int d3q19_nt_v[] = {1, 2, 3, 0x04, 0x08, 0x0C, 0x10, 0x14, 0x18, 0x20};
const int d3q19_nt_m[] = {3, 3, 3, 0x1C, 0x1C, 0x1C, 0x1C, 0x1C, 0x1C, 0x20};
const char* const d3q19_q[] = {"P", "U"};
const int d3q19_qv[] = {0, 1};

const char* const d3q27c_set[] = {"nu", "nubuffer", "GalileanCorrection", "ForceX", "ForceY", "ForceZ", "Omega",
                                  "Threshold"};
const double d3q27c_set_def[] = {0.16666666, 0.01, 1, 0, 0, 0, 1, 0.5};
const int d3q27c_set_der[] = {-1, -1, -1, -1, -1, -1, -1, -1};
const char* const d3q27c_zs[] = {"Velocity",    "Pressure",   "Turbulence", "DensityInObj",
                                 "FluxInObj",   "DragInObj",  "LiftInObj",  "LateralInObj",
                                 "MassInObj",   "XMomentumInObj", "YMomentumInObj", "ZMomentumInObj"};
const double d3q27c_zs_def[12] = {0};
const char* const d3q27c_gl[] = {"Density", "Flux", "Drag", "Lift", "Lateral", "Mass", "XMomentum", "YMomentum",
                                 "ZMomentum", "Objective"};
const char* const d3q27c_nt[] = {"NSymmetry", "SSymmetry", "Body", "Buffer", "WVelocityTurbulent", "NVelocity",
                                 "SVelocity", "NPressure", "SPressure", "EPressure", "EVelocity", "Solid", "Wall",
                                 "WPressure", "WVelocity", "MRT"};
const int d3q27c_nt_v[] = {1, 2, 4, 0x08, 0x10, 0x18, 0x20, 0x28, 0x30, 0x38, 0x40, 0x48, 0x50, 0x58, 0x60, 0x80};
const int d3q27c_nt_m[] = {3, 3, 4, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x78, 0x80};
const char* const d3q27c_q[] = {"P", "U", "Solid"};
const int d3q27c_qv[] = {0, 1, 0};

const char* const d2q9_grp[] = {"BOUNDARY", "COLLISION", "OBJECTIVE"};
const int d2q9_grp_m[] = {0xF, 0x10, 0x60};
const char* const d3q19_grp[] = {"ADDITIONALS", "BOUNDARY", "COLLISION"};
const int d3q19_grp_m[] = {0x3, 0x1C, 0x20};
const char* const d3q27c_grp[] = {"ADDITIONALS", "BODY", "BOUNDARY", "COLLISION"};
const int d3q27c_grp_m[] = {0x3, 0x4, 0x78, 0x80};

const ModelTable TABLES[3] = {
    {"d2q9", 9, 2, d2q9::NSET, d2q9::NZS, d2q9::NG, d2q9::NSUM, d2q9::G_Objective, d2q9::IN_OBJ_OFFSET,
     d2q9::ZONE_SHIFT, d2q9_set, d2q9_set_def, d2q9_set_der, d2q9_zs, d2q9_zs_def, d2q9_gl, d2q9_nt, d2q9_nt_v,
     d2q9_nt_m, 13, d2q9_q, d2q9_qv, 2, d2q9_grp, d2q9_grp_m, 3},
    {"d3q19", 19, 3, d3q19::NSET, d3q19::NZS, d3q19::NG, d3q19::NSUM, d3q19::G_Objective, d3q19::IN_OBJ_OFFSET,
     d3q19::ZONE_SHIFT, d3q19_set, d3q19_set_def, d3q19_set_der, d3q19_zs, d3q19_zs_def, d3q19_gl, d3q19_nt,
     d3q19_nt_v, d3q19_nt_m, 10, d3q19_q, d3q19_qv, 2, d3q19_grp, d3q19_grp_m, 3},
    {"d3q27_cumulant", 27, 3, d3q27c::NSET, d3q27c::NZS, d3q27c::NG, d3q27c::NSUM, d3q27c::G_Objective,
     d3q27c::IN_OBJ_OFFSET, d3q27c::ZONE_SHIFT, d3q27c_set, d3q27c_set_def, d3q27c_set_der, d3q27c_zs, d3q27c_zs_def,
     d3q27c_gl, d3q27c_nt, d3q27c_nt_v, d3q27c_nt_m, 16, d3q27c_q, d3q27c_qv, 3, d3q27c_grp, d3q27c_grp_m, 4},
};

// Derived-setting equations (each model's Dynamics.R AddSetting(..., X='expr'))
double derive_value(int model, int from, double v) {
  if (model == MODEL_D2Q9) {
    if (from == d2q9::S_Viscosity) return 1.0 / (3 * v + 0.5);
    if (from == d2q9::S_RelaxationRate) return 1 - v;
  } else if (model == MODEL_D3Q19) {
    if (from == d3q19::S_nu) return 1.0 / (3 * v + 0.5);
    if (from == d3q19::S_InletPressure) return 1.0 + v * 3;
  }
  return v;
}

}  // namespace

namespace tclb {
const ModelTable* model_table(int model) { return (model >= 0 && model < 3) ? &TABLES[model] : nullptr; }
}  // namespace tclb

// ------------------------------------------------------------------ lattice
struct Impl;

struct tclb_lattice {
  int model, precision, storage, device;
  int nx, ny, nz;
  size_t N, stride, elem;
  const ModelTable* T;
  int nzones;
  char* pool = nullptr;
  void* buf[2] = {nullptr, nullptr};
  int cur = 0;
  flag_t* flags = nullptr;
  void* zone_dev = nullptr;
  double* glob_dev = nullptr;
  std::vector<double> settings, zone, globals;
  cudaStream_t stream = nullptr;
  long long iter = 0;
  int bx = 128, by = 2;
  void* qbuf = nullptr;
  size_t qbuf_bytes = 0;
  const Impl* impl = nullptr;
  // CUDA graphs of GRAPH_CHUNK plain iterations starting from snapshot 0 / 1;
  // settings travel as kernel parameters, so a settings change drops them.
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int use_graphs = 1;
  int use_pairs = 1;  // 16-bit storage: two nodes per thread when nx % 64 == 0
  // 16-bit storage: tile-staged TMA kernel (tma_rows rows per tile; tma[b]
  // describes snapshot b as the source), and its error word in the pool
  int use_tma = 1, tma_ok = 0, tma_rows = 0, tma_grid = 0;
  // shapes where a model's register pair kernel measured faster (d3q19: rows
  // wider than 256, under-filled or too few tiles): plain iterations take
  // that kernel unless tma_always
  int tma_pref_pairs = 0, tma_always = 0;
  // node pairs of which one node collides and the other not make up at least
  // 1% of the lattice (porous media): the tile-staged kernel of a model with
  // identity-rate lanes runs the other node at identity rates instead of
  // parking it (measured on B200, d3q19 porous 256^3 FP16-shift: 2% solids
  // 66.1k -> 67.5k MLUPS, 8.5% 62.1k -> 64.6-64.9k, 15% 61.3-61.6k ->
  // 64.5-65.1k; without such pairs, Taylor-Green, parking is 1.3% faster)
  int lanes = 0;
  unsigned* count_dev = nullptr;  // device word for the count
  TmaMaps tma[2];
  int* err_dev = nullptr;
  // failure-path test of the tile-staged kernel (tclb_set_fault_injection):
  // the tile whose copies are not issued (-1: none) and the wait bound
  int fault_tile = -1;
  long long wait_cycles = TMA_WAIT_CYCLES;
};

struct Impl {
  void (*iterate)(tclb_lattice*, bool, cudaStream_t);
  int (*flags_changed)(tclb_lattice*);  // after new node types: the kernel choices that depend on them
  void (*init)(tclb_lattice*, cudaStream_t);
  void (*quantity)(tclb_lattice*, int, int, const int*, double, void*, cudaStream_t);
  void (*equilibrium)(tclb_lattice*, const void*, const void*, cudaStream_t);
  void (*color)(tclb_lattice*, int, void*, cudaStream_t);
  void (*to_double)(const void*, size_t, size_t, size_t, int, double*);   // storage -> double SoA
  void (*from_double)(const double*, size_t, size_t, size_t, int, void*);  // double SoA -> storage
  void (*prepare)(tclb_lattice*);
  size_t real_size;
};

namespace {

template <class M, class R>
Args<R, M::NSET> make_args(const tclb_lattice* L, const void* src, void* dst) {
  Args<R, M::NSET> a;
  a.src = src;
  a.dst = dst;
  a.stride = L->stride;
  a.flags = L->flags;
  a.nx = L->nx;
  a.ny = L->ny;
  a.nz = L->nz;
  a.zone = static_cast<const R*>(L->zone_dev);
  a.glob = L->glob_dev;
  for (int i = 0; i < M::NSET; i++) a.s[i] = (R)L->settings[i];
  M::template derived<R>(a.s, a.k);
  return a;
}

// Plain iterations of 16-bit storage take the tile-staged kernel.
inline bool tma_path(const tclb_lattice* L) {
  return L->use_tma && L->tma_ok && L->tma_grid > 0 &&
         (L->tma_always || !L->tma_pref_pairs || !(L->use_pairs && L->nx % 64 == 0));
}

// A kernel launch on stream s whose grid may be scheduled while the previous
// kernel on the stream drains (the kernel itself waits for it with
// griddepcontrol.wait); captured into CUDA graphs as a programmatic edge.
template <class... KArgs, class... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <class M>
inline bool tma_lanes(const tclb_lattice* L) {
  return M::identity_lanes && L->lanes;
}

inline dim3 grid_of(const tclb_lattice* L) {
  return dim3((L->nx + L->bx - 1) / L->bx, (L->ny + L->by - 1) / L->by, L->nz);
}

template <class M, class R, class St>
struct Launch {
  static void iterate(tclb_lattice* L, bool glob, cudaStream_t s) {
    const void* src = L->buf[L->cur];
    void* dst = L->buf[1 - L->cur];
    auto a = make_args<M, R>(L, src, dst);
    // Addressing by storage width (measured on B200): the issue-bound 16-bit
    // kernels gain from per-plane base pointers (fewer integer instructions
    // per access); the memory-bound 32/64-bit kernels run faster with one
    // pointer and the plane stride.
    using T = typename St::T;
    if constexpr (sizeof(T) == 2) {
      PlaneAddr<T, M::Q> P;
      for (int i = 0; i < M::Q; i++) {
        P.s[i] = static_cast<const T*>(src) + (size_t)i * L->stride;
        P.d[i] = static_cast<T*>(dst) + (size_t)i * L->stride;
      }
      if (tma_path(L) && !glob) {  // tiles staged in shared memory by TMA
        const int rows = L->tma_rows, threads = tma_threads(rows, L->nx);
        const size_t smem = tma_smem_bytes<M>();
        if (L->tma_grid > 0) {
          const bool partial = (rows * L->nx / 2) % 32 != 0;  // pairs that do not fill whole warps
          if (L->fault_tile >= 0 || L->wait_cycles != TMA_WAIT_CYCLES)  // the failure-path test
            k_iterate_tma<M, R, St, true, true><<<L->tma_grid, threads, smem, s>>>(
                a, L->tma[L->cur], P, rows, L->err_dev, L->wait_cycles, L->fault_tile);
          else if (partial)
            k_iterate_tma<M, R, St, false, true><<<L->tma_grid, threads, smem, s>>>(a, L->tma[L->cur], P, rows,
                                                                                   L->err_dev, TMA_WAIT_CYCLES, -1);
          else if (tma_lanes<M>(L))
            k_iterate_tma<M, R, St, false, false, M::identity_lanes><<<L->tma_grid, threads, smem, s>>>(
                a, L->tma[L->cur], P, rows, L->err_dev, TMA_WAIT_CYCLES, -1);
          else
            k_iterate_tma<M, R, St><<<L->tma_grid, threads, smem, s>>>(a, L->tma[L->cur], P, rows, L->err_dev,
                                                                        TMA_WAIT_CYCLES, -1);
          return;
        }
      }
      if (L->use_pairs && !glob && L->nx % 64 == 0) {  // two nodes per thread, 32-bit accesses
        constexpr int by = M::PAIR_THREADS / 32;
        const dim3 blk(32, by), grd(L->nx / 64, (L->ny + by - 1) / by, L->nz);
        k_iterate_pair<M, R, St><<<grd, blk, 0, s>>>(a, P);
        return;
      }
      if (glob) launch_pdl(k_iterate<M, R, St, true, PlaneAddr<T, M::Q>>, grid_of(L), dim3(L->bx, L->by), s, a, P);
      else launch_pdl(k_iterate<M, R, St, false, PlaneAddr<T, M::Q>>, grid_of(L), dim3(L->bx, L->by), s, a, P);
    } else {
      const StrideAddr<T> P{static_cast<const T*>(src), static_cast<T*>(dst), L->stride};
      if (glob) launch_pdl(k_iterate<M, R, St, true, StrideAddr<T>>, grid_of(L), dim3(L->bx, L->by), s, a, P);
      else launch_pdl(k_iterate<M, R, St, false, StrideAddr<T>>, grid_of(L), dim3(L->bx, L->by), s, a, P);
    }
  }
  // Once at creation: the dynamic shared-memory limit and persistent grid of the
  // tile-staged kernel (resident blocks per SM x SMs, at most one per tile).
  static void prepare(tclb_lattice* L) {
    using T = typename St::T;
    if constexpr (sizeof(T) == 2) {
      if (!L->tma_ok) return;
      const int rows = L->tma_rows, threads = tma_threads(rows, L->nx);
      const size_t smem = tma_smem_bytes<M>();
      int per_sm = 0, sms = 0;
      if (cudaFuncSetAttribute(k_iterate_tma<M, R, St>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
              cudaSuccess ||
          cudaFuncSetAttribute(k_iterate_tma<M, R, St, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(k_iterate_tma<M, R, St, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(k_iterate_tma<M, R, St, false, false, M::identity_lanes>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_iterate_tma<M, R, St>, threads, smem) !=
              cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, L->device) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        L->tma_ok = 0;
        return;
      }
      const int tiles = L->nz * (L->ny / rows);
      L->tma_grid = std::min(tiles, per_sm * sms);
      // d3q19 (register pair kernel with identity-rate lanes) takes that kernel
      // where nx % 64 == 0 and the staged tiles would be under-filled or too
      // few, as measured on B200 (porous boxes, FP16-shift): rows wider than
      // 256 (one-row tiles, six consumer warps per block; 384x192x192: 57.7k
      // against 51.6k MLUPS), tiles of fewer than 448 nodes (192^3: 56.4k
      // against 50.2k), fewer than four tiles per resident block (64^3: 45.8k
      // against 27.8k)
      if constexpr (M::identity_lanes)
        L->tma_pref_pairs = L->nx % 64 == 0 && (tma_wide(L->nx) || rows * L->nx < 448 || tiles < 4 * per_sm * sms);
    }
  }
  // Count the node pairs (x, x+1), x even, of which exactly one node
  // collides; with 16-bit storage and identity-rate lanes, set L->lanes.
  static int flags_changed(tclb_lattice* L) {
    L->lanes = 0;
    if constexpr (M::identity_lanes && sizeof(typename St::T) == 2) {
      if (L->nx % 2) return TCLB_OK;
      const unsigned npairs = (unsigned)(L->N / 2);
      TCLB_CK(cudaMemsetAsync(L->count_dev, 0, sizeof(unsigned), L->stream));
      k_count_mixed_pairs<M><<<std::min<unsigned>((npairs + 255) / 256, 1184), 256, 0, L->stream>>>(
          L->flags, npairs, L->count_dev);
      TCLB_CK(cudaGetLastError());
      unsigned mixed = 0;
      TCLB_CK(cudaMemcpyAsync(&mixed, L->count_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, L->stream));
      TCLB_CK(cudaStreamSynchronize(L->stream));
      L->lanes = (unsigned long long)mixed * 100 >= npairs ? 1 : 0;
    }
    return TCLB_OK;
  }
  static void init(tclb_lattice* L, cudaStream_t s) {
    auto a = make_args<M, R>(L, nullptr, L->buf[L->cur]);
    k_init<M, R, St><<<grid_of(L), dim3(L->bx, L->by), 0, s>>>(a);
  }
  static void quantity(tclb_lattice* L, int q, int vec, const int* r, double scale, void* out, cudaStream_t s) {
    auto a = make_args<M, R>(L, L->buf[L->cur], nullptr);
    dim3 blk(32, 4);
    dim3 grd((r[3] + 31) / 32, (r[4] + 3) / 4, r[5]);
    k_quantity<M, R, St><<<grd, blk, 0, s>>>(a, q, vec, r[0], r[1], r[2], r[3], r[4], r[5], (R)scale,
                                               static_cast<R*>(out));
  }
  static void equilibrium(tclb_lattice* L, const void* rho, const void* u, cudaStream_t s) {
    auto a = make_args<M, R>(L, nullptr, L->buf[L->cur]);
    k_equilibrium<M, R, St><<<grid_of(L), dim3(L->bx, L->by), 0, s>>>(a, static_cast<const R*>(rho),
                                                                       static_cast<const R*>(u));
  }
  static void color(tclb_lattice* L, int z, void* out, cudaStream_t s) {
    auto a = make_args<M, R>(L, L->buf[L->cur], nullptr);
    k_color<M, R, St><<<dim3((L->nx + 127) / 128, L->ny), 128, 0, s>>>(a, z, static_cast<uchar4*>(out));
  }
  static void to_double(const void* raw, size_t N, size_t stride, size_t, int Q, double* out) {
    const typename St::T* p = static_cast<const typename St::T*>(raw);
    for (int q = 0; q < Q; q++)
      for (size_t n = 0; n < N; n++) out[(size_t)q * N + n] = St::to_double(p[(size_t)q * stride + n], M::w(q));
  }
  static void from_double(const double* in, size_t N, size_t stride, size_t, int Q, void* raw) {
    typename St::T* p = static_cast<typename St::T*>(raw);
    for (int q = 0; q < Q; q++)
      for (size_t n = 0; n < N; n++) p[(size_t)q * stride + n] = St::from_double(in[(size_t)q * N + n], M::w(q));
  }
  static const Impl* get() {
    static const Impl impl = {iterate,     flags_changed, init,    quantity, equilibrium, color,
                              to_double,   from_double,   prepare, sizeof(R)};
    return &impl;
  }
};

template <class M>
const Impl* impl_for_model(int precision, int storage) {
  if (precision == TCLB_FP64) return storage == TCLB_STORAGE_SAME ? Launch<M, double, StoreF64>::get() : nullptr;
  switch (storage) {
    case TCLB_STORAGE_SAME: return Launch<M, float, StoreF32>::get();
    case TCLB_STORAGE_FP16: return Launch<M, float, StoreF16<false>>::get();
    case TCLB_STORAGE_FP16_SHIFT: return Launch<M, float, StoreF16<true>>::get();
    case TCLB_STORAGE_BF16: return Launch<M, float, StoreBF16<false>>::get();
    case TCLB_STORAGE_BF16_SHIFT: return Launch<M, float, StoreBF16<true>>::get();
  }
  return nullptr;
}

const Impl* impl_for(int model, int precision, int storage) {
  switch (model) {
    case MODEL_D2Q9: return impl_for_model<D2Q9>(precision, storage);
    case MODEL_D3Q19: return impl_for_model<D3Q19>(precision, storage);
    case MODEL_D3Q27C: return impl_for_model<D3Q27C>(precision, storage);
  }
  return nullptr;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Tensor maps of the tile-staged kernel (16-bit storage, nx a multiple of 32
// and at most 512, R <= 512 / nx rows per tile dividing ny). When anything
// does not fit, tma_ok stays 0 and the register kernels run.
void setup_tma(tclb_lattice* L) {
  L->tma_ok = 0;
  // Tiles of at most 512 nodes (R whole rows; one row when nx > 256, copied
  // as one split-x box). Longer rows take the register pair kernel.
  const int R = tma_rows_for(L->elem, L->nx, L->ny);
  if (!R) return;
  for (int b = 0; b < 2; b++)
    if (!encode_tile_maps(L->buf[b], L->flags, L->nx, L->ny, L->nz, L->T->Q, L->stride, R, &L->tma[b].rows,
                          &L->tma[b].row1, &L->tma[b].flags))
      return;
  L->tma_rows = R;
  L->tma_ok = 1;
}

// An mbarrier wait of the tile-staged kernel ran out: the iteration it was in
// did not update every node.
int check_device_error(tclb_lattice* L, cudaStream_t s) {
  int e = 0;
  TCLB_CK(cudaMemcpyAsync(&e, L->err_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  TCLB_CK(cudaStreamSynchronize(s));
  if (e == TMA_ERR_TIMEOUT) {
    TCLB_CK(cudaMemsetAsync(L->err_dev, 0, sizeof(int), s));
    return fail(TCLB_ERR_CUDA, "tile pipeline: a wait for staged tiles ran out; the state is not valid");
  }
  return TCLB_OK;
}

int upload_zone(tclb_lattice* L) {
  const size_t n = L->zone.size();
  if (L->precision == TCLB_FP64) {
    TCLB_CK(cudaMemcpyAsync(L->zone_dev, L->zone.data(), n * sizeof(double), cudaMemcpyHostToDevice, L->stream));
  } else {
    std::vector<float> z(n);
    for (size_t i = 0; i < n; i++) z[i] = (float)L->zone[i];
    TCLB_CK(cudaMemcpyAsync(L->zone_dev, z.data(), n * sizeof(float), cudaMemcpyHostToDevice, L->stream));
    TCLB_CK(cudaStreamSynchronize(L->stream));
    return TCLB_OK;
  }
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return TCLB_OK;
}

constexpr int GRAPH_CHUNK = 32;

void drop_graphs(tclb_lattice* L) {
  for (int p = 0; p < 2; p++)
    if (L->graph[p]) {
      cudaGraphExecDestroy(L->graph[p]);
      L->graph[p] = nullptr;
    }
}

// Capture GRAPH_CHUNK plain iterations starting from the current snapshot.
int ensure_iter_graph(tclb_lattice* L, cudaStream_t s) {
  const int p = L->cur;
  if (L->graph[p]) return TCLB_OK;
  cudaStream_t cs;
  TCLB_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int k = 0; k < GRAPH_CHUNK; k++) {
      L->impl->iterate(L, false, cs);
      L->cur = 1 - L->cur;
    }
    e = cudaStreamEndCapture(cs, &g);
  }
  L->cur = p;  // capture recorded the launches without running them
  if (e == cudaSuccess) e = cudaGraphInstantiate(&L->graph[p], g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    L->graph[p] = nullptr;
    return fail(TCLB_ERR_CUDA, std::string("iteration graph: ") + cudaGetErrorString(e));
  }
  (void)s;
  return TCLB_OK;
}

int set_setting_rec(tclb_lattice* L, int i, double v, int depth) {
  if (depth > 8) return fail(TCLB_ERR_STATE, "derived-setting chain too deep");
  L->settings[i] = v;
  const int t = L->T->setting_derives[i];
  if (t >= 0) return set_setting_rec(L, t, derive_value(L->model, i, v), depth + 1);
  return TCLB_OK;
}

// Lattice::calcGlobals (src/Lattice.cu.Rt:1299-1315): device Globals -> host
// accumulators, then clear the device copy.
int calc_globals(tclb_lattice* L, cudaStream_t s) {
  std::vector<double> tab(L->T->nglobals);
  TCLB_CK(cudaMemcpyAsync(tab.data(), L->glob_dev, tab.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  TCLB_CK(cudaStreamSynchronize(s));
  for (size_t i = 0; i < tab.size(); i++) L->globals[i] += tab[i];
  TCLB_CK(cudaMemsetAsync(L->glob_dev, 0, tab.size() * sizeof(double), s));
  return check_device_error(L, s);
}

#define CHECK_H(h) \
  if (!(h)) return fail(TCLB_ERR_ARG, "null lattice handle")

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* tclb_last_error(void) { return g_err.c_str(); }

int tclb_model_info(int model, int* Q, int* nsettings, int* nzonesettings, int* nglobals, int* nquantities,
                    int* zone_shift) {
  const ModelTable* T = model_table(model);
  if (!T) return fail(TCLB_ERR_ARG, "unknown model");
  if (Q) *Q = T->Q;
  if (nsettings) *nsettings = T->nsettings;
  if (nzonesettings) *nzonesettings = T->nzonesettings;
  if (nglobals) *nglobals = T->nglobals;
  if (nquantities) *nquantities = T->nquantities;
  if (zone_shift) *zone_shift = T->zone_shift;
  return TCLB_OK;
}

int tclb_model_item(int model, int kind, int i, const char** name, int* value, int* mask) {
  const ModelTable* T = model_table(model);
  if (!T) return fail(TCLB_ERR_ARG, "unknown model");
  const char* const* names = nullptr;
  int n = 0;
  switch (kind) {
    case 0: names = T->setting_names; n = T->nsettings; break;
    case 1: names = T->zone_setting_names; n = T->nzonesettings; break;
    case 2: names = T->global_names; n = T->nglobals; break;
    case 3: names = T->node_type_names; n = T->n_node_types; break;
    case 4: names = T->quantity_names; n = T->nquantities; break;
    default: return fail(TCLB_ERR_ARG, "unknown item kind");
  }
  if (i < 0 || i >= n) return fail(TCLB_ERR_ARG, "item index out of range");
  if (name) *name = names[i];
  if (value) *value = kind == 3 ? T->node_type_values[i] : (kind == 4 ? T->quantity_vector[i] : 0);
  if (mask) *mask = kind == 3 ? T->node_type_masks[i] : 0;
  return TCLB_OK;
}

int tclb_create(tclb_h* out, int model, int nx, int ny, int nz, int precision, int storage) {
  if (!out) return fail(TCLB_ERR_ARG, "null output handle");
  *out = nullptr;
  const ModelTable* T = model_table(model);
  if (!T) return fail(TCLB_ERR_ARG, "unknown model");
  if (nx < 1 || ny < 1 || nz < 1) return fail(TCLB_ERR_ARG, "lattice size must be positive");
  if (T->dim == 2 && nz != 1) return fail(TCLB_ERR_ARG, "2D model needs nz == 1");
  if (nz > 65535) return fail(TCLB_ERR_ARG, "nz above 65535");
  const size_t N = (size_t)nx * ny * nz;
  if (N >= (size_t)1 << 31) return fail(TCLB_ERR_ARG, "lattice above 2^31 nodes");
  if (precision != TCLB_FP32 && precision != TCLB_FP64) return fail(TCLB_ERR_ARG, "unknown precision");
  const Impl* impl = impl_for(model, precision, storage);
  if (!impl) return fail(TCLB_ERR_ARG, "unsupported precision/storage combination");
  tclb_lattice* L = new tclb_lattice();
  L->model = model;
  L->precision = precision;
  L->storage = storage;
  L->nx = nx;
  L->ny = ny;
  L->nz = nz;
  L->N = N;
  L->T = T;
  L->impl = impl;
  L->elem = precision == TCLB_FP64 ? 8 : (storage == TCLB_STORAGE_SAME ? 4 : 2);
  L->stride = align_up(N, 256 / L->elem);  // 256-byte aligned population planes
  L->nzones = 1 << (16 - T->zone_shift);
  cudaGetDevice(&L->device);
  const size_t bufb = L->stride * T->Q * L->elem;
  const size_t flagb = align_up(N * sizeof(flag_t), 256);
  const size_t zoneb = align_up((size_t)L->nzones * T->nzonesettings * impl->real_size, 256);
  const size_t globb = align_up(T->nglobals * sizeof(double), 256);
  const size_t total = 2 * bufb + flagb + zoneb + globb + 256;
  cudaError_t e = cudaMalloc((void**)&L->pool, total);
  if (e != cudaSuccess) {
    delete L;
    cudaGetLastError();
    return fail(TCLB_ERR_MEMORY, std::string("cudaMalloc of lattice pool failed: ") + cudaGetErrorString(e));
  }
  L->buf[0] = L->pool;
  L->buf[1] = L->pool + bufb;
  L->flags = reinterpret_cast<flag_t*>(L->pool + 2 * bufb);
  L->zone_dev = L->pool + 2 * bufb + flagb;
  L->glob_dev = reinterpret_cast<double*>(L->pool + 2 * bufb + flagb + zoneb);
  L->err_dev = reinterpret_cast<int*>(L->pool + 2 * bufb + flagb + zoneb + globb);
  L->count_dev = reinterpret_cast<unsigned*>(L->pool + 2 * bufb + flagb + zoneb + globb + 64);
  e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaFree(L->pool);
    delete L;
    return fail(TCLB_ERR_CUDA, std::string("stream create failed: ") + cudaGetErrorString(e));
  }
  // launch shape: a row of x (multiple of 32), 256 threads per block
  L->bx = nx >= 128 ? 128 : (nx >= 64 ? 64 : 32);
  L->by = 256 / L->bx;
  // settings defaults (src/Solver.cpp.Rt:276-281) and zonal defaults (:393)
  L->settings.assign(T->nsettings, 0.0);
  for (int i = 0; i < T->nsettings; i++)
    if (!std::isnan(T->setting_defaults[i])) L->settings[i] = T->setting_defaults[i];
  L->zone.assign((size_t)L->nzones * T->nzonesettings, 0.0);
  for (int z = 0; z < L->nzones; z++)
    for (int s = 0; s < T->nzonesettings; s++) L->zone[(size_t)z * T->nzonesettings + s] = T->zone_setting_defaults[s];
  L->globals.assign(T->nglobals, 0.0);
  int rc = TCLB_OK;
  if (cudaMemsetAsync(L->pool, 0, total, L->stream) != cudaSuccess) rc = fail(TCLB_ERR_CUDA, "memset of pool failed");
  if (rc == TCLB_OK) rc = upload_zone(L);
  if (rc != TCLB_OK) {
    cudaStreamDestroy(L->stream);
    cudaFree(L->pool);
    delete L;
    return rc;
  }
  setup_tma(L);
  impl->prepare(L);
  *out = L;
  return TCLB_OK;
}

int tclb_destroy(tclb_h L) {
  CHECK_H(L);
  cudaStreamSynchronize(L->stream);
  drop_graphs(L);
  if (L->qbuf) cudaFree(L->qbuf);
  cudaFree(L->pool);
  cudaStreamDestroy(L->stream);
  delete L;
  return TCLB_OK;
}

int tclb_get_size(tclb_h L, int* nx, int* ny, int* nz) {
  CHECK_H(L);
  if (nx) *nx = L->nx;
  if (ny) *ny = L->ny;
  if (nz) *nz = L->nz;
  return TCLB_OK;
}

int tclb_set_flags(tclb_h L, const uint16_t* flags, int dx, int dy, int dz, int nx, int ny, int nz) {
  CHECK_H(L);
  if (!flags) return fail(TCLB_ERR_ARG, "null flags");
  if (dx < 0 || dy < 0 || dz < 0 || nx < 0 || ny < 0 || nz < 0 || dx + nx > L->nx || dy + ny > L->ny ||
      dz + nz > L->nz)
    return fail(TCLB_ERR_ARG, "flag box outside the lattice");
  if (dx == 0 && dy == 0 && dz == 0 && nx == L->nx && ny == L->ny && nz == L->nz) {
    TCLB_CK(cudaMemcpyAsync(L->flags, flags, L->N * sizeof(flag_t), cudaMemcpyHostToDevice, L->stream));
  } else {
    for (int z = 0; z < nz; z++) {
      flag_t* d = L->flags + (size_t)dx + (size_t)L->nx * ((size_t)dy + (size_t)L->ny * (dz + z));
      TCLB_CK(cudaMemcpy2DAsync(d, L->nx * sizeof(flag_t), flags + (size_t)z * nx * ny, nx * sizeof(flag_t),
                                nx * sizeof(flag_t), ny, cudaMemcpyHostToDevice, L->stream));
    }
  }
  TCLB_CK(cudaStreamSynchronize(L->stream));
  const int lanes = L->lanes;
  const int rc = L->impl->flags_changed(L);
  if (rc != TCLB_OK) return rc;
  if (L->lanes != lanes) drop_graphs(L);  // the captured launches name the other kernel
  return TCLB_OK;
}

int tclb_get_flags(tclb_h L, uint16_t* flags) {
  CHECK_H(L);
  TCLB_CK(cudaMemcpyAsync(flags, L->flags, L->N * sizeof(flag_t), cudaMemcpyDeviceToHost, L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return TCLB_OK;
}

int tclb_set_setting(tclb_h L, int i, double v) {
  CHECK_H(L);
  if (i < 0 || i >= L->T->nsettings) return fail(TCLB_ERR_ARG, "setting index out of range");
  drop_graphs(L);
  return set_setting_rec(L, i, v, 0);
}

int tclb_get_setting(tclb_h L, int i, double* v) {
  CHECK_H(L);
  if (i < 0 || i >= L->T->nsettings || !v) return fail(TCLB_ERR_ARG, "setting index out of range");
  *v = L->settings[i];
  return TCLB_OK;
}

int tclb_set_zone_setting(tclb_h L, int s, int zone, double v) {
  CHECK_H(L);
  if (s < 0 || s >= L->T->nzonesettings) return fail(TCLB_ERR_ARG, "zone setting index out of range");
  if (zone < -1 || zone >= L->nzones) return fail(TCLB_ERR_ARG, "zone out of range");
  const int nzs = L->T->nzonesettings;
  if (zone < 0)
    for (int z = 0; z < L->nzones; z++) L->zone[(size_t)z * nzs + s] = v;
  else
    L->zone[(size_t)zone * nzs + s] = v;
  return upload_zone(L);
}

int tclb_get_zone_setting(tclb_h L, int s, int zone, double* v) {
  CHECK_H(L);
  if (s < 0 || s >= L->T->nzonesettings || zone < 0 || zone >= L->nzones || !v)
    return fail(TCLB_ERR_ARG, "zone setting or zone out of range");
  *v = L->zone[(size_t)zone * L->T->nzonesettings + s];
  return TCLB_OK;
}

int tclb_init(tclb_h L) {
  CHECK_H(L);
  L->impl->init(L, L->stream);
  TCLB_CK(cudaGetLastError());
  L->iter = 0;
  std::fill(L->globals.begin(), L->globals.end(), 0.0);
  TCLB_CK(cudaMemsetAsync(L->glob_dev, 0, L->T->nglobals * sizeof(double), L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return TCLB_OK;
}

int tclb_init_equilibrium(tclb_h L, const void* rho, const void* u, void* stream) {
  CHECK_H(L);
  if (!rho || !u) return fail(TCLB_ERR_ARG, "null field");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const size_t rs = L->impl->real_size;
  const size_t bytes = align_up(L->N * rs, 256) + 3 * L->N * rs;
  if (bytes > L->qbuf_bytes) {
    if (L->qbuf) TCLB_CK(cudaFree(L->qbuf));
    L->qbuf = nullptr;
    L->qbuf_bytes = 0;
    TCLB_CK(cudaMalloc(&L->qbuf, bytes));
    L->qbuf_bytes = bytes;
  }
  char* d_rho = static_cast<char*>(L->qbuf);
  char* d_u = d_rho + align_up(L->N * rs, 256);
  TCLB_CK(cudaMemcpyAsync(d_rho, rho, L->N * rs, cudaMemcpyHostToDevice, s));
  TCLB_CK(cudaMemcpyAsync(d_u, u, 3 * L->N * rs, cudaMemcpyHostToDevice, s));
  L->impl->equilibrium(L, d_rho, d_u, s);
  TCLB_CK(cudaGetLastError());
  L->iter = 0;
  std::fill(L->globals.begin(), L->globals.end(), 0.0);
  TCLB_CK(cudaMemsetAsync(L->glob_dev, 0, L->T->nglobals * sizeof(double), s));
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

int tclb_iterate(tclb_h L, int niter, int iter_type, void* stream) {
  CHECK_H(L);
  if (niter < 0) return fail(TCLB_ERR_ARG, "negative iteration count");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  int last_glob = iter_type & TCLB_ITER_LASTGLOB;
  const bool integ = (iter_type & TCLB_ITER_INTEG) == TCLB_ITER_INTEG;
  if (integ) last_glob = 0;
  bool globs = (iter_type & TCLB_ITER_GLOBS) != 0;
  int i = 0;
  if (!globs && L->use_graphs) {
    // plain iterations in graph replays of GRAPH_CHUNK (even: the snapshot
    // parity is unchanged by a replay)
    const int plain = niter - (last_glob ? 1 : 0);
    while (plain - i >= GRAPH_CHUNK) {
      int rc = ensure_iter_graph(L, s);
      if (rc) return rc;
      TCLB_CK(cudaGraphLaunch(L->graph[L->cur], s));
      i += GRAPH_CHUNK;
      L->iter += GRAPH_CHUNK;
    }
  }
  for (; i < niter; i++) {
    if (last_glob && i == niter - 1) {
      TCLB_CK(cudaMemsetAsync(L->glob_dev, 0, L->T->nglobals * sizeof(double), s));
      globs = true;
    }
    L->impl->iterate(L, globs, s);
    L->cur = 1 - L->cur;
    L->iter++;
  }
  TCLB_CK(cudaGetLastError());
  if (last_glob && niter > 0) {
    std::fill(L->globals.begin(), L->globals.end(), 0.0);
    return calc_globals(L, s);
  } else if (integ && niter > 0) {
    return calc_globals(L, s);
  }
  return TCLB_OK;
}

int tclb_get_globals(tclb_h L, double* out) {
  CHECK_H(L);
  if (!out) return fail(TCLB_ERR_ARG, "null output");
  std::copy(L->globals.begin(), L->globals.end(), out);
  return TCLB_OK;
}

int tclb_clear_globals(tclb_h L) {
  CHECK_H(L);
  std::fill(L->globals.begin(), L->globals.end(), 0.0);
  return TCLB_OK;
}

int tclb_get_quantity(tclb_h L, int q, const int region[6], void* out, double scale, void* stream) {
  CHECK_H(L);
  if (q < 0 || q >= L->T->nquantities) return fail(TCLB_ERR_ARG, "quantity index out of range");
  if (!out) return fail(TCLB_ERR_ARG, "null output");
  int r[6] = {0, 0, 0, L->nx, L->ny, L->nz};
  if (region) std::memcpy(r, region, sizeof(r));
  if (r[0] < 0 || r[1] < 0 || r[2] < 0 || r[3] < 1 || r[4] < 1 || r[5] < 1 || r[0] + r[3] > L->nx ||
      r[1] + r[4] > L->ny || r[2] + r[5] > L->nz)
    return fail(TCLB_ERR_ARG, "quantity region outside the lattice");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const int vec = L->T->quantity_vector[q];
  const size_t bytes = (size_t)r[3] * r[4] * r[5] * (vec ? 3 : 1) * L->impl->real_size;
  if (bytes > L->qbuf_bytes) {
    if (L->qbuf) TCLB_CK(cudaFree(L->qbuf));
    L->qbuf = nullptr;
    L->qbuf_bytes = 0;
    TCLB_CK(cudaMalloc(&L->qbuf, bytes));
    L->qbuf_bytes = bytes;
  }
  L->impl->quantity(L, q, vec, r, scale, L->qbuf, s);
  TCLB_CK(cudaGetLastError());
  TCLB_CK(cudaMemcpyAsync(out, L->qbuf, bytes, cudaMemcpyDeviceToHost, s));
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

int tclb_energy_enstrophy(tclb_h L, double* out, void* stream) {
  CHECK_H(L);
  if (!out) return fail(TCLB_ERR_ARG, "null output");
  int q = -1;
  for (int i = 0; i < L->T->nquantities; i++)
    if (std::strcmp(L->T->quantity_names[i], "U") == 0) q = i;
  if (q < 0) return fail(TCLB_ERR_ARG, "model has no U quantity");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const size_t ub = align_up(3 * L->N * L->impl->real_size, 256);
  const size_t bytes = ub + 256;
  if (bytes > L->qbuf_bytes) {
    if (L->qbuf) TCLB_CK(cudaFree(L->qbuf));
    L->qbuf = nullptr;
    L->qbuf_bytes = 0;
    TCLB_CK(cudaMalloc(&L->qbuf, bytes));
    L->qbuf_bytes = bytes;
  }
  const int r[6] = {0, 0, 0, L->nx, L->ny, L->nz};
  L->impl->quantity(L, q, 1, r, 1.0, L->qbuf, s);
  double* acc = reinterpret_cast<double*>(static_cast<char*>(L->qbuf) + ub);
  TCLB_CK(cudaMemsetAsync(acc, 0, 2 * sizeof(double), s));
  const int blocks = (int)std::min<size_t>((L->N + 255) / 256, 148 * 8);
  if (L->precision == TCLB_FP64)
    k_energy_enstrophy<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(L->qbuf), L->nx, L->ny, L->nz, acc);
  else
    k_energy_enstrophy<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(L->qbuf), L->nx, L->ny, L->nz, acc);
  TCLB_CK(cudaGetLastError());
  TCLB_CK(cudaMemcpyAsync(out, acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

int tclb_color(tclb_h L, void* rgba, int z, int on_host, void* stream) {
  CHECK_H(L);
  if (!rgba) return fail(TCLB_ERR_ARG, "null output");
  if (z < 0) z = L->nz / 2;  // LatticeContainer::Color draws plane nz/2
  if (z >= L->nz) return fail(TCLB_ERR_ARG, "plane outside the lattice");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const size_t bytes = (size_t)L->nx * L->ny * 4;
  if (!on_host) {
    L->impl->color(L, z, rgba, s);
    TCLB_CK(cudaGetLastError());
    return TCLB_OK;
  }
  if (bytes > L->qbuf_bytes) {
    if (L->qbuf) TCLB_CK(cudaFree(L->qbuf));
    L->qbuf = nullptr;
    L->qbuf_bytes = 0;
    TCLB_CK(cudaMalloc(&L->qbuf, bytes));
    L->qbuf_bytes = bytes;
  }
  L->impl->color(L, z, L->qbuf, s);
  TCLB_CK(cudaGetLastError());
  TCLB_CK(cudaMemcpyAsync(rgba, L->qbuf, bytes, cudaMemcpyDeviceToHost, s));
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

int tclb_get_densities(tclb_h L, double* out) {
  CHECK_H(L);
  if (!out) return fail(TCLB_ERR_ARG, "null output");
  std::vector<char> raw(L->stride * L->T->Q * L->elem);
  TCLB_CK(cudaMemcpyAsync(raw.data(), L->buf[L->cur], raw.size(), cudaMemcpyDeviceToHost, L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  L->impl->to_double(raw.data(), L->N, L->stride, L->elem, L->T->Q, out);
  return TCLB_OK;
}

int tclb_set_densities(tclb_h L, const double* in) {
  CHECK_H(L);
  if (!in) return fail(TCLB_ERR_ARG, "null input");
  std::vector<char> raw(L->stride * L->T->Q * L->elem, 0);
  L->impl->from_double(in, L->N, L->stride, L->elem, L->T->Q, raw.data());
  TCLB_CK(cudaMemcpyAsync(L->buf[L->cur], raw.data(), raw.size(), cudaMemcpyHostToDevice, L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return TCLB_OK;
}

size_t tclb_snapshot_bytes(tclb_h L) { return L ? L->N * L->T->Q * L->elem : 0; }

int tclb_save(tclb_h L, void* host, size_t bytes, void* stream) {
  CHECK_H(L);
  if (!host || bytes != tclb_snapshot_bytes(L)) return fail(TCLB_ERR_ARG, "snapshot buffer size mismatch");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const size_t plane = L->N * L->elem;
  if (L->stride == L->N) {
    TCLB_CK(cudaMemcpyAsync(host, L->buf[L->cur], bytes, cudaMemcpyDeviceToHost, s));
  } else {
    for (int q = 0; q < L->T->Q; q++)
      TCLB_CK(cudaMemcpyAsync(static_cast<char*>(host) + q * plane,
                              static_cast<char*>(L->buf[L->cur]) + q * L->stride * L->elem, plane,
                              cudaMemcpyDeviceToHost, s));
  }
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

int tclb_load(tclb_h L, const void* host, size_t bytes, void* stream) {
  CHECK_H(L);
  if (!host || bytes != tclb_snapshot_bytes(L)) return fail(TCLB_ERR_ARG, "snapshot buffer size mismatch");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
  const size_t plane = L->N * L->elem;
  if (L->stride == L->N) {
    TCLB_CK(cudaMemcpyAsync(L->buf[L->cur], host, bytes, cudaMemcpyHostToDevice, s));
  } else {
    for (int q = 0; q < L->T->Q; q++)
      TCLB_CK(cudaMemcpyAsync(static_cast<char*>(L->buf[L->cur]) + q * L->stride * L->elem,
                              static_cast<const char*>(host) + q * plane, plane, cudaMemcpyHostToDevice, s));
  }
  TCLB_CK(cudaStreamSynchronize(s));
  return TCLB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// TCLB's .pri snapshot (Lattice::save / load, src/Lattice.cu.Rt:642-769): the
// non-empty margin blocks of a snapshot, block k = 1..27 with offsets
// (dx,dy,dz) = ((k-1)%3-1, ((k-1)/3)%3-1, (k-1)/9-1), concatenated. Block
// (0,0,0) is the interior. Density i (velocity e) is a field spanning
// offsets -e (src/conf.R:65-100, AddDensity -> AddField(dx=-dx)), so it owns
// a box in every block d with d_a in {0, -e_a} on each axis; boxes are
// x-fastest, fields in density order within a block, values in storage_t
// (src/conf.R:905-1000, default GPU layout: no X_MOD, no CPU layout).
//
// Where a node's value is written (the put of src/conf.R:978-983 driven by
// if.apply in src/LatticeAccess.inc.cpp.Rt:83-117): a node on the outgoing
// edge of axis a (e_a = +1 at n_a-1, e_a = -1 at 0) writes density i into
// the margin d_a = -e_a at position 0; every other node writes it in place.
// Models that also register the densities as unshifted fields (d3q27_cumulant,
// models/flow/d3q27_cumulant/Dynamics.R:51) write the edge node in place too,
// so their interior is complete; in d2q9 and d3q19 those interior slots are
// never written and stay zero (the snapshot is zeroed at allocation,
// src/LatticeContainer.inc.cpp.Rt:119). On one rank the margin d_a = -1
// is what node 0 pulls: the periodic wrap.
// ---------------------------------------------------------------------------
namespace {
struct PriBlock {
  int d[3];
  std::vector<int> fields;
  int n[3];
};

struct PriLayout {
  std::vector<PriBlock> blocks;
  std::vector<std::array<int, 3>> e;  // velocity of each density
  bool interior_copy;                 // edge nodes also written in place
  int dims[3];

  // true when slot (block b, density i, node n) is written by node n's put
  bool written(const PriBlock& b, int i, const int* n) const {
    for (int a = 0; a < 3; a++) {
      if (b.d[a] != 0) continue;
      const bool outgoing = (e[i][a] == 1 && n[a] == dims[a] - 1) || (e[i][a] == -1 && n[a] == 0);
      if (outgoing && !interior_copy) return false;
    }
    return true;
  }
  // true when block b is where node n's density i is pulled from
  bool primary(const PriBlock& b, int i, const int* n) const {
    for (int a = 0; a < 3; a++) {
      const bool outgoing = (e[i][a] == 1 && n[a] == dims[a] - 1) || (e[i][a] == -1 && n[a] == 0);
      if (b.d[a] != (outgoing ? -e[i][a] : 0)) return false;
    }
    return true;
  }
};

template <class M>
PriLayout pri_layout_m(int nx, int ny, int nz, bool interior_copy) {
  PriLayout L;
  L.dims[0] = nx;
  L.dims[1] = ny;
  L.dims[2] = nz;
  L.interior_copy = interior_copy;
  for (int i = 0; i < M::Q; i++) L.e.push_back({M::ex(i), M::ey(i), M::ez(i)});
  for (int k = 0; k < 27; k++) {
    PriBlock b;
    b.d[0] = k % 3 - 1;
    b.d[1] = (k / 3) % 3 - 1;
    b.d[2] = k / 9 - 1;
    for (int i = 0; i < M::Q; i++) {
      bool in = true;
      for (int a = 0; a < 3; a++) in = in && (b.d[a] == 0 || L.e[i][a] == -b.d[a]);
      if (in) b.fields.push_back(i);
    }
    for (int a = 0; a < 3; a++) b.n[a] = b.d[a] == 0 ? L.dims[a] : 1;
    if (!b.fields.empty()) L.blocks.push_back(b);
  }
  return L;
}

PriLayout pri_layout(const tclb_lattice* L) {
  switch (L->model) {
    case MODEL_D2Q9: return pri_layout_m<D2Q9>(L->nx, L->ny, L->nz, false);
    case MODEL_D3Q19: return pri_layout_m<D3Q19>(L->nx, L->ny, L->nz, false);
    default: return pri_layout_m<D3Q27C>(L->nx, L->ny, L->nz, true);
  }
}

size_t pri_size(const tclb_lattice* L) {
  size_t s = 0;
  for (const auto& b : pri_layout(L).blocks) s += b.fields.size() * (size_t)b.n[0] * b.n[1] * b.n[2] * L->elem;
  return s;
}

// Calls f(block, density, node, byte offset in the file) for every slot.
template <class F>
void pri_for_each(const tclb_lattice* L, const PriLayout& P, F&& f) {
  size_t off = 0;
  for (const auto& b : P.blocks)
    for (int i : b.fields)
      for (int z = 0; z < b.n[2]; z++)
        for (int y = 0; y < b.n[1]; y++)
          for (int x = 0; x < b.n[0]; x++) {
            const int p[3] = {x, y, z};
            int n[3];
            for (int a = 0; a < 3; a++) n[a] = b.d[a] < 0 ? P.dims[a] - 1 : (b.d[a] > 0 ? 0 : p[a]);
            f(b, i, n, off);
            off += L->elem;
          }
}
}  // namespace

extern "C" {

size_t tclb_pri_bytes(tclb_h L) { return L ? pri_size(L) : 0; }

int tclb_save_pri(tclb_h L, void* host, size_t bytes) {
  CHECK_H(L);
  if (!host || bytes != pri_size(L)) return fail(TCLB_ERR_ARG, ".pri buffer size mismatch");
  std::vector<char> raw(L->stride * L->T->Q * L->elem);
  TCLB_CK(cudaMemcpyAsync(raw.data(), L->buf[L->cur], raw.size(), cudaMemcpyDeviceToHost, L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  char* o = static_cast<char*>(host);
  const size_t e = L->elem;
  const PriLayout P = pri_layout(L);
  pri_for_each(L, P, [&](const PriBlock& b, int i, const int* n, size_t off) {
    if (P.written(b, i, n)) {
      const size_t node = (size_t)n[0] + (size_t)L->nx * ((size_t)n[1] + (size_t)L->ny * n[2]);
      std::memcpy(o + off, raw.data() + ((size_t)i * L->stride + node) * e, e);
    } else {
      std::memset(o + off, 0, e);
    }
  });
  return TCLB_OK;
}

int tclb_load_pri(tclb_h L, const void* host, size_t bytes) {
  CHECK_H(L);
  if (!host || bytes != pri_size(L)) return fail(TCLB_ERR_ARG, ".pri buffer size mismatch");
  const char* in = static_cast<const char*>(host);
  const size_t e = L->elem;
  std::vector<char> raw(L->stride * L->T->Q * L->elem, 0);
  const PriLayout P = pri_layout(L);
  pri_for_each(L, P, [&](const PriBlock& b, int i, const int* n, size_t off) {
    if (!P.primary(b, i, n)) return;  // each node's value is taken from the block it is pulled from
    const size_t node = (size_t)n[0] + (size_t)L->nx * ((size_t)n[1] + (size_t)L->ny * n[2]);
    std::memcpy(raw.data() + ((size_t)i * L->stride + node) * e, in + off, e);
  });
  TCLB_CK(cudaMemcpyAsync(L->buf[L->cur], raw.data(), raw.size(), cudaMemcpyHostToDevice, L->stream));
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return TCLB_OK;
}

int tclb_get_iteration(tclb_h L, long long* iter) {
  CHECK_H(L);
  if (iter) *iter = L->iter;
  return TCLB_OK;
}

double tclb_bytes_per_update(tclb_h L) { return L ? 2.0 * L->T->Q * L->elem + sizeof(flag_t) : 0.0; }

int tclb_set_launch(tclb_h L, int bx, int by, int flags) {
  CHECK_H(L);
  if (bx < 32 || bx % 32 || by < 1 || bx * by > 256) return fail(TCLB_ERR_ARG, "bad block shape");
  drop_graphs(L);
  L->bx = bx;
  L->by = by;
  L->use_graphs = (flags & TCLB_LAUNCH_GRAPHS) ? 1 : 0;
  L->use_pairs = (flags & TCLB_LAUNCH_PAIRS) ? 1 : 0;
  L->use_tma = (flags & TCLB_LAUNCH_TMA) ? 1 : 0;
  L->tma_always = (flags & TCLB_LAUNCH_TMA_ALWAYS) ? 1 : 0;
  return TCLB_OK;
}

int tclb_set_fault_injection(tclb_h L, int tile, long long wait_cycles) {
  CHECK_H(L);
  if (tile < -1) return fail(TCLB_ERR_ARG, "fault injection: tile must be -1 (off) or a tile index");
  if (wait_cycles < 0 || wait_cycles > TMA_WAIT_CYCLES) return fail(TCLB_ERR_ARG, "fault injection: wait bound out of range");
  drop_graphs(L);  // the kernel parameters are part of the captured launches
  L->fault_tile = tile;
  L->wait_cycles = wait_cycles ? wait_cycles : TMA_WAIT_CYCLES;
  return TCLB_OK;
}

int tclb_get_launch(tclb_h L, int* bx, int* by, int* flags) {
  CHECK_H(L);
  if (bx) *bx = L->bx;
  if (by) *by = L->by;
  if (flags) {
    const bool tma = tma_path(L);
    const bool pairs = !tma && L->use_pairs && L->elem == 2 && L->nx % 64 == 0;
    *flags = (L->use_graphs ? TCLB_LAUNCH_GRAPHS : 0) | (pairs ? TCLB_LAUNCH_PAIRS : 0) | (tma ? TCLB_LAUNCH_TMA : 0);
  }
  return TCLB_OK;
}

int tclb_sync(tclb_h L) {
  CHECK_H(L);
  TCLB_CK(cudaStreamSynchronize(L->stream));
  return check_device_error(L, L->stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Quantity read-out that allocates no device memory.
//
// tclb_get_quantity stages the quantity in a device buffer that it grows with
// cudaMalloc. Some callers cannot allow that: a host application that has
// handed the whole GPU to its own memory pool or admission budget (a
// cudaMalloc there can fail, or break the budget the pool enforces), and code
// on a latency-critical path, where cudaMalloc/cudaFree may synchronise the
// device and stall unrelated streams. For them this variant stages the
// quantity in a fixed device array that is part of the library image.
//
// The array is TCLB_NOALLOC_SCRATCH_BYTES (8 MiB) of device memory held by
// every GPU that loads the library, until the process exits. Regions whose
// quantity needs more are rejected. All calls share the array and it keeps
// the last call's contents; the quantity kernel overwrites every byte a call
// reads back, so nothing needs clearing. Calls that overlap on the GPU (other
// host threads, or other streams without ordering between them) race on the
// array.
// ---------------------------------------------------------------------------
#define TCLB_NOALLOC_SCRATCH_BYTES (8u << 20)
#define TCLB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[TCLB_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_address[TCLB_NOALLOC_MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on `dev`, which must be current. In host
// code the array's name is only a host-side stand-in, so the address is looked
// up once per device with cudaGetSymbolAddress and cached.
int noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= TCLB_NOALLOC_MAX_DEVICES) return fail(TCLB_ERR_ARG, "device ordinal above the no-allocation table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_address[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(TCLB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
    g_noalloc_address[dev] = p;
  }
  *out = g_noalloc_address[dev];
  return TCLB_OK;
}
}  // namespace

extern "C" int tclb_get_quantity_noalloc(tclb_h L, int q, const int region[6], void* out, double scale,
                                         void* stream) {
  CHECK_H(L);
  if (q < 0 || q >= L->T->nquantities) return fail(TCLB_ERR_ARG, "quantity index out of range");
  if (!out) return fail(TCLB_ERR_ARG, "null output");
  int r[6] = {0, 0, 0, L->nx, L->ny, L->nz};
  if (region) std::memcpy(r, region, sizeof(r));
  if (r[0] < 0 || r[1] < 0 || r[2] < 0 || r[3] < 1 || r[4] < 1 || r[5] < 1 || r[0] + r[3] > L->nx ||
      r[1] + r[4] > L->ny || r[2] + r[5] > L->nz)
    return fail(TCLB_ERR_ARG, "quantity region outside the lattice");
  const int vec = L->T->quantity_vector[q];
  const size_t bytes = (size_t)r[3] * r[4] * r[5] * (vec ? 3 : 1) * L->impl->real_size;
  if (bytes > TCLB_NOALLOC_SCRATCH_BYTES)
    return fail(TCLB_ERR_ARG, "region needs " + std::to_string(bytes) +
                                  " bytes of scratch, above the no-allocation limit of " +
                                  std::to_string(TCLB_NOALLOC_SCRATCH_BYTES) + " bytes; use tclb_get_quantity");
  int prev = -1;
  TCLB_CK(cudaGetDevice(&prev));
  if (prev != L->device) TCLB_CK(cudaSetDevice(L->device));
  void* scratch = nullptr;
  int rc = noalloc_scratch(L->device, &scratch);
  if (rc == TCLB_OK) {
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    L->impl->quantity(L, q, vec, r, scale, scratch, s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(TCLB_ERR_CUDA, std::string("no-allocation quantity: ") + cudaGetErrorString(e));
  }
  if (prev != L->device) {
    const cudaError_t e = cudaSetDevice(prev);
    if (e != cudaSuccess && rc == TCLB_OK)
      rc = fail(TCLB_ERR_CUDA, std::string("no-allocation quantity: could not restore the caller's device: ") +
                                   cudaGetErrorString(e));
  }
  return rc;
}
