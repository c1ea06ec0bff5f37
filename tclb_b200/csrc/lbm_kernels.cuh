// Device code of the B200 lattice-Boltzmann engine: storage policies, the
// per-node physics of the d2q9, d3q19 and d3q27_cumulant models, and the
// fused pull-stream + collide + Globals kernel.
//
// Layout: densities are SoA, one plane of N = nx*ny*nz values per population,
// planes 256-byte aligned (stride in elements), node index x + nx*(y + ny*z).
// Two snapshots are kept (A/B); an iteration pulls f_i(x) from A at x - e_i
// with periodic wrap on every axis (TCLB's single-rank margins,
// src/Global.cpp.Rt:61-82, src/Lattice.cu.Rt:439-456), runs the node update
// and stores f_i(x) into B (src/LatticeAccess.inc.cpp.Rt:299-347).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

#include "f32x2.cuh"
#include "tclb_models.h"

namespace tclb {

// ---------------------------------------------------------------------------
// Storage policies: storage_t <-> real_t (src/LatticeAccess.inc.cpp.Rt:14-35).
// Shifted formats store (f - w_i) and add w_i back on load.
// ---------------------------------------------------------------------------
struct StoreF64 {
  typedef double T;
  static constexpr bool shifted = false;
  template <class R>
  __device__ __forceinline__ static R load(const T* p, R) { return (R)__ldg(p); }
  template <class R>
  __device__ __forceinline__ static void store(T* p, R v, R) { __stcs(p, (double)v); }
  __host__ static T from_double(double v, double) { return v; }
  __host__ static double to_double(T v, double) { return v; }
};
struct StoreF32 {
  typedef float T;
  static constexpr bool shifted = false;
  template <class R>
  __device__ __forceinline__ static R load(const T* p, R) { return (R)__ldg(p); }
  template <class R>
  __device__ __forceinline__ static void store(T* p, R v, R) { __stcs(p, (float)v); }
  __host__ static T from_double(double v, double) { return (float)v; }
  __host__ static double to_double(T v, double) { return v; }
};
template <bool SHIFT>
struct StoreF16 {
  typedef __half T;
  static constexpr bool shifted = SHIFT;
  template <class R>
  __device__ __forceinline__ static R load(const T* p, R s) {
    float v = __half2float(__ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(p))));
    return SHIFT ? (R)v + s : (R)v;
  }
  template <class R>
  __device__ __forceinline__ static void store(T* p, R v, R s) {
    __half h = __float2half_rn((float)(SHIFT ? v - s : v));
    __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(h));
  }
  __host__ static T from_double(double v, double s) { return __float2half_rn((float)(SHIFT ? v - s : v)); }
  __host__ static double to_double(T v, double s) { return (double)__half2float(v) + (SHIFT ? s : 0.0); }
};
template <bool SHIFT>
struct StoreBF16 {
  typedef __nv_bfloat16 T;
  static constexpr bool shifted = SHIFT;
  template <class R>
  __device__ __forceinline__ static R load(const T* p, R s) {
    unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
    float v = __uint_as_float(((unsigned)u) << 16);
    return SHIFT ? (R)v + s : (R)v;
  }
  template <class R>
  __device__ __forceinline__ static void store(T* p, R v, R s) {
    __nv_bfloat16 h = __float2bfloat16_rn((float)(SHIFT ? v - s : v));
    __stcs(reinterpret_cast<unsigned short*>(p), *reinterpret_cast<unsigned short*>(&h));
  }
  __host__ static T from_double(double v, double s) { return __float2bfloat16_rn((float)(SHIFT ? v - s : v)); }
  __host__ static double to_double(T v, double s) { return (double)__bfloat162float(v) + (SHIFT ? s : 0.0); }
};

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------
template <class R, int NSET>
struct Args {
  typedef R real;
  const void* src;
  void* dst;
  size_t stride;  // elements between population planes
  const flag_t* flags;
  int nx, ny, nz;
  const R* zone;  // [zones][NZS] zonal settings
  double* glob;   // device Globals (FP64)
  R s[NSET];      // settings
  R k[4];         // per-launch constants derived from the settings (Model::derived)
};

// AddTo<Global>(x) with TCLB's Objective rule: every AddTo of a SUM Global
// also adds that Global's zonal <Global>InObj weight to Objective
// (src/cuda.cu.Rt:114-119).
template <int NSUM, int OBJ, int INOBJ, class R>
__device__ __forceinline__ void add_glob(R* g, int i, R x, const R* zs) {
  g[i] += x;
  if (i < NSUM) g[OBJ] += zs[i + INOBJ];
}

// ---------------------------------------------------------------------------
// d2q9 (models/flow/d2q9/Dynamics.c.Rt), plain variant (bc=FALSE)
// ---------------------------------------------------------------------------
struct D2Q9 {
  static constexpr int Q = 9, DIM = 2, NSET = d2q9::NSET, NZS = d2q9::NZS, NG = d2q9::NG, NSUM = d2q9::NSUM,
                       ZONE_SHIFT = d2q9::ZONE_SHIFT;
  // staged batch cases keep their own settings (no shared settings group):
  // the cases of a batch differ in viscosity
  static constexpr bool has_bulk = false;
  static constexpr bool packed = true;  // one packed FP32x2 collision for a node pair
  static constexpr bool identity_lanes = false;
  static constexpr int PAIR_THREADS = 256, PAIR_MIN_BLOCKS = 4;  // <= 64 registers
  static constexpr int BATCH_MIN_BLOCKS = 6;  // one-tile batch kernel: <= 40 registers
  template <class R>
  __host__ __device__ static void derived(const R*, R* k) { k[0] = k[1] = k[2] = k[3] = R(0); }
  __host__ __device__ static constexpr int ex(int i) { return (i == 1 || i == 5 || i == 8) ? 1 : ((i == 3 || i == 6 || i == 7) ? -1 : 0); }
  __host__ __device__ static constexpr int ey(int i) { return (i == 2 || i == 5 || i == 6) ? 1 : ((i == 4 || i == 7 || i == 8) ? -1 : 0); }
  __host__ __device__ static constexpr int ez(int) { return 0; }
  __host__ __device__ static constexpr int opp(int i) { return i == 0 ? 0 : (i <= 4 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5); }
  __host__ __device__ static constexpr double w(int i) { return i == 0 ? 4.0 / 9.0 : (i <= 4 ? 1.0 / 9.0 : 1.0 / 36.0); }

  template <class R>
  __device__ __forceinline__ static void glob(R* g, int i, R x, const R* zs) {
    add_glob<NSUM, d2q9::G_Objective, d2q9::IN_OBJ_OFFSET>(g, i, x, zs);
  }

  template <class R>
  __device__ __forceinline__ static void bounce(R (&f)[Q]) {
    R t;
    t = f[1]; f[1] = f[3]; f[3] = t;
    t = f[2]; f[2] = f[4]; f[4] = t;
    t = f[5]; f[5] = f[7]; f[7] = t;
    t = f[6]; f[6] = f[8]; f[8] = t;
  }

  // ZouHeRewrite (lib/boundary.R:143-198) solved in closed form for the D2Q9
  // second-order equilibrium. Outward normal n = SG*e_AX; unknowns have
  // e.n < 0 and become f_opp + (feq_i - feq_opp)(R) = f_opp + 6 w_i e_i.R.
  template <int AX, int SG, bool VEL, class R>
  __device__ __forceinline__ static void zouhe(R (&f)[Q], R vx, R vy, R rho0) {
    R S = 0, T = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) {
      const int ea = AX == 0 ? ex(i) : ey(i), et = AX == 0 ? ey(i) : ex(i);
      if (ea == 0) { S += f[i]; T += (R)et * f[i]; }
      else if (SG * ea > 0) S += R(2) * f[i];
    }
    R Rn, Rt;
    if (VEL) {
      const R vn = AX == 0 ? vx : vy, vt = AX == 0 ? vy : vx;
      Rn = vn * S / (R(1) + R(SG) * vn);
      const R rho = S - R(SG) * Rn;
      Rt = R(3) * (vt * rho - T);
    } else {
      Rn = R(SG) * (S - rho0);
      Rt = R(-3) * T;
    }
#pragma unroll
    for (int i = 0; i < Q; i++) {
      const int ea = AX == 0 ? ex(i) : ey(i), et = AX == 0 ? ey(i) : ex(i);
      if (SG * ea < 0) f[i] = f[opp(i)] + R(6.0 * w(i)) * (R(ea) * Rn + R(et) * Rt);
    }
  }

  // Equilibrium / MRT moments in the Cholesky-weighted basis
  // (d2q9/Dynamics.c.Rt:8-23): columns 1, x, y, 3x^2-1, 3y^2-1, 3xy,
  // 3x^2y-y, 3xy^2-x, 9x^2y^2-3x^2-3y^2+1 with norms 1,1/3,1/3,2,2,1,2/3,2/3,4.
  template <class R>
  __device__ __forceinline__ static void from_moments(R (&f)[Q], R rho, R jx, R jy, R m3, R m4, R m5, R m6, R m7, R m8) {
    const R r0 = rho, r1 = R(3) * jx, r2 = R(3) * jy, r3 = R(0.5) * m3, r4 = R(0.5) * m4, r5 = m5, r6 = R(1.5) * m6,
            r7 = R(1.5) * m7, r8 = R(0.25) * m8;
    const R a = r0 + R(2) * (r3 + r4) + R(4) * r8;
    f[0] = R(4.0 / 9.0) * (r0 - r3 - r4 + r8);
    f[1] = R(1.0 / 9.0) * (r0 + r1 + R(2) * r3 - r4 - r7 - R(2) * r8);
    f[2] = R(1.0 / 9.0) * (r0 + r2 - r3 + R(2) * r4 - r6 - R(2) * r8);
    f[3] = R(1.0 / 9.0) * (r0 - r1 + R(2) * r3 - r4 + r7 - R(2) * r8);
    f[4] = R(1.0 / 9.0) * (r0 - r2 - r3 + R(2) * r4 + r6 - R(2) * r8);
    f[5] = R(1.0 / 36.0) * (a + r1 + r2 + R(3) * r5 + R(2) * r6 + R(2) * r7);
    f[6] = R(1.0 / 36.0) * (a - r1 + r2 - R(3) * r5 + R(2) * r6 - R(2) * r7);
    f[7] = R(1.0 / 36.0) * (a - r1 - r2 + R(3) * r5 - R(2) * r6 - R(2) * r7);
    f[8] = R(1.0 / 36.0) * (a + r1 - r2 - R(3) * r5 - R(2) * r6 + R(2) * r7);
  }

  template <class R, bool G>
  __device__ __forceinline__ static void mrt(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g, const R* zs) {
    const R d = f[5] + f[6] + f[7] + f[8];
    const R rho = f[0] + f[1] + f[2] + f[3] + f[4] + d;
    R jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    R jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    R m3 = -f[0] + R(2) * (f[1] + f[3]) - f[2] - f[4] + R(2) * d;
    R m4 = -f[0] - f[1] - f[3] + R(2) * (f[2] + f[4]) + R(2) * d;
    R m5 = R(3) * (f[5] - f[6] + f[7] - f[8]);
    R m6 = f[4] - f[2] + R(2) * (f[5] + f[6] - f[7] - f[8]);
    R m7 = f[3] - f[1] + R(2) * (f[5] - f[6] - f[7] + f[8]);
    R m8 = f[0] - R(2) * (f[1] + f[2] + f[3] + f[4]) + R(4) * d;
    const R irho = R(1) / rho;
    if (G) {  // d2q9/Dynamics.c.Rt:228-246 (pre-relaxation rho, J)
      const unsigned obj = fl & d2q9::OBJECTIVE;
      if (obj) {
        const R usq = (jx * jx + jy * jy) / (rho * rho);
        const R flux = jx / rho / rho;
        const R pl = flux * ((rho - R(1)) / R(3) + usq / rho / R(2));
        if (obj == d2q9::Outlet) { glob(g, d2q9::G_OutletFlux, flux, zs); glob(g, d2q9::G_PressureLoss, -pl, zs); }
        else if (obj == d2q9::Inlet) { glob(g, d2q9::G_InletFlux, flux, zs); glob(g, d2q9::G_PressureLoss, pl, zs); }
      }
    }
    const R S2 = a.s[d2q9::S_S2], S3 = a.s[d2q9::S_S3], S4 = a.s[d2q9::S_S4];
    m3 = S2 * (m3 - R(3) * jx * jx * irho);
    m4 = S2 * (m4 - R(3) * jy * jy * irho);
    m5 = S2 * (m5 - R(3) * jx * jy * irho);
    m6 = S3 * m6;
    m7 = S3 * m7;
    m8 = S4 * m8;
    jx = jx + a.s[d2q9::S_GravitationX] * rho;
    jy = jy + a.s[d2q9::S_GravitationY] * rho;
    m3 += R(3) * jx * jx * irho;
    m4 += R(3) * jy * jy * irho;
    m5 += R(3) * jx * jy * irho;
    from_moments(f, rho, jx, jy, m3, m4, m5, m6, m7, m8);
  }

  template <class R, bool G>
  __device__ __forceinline__ static void run(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g) {
    boundaries(f, fl, a);
    if (fl & d2q9::MRT) mrt<R, G>(f, fl, a, g, a.zone + (fl >> ZONE_SHIFT) * NZS);
  }

  template <class R, class AR>
  __device__ __forceinline__ static void boundaries(R (&f)[Q], flag_t fl, const AR& a) {
    const unsigned b = fl & d2q9::BOUNDARY;
    if (b) {
      const auto* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
      const R vx = zs[d2q9::Z_VelocityX], vy = zs[d2q9::Z_VelocityY], rho0 = zs[d2q9::Z_Pressure] * R(3) + R(1);
      switch (b) {  // d2q9/Dynamics.c.Rt:108-138
        case d2q9::Solid:
        case d2q9::Wall: bounce(f); break;
        case d2q9::EVelocity: zouhe<0, 1, true>(f, vx, vy, rho0); break;
        case d2q9::WPressure: zouhe<0, -1, false>(f, vx, vy, rho0); break;
        case d2q9::WVelocity: zouhe<0, -1, true>(f, vx, vy, rho0); break;
        case d2q9::EPressure: zouhe<0, 1, false>(f, vx, vy, rho0); break;
        case d2q9::NVelocity: zouhe<1, 1, true>(f, vx, vy, rho0); break;
        case d2q9::SVelocity: zouhe<1, -1, true>(f, vx, vy, rho0); break;
        case d2q9::NSymmetry: f[4] = f[2]; f[7] = f[6]; f[8] = f[5]; break;  // Symmetry(2,-1)
        case d2q9::SSymmetry: f[2] = f[4]; f[6] = f[7]; f[5] = f[8]; break;  // Symmetry(2, 1)
        default: break;
      }
    }
  }

  // Two nodes with one packed collision (plain iterations): boundaries per
  // node, then the MRT update of mrt() on both lanes; a lane whose node does
  // not collide keeps its values (pair_update_store parks them). With DEV the
  // values are deviations g = f - w: the weights' MRT moments are all zero
  // but the density (1), so the moments of g are those of f with rho - 1,
  // which enters the linear terms (from_moments is linear, its rho part
  // weighted by w), while the quadratic equilibrium terms and the force use
  // the true density.
  __device__ __forceinline__ static bool collides(flag_t fl) { return (fl & d2q9::MRT) != 0; }
  __device__ __forceinline__ static bool has_boundary(flag_t fl) { return (fl & d2q9::BOUNDARY) != 0; }
  template <class R, class AR>
  __device__ __forceinline__ static void pre_collision(R (&f)[Q], flag_t fl, const AR& a) {
    boundaries(f, fl, a);
  }
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair(F2 (&f)[Q], flag_t, flag_t, const AR& a) {
    const F2 d = f[5] + f[6] + f[7] + f[8];
    const F2 rho = f[0] + f[1] + f[2] + f[3] + f[4] + d;  // rho - 1 with DEV
    F2 jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    F2 jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    F2 m3 = -f[0] + F2(2.0f) * (f[1] + f[3]) - f[2] - f[4] + F2(2.0f) * d;
    F2 m4 = -f[0] - f[1] - f[3] + F2(2.0f) * (f[2] + f[4]) + F2(2.0f) * d;
    F2 m5 = F2(3.0f) * (f[5] - f[6] + f[7] - f[8]);
    F2 m6 = f[4] - f[2] + F2(2.0f) * (f[5] + f[6] - f[7] - f[8]);
    F2 m7 = f[3] - f[1] + F2(2.0f) * (f[5] - f[6] - f[7] + f[8]);
    F2 m8 = f[0] - F2(2.0f) * (f[1] + f[2] + f[3] + f[4]) + F2(4.0f) * d;
    const F2 rho_t = DEV ? rho + F2(1.0f) : rho;  // true density
    const F2 irho = recip(rho_t);
    const F2 S2((float)a.s[d2q9::S_S2]), S3((float)a.s[d2q9::S_S3]), S4((float)a.s[d2q9::S_S4]);
    const F2 gx((float)a.s[d2q9::S_GravitationX]), gy((float)a.s[d2q9::S_GravitationY]);
    m3 = S2 * (m3 - F2(3.0f) * jx * jx * irho);
    m4 = S2 * (m4 - F2(3.0f) * jy * jy * irho);
    m5 = S2 * (m5 - F2(3.0f) * jx * jy * irho);
    m6 = S3 * m6;
    m7 = S3 * m7;
    m8 = S4 * m8;
    jx = jx + gx * rho_t;
    jy = jy + gy * rho_t;
    m3 += F2(3.0f) * jx * jx * irho;
    m4 += F2(3.0f) * jy * jy * irho;
    m5 += F2(3.0f) * jx * jy * irho;
    from_moments(f, rho, jx, jy, m3, m4, m5, m6, m7, m8);
  }
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair_lanes(F2 (&)[Q], bool, bool, const AR&) {}

  // SetEquilibrum (:73-89): f = Req(rho, J) in the MRT basis, mapped back
  template <class R>
  __device__ __forceinline__ static void equilibrium(R (&f)[Q], R rho, R jx, R jy, R) {
    const R irho = R(1) / rho;
    from_moments(f, rho, jx, jy, R(3) * jx * jx * irho, R(3) * jy * jy * irho, R(3) * jx * jy * irho, R(0), R(0), R(0));
  }

  template <class R>
  __device__ __forceinline__ static void init(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, int, int, int) {
    const R* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
    R rho = R(1) + zs[d2q9::Z_Pressure] * R(3), ux = zs[d2q9::Z_VelocityX], uy = zs[d2q9::Z_VelocityY];
    if ((fl & d2q9::BOUNDARY) == d2q9::Wall) { rho = 1; ux = 0; uy = 0; }
    equilibrium(f, rho, ux * rho, uy * rho, R(0));
  }

  // Quantities (d2q9/Dynamics.c.Rt:39-59): 0 Rho, 1 U
  template <class R>
  __device__ __forceinline__ static void quantity(int q, R (&f)[Q], flag_t, const Args<R, NSET>& a, R* out) {
    R rho = 0, jx = 0, jy = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) { rho += f[i]; jx += R(ex(i)) * f[i]; jy += R(ey(i)) * f[i]; }
    if (q == 0) { out[0] = rho; return; }
    out[0] = jx / rho + a.s[d2q9::S_GravitationX] * R(0.5);
    out[1] = jy / rho + a.s[d2q9::S_GravitationY] * R(0.5);
    out[2] = 0;
  }
  // Color() (:61-71): |U| shaded, the whole flag equal to Solid drawn blank
  __device__ __forceinline__ static float color_weight(flag_t fl) { return fl == d2q9::Solid ? 0.f : 1.f; }
};

// ---------------------------------------------------------------------------
// d3q19 (models/flow/d3q19/Dynamics.c.Rt)
// ---------------------------------------------------------------------------


struct D3Q19 {
  static constexpr int Q = 19, DIM = 3, NSET = d3q19::NSET, NZS = d3q19::NZS, NG = d3q19::NG, NSUM = d3q19::NSUM,
                       ZONE_SHIFT = d3q19::ZONE_SHIFT;
  static constexpr bool has_bulk = true;
  static constexpr bool packed = true;
  // two-node kernel: 256 threads, <= 80 registers (3 blocks per SM), no spills
  static constexpr int PAIR_THREADS = 256, PAIR_MIN_BLOCKS = 3;
  static constexpr int BATCH_MIN_BLOCKS = 5;  // one-tile batch kernel: <= 48 registers
  // gamma1 = 1 - omega and gamma2 = 1 - 8(2 - omega)/(8 - omega), once per launch
  template <class R>
  __host__ __device__ static void derived(const R* s, R* k) {
    const R omega = s[d3q19::S_omega];
    k[0] = R(1) - omega;
    k[1] = R(1) - R(8) * (R(2) - omega) / (R(8) - omega);
    k[2] = k[3] = R(0);
  }
  // directions: columns 4, 6, 8 of MRTMAT (d3q19/Dynamics.R:26-35)
  __host__ __device__ static constexpr int ex(int i) {
    return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1 : ((i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0);
  }
  __host__ __device__ static constexpr int ey(int i) {
    return (i == 3 || i == 7 || i == 8 || i == 15 || i == 17) ? 1 : ((i == 4 || i == 9 || i == 10 || i == 16 || i == 18) ? -1 : 0);
  }
  __host__ __device__ static constexpr int ez(int i) {
    return (i == 5 || i == 11 || i == 12 || i == 15 || i == 16) ? 1 : ((i == 6 || i == 13 || i == 14 || i == 17 || i == 18) ? -1 : 0);
  }
  __host__ __device__ static constexpr int opp(int i) {
    return i == 0 ? 0 : (i <= 6 ? (i % 2 ? i + 1 : i - 1) : (i <= 10 ? 17 - i : (i <= 14 ? 25 - i : 33 - i)));
  }
  __host__ __device__ static constexpr double w(int i) { return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }

  template <class R>
  __device__ __forceinline__ static void glob(R* g, int i, R x, const R* zs) {
    add_glob<NSUM, d3q19::G_Objective, d3q19::IN_OBJ_OFFSET>(g, i, x, zs);
  }

  template <class R>
  __device__ __forceinline__ static void bounce(R (&f)[Q]) {
    R t;
#pragma unroll
    for (int i = 1; i < Q; i++)
      if (opp(i) > i) { t = f[i]; f[i] = f[opp(i)]; f[opp(i)] = t; }
  }
  // sum f over directions with sign(e_x) == SX
  template <int SX, class R>
  __device__ __forceinline__ static R sumx(const R (&f)[Q]) {
    R s = 0;
#pragma unroll
    for (int i = 0; i < Q; i++)
      if ((ex(i) > 0 ? 1 : (ex(i) < 0 ? -1 : 0)) == SX) s += f[i];
    return s;
  }
  template <class R>
  __device__ __forceinline__ static void nxy(const R (&f)[Q], R& Nxy, R& Nxz) {
    Nxy = (f[3] + f[15] + f[17] - f[4] - f[16] - f[18]) / R(2);
    Nxz = (f[5] + f[15] + f[16] - f[6] - f[17] - f[18]) / R(2);
  }
  template <class R>
  __device__ __forceinline__ static void inlet(R (&f)[Q], R rho, R ux) {  // :98-108
    R Nxy, Nxz;
    nxy(f, Nxy, Nxz);
    f[1] = f[2] + rho * ux / R(3);
    f[9] = f[8] + rho * ux / R(6) + Nxy;
    f[7] = f[10] + rho * ux / R(6) - Nxy;
    f[11] = f[14] + rho * ux / R(6) - Nxz;
    f[13] = f[12] + rho * ux / R(6) + Nxz;
  }

  // <plane>vx, vy, vz, rho, area of one slice (:271-279)
  template <int B, class R>
  __device__ __forceinline__ static void plane(R* g, R ux, R uy, R uz, R rs, const R* zs) {
    glob(g, B + 0, ux, zs);
    glob(g, B + 1, uy, zs);
    glob(g, B + 2, uz, zs);
    glob(g, B + 3, rs, zs);
    glob(g, B + 4, R(1), zs);
  }

  // Pairs (i, opposite of i); pair p has direction e of its first member.
  __host__ __device__ static constexpr int pair_a(int p) { return p < 3 ? 1 + 2 * p : (p < 5 ? 4 + p : (p < 7 ? 6 + p : 8 + p)); }
  __host__ __device__ static constexpr int pair_b(int p) { return opp(pair_a(p)); }

  // TCLB's d3q19 equilibrium (Req . MRTMAT^-1, lib/d3q19.R:40-62) split into
  // the part even under e -> -e (e[p], e0 for the rest population) and the
  // odd part o[p] of the first member of each pair. With X = Jx^2/rho etc.:
  //   rest:        rho/3 - (X+Y+Z)/3
  //   +-x axis:    rho/18 + X/6 - (Y+Z)/6     +-  Jx/6
  //   (sx,sy,0):   rho/36 + (X+Y)/12 + sx*sy*Jx*Jy/(4 rho)  +  (sx*Jx + sy*Jy)/12
  // (and the same with the axes permuted).
  // With EXACT_SUM the rest part is rho - 2 sum(e): the equilibrium then sums
  // to rho up to the rounding of that sum, not to rho times the rounded
  // weights' sum (1/3, 1/18, 1/36 are inexact in binary), which as a bias of
  // ~1e-8 per iteration drifts the mass of a long FP32 run (5000 iterations:
  // ~2e-4). Deviation storage (rho - 1 in place of rho) does not need it.
  template <bool EXACT_SUM = false, class R>
  __device__ __forceinline__ static void feq_parts(R rho, R irho, R jx, R jy, R jz, R& e0, R (&e)[9], R (&o)[9]) {
    const R X = jx * jx * irho, Y = jy * jy * irho, Z = jz * jz * irho;
    const R c18 = rho * R(1.0 / 18.0), c36 = rho * R(1.0 / 36.0);
    if (!EXACT_SUM) e0 = (rho - X - Y - Z) * R(1.0 / 3.0);
    e[0] = c18 + (X - Y - Z) * R(1.0 / 6.0);
    e[1] = c18 + (Y - X - Z) * R(1.0 / 6.0);
    e[2] = c18 + (Z - X - Y) * R(1.0 / 6.0);
    const R xy = c36 + (X + Y) * R(1.0 / 12.0), pxy = R(0.25) * jx * jy * irho;
    const R xz = c36 + (X + Z) * R(1.0 / 12.0), pxz = R(0.25) * jx * jz * irho;
    const R yz = c36 + (Y + Z) * R(1.0 / 12.0), pyz = R(0.25) * jy * jz * irho;
    e[3] = xy + pxy;  // 7 (1,1,0)
    e[4] = xy - pxy;  // 8 (-1,1,0)
    e[5] = xz + pxz;  // 11 (1,0,1)
    e[6] = xz - pxz;  // 12 (-1,0,1)
    e[7] = yz + pyz;  // 15 (0,1,1)
    e[8] = yz - pyz;  // 16 (0,-1,1)
    o[0] = jx * R(1.0 / 6.0);
    o[1] = jy * R(1.0 / 6.0);
    o[2] = jz * R(1.0 / 6.0);
    o[3] = (jx + jy) * R(1.0 / 12.0);
    o[4] = (jy - jx) * R(1.0 / 12.0);
    o[5] = (jx + jz) * R(1.0 / 12.0);
    o[6] = (jz - jx) * R(1.0 / 12.0);
    o[7] = (jy + jz) * R(1.0 / 12.0);
    o[8] = (jz - jy) * R(1.0 / 12.0);
    if (EXACT_SUM) e0 = rho - R(2) * ((e[0] + e[1] + e[2]) + ((e[3] + e[4]) + (e[5] + e[6]) + (e[7] + e[8])));
  }

  // CollisionMRT (:223-290). The d'Humieres rates of TCLB's d3q19 give every
  // non-conserved moment that is even under e -> -e the rate gamma1 = 1-omega
  // and every non-conserved odd moment gamma2 = 1 - 8(2-omega)/(8-omega);
  // the conserved ones are rho (even) and J (odd). The moment-space update
  //   R <- S (R - Req(J)) + Req(J + rho F),  f = R . MRTMAT^-1
  // is therefore the same linear map as, in population space,
  //   f_i <- feq_i(J') + gamma1 (f - feq(J))_i^even + gamma2 (f - feq(J))_i^odd
  // with even/odd parts taken over each pair (i, opposite i). It is evaluated
  // that way here: pair sums and differences instead of two 19x19 transforms.
  // The two-rate update for value type V (R, or F2 for two nodes); leaves
  // rho and the forced momentum J' for the Globals. With DEV the values are
  // deviations g = f - w: the sum of g is rho - 1, which enters the
  // equilibrium's terms linear in rho (giving feq - w), while the quadratic
  // terms and the force use the true density.
  // `lanes` (two-node form only) gives per-lane rates and force: a lane whose
  // node does not collide gets gamma1 = gamma2 = 1 and no force, which maps its
  // values onto themselves up to FP32 rounding (far below the 16-bit storage
  // the two-node form serves).
  struct Lanes { F2 g1, g2, fx, fy, fz; };
  template <bool DEV = false, class V, class AR>
  __device__ __forceinline__ static void trt(V (&f)[Q], const AR& a, V& rho, V& jx, V& jy, V& jz,
                                             const Lanes* lanes = nullptr) {
    V s[9], d[9];
#pragma unroll
    for (int p = 0; p < 9; p++) {
      s[p] = f[pair_a(p)] + f[pair_b(p)];
      d[p] = f[pair_a(p)] - f[pair_b(p)];
    }
    rho = f[0] + (s[0] + s[1] + s[2]) + ((s[3] + s[4]) + (s[5] + s[6]) + (s[7] + s[8]));
    jx = d[0] + d[3] - d[4] + d[5] - d[6];
    jy = d[1] + d[3] + d[4] + d[7] - d[8];
    jz = d[2] + d[5] + d[6] + d[7] + d[8];
    V g1, g2, fx, fy, fz;
    if constexpr (std::is_same<V, F2>::value) {
      if (lanes) {
        g1 = lanes->g1, g2 = lanes->g2, fx = lanes->fx, fy = lanes->fy, fz = lanes->fz;
      } else {
        g1 = V(a.k[0]), g2 = V(a.k[1]);
        fx = V(a.s[d3q19::S_ForceX]), fy = V(a.s[d3q19::S_ForceY]), fz = V(a.s[d3q19::S_ForceZ]);
      }
    } else {
      g1 = V(a.k[0]), g2 = V(a.k[1]);
      fx = V(a.s[d3q19::S_ForceX]), fy = V(a.s[d3q19::S_ForceY]), fz = V(a.s[d3q19::S_ForceZ]);
    }
    const V rho_t = DEV ? rho + V(1) : rho;  // true density
    const V irho = recip(rho_t);
    V e0, e[9], o[9];
    feq_parts<!DEV>(rho, irho, jx, jy, jz, e0, e, o);
    jx += rho_t * fx;
    jy += rho_t * fy;
    jz += rho_t * fz;
    V e0n, en[9], on[9];
    feq_parts<!DEV>(rho, irho, jx, jy, jz, e0n, en, on);
    f[0] = e0n + g1 * (f[0] - e0);
#pragma unroll
    for (int p = 0; p < 9; p++) {
      const V E = en[p] + g1 * (V(0.5) * s[p] - e[p]);
      const V O = on[p] + g2 * (V(0.5) * d[p] - o[p]);
      f[pair_a(p)] = E + O;
      f[pair_b(p)] = E - O;
    }
  }

  template <class R, bool G>
  __device__ __forceinline__ static void mrt(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g, const R* zs) {
    R rho, jx, jy, jz;
    trt(f, a, rho, jx, jy, jz);
    if (G) {  // :266-289, with rho and J already divided by Mw = 19, 10 (C(R, Mw, eq="/="))
      const R rs = rho * R(1.0 / 19.0), px = jx * R(0.1), py = jy * R(0.1), pz = jz * R(0.1);
      const R ux = px / rs, uy = py / rs, uz = pz / rs;
      switch (fl & d3q19::ADDITIONALS) {  // constant indices keep g[] in registers
        case d3q19::XYslice: plane<d3q19::G_XY>(g, ux, uy, uz, rs, zs); break;
        case d3q19::XZslice: plane<d3q19::G_XZ>(g, ux, uy, uz, rs, zs); break;
        case d3q19::YZslice: plane<d3q19::G_YZ>(g, ux, uy, uz, rs, zs); break;
        default: break;
      }
      glob(g, d3q19::G_VOLvx, ux, zs);
      glob(g, d3q19::G_VOLvy, uy, zs);
      glob(g, d3q19::G_VOLvz, uz, zs);
      glob(g, d3q19::G_VOLpx, px, zs);
      glob(g, d3q19::G_VOLpy, py, zs);
      glob(g, d3q19::G_VOLpz, pz, zs);
      glob(g, d3q19::G_VOLrho, rs, zs);
      glob(g, d3q19::G_VOLvolume, R(1), zs);
      const R v = sqrt(ux * ux + uy * uy + uz * uz);
      g[d3q19::G_MaxV] = g[d3q19::G_MaxV] > v ? g[d3q19::G_MaxV] : v;
    }
  }

  template <class R, bool G>
  __device__ __forceinline__ static void run(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g) {
    const R* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
    boundaries(f, fl, a);
    if ((fl & d3q19::COLLISION) == d3q19::MRT) mrt<R, G>(f, fl, a, g, zs);
  }

  // BOUNDARY group of Run (:181-204)
  template <class R, class AR>
  __device__ __forceinline__ static void boundaries(R (&f)[Q], flag_t fl, const AR& a) {
    const unsigned b = fl & d3q19::BOUNDARY;
    if (b) {
      switch (b) {  // :181-204
        case d3q19::WPressureL: {  // :138-153
          R SF = sumx<-1>(f);
          SF = sumx<0>(f) + R(2) * SF;
          R rho = a.s[d3q19::S_InletDensity];
          R ux = R(1) - SF / rho;
          if (ux > a.s[d3q19::S_InletVelocity]) { ux = a.s[d3q19::S_InletVelocity]; rho = SF / (R(1) - ux); }
          inlet(f, rho, ux);
          break;
        }
        case d3q19::WPressure: {  // :124-136
          const R rho = a.s[d3q19::S_InletDensity];
          R ux = sumx<-1>(f);
          ux = sumx<0>(f) + R(2) * ux;
          ux = R(1) - ux / rho;
          inlet(f, rho, ux);
          break;
        }
        case d3q19::WVelocity: {  // :110-122
          const R ux = a.s[d3q19::S_InletVelocity];
          R rho = sumx<-1>(f);
          rho = sumx<0>(f) + R(2) * rho;
          rho = rho / (R(1) - ux);
          inlet(f, rho, ux);
          break;
        }
        case d3q19::EPressure: {  // :157-179
          const R rho = 1;
          R ux = sumx<1>(f);
          ux = sumx<0>(f) + R(2) * ux;
          ux = R(-1) + ux / rho;
          R Nxy, Nxz;
          nxy(f, Nxy, Nxz);
          f[2] = f[1] - rho * ux / R(3);
          f[8] = f[9] - rho * ux / R(6) - Nxy;
          f[10] = f[7] - rho * ux / R(6) + Nxy;
          f[14] = f[11] - rho * ux / R(6) + Nxz;
          f[12] = f[13] - rho * ux / R(6) - Nxz;
          break;
        }
        case d3q19::Wall:
        case d3q19::Solid: bounce(f); break;
        default: break;
      }
    }
  }

  // Two nodes with one packed collision: boundaries per node, then the
  // two-rate update on both lanes (a lane whose node does not collide keeps
  // its values; the rates are the same for every node).
  __device__ __forceinline__ static bool collides(flag_t fl) { return (fl & d3q19::COLLISION) == d3q19::MRT; }
  __device__ __forceinline__ static bool has_boundary(flag_t fl) { return (fl & d3q19::BOUNDARY) != 0; }
  template <class R, class AR>
  __device__ __forceinline__ static void pre_collision(R (&f)[Q], flag_t fl, const AR& a) {
    boundaries(f, fl, a);
  }
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair(F2 (&f)[Q], flag_t, flag_t, const AR& a) {
    F2 rho, jx, jy, jz;
    trt<DEV>(f, a, rho, jx, jy, jz);
  }
  // A pair where one node collides and the other does not (fluid next to a
  // wall or a solid): the other lane takes the identity rates, so no copy of
  // it is kept across the collision. Rates and force are selected per lane
  // for every pair (exact selects), so all pairs take the same path.
  static constexpr bool identity_lanes = true;
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair_lanes(F2 (&f)[Q], bool ca, bool cb, const AR& a) {
    F2 rho, jx, jy, jz;
    const float g1 = (float)a.k[0], g2 = (float)a.k[1];
    const float fx = (float)a.s[d3q19::S_ForceX], fy = (float)a.s[d3q19::S_ForceY], fz = (float)a.s[d3q19::S_ForceZ];
    const Lanes L{F2(ca ? g1 : 1.0f, cb ? g1 : 1.0f), F2(ca ? g2 : 1.0f, cb ? g2 : 1.0f),
                  F2(ca ? fx : 0.0f, cb ? fx : 0.0f), F2(ca ? fy : 0.0f, cb ? fy : 0.0f),
                  F2(ca ? fz : 0.0f, cb ? fz : 0.0f)};
    trt<DEV>(f, a, rho, jx, jy, jz, &L);
  }

  // SetEquilibrum (:212-217): f = Req(rho, J) . MRTMAT.inv
  template <class R>
  __device__ __forceinline__ static void equilibrium(R (&f)[Q], R rho, R jx, R jy, R jz) {
    R e0, e[9], o[9];
    feq_parts(rho, R(1) / rho, jx, jy, jz, e0, e, o);
    f[0] = e0;
#pragma unroll
    for (int p = 0; p < 9; p++) {
      f[pair_a(p)] = e[p] + o[p];
      f[pair_b(p)] = e[p] - o[p];
    }
  }

  template <class R>
  __device__ __forceinline__ static void init(R (&f)[Q], flag_t, const Args<R, NSET>& a, int, int, int) {
    // SetEquilibrum(1, InletVelocity, 0, 0) (:219-221)
    equilibrium(f, R(1), a.s[d3q19::S_InletVelocity], R(0), R(0));
  }

  // Quantities (:23-40): 0 P, 1 U
  template <class R>
  __device__ __forceinline__ static void quantity(int q, R (&f)[Q], flag_t fl, const Args<R, NSET>&, R* out) {
    R rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) { rho += f[i]; jx += R(ex(i)) * f[i]; jy += R(ey(i)) * f[i]; jz += R(ez(i)) * f[i]; }
    if (q == 0) { out[0] = (rho - R(1)) / R(3); return; }
    if ((fl & d3q19::BOUNDARY) == d3q19::Wall) { out[0] = out[1] = out[2] = 0; return; }
    out[0] = jx / rho; out[1] = jy / rho; out[2] = jz / rho;
  }
  // Color() (:42-52): walls drawn blank
  __device__ __forceinline__ static float color_weight(flag_t fl) {
    return (fl & d3q19::BOUNDARY) == d3q19::Wall ? 0.f : 1.f;
  }
};

// ---------------------------------------------------------------------------
// d3q27_cumulant (models/flow/d3q27_cumulant/Dynamics.c.Rt), plain variant
// ---------------------------------------------------------------------------
#include "cumulant_gen.cuh"

struct D3Q27C {
  static constexpr int Q = 27, DIM = 3, NSET = d3q27c::NSET, NZS = d3q27c::NZS, NG = d3q27c::NG,
                       NSUM = d3q27c::NSUM, ZONE_SHIFT = d3q27c::ZONE_SHIFT;
  static constexpr bool has_bulk = true;
  static constexpr bool packed = true;
  // two-node kernel: 128 threads, <= 96 registers (5 blocks per SM), no spills
  static constexpr int PAIR_THREADS = 128, PAIR_MIN_BLOCKS = 5;
  static constexpr int BATCH_MIN_BLOCKS = 4;  // one-tile batch kernel: <= 64 registers
  // relaxation rates of the bulk (nu) and of BOUNDARY nodes (nubuffer), once per launch
  template <class R>
  __host__ __device__ static void derived(const R* s, R* k) {
    k[0] = R(1) / (R(3) * s[d3q27c::S_nu] + R(0.5));
    k[1] = R(1) / (R(3) * s[d3q27c::S_nubuffer] + R(0.5));
    k[2] = k[3] = R(0);
  }
  // f<a><b><c>: index a + 3b + 9c, digit 0 -> 0, 1 -> +1, 2 -> -1
  __host__ __device__ static constexpr int dg(int v) { return v == 1 ? 1 : (v == 2 ? -1 : 0); }
  __host__ __device__ static constexpr int ex(int i) { return dg(i % 3); }
  __host__ __device__ static constexpr int ey(int i) { return dg((i / 3) % 3); }
  __host__ __device__ static constexpr int ez(int i) { return dg(i / 9); }
  __host__ __device__ static constexpr int od(int v) { return (3 - v) % 3; }
  __host__ __device__ static constexpr int opp(int i) { return od(i % 3) + 3 * od((i / 3) % 3) + 9 * od(i / 9); }
  __host__ __device__ static constexpr int mirror_y(int i) { return i % 3 + 3 * od((i / 3) % 3) + 9 * (i / 9); }
  __host__ __device__ static constexpr int nnz(int i) { return (i % 3 != 0) + ((i / 3) % 3 != 0) + (i / 9 != 0); }
  __host__ __device__ static constexpr double w(int i) {
    return nnz(i) == 0 ? 8.0 / 27.0 : (nnz(i) == 1 ? 2.0 / 27.0 : (nnz(i) == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
  }
  __host__ __device__ static constexpr int ea(int i, int ax) { return ax == 0 ? ex(i) : (ax == 1 ? ey(i) : ez(i)); }

  template <class R>
  __device__ __forceinline__ static void glob(R* g, int i, R x, const R* zs) {
    add_glob<NSUM, d3q27c::G_Objective, d3q27c::IN_OBJ_OFFSET>(g, i, x, zs);
  }

  // ZouHe (lib/boundary.R:67-108) in closed form: unknowns SG*e_AX > 0 become
  // f_opp + 6 w_i e_i.J; rho/J_AX from the density equation, tangential J
  // from zero tangential momentum.
  template <int AX, int SG, bool VEL, class R>
  __device__ __forceinline__ static void zouhe(R (&f)[Q], R P, R V) {
    R S = 0, T1 = 0, T2 = 0;
    constexpr int A1 = (AX + 1) % 3, A2 = (AX + 2) % 3;
#pragma unroll
    for (int i = 0; i < Q; i++) {
      const int e = ea(i, AX);
      if (e == 0) { S += f[i]; T1 += R(ea(i, A1)) * f[i]; T2 += R(ea(i, A2)) * f[i]; }
      else if (SG * e < 0) S += R(2) * f[i];
    }
    R J[3];
    if (VEL) {
      const R rho = S / (R(1) - R(SG) * V);
      J[AX] = rho * V;
    } else {
      const R rho = P * R(3) + R(1);
      J[AX] = R(SG) * (rho - S);
    }
    J[A1] = R(-3) * T1;
    J[A2] = R(-3) * T2;
#pragma unroll
    for (int i = 0; i < Q; i++)
      if (SG * ea(i, AX) > 0)
        f[i] = f[opp(i)] + R(6.0 * w(i)) * (R(ex(i)) * J[0] + R(ey(i)) * J[1] + R(ez(i)) * J[2]);
  }

  template <class R, bool G>
  __device__ __forceinline__ static void bounce_drag(R (&f)[Q], flag_t fl, R* g, const R* zs) {
    R p1x = 0, p1y = 0, p1z = 0, p2x = 0, p2y = 0, p2z = 0;
    if (G) {
#pragma unroll
      for (int i = 0; i < Q; i++) { p1x += R(ex(i)) * f[i]; p1y += R(ey(i)) * f[i]; p1z += R(ez(i)) * f[i]; }
    }
#pragma unroll
    for (int i = 1; i < Q; i++)
      if (opp(i) > i) { const R t = f[i]; f[i] = f[opp(i)]; f[opp(i)] = t; }
    if (G && (fl & d3q27c::BODY) == d3q27c::Body) {  // :121-126
#pragma unroll
      for (int i = 0; i < Q; i++) { p2x += R(ex(i)) * f[i]; p2y += R(ey(i)) * f[i]; p2z += R(ez(i)) * f[i]; }
      glob(g, d3q27c::G_Drag, -(p2x - p1x), zs);
      glob(g, d3q27c::G_Lateral, -(p2y - p1y), zs);
      glob(g, d3q27c::G_Lift, -(p2z - p1z), zs);
    }
  }

  template <class R, bool G>
  __device__ __forceinline__ static void boundaries(R (&f)[Q], flag_t fl, R* g, const R* zs) {  // :224-272
    const unsigned ad = fl & d3q27c::ADDITIONALS;
    if (ad == d3q27c::NSymmetry) {
#pragma unroll
      for (int i = 0; i < Q; i++) if (ey(i) < 0) f[i] = f[mirror_y(i)];
    } else if (ad == d3q27c::SSymmetry) {
#pragma unroll
      for (int i = 0; i < Q; i++) if (ey(i) > 0) f[i] = f[mirror_y(i)];
    }
    const unsigned b = fl & d3q27c::BOUNDARY;
    if (!b) return;
    const R V = zs[d3q27c::Z_Velocity], P = zs[d3q27c::Z_Pressure];
    switch (b) {
      case d3q27c::WVelocityTurbulent: zouhe<0, 1, true>(f, P, V); break;  // zero turbulence intensity
      case d3q27c::EPressure: zouhe<0, -1, false>(f, P, V); break;
      case d3q27c::WPressure: zouhe<0, 1, false>(f, P, V); break;
      case d3q27c::SPressure: zouhe<1, 1, false>(f, P, V); break;
      case d3q27c::NPressure: zouhe<1, -1, false>(f, P, V); break;
      case d3q27c::WVelocity: zouhe<0, 1, true>(f, P, V); break;
      case d3q27c::NVelocity: zouhe<1, -1, true>(f, P, V); break;
      case d3q27c::SVelocity: zouhe<1, 1, true>(f, P, V); break;
      case d3q27c::EVelocity: zouhe<0, -1, true>(f, P, V); break;
      case d3q27c::Wall: bounce_drag<R, G>(f, fl, g, zs); break;
      default: break;
    }
  }

  // 1D raw-moment transform of a (0, +1, -1) triple and its inverse
  // (:323-349 and :479-505)
  template <class R>
  __device__ __forceinline__ static void raw3(R& a0, R& a1, R& a2) {
    a0 = a2 + a1 + a0;
    a1 = a1 - a2;
    a2 = a1 + a2 * R(2);
  }
  template <class R>
  __device__ __forceinline__ static void unraw3(R& a0, R& a1, R& a2) {
    a0 = a0 - a2;
    a1 = (a2 + a1) * R(0.5);
    a2 = a2 - a1;
  }

  template <class R, bool G>
  __device__ __forceinline__ static void collide(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g, const R* zs) {
    const R Fx = a.s[d3q27c::S_ForceX], Fy = a.s[d3q27c::S_ForceY], Fz = a.s[d3q27c::S_ForceZ];
    const R w0 = (fl & d3q27c::BOUNDARY) ? a.k[1] : a.k[0];
    to_raw(f);
    if (G) {  // :311-319 with getU_ (:30-45); rho and J are the raw moments m000, m100, m010, m001
      const R rho = f[0], jx = f[1], jy = f[3], jz = f[9];
      R ux = (jx + Fx / R(2)) / rho, uy = (jy + Fy / R(2)) / rho, uz = (jz + Fz / R(2)) / rho;
      if ((fl & d3q27c::BOUNDARY) == d3q27c::Wall) ux = uy = uz = 0;
      glob(g, d3q27c::G_Density, rho, zs);
      glob(g, d3q27c::G_Flux, ux, zs);
      glob(g, d3q27c::G_Mass, rho, zs);
      glob(g, d3q27c::G_XMomentum, rho * ux, zs);
      glob(g, d3q27c::G_YMomentum, rho * uy, zs);
      glob(g, d3q27c::G_ZMomentum, rho * uz, zs);
    }
    // Cumulants of order >= 4 are set to zero by the collision and those of
    // order 3 are scaled by (1 - Omega): with the default Omega = 1 they vanish
    // too, so only orders <= 2 are converted (a branch uniform over the launch).
    if (a.s[d3q27c::S_Omega] == R(1)) relax<R, Args<R, NSET>, false>(f, a, w0);
    else relax<R, Args<R, NSET>, true>(f, a, w0);
    from_raw(f);
  }

  // populations -> raw moments (x, y, z passes) and back
  template <class V>
  __device__ __forceinline__ static void to_raw(V (&f)[Q]) {
#pragma unroll
    for (int r = 0; r < 27; r += 3) raw3(f[r], f[r + 1], f[r + 2]);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int x = 0; x < 3; x++) raw3(f[x + 9 * c], f[x + 3 + 9 * c], f[x + 6 + 9 * c]);
#pragma unroll
    for (int r = 0; r < 9; r++) raw3(f[r], f[r + 9], f[r + 18]);
  }
  template <class V>
  __device__ __forceinline__ static void from_raw(V (&f)[Q]) {
#pragma unroll
    for (int r = 0; r < 27; r += 3) unraw3(f[r], f[r + 1], f[r + 2]);
#pragma unroll
    for (int cc = 0; cc < 3; cc++)
#pragma unroll
      for (int x = 0; x < 3; x++) unraw3(f[x + 9 * cc], f[x + 3 + 9 * cc], f[x + 6 + 9 * cc]);
#pragma unroll
    for (int r = 0; r < 9; r++) unraw3(f[r], f[r + 9], f[r + 18]);
  }

  // Two nodes with one packed collision: boundaries per node (no Globals),
  // then the cumulant collision on both lanes with each node's rate (nubuffer
  // on BOUNDARY nodes); a lane whose node does not collide keeps its values.
  __device__ __forceinline__ static bool collides(flag_t fl) { return (fl & d3q27c::COLLISION) == d3q27c::MRT; }
  __device__ __forceinline__ static bool has_boundary(flag_t fl) {
    return (fl & (d3q27c::ADDITIONALS | d3q27c::BOUNDARY)) != 0;
  }
  template <class R, class AR>
  __device__ __forceinline__ static void pre_collision(R (&f)[Q], flag_t fl, const AR& a) {
    if (fl & (d3q27c::ADDITIONALS | d3q27c::BOUNDARY)) {
      R g[1];
      boundaries<R, false>(f, fl, g, a.zone + (fl >> ZONE_SHIFT) * NZS);
    }
  }
  // With DEV the values are deviations g = f - w. The raw-moment transform is
  // linear, so the weights' raw moments (per axis (1, 0, 1/3): m000 = 1,
  // m200 = m020 = m002 = 1/3, m220 = m202 = m022 = 1/9, m222 = 1/27) are added
  // after the forward transform and taken off before the backward one,
  // instead of adding and removing w on all 27 populations.
  template <class V>
  __device__ __forceinline__ static void weight_moments(V (&m)[Q], float sign) {
    m[0] += V(sign);
    m[2] += V(sign * (1.0f / 3.0f));
    m[6] += V(sign * (1.0f / 3.0f));
    m[18] += V(sign * (1.0f / 3.0f));
    m[8] += V(sign * (1.0f / 9.0f));
    m[20] += V(sign * (1.0f / 9.0f));
    m[24] += V(sign * (1.0f / 9.0f));
    m[26] += V(sign * (1.0f / 27.0f));
  }
  static constexpr bool identity_lanes = false;  // orders above 3 are set to zero: no identity rates
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair_lanes(F2 (&)[Q], bool, bool, const AR&) {}
  template <bool DEV, class AR>
  __device__ __forceinline__ static void collide_pair(F2 (&f)[Q], flag_t fla, flag_t flb, const AR& a) {
    typedef typename AR::real R;
    const F2 w0((float)((fla & d3q27c::BOUNDARY) ? a.k[1] : a.k[0]), (float)((flb & d3q27c::BOUNDARY) ? a.k[1] : a.k[0]));
    to_raw(f);
    if (DEV) weight_moments(f, 1.0f);
    if (a.s[d3q27c::S_Omega] == R(1)) relax<F2, AR, false>(f, a, w0);
    else relax<F2, AR, true>(f, a, w0);
    if (DEV) weight_moments(f, -1.0f);
    from_raw(f);
  }

  // Raw moments f -> cumulants -> relaxed cumulants -> raw moments (:359-477).
  template <class V, class AR, bool THIRD>
  __device__ __forceinline__ static void relax(V (&f)[Q], const AR& a, V w0) {
    typedef typename AR::real R;
    const V Fx = V(a.s[d3q27c::S_ForceX]), Fy = V(a.s[d3q27c::S_ForceY]), Fz = V(a.s[d3q27c::S_ForceZ]);
    const V w1 = V(1);
    V c[Q];
    const V m0 = f[0], im0 = recip(m0);
    if (THIRD) cum_from_raw_o3(f, c, im0);
    else cum_from_raw_o2(f, c, im0);
    // relaxation (:386-449); x/2 written as x*0.5 (exact)
    const V ux = c[1] + Fx * V(0.5) * im0, uy = c[3] + Fy * V(0.5) * im0, uz = c[9] + Fz * V(0.5) * im0;
    const V c200 = c[2], c020 = c[6], c002 = c[18];
    const V dxu = -w0 * V(0.5) * (V(2) * c200 - c020 - c002) - w1 * V(0.5) * (c200 + c020 + c002 - V(1));
    const V dyv = dxu + V(3) * w0 * V(0.5) * (c200 - c020);
    const V dzw = dxu + V(3) * w0 * V(0.5) * (c200 - c002);
    const V gcor1 = V(3) * (V(1) - w0 * V(0.5)) * (ux * ux * dxu - uy * uy * dyv);
    const V gcor2 = V(3) * (V(1) - w0 * V(0.5)) * (ux * ux * dxu - uz * uz * dzw);
    const V gcor3 = V(3) * (V(1) - w1 * V(0.5)) * (ux * ux * dxu + uy * uy * dyv + uz * uz * dzw);
    const V GC = V(a.s[d3q27c::S_GalileanCorrection]);
    const V A = (V(1) - w0) * (c200 - c020) - gcor1 * GC;
    const V B = (V(1) - w0) * (c200 - c002) - gcor2 * GC;
    const V CC = w1 + (V(1) - w1) * (c200 + c020 + c002) - gcor3 * GC;
    c[1] += Fx;
    c[2] = (A + B + CC) * V(1.0 / 3.0);
    c[6] = (CC - V(2) * A + B) * V(1.0 / 3.0);
    c[18] = (CC - V(2) * B + A) * V(1.0 / 3.0);
    c[3] += Fy;
    c[9] += Fz;
    c[4] *= (V(1) - w0);
    c[12] *= (V(1) - w0);
    c[10] *= (V(1) - w0);
    if (THIRD) {
      const V om3 = V(R(1) - a.s[d3q27c::S_Omega]);
#pragma unroll
      for (int n = 1; n < Q; n++)
        if (n % 3 + (n / 3) % 3 + n / 9 == 3) c[n] = om3 * c[n];
      raw_from_cum_o3(c, f, m0);
    } else {
      raw_from_cum_o2(c, f, m0);
    }
  }

  template <class R, bool G>
  __device__ __forceinline__ static void run(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* g) {
    const R* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
    if (fl & (d3q27c::ADDITIONALS | d3q27c::BOUNDARY)) boundaries<R, G>(f, fl, g, zs);
    if ((fl & d3q27c::COLLISION) == d3q27c::MRT) collide<R, G>(f, fl, a, g, zs);
  }

  template <class R>
  __device__ __forceinline__ static void equilibrium(R (&f)[Q], R rho, R jx, R jy, R jz) {
    const R irho = R(1) / rho, j2 = (jx * jx + jy * jy + jz * jz) * irho;
#pragma unroll
    for (int i = 0; i < Q; i++) {
      const R eu = R(ex(i)) * jx + R(ey(i)) * jy + R(ez(i)) * jz;
      f[i] = R(w(i)) * (rho + R(3) * eu + R(4.5) * eu * eu * irho - R(1.5) * j2);
    }
  }

  template <class R>
  __device__ __forceinline__ static void init(R (&f)[Q], flag_t fl, const Args<R, NSET>& a, int, int, int) {
    // :290-299 with zero synthetic turbulence: SetEquilibrum(1+3P, Velocity, 0, 0)
    const R* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
    if ((fl & d3q27c::BOUNDARY) == d3q27c::Wall) equilibrium(f, R(1), R(0), R(0), R(0));
    else equilibrium(f, R(1) + zs[d3q27c::Z_Pressure] * R(3), zs[d3q27c::Z_Velocity], R(0), R(0));
  }

  // Quantities (:23-60): 0 P, 1 U (after RunBoundaries), 2 Solid
  template <class R>
  __device__ __forceinline__ static void quantity(int q, R (&f)[Q], flag_t fl, const Args<R, NSET>& a, R* out) {
    const bool wall = (fl & d3q27c::BOUNDARY) == d3q27c::Wall;
    if (q == 2) { out[0] = wall ? R(1) : R(0); return; }
    if (q == 1) {
      const R* zs = a.zone + (fl >> ZONE_SHIFT) * NZS;
      boundaries<R, false>(f, fl, nullptr, zs);
    }
    R rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) { rho += f[i]; jx += R(ex(i)) * f[i]; jy += R(ey(i)) * f[i]; jz += R(ez(i)) * f[i]; }
    if (q == 0) { out[0] = (rho - R(1)) / R(3); return; }
    if (wall) { out[0] = out[1] = out[2] = 0; return; }
    out[0] = (jx + a.s[d3q27c::S_ForceX] / R(2)) / rho;
    out[1] = (jy + a.s[d3q27c::S_ForceY] / R(2)) / rho;
    out[2] = (jz + a.s[d3q27c::S_ForceZ] / R(2)) / rho;
  }
  // Color() (:101-111): the whole flag equal to Solid drawn blank
  __device__ __forceinline__ static float color_weight(flag_t fl) { return fl == d3q27c::Solid ? 0.f : 1.f; }
};

// ---------------------------------------------------------------------------
// Globals: warp shuffle -> shared memory -> one FP64 atomic per Global per
// block (replaces CudaAtomicAddReduceWarp / MaxReduceWarp, src/cross.hpp:163-181).
// MAX Globals are non-negative here, so an integer max on the FP64 bits orders
// them correctly.
// ---------------------------------------------------------------------------
template <int NG, int NSUM, class R>
__device__ __forceinline__ void reduce_globals(const R (&g)[NG], double* out) {
  __shared__ double sh[32][NG];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NG; i++) {
    double v = (double)g[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_down_sync(0xffffffffu, v, o);
      v = i < NSUM ? v + u : (u > v ? u : v);
    }
    if (lane == 0) sh[warp][i] = v;
  }
  __syncthreads();
  if (tid < NG) {
    double v = sh[0][tid];
    for (int w = 1; w < nwarps; w++) v = tid < NSUM ? v + sh[w][tid] : (sh[w][tid] > v ? sh[w][tid] : v);
    if (tid < NSUM) {
      if (v != 0.0) atomicAdd(out + tid, v);
    } else if (v > 0.0) {
      atomicMax(reinterpret_cast<unsigned long long*>(out + tid), (unsigned long long)__double_as_longlong(v));
    }
  }
}

// ---------------------------------------------------------------------------
// The fused iteration kernel: one thread per node.
// ---------------------------------------------------------------------------
// Where the population planes are. StrideAddr derives plane i from one base
// pointer and the plane stride (the batch kernel, whose case descriptors are
// read from device memory); PlaneAddr carries all 2*Q plane base pointers as
// a kernel parameter, so each load or store needs only its 32-bit node index
// scaled onto a base that every thread shares.
template <class T>
struct StrideAddr {
  static constexpr bool per_plane = false;
  const T* s;
  T* d;
  size_t stride;
  __device__ __forceinline__ const T* src(int i) const { return s + (size_t)i * stride; }
  __device__ __forceinline__ T* dst(int i) const { return d + (size_t)i * stride; }
};
template <class T, int Q>
struct PlaneAddr {
  static constexpr bool per_plane = true;
  const T* s[Q];
  T* d[Q];
  __device__ __forceinline__ const T* src(int i) const { return s[i]; }
  __device__ __forceinline__ T* dst(int i) const { return d[i]; }
};

// One node: pull from the source planes with periodic wrap, run the model,
// store to the destination planes.
//
// Addressing: the source of population i is node - e_i with periodic wrap.
// Per axis the two possible offsets (pulling from the lower / upper
// neighbour, wrapped at the faces) are computed once; each population's
// offset is then the sum of three of them, chosen at compile time. Node
// indices are unsigned 32-bit (a lattice has fewer than 2^32 nodes); a
// negative offset wraps modulo 2^32 and lands on the right node.
template <class M, class R, class St, bool G, class A>
__device__ __forceinline__ void node_update(const Args<R, M::NSET>& a, const A& P, int x, int y, int z, R* g) {
  const unsigned nx = a.nx, ny = a.ny, nz = a.nz;
  const unsigned sxy = nx * ny;
  const unsigned node = x + nx * y + sxy * z;
  const unsigned ox_lo = x == 0 ? nx - 1 : 0u - 1u, ox_hi = x + 1 == (int)nx ? 1u - nx : 1u;  // e_x = +1 / -1
  const unsigned oy_lo = y == 0 ? nx * (ny - 1) : 0u - nx, oy_hi = y + 1 == (int)ny ? nx * (1u - ny) : nx;
  const unsigned oz_lo = z == 0 ? sxy * (nz - 1) : 0u - sxy, oz_hi = z + 1 == (int)nz ? sxy * (1u - nz) : sxy;
  const flag_t fl = a.flags[node];
  R f[M::Q];
  using T = typename St::T;
  if constexpr (A::per_plane) {
#pragma unroll
    for (int i = 0; i < M::Q; i++) {
      const unsigned o = (M::ex(i) > 0 ? ox_lo : (M::ex(i) < 0 ? ox_hi : 0u)) +
                         (M::ey(i) > 0 ? oy_lo : (M::ey(i) < 0 ? oy_hi : 0u)) +
                         (M::DIM == 2 ? 0u : (M::ez(i) > 0 ? oz_lo : (M::ez(i) < 0 ? oz_hi : 0u)));
      f[i] = St::template load<R>(P.src(i) + (node + o), R(M::w(i)));
    }
    M::template run<R, G>(f, fl, a, g);
#pragma unroll
    for (int i = 0; i < M::Q; i++) St::template store<R>(P.dst(i) + node, f[i], R(M::w(i)));
  } else {
    // one pointer at the node, planes reached by adding the stride
    const T* __restrict__ src = P.s + node;
    T* __restrict__ dst = P.d + node;
    const size_t stride = P.stride;
#pragma unroll
    for (int i = 0; i < M::Q; i++) {
      const int o = (int)((M::ex(i) > 0 ? ox_lo : (M::ex(i) < 0 ? ox_hi : 0u)) +
                          (M::ey(i) > 0 ? oy_lo : (M::ey(i) < 0 ? oy_hi : 0u)) +
                          (M::DIM == 2 ? 0u : (M::ez(i) > 0 ? oz_lo : (M::ez(i) < 0 ? oz_hi : 0u))));
      f[i] = St::template load<R>(src + i * stride + o, R(M::w(i)));
    }
    M::template run<R, G>(f, fl, a, g);
#pragma unroll
    for (int i = 0; i < M::Q; i++) St::template store<R>(dst + i * stride, f[i], R(M::w(i)));
  }
}

// Two nodes per thread for 16-bit storage: (x, x+1) with x even, so every
// population is one aligned 32-bit load and store and a warp moves 128 bytes
// per request (with 2-byte values one node per thread moves only 64). The
// pull shifts e_x = +1 / -1 take the neighbouring pair from the adjacent lane
// by a shuffle; the lanes at the warp edges load their halo pair directly
// (with the periodic wrap). Requires nx % 64 == 0 and whole warps on one row.
template <class St>
struct Pack16;
template <bool SH>
struct Pack16<StoreF16<SH>> {
  __device__ __forceinline__ static float2 unpack(unsigned w) { return __half22float2(*reinterpret_cast<__half2*>(&w)); }
  __device__ __forceinline__ static float lo(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
  __device__ __forceinline__ static float hi(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }
  __device__ __forceinline__ static unsigned pack(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<unsigned*>(&h);
  }
};
template <bool SH>
struct Pack16<StoreBF16<SH>> {
  __device__ __forceinline__ static float lo(unsigned w) { return __uint_as_float(w << 16); }
  __device__ __forceinline__ static float hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }
  __device__ __forceinline__ static float2 unpack(unsigned w) { return make_float2(lo(w), hi(w)); }
  __device__ __forceinline__ static unsigned pack(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<unsigned*>(&h);
  }
};

// Update and store two neighbouring nodes (x, x+1) of one row whose pulled
// densities, as stored (shift not yet added), are v[i] = (node x, node x+1).
// Models with a packed collision: boundary conditions per node, then one
// FP32x2 collision for both; others: the scalar node update twice. Plain
// iterations (no Globals).
// AR: Args<R, M::NSET>, or for the packed models a view with the same
// members s[], k[], zone (SharedArgsView).
// LANES (models with identity rates, d3q19): a pair where one node collides
// runs the other lane at the identity rates instead of parking it. The
// register pair kernels always do; the one-lattice tile-staged kernel does
// when such pairs are at least 1% of the lattice (at its 96-register cap the
// per-lane rates spill, which costs more than parking when they are rare);
// the batch tile-staged kernel, with more state per warp, parks.
template <class M, class R, class St, class A, class AR, bool LANES = false>
__device__ __forceinline__ void pair_update_store(float2 (&v)[M::Q], flag_t fla, flag_t flb, const AR& a, const A& P,
                                                  unsigned node) {
  using P16 = Pack16<St>;
  if constexpr (M::packed && sizeof(R) == 4) {
    // Values stay packed (node x, node x+1). A node with a boundary type has
    // its lane taken out, updated by the scalar boundary code and put back;
    // then one packed FP32x2 collision serves both nodes, so bulk and
    // boundary pairs do not diverge in the collision.
    // With shifted storage the packed values stay deviations g = f - w
    // (the collision works on them directly); the scalar boundary code sees f.
    constexpr float SH = St::shifted ? 1.0f : 0.0f;
    F2 f2[M::Q];
#pragma unroll
    for (int i = 0; i < M::Q; i++) f2[i] = F2(v[i]);
    if (M::has_boundary(fla)) {
      float t[M::Q];
#pragma unroll
      for (int i = 0; i < M::Q; i++) t[i] = f2[i].v.x + SH * (float)M::w(i);
      M::pre_collision(t, fla, a);
#pragma unroll
      for (int i = 0; i < M::Q; i++) f2[i].v.x = t[i] - SH * (float)M::w(i);
    }
    if (M::has_boundary(flb)) {
      float t[M::Q];
#pragma unroll
      for (int i = 0; i < M::Q; i++) t[i] = f2[i].v.y + SH * (float)M::w(i);
      M::pre_collision(t, flb, a);
#pragma unroll
      for (int i = 0; i < M::Q; i++) f2[i].v.y = t[i] - SH * (float)M::w(i);
    }
    const bool ca = M::collides(fla), cb = M::collides(flb);
    if constexpr (LANES && M::identity_lanes) {
      if (ca || cb) M::template collide_pair_lanes<St::shifted>(f2, ca, cb, a);
    } else if (ca || cb) {
      // A pair where only one node collides (fluid next to a wall) parks the
      // other node's values in thread-local memory across the collision; a
      // volatile array keeps them out of the registers every pair would pay.
      float keep_mem[M::Q];
      volatile float* keep = keep_mem;
      const bool mixed = ca != cb;
      if (mixed) {
#pragma unroll
        for (int i = 0; i < M::Q; i++) keep[i] = ca ? f2[i].v.y : f2[i].v.x;
      }
      M::template collide_pair<St::shifted>(f2, fla, flb, a);
      if (mixed) {
#pragma unroll
        for (int i = 0; i < M::Q; i++) {
          if (ca) f2[i].v.y = keep[i];
          else f2[i].v.x = keep[i];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < M::Q; i++) v[i] = f2[i].v;
  } else {
    R fa[M::Q], fb[M::Q];
#pragma unroll
    for (int i = 0; i < M::Q; i++) {
      const R sh = St::shifted ? R(M::w(i)) : R(0);
      fa[i] = R(v[i].x) + sh;
      fb[i] = R(v[i].y) + sh;
    }
    R g[1];
    M::template run<R, false>(fa, fla, a, g);
    M::template run<R, false>(fb, flb, a, g);
#pragma unroll
    for (int i = 0; i < M::Q; i++) {
      const R sh = St::shifted ? R(M::w(i)) : R(0);
      v[i] = make_float2((float)(fa[i] - sh), (float)(fb[i] - sh));
    }
  }
#pragma unroll
  for (int i = 0; i < M::Q; i++) {
    unsigned short* base = reinterpret_cast<unsigned short*>(P.dst(i));
    __stcs(reinterpret_cast<unsigned*>(base + node), P16::pack(v[i].x, v[i].y));
  }
}

// PARTIAL: x may lie past the row (the last tile of a row whose width is not
// a multiple of 64); such a lane loads the pair at x mod nx, which its
// neighbours' shuffles need, and stores nothing.
template <class M, class R, class St, class A, bool PARTIAL = false>
__device__ __forceinline__ void node_update_pair(const Args<R, M::NSET>& a, const A& P, int x, int y, int z,
                                                 int lane) {
  using P16 = Pack16<St>;
  const unsigned nx = a.nx, ny = a.ny, nz = a.nz;
  bool store = true;
  if constexpr (PARTIAL) {
    if (x >= a.nx) {
      x = (unsigned)x % nx;
      store = false;
    }
  }
  const unsigned sxy = nx * ny;
  const unsigned node = x + nx * y + sxy * z;  // even
  const unsigned oy_lo = y == 0 ? nx * (ny - 1) : 0u - nx, oy_hi = y + 1 == (int)ny ? nx * (1u - ny) : nx;
  const unsigned oz_lo = z == 0 ? sxy * (nz - 1) : 0u - sxy, oz_hi = z + 1 == (int)nz ? sxy * (1u - nz) : sxy;
  const unsigned o_prev = x == 0 ? nx - 2 : 0u - 2u;       // pair (x-2, x-1), wrapped
  const unsigned o_next = x + 2 == (int)nx ? 2u - nx : 2u;  // pair (x+2, x+3), wrapped
  const unsigned fl2 = __ldg(reinterpret_cast<const unsigned*>(a.flags + node));
  const flag_t fla = (flag_t)(fl2 & 0xffffu), flb = (flag_t)(fl2 >> 16);
  float2 v[M::Q];  // (node x, node x+1)
#pragma unroll
  for (int i = 0; i < M::Q; i++) {
    const unsigned o = (M::ey(i) > 0 ? oy_lo : (M::ey(i) < 0 ? oy_hi : 0u)) +
                       (M::DIM == 2 ? 0u : (M::ez(i) > 0 ? oz_lo : (M::ez(i) < 0 ? oz_hi : 0u)));
    const unsigned short* base = reinterpret_cast<const unsigned short*>(P.src(i));
    const unsigned idx = node + o;
    const unsigned w = __ldg(reinterpret_cast<const unsigned*>(base + idx));
    if (M::ex(i) == 0) {
      v[i] = P16::unpack(w);
    } else if (M::ex(i) > 0) {  // from x-1: (prev.hi, w.lo)
      unsigned prev = __shfl_up_sync(0xffffffffu, w, 1);
      if (lane == 0) prev = __ldg(reinterpret_cast<const unsigned*>(base + (idx + o_prev)));
      v[i] = make_float2(P16::hi(prev), P16::lo(w));
    } else {  // from x+1: (w.hi, next.lo)
      unsigned next = __shfl_down_sync(0xffffffffu, w, 1);
      if (lane == 31) next = __ldg(reinterpret_cast<const unsigned*>(base + (idx + o_next)));
      v[i] = make_float2(P16::hi(w), P16::lo(next));
    }
  }
  if (!PARTIAL || store) pair_update_store<M, R, St, A, Args<R, M::NSET>, true>(v, fla, flb, a, P, node);
}

// Node pairs (2p, 2p+1) of the flat node index, p < npairs, of which exactly
// one node collides (a pair of one row when nx is even); the count is added
// to *count.
template <class M>
__global__ void k_count_mixed_pairs(const flag_t* __restrict__ flags, unsigned npairs, unsigned* count) {
  unsigned c = 0;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) {
    const unsigned w = __ldg(reinterpret_cast<const unsigned*>(flags) + p);
    c += M::collides((flag_t)(w & 0xffffu)) != M::collides((flag_t)(w >> 16)) ? 1u : 0u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Block (32, M::PAIR_THREADS / 32): each warp covers 64 consecutive x of one
// row. Plain iterations only (Globals iterations use k_iterate).
template <class M, class R, class St>
__global__ void __launch_bounds__(M::PAIR_THREADS, M::PAIR_MIN_BLOCKS)
    k_iterate_pair(const Args<R, M::NSET> a, const PlaneAddr<typename St::T, M::Q> P) {
  const int lane = threadIdx.x;
  const int x = 2 * (blockIdx.x * 32 + lane);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (y < a.ny) node_update_pair<M, R, St, PlaneAddr<typename St::T, M::Q>>(a, P, x, y, z, lane);  // y is uniform per warp
}

// Launched with programmatic stream serialization (launch_pdl), the next
// iteration's grid is scheduled while this one drains: griddepcontrol.wait
// returns once the previous grid has completed and its writes are visible,
// and launch_dependents lets the next grid start launching at once. Both are
// no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait_and_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class M, class R, class St, bool G, class A>
__global__ void __launch_bounds__(256) k_iterate(const Args<R, M::NSET> a, const A P) {
  pdl_wait_and_release();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool act = (x < a.nx) && (y < a.ny);
  R g[G ? M::NG : 1];
#pragma unroll
  for (int i = 0; i < (G ? M::NG : 1); i++) g[i] = 0;
  if (act) node_update<M, R, St, G>(a, P, x, y, z, g);
  if constexpr (G) reduce_globals<M::NG, M::NSUM, R>(g, a.glob);
}

// BaseInit stage: equilibrium from settings, written to the current snapshot.
template <class M, class R, class St>
__global__ void k_init(const Args<R, M::NSET> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= a.nx || y >= a.ny) return;
  const int node = x + a.nx * (y + a.ny * z);
  R f[M::Q];
  M::template init<R>(f, a.flags[node], a, x, y, z);
  typename St::T* dst = static_cast<typename St::T*>(a.dst);
#pragma unroll
  for (int i = 0; i < M::Q; i++) St::template store<R>(dst + (size_t)i * a.stride + node, f[i], R(M::w(i)));
}

// Equilibrium from density and velocity fields (J = rho u), the initial
// condition of cases that TCLB loads through <LoadBinary>.
template <class M, class R, class St>
__global__ void k_equilibrium(const Args<R, M::NSET> a, const R* __restrict__ rho, const R* __restrict__ u) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= a.nx || y >= a.ny) return;
  const int node = x + a.nx * (y + a.ny * z);
  const R r = rho[node];
  R f[M::Q];
  M::template equilibrium<R>(f, r, r * u[3 * (size_t)node], r * u[3 * (size_t)node + 1], r * u[3 * (size_t)node + 2]);
  typename St::T* dst = static_cast<typename St::T*>(a.dst);
#pragma unroll
  for (int i = 0; i < M::Q; i++) St::template store<R>(dst + (size_t)i * a.stride + node, f[i], R(M::w(i)));
}

// Quantity over a region (LatticeContainer.inc.cpp.Rt:437-473): pull, then
// the model's get<Q>(), times scale. Region origin (rx,ry,rz), size (rnx,rny).
template <class M, class R, class St>
__global__ void k_quantity(const Args<R, M::NSET> a, int q, int vec, int rx, int ry, int rz, int rnx, int rny,
                           int rnz, R scale, R* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= rnx || j >= rny || k >= rnz) return;
  const int x = rx + i, y = ry + j, z = rz + k;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int xm = (x == 0 ? nx : x) - 1, xp = (x + 1 == nx) ? 0 : x + 1;
  const int ym = (y == 0 ? ny : y) - 1, yp = (y + 1 == ny) ? 0 : y + 1;
  const int zm = (z == 0 ? nz : z) - 1, zp = (z + 1 == nz) ? 0 : z + 1;
  const typename St::T* src = static_cast<const typename St::T*>(a.src);
  R f[M::Q];
#pragma unroll
  for (int d = 0; d < M::Q; d++) {
    const int sx = M::ex(d) == 0 ? x : (M::ex(d) > 0 ? xm : xp);
    const int sy = M::ey(d) == 0 ? y : (M::ey(d) > 0 ? ym : yp);
    const int sz = M::DIM == 2 ? z : (M::ez(d) == 0 ? z : (M::ez(d) > 0 ? zm : zp));
    f[d] = St::template load<R>(src + (size_t)d * a.stride + (sx + nx * (sy + ny * sz)), R(M::w(d)));
  }
  R v[3];
  M::template quantity<R>(q, f, a.flags[x + nx * (y + ny * z)], a, v);
  const size_t o = (size_t)i + (size_t)rnx * ((size_t)j + (size_t)rny * k);
  if (vec) {
    out[3 * o] = v[0] * scale;
    out[3 * o + 1] = v[1] * scale;
    out[3 * o + 2] = v[2] * scale;
  } else {
    out[o] = v[0] * scale;
  }
}

// Headless ColorKernel (src/LatticeContainer.inc.cpp.Rt:350-412): one RGBA
// byte quadruple per node of plane z, x fastest. The model's Color() gives
// l = |U| (U as the quantity export computes it, from the pulled densities)
// and a weight w; l * 111 goes through TCLB's piecewise-linear map (white /
// cyan / blue for negative, red / yellow / white for positive values), w = 0
// paints the node green and a non-finite l magenta. The arithmetic is float
// with explicitly rounded operations, so a CPU restatement reproduces every
// byte.
__device__ __forceinline__ uchar4 color_map(float l, float w) {
  int r = 0, g = 0, b = 0;
  if (isfinite(l)) {
    l = __fmul_rn(l, 111.f);
    if (l < -111.f) { r = 255; g = 255; b = 255; }
    else if (l < -11.f) { r = (int)__fdiv_rn(__fmul_rn(255.f, __fadd_rn(-l, -11.f)), 100.f); g = 255; b = 255; }
    else if (l < -1.f) { r = 0; g = (int)__fdiv_rn(__fmul_rn(255.f, __fadd_rn(-l, -1.f)), 10.f); b = 255; }
    else if (l < 0.f) { r = 0; g = 0; b = (int)__fmul_rn(255.f, -l); }
    else if (l < 1.f) { r = (int)__fmul_rn(255.f, l); g = 0; b = 0; }
    else if (l < 11.f) { r = 255; g = (int)__fdiv_rn(__fmul_rn(255.f, __fadd_rn(l, -1.f)), 10.f); b = 0; }
    else if (l < 111.f) { r = 255; g = 255; b = (int)__fdiv_rn(__fmul_rn(255.f, __fadd_rn(l, -11.f)), 100.f); }
    else { r = 255; g = 255; b = 255; }
    r = (int)__fmul_rn((float)r, w);
    g = (int)__fadd_rn(__fmul_rn((float)g, w), __fmul_rn(__fadd_rn(1.f, -w), 255.f));
    b = (int)__fmul_rn((float)b, w);
  } else {
    r = 255; g = 0; b = 255;
  }
  return make_uchar4((unsigned char)r, (unsigned char)g, (unsigned char)b, 255);
}

template <class R>
__device__ __forceinline__ float speed(const R* u, bool three) {
  if constexpr (sizeof(R) == 8) {
    double s = __dadd_rn(__dmul_rn(u[0], u[0]), __dmul_rn(u[1], u[1]));
    if (three) s = __dadd_rn(s, __dmul_rn(u[2], u[2]));
    return (float)sqrt(s);
  } else {
    float s = __fadd_rn(__fmul_rn(u[0], u[0]), __fmul_rn(u[1], u[1]));
    if (three) s = __fadd_rn(s, __fmul_rn(u[2], u[2]));
    return __fsqrt_rn(s);
  }
}

template <class M, class R, class St>
__global__ void k_color(const Args<R, M::NSET> a, int z, uchar4* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= a.nx || y >= a.ny) return;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int xm = (x == 0 ? nx : x) - 1, xp = (x + 1 == nx) ? 0 : x + 1;
  const int ym = (y == 0 ? ny : y) - 1, yp = (y + 1 == ny) ? 0 : y + 1;
  const int zm = (z == 0 ? nz : z) - 1, zp = (z + 1 == nz) ? 0 : z + 1;
  const typename St::T* src = static_cast<const typename St::T*>(a.src);
  R f[M::Q];
#pragma unroll
  for (int d = 0; d < M::Q; d++) {
    const int sx = M::ex(d) == 0 ? x : (M::ex(d) > 0 ? xm : xp);
    const int sy = M::ey(d) == 0 ? y : (M::ey(d) > 0 ? ym : yp);
    const int sz = M::DIM == 2 ? z : (M::ez(d) == 0 ? z : (M::ez(d) > 0 ? zm : zp));
    f[d] = St::template load<R>(src + (size_t)d * a.stride + (sx + nx * (sy + ny * sz)), R(M::w(d)));
  }
  const flag_t fl = a.flags[x + nx * (y + ny * z)];
  R u[3];
  M::template quantity<R>(1, f, fl, a, u);
  out[x + (size_t)nx * y] = color_map(speed<R>(u, M::DIM == 3), M::color_weight(fl));
}

// Kinetic energy and enstrophy of a velocity field (3 values per node, x
// fastest): E = 1/2 sum |u|^2 and Omega = 1/2 sum |curl u|^2 with second-order
// central differences on the periodic lattice (lattice units, dx = 1). FP64
// per-thread values, block reduction in shared memory, one FP64 atomic per
// block and quantity. 2D lattices (nz = 1) have only the z vorticity.
template <class R>
__global__ void __launch_bounds__(256) k_energy_enstrophy(const R* __restrict__ u, int nx, int ny, int nz,
                                                          double* out) {
  __shared__ double sh[2][256];
  const int tid = threadIdx.x;
  const size_t N = (size_t)nx * ny * nz;
  double e = 0.0, w = 0.0;
  for (size_t n = (size_t)blockIdx.x * blockDim.x + tid; n < N; n += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(n % nx), y = (int)((n / nx) % ny), z = (int)(n / ((size_t)nx * ny));
    const size_t sy = nx, sz = (size_t)nx * ny;
    const size_t xm = n - x + (x == 0 ? nx - 1 : x - 1), xp = n - x + (x + 1 == nx ? 0 : x + 1);
    const size_t ym = n + ((y == 0 ? ny - 1 : y - 1) - y) * sy, yp = n + ((y + 1 == ny ? 0 : y + 1) - y) * sy;
    const size_t zm = n + ((z == 0 ? nz - 1 : z - 1) - z) * sz, zp = n + ((z + 1 == nz ? 0 : z + 1) - z) * sz;
    const double ux = u[3 * n], uy = u[3 * n + 1], uz = u[3 * n + 2];
    e += 0.5 * (ux * ux + uy * uy + uz * uz);
    // d(u_c)/d(axis) = (u_c(+1) - u_c(-1)) / 2
    const double duz_dy = 0.5 * ((double)u[3 * yp + 2] - (double)u[3 * ym + 2]);
    const double duy_dz = nz > 1 ? 0.5 * ((double)u[3 * zp + 1] - (double)u[3 * zm + 1]) : 0.0;
    const double dux_dz = nz > 1 ? 0.5 * ((double)u[3 * zp] - (double)u[3 * zm]) : 0.0;
    const double duz_dx = 0.5 * ((double)u[3 * xp + 2] - (double)u[3 * xm + 2]);
    const double duy_dx = 0.5 * ((double)u[3 * xp + 1] - (double)u[3 * xm + 1]);
    const double dux_dy = 0.5 * ((double)u[3 * yp] - (double)u[3 * ym]);
    const double wx = duz_dy - duy_dz, wy = dux_dz - duz_dx, wz = duy_dx - dux_dy;
    w += 0.5 * (wx * wx + wy * wy + wz * wz);
  }
  sh[0][tid] = e;
  sh[1][tid] = w;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s) {
      sh[0][tid] += sh[0][tid + s];
      sh[1][tid] += sh[1][tid + s];
    }
    __syncthreads();
  }
  if (tid == 0) {
    atomicAdd(out, sh[0][0]);
    atomicAdd(out + 1, sh[1][0]);
  }
}

}  // namespace tclb
