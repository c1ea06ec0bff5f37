// CPU oracle for the TCLB lattice-Boltzmann hot path (d2q9, d3q19, d3q27_cumulant).
//
// TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA library is
// compared against; it is never linked into, loaded by, or called from the
// product library. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it.
//
// It restates, in plain C++ with OpenMP over nodes, the algorithm that TCLB's
// R templates expand into per-model C/CUDA code. Where TCLB generates closed
// forms symbolically (polyAlgebra), this oracle recomputes the same objects
// numerically and generically (moment matrices, Cholesky-weighted bases,
// Zou-He linear solves, moment/cumulant recursions), so that the product's
// hand-derived closed forms are checked against an independent construction.
//
// Parity status: pinned only by analytic invariants and by the hand-written
// closed forms in the reference (models/flow/d2q9_SRT/Dynamics.c:120-176); the
// reference ships no golden vectors for these models (tests/external is an
// absent submodule) and its build needs R + polyAlgebra, which are absent.
//
// Reference citations use paths inside the TCLB source tree.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

typedef uint16_t flag_t;

// ---------------------------------------------------------------------------
// Dense linear algebra helpers (double)
// ---------------------------------------------------------------------------
static std::vector<double> mat_inverse(std::vector<double> A, int n) {
  std::vector<double> I(n * n, 0.0);
  for (int i = 0; i < n; i++) I[i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (std::fabs(A[p * n + c]) < 1e-300) throw std::runtime_error("singular matrix");
    if (p != c)
      for (int k = 0; k < n; k++) {
        std::swap(A[p * n + k], A[c * n + k]);
        std::swap(I[p * n + k], I[c * n + k]);
      }
    double d = A[c * n + c];
    for (int k = 0; k < n; k++) { A[c * n + k] /= d; I[c * n + k] /= d; }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      double m = A[r * n + c];
      if (m == 0) continue;
      for (int k = 0; k < n; k++) { A[r * n + k] -= m * A[c * n + k]; I[r * n + k] -= m * I[c * n + k]; }
    }
  }
  return I;
}

static std::vector<double> mat_mul(const std::vector<double>& A, const std::vector<double>& B, int n, int m, int p) {
  std::vector<double> C(n * p, 0.0);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < m; k++)
      for (int j = 0; j < p; j++) C[i * p + j] += A[i * m + k] * B[k * p + j];
  return C;
}

static std::vector<double> transpose(const std::vector<double>& A, int n, int m) {
  std::vector<double> T(m * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++) T[j * n + i] = A[i * m + j];
  return T;
}

// Cholesky, upper factor U with A = U^T U (R's chol()).
static std::vector<double> chol_upper(const std::vector<double>& A, int n) {
  std::vector<double> U(n * n, 0.0);
  for (int j = 0; j < n; j++) {
    double s = A[j * n + j];
    for (int k = 0; k < j; k++) s -= U[k * n + j] * U[k * n + j];
    if (s <= 0) throw std::runtime_error("cholesky: not positive definite");
    U[j * n + j] = std::sqrt(s);
    for (int i = j + 1; i < n; i++) {
      double t = A[j * n + i];
      for (int k = 0; k < j; k++) t -= U[k * n + j] * U[k * n + i];
      U[j * n + i] = t / U[j * n + j];
    }
  }
  return U;
}

// ---------------------------------------------------------------------------
// Second-order equilibrium in a moment basis (src/lib/feq.R:9-82).
//
// A quantity that is a polynomial of (rho, J) truncated at J-degree 2 is
// stored as: a*rho + sum_d b[d]*J_d + sum_{d,e} c[d][e]*J_d*J_e/rho.
// ---------------------------------------------------------------------------
struct Poly2 {
  double a = 0, b[3] = {0, 0, 0}, c[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  void add(const Poly2& o, double s) {
    a += s * o.a;
    for (int d = 0; d < 3; d++) b[d] += s * o.b[d];
    for (int d = 0; d < 3; d++)
      for (int e = 0; e < 3; e++) c[d][e] += s * o.c[d][e];
  }
};

// Moment of the product-form equilibrium for exponent vector p, with
// sigma2 = 1/3, truncated to J-degree <= 2 (MRT_eq: feq.R:41-57;
// d3q19_MRT: d3q19.R:47-62).
static Poly2 eq_moment(const int* p, int D) {
  const double sig = 1.0 / 3.0;
  int n1 = 0, n2 = 0, a1[3], a2[3];
  for (int d = 0; d < D; d++) {
    if (p[d] == 1) a1[n1++] = d;
    if (p[d] == 2) a2[n2++] = d;
  }
  Poly2 h;
  if (n1 == 0) {
    h.a = std::pow(sig, n2);
    for (int i = 0; i < n2; i++) h.c[a2[i]][a2[i]] = std::pow(sig, n2 - 1);
  } else if (n1 == 1) {
    h.b[a1[0]] = std::pow(sig, n2);
  } else if (n1 == 2) {
    h.c[a1[0]][a1[1]] = std::pow(sig, n2);
  }
  return h;
}

struct Lattice_desc {
  int Q, D;
  std::vector<int> e;  // Q*3
  std::vector<int> opp;
};

// Velocity set exponent table, MRT_polyMatrix (feq.R:9-21): p = U with -1 -> 2.
// If 'sorted', rows are sorted by total order (stable), as MRT_polyMatrix does.
static void poly_matrix(const Lattice_desc& L, bool sorted, std::vector<int>& P, std::vector<int>& order,
                        std::vector<double>& M) {
  int Q = L.Q;
  std::vector<int> raw(Q * 3);
  for (int j = 0; j < Q; j++)
    for (int d = 0; d < 3; d++) raw[j * 3 + d] = L.e[j * 3 + d] < 0 ? 2 : L.e[j * 3 + d];
  std::vector<int> idx(Q);
  for (int i = 0; i < Q; i++) idx[i] = i;
  if (sorted)
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
      return raw[x * 3] + raw[x * 3 + 1] + raw[x * 3 + 2] < raw[y * 3] + raw[y * 3 + 1] + raw[y * 3 + 2];
    });
  P.assign(Q * 3, 0);
  order.assign(Q, 0);
  for (int i = 0; i < Q; i++) {
    for (int d = 0; d < 3; d++) P[i * 3 + d] = raw[idx[i] * 3 + d];
    order[i] = P[i * 3] + P[i * 3 + 1] + P[i * 3 + 2];
  }
  M.assign(Q * Q, 0.0);
  for (int j = 0; j < Q; j++)
    for (int i = 0; i < Q; i++) {
      double v = 1;
      for (int d = 0; d < 3; d++) v *= std::pow((double)L.e[j * 3 + d], P[i * 3 + d]);  // 0^0 = 1
      M[j * Q + i] = v;
    }
}

// Equilibrium distribution coefficients: feq_j = H . Minv[:, j].
static std::vector<Poly2> feq_from_moments(const Lattice_desc& L, const std::vector<int>& P, const std::vector<double>& Minv) {
  int Q = L.Q;
  std::vector<Poly2> H(Q), feq(Q);
  for (int i = 0; i < Q; i++) H[i] = eq_moment(&P[i * 3], L.D);
  for (int j = 0; j < Q; j++)
    for (int i = 0; i < Q; i++) feq[j].add(H[i], Minv[i * Q + j]);
  return feq;
}

template <class R>
struct PolyR {  // Poly2 evaluated in arithmetic type R
  R a, b[3], c[3][3];
  void set(const Poly2& p) {
    a = (R)p.a;
    for (int d = 0; d < 3; d++) b[d] = (R)p.b[d];
    for (int d = 0; d < 3; d++)
      for (int e = 0; e < 3; e++) c[d][e] = (R)p.c[d][e];
  }
  R eval(R rho, const R* J, int D) const {
    R s = a * rho, q = 0;
    for (int d = 0; d < D; d++) s += b[d] * J[d];
    for (int d = 0; d < D; d++)
      for (int e = 0; e < D; e++) q += c[d][e] * J[d] * J[e];
    return s + q / rho;
  }
};

// ---------------------------------------------------------------------------
// Model tables. Node-type values follow the packing rule of src/conf.R:600-699
// (groups in alphabetical order, ceil(log2(n+1)) bits per group, zone index in
// the remaining high bits).
// ---------------------------------------------------------------------------
enum { M_D2Q9 = 0, M_D3Q19 = 1, M_D3Q27C = 2 };

struct NodeTypeDef { const char* name; const char* group; int value; int mask; };

// d2q9: models/flow/d2q9/Dynamics.R:69-88
static const NodeTypeDef nt_d2q9[] = {
    {"EPressure", "BOUNDARY", 1, 0xF},  {"WPressure", "BOUNDARY", 2, 0xF}, {"NVelocity", "BOUNDARY", 3, 0xF},
    {"SVelocity", "BOUNDARY", 4, 0xF},  {"WVelocity", "BOUNDARY", 5, 0xF}, {"EVelocity", "BOUNDARY", 6, 0xF},
    {"NSymmetry", "BOUNDARY", 7, 0xF},  {"SSymmetry", "BOUNDARY", 8, 0xF}, {"Solid", "BOUNDARY", 9, 0xF},
    {"Wall", "BOUNDARY", 10, 0xF},      {"MRT", "COLLISION", 0x10, 0x10},  {"Inlet", "OBJECTIVE", 0x20, 0x60},
    {"Outlet", "OBJECTIVE", 0x40, 0x60}};
// d3q19: models/flow/d3q19/Dynamics.R:44-92
static const NodeTypeDef nt_d3q19[] = {
    {"XYslice", "ADDITIONALS", 1, 3},      {"XZslice", "ADDITIONALS", 2, 3},    {"YZslice", "ADDITIONALS", 3, 3},
    {"EPressure", "BOUNDARY", 0x04, 0x1C}, {"Solid", "BOUNDARY", 0x08, 0x1C},   {"Wall", "BOUNDARY", 0x0C, 0x1C},
    {"WPressure", "BOUNDARY", 0x10, 0x1C}, {"WPressureL", "BOUNDARY", 0x14, 0x1C}, {"WVelocity", "BOUNDARY", 0x18, 0x1C},
    {"MRT", "COLLISION", 0x20, 0x20}};
// d3q27_cumulant: models/flow/d3q27_cumulant/Dynamics.R:37-98
static const NodeTypeDef nt_d3q27c[] = {
    {"NSymmetry", "ADDITIONALS", 1, 3},     {"SSymmetry", "ADDITIONALS", 2, 3},
    {"Body", "BODY", 4, 4},                 {"Buffer", "BOUNDARY", 0x08, 0x78},
    {"WVelocityTurbulent", "BOUNDARY", 0x10, 0x78}, {"NVelocity", "BOUNDARY", 0x18, 0x78},
    {"SVelocity", "BOUNDARY", 0x20, 0x78},  {"NPressure", "BOUNDARY", 0x28, 0x78},
    {"SPressure", "BOUNDARY", 0x30, 0x78},  {"EPressure", "BOUNDARY", 0x38, 0x78},
    {"EVelocity", "BOUNDARY", 0x40, 0x78},  {"Solid", "BOUNDARY", 0x48, 0x78},
    {"Wall", "BOUNDARY", 0x50, 0x78},       {"WPressure", "BOUNDARY", 0x58, 0x78},
    {"WVelocity", "BOUNDARY", 0x60, 0x78},  {"MRT", "COLLISION", 0x80, 0x80}};

static int nt_value(int model, const char* name) {
  const NodeTypeDef* t;
  int n;
  if (model == M_D2Q9) { t = nt_d2q9; n = sizeof(nt_d2q9) / sizeof(*t); }
  else if (model == M_D3Q19) { t = nt_d3q19; n = sizeof(nt_d3q19) / sizeof(*t); }
  else { t = nt_d3q27c; n = sizeof(nt_d3q27c) / sizeof(*t); }
  for (int i = 0; i < n; i++)
    if (!strcmp(t[i].name, name)) return t[i].value;
  throw std::runtime_error(std::string("unknown node type ") + name);
}

struct SettingDef { const char* name; double def; int has_default; int unused; };

// Settings (non-zonal) in TCLB index order, with defaults applied only to
// settings that derive nothing (src/Solver.cpp.Rt:276-281).
static const SettingDef st_d2q9[] = {{"RelaxationRate", 0, 0, 4}, {"Viscosity", 0.16666666, 0, 0},
                                     {"GravitationX", 0, 1, -1},  {"GravitationY", 0, 1, -1},
                                     {"S2", 0, 1, -1},            {"S3", 0, 1, -1},
                                     {"S4", 0, 1, -1},            {"Threshold", 0.5, 1, -1}};
static const SettingDef st_d3q19[] = {{"omega", 0, 1, -1},        {"nu", 0.16666666, 0, 0},
                                      {"InletVelocity", 0, 1, -1}, {"InletPressure", 0, 0, 4},
                                      {"InletDensity", 1, 1, -1},  {"ForceX", 0, 1, -1},
                                      {"ForceY", 0, 1, -1},        {"ForceZ", 0, 1, -1},
                                      {"Threshold", 0.5, 1, -1}};
static const SettingDef st_d3q27c[] = {{"nu", 0.16666666, 1, -1}, {"nubuffer", 0.01, 1, -1},
                                       {"GalileanCorrection", 1, 1, -1}, {"ForceX", 0, 1, -1},
                                       {"ForceY", 0, 1, -1},      {"ForceZ", 0, 1, -1},
                                       {"Omega", 1, 1, -1},       {"Threshold", 0.5, 1, -1}};

// Derived-setting equations (Dynamics.R AddSetting(..., X='expr')).
static double derive(int model, int from, double v) {
  if (model == M_D2Q9) {
    if (from == 1) return 1.0 / (3 * v + 0.5);  // Viscosity -> RelaxationRate
    if (from == 0) return 1 - v;                // RelaxationRate -> S2
  } else if (model == M_D3Q19) {
    if (from == 1) return 1.0 / (3 * v + 0.5);  // nu -> omega
    if (from == 3) return 1.0 + v * 3;          // InletPressure -> InletDensity
  }
  return v;
}
static int derived_target(int model, int from) {
  if (model == M_D2Q9) { if (from == 1) return 0; if (from == 0) return 4; }
  if (model == M_D3Q19) { if (from == 1) return 0; if (from == 3) return 4; }
  return -1;
}

struct ModelInfo {
  int Q, D, nset, nzs, nglob, nsum, zone_shift, in_obj_offset, obj_idx;
  const SettingDef* st;
  std::vector<double> zs_default;
};

static ModelInfo model_info(int model) {
  ModelInfo m;
  if (model == M_D2Q9) {
    m.Q = 9; m.D = 2; m.nset = 8; m.nzs = 6; m.nglob = 4; m.nsum = 4; m.zone_shift = 7; m.in_obj_offset = 3;
    m.obj_idx = 3; m.st = st_d2q9; m.zs_default.assign(6, 0.0);
  } else if (model == M_D3Q19) {
    m.Q = 19; m.D = 3; m.nset = 9; m.nzs = 24; m.nglob = 26; m.nsum = 25; m.zone_shift = 6; m.in_obj_offset = 0;
    m.obj_idx = 24; m.st = st_d3q19; m.zs_default.assign(24, 0.0);
  } else if (model == M_D3Q27C) {
    m.Q = 27; m.D = 3; m.nset = 8; m.nzs = 12; m.nglob = 10; m.nsum = 10; m.zone_shift = 8; m.in_obj_offset = 3;
    m.obj_idx = 9; m.st = st_d3q27c; m.zs_default.assign(12, 0.0);
  } else throw std::runtime_error("bad model");
  return m;
}

// ---------------------------------------------------------------------------
// Velocity sets
// ---------------------------------------------------------------------------
static Lattice_desc make_lattice(int model) {
  Lattice_desc L;
  if (model == M_D2Q9) {  // models/flow/d2q9/Dynamics.R:6-14
    const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    L.Q = 9; L.D = 2;
    for (int i = 0; i < 9; i++) { L.e.push_back(ex[i]); L.e.push_back(ey[i]); L.e.push_back(0); }
  } else if (model == M_D3Q19) {  // d3q19/Dynamics.R:26-35 (columns 4,6,8 of MRTMAT)
    const int e[19][3] = {{0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                          {1, 1, 0},  {-1, 1, 0},  {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1}, {1, 0, -1},
                          {-1, 0, -1}, {0, 1, 1},  {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
    L.Q = 19; L.D = 3;
    for (int i = 0; i < 19; i++)
      for (int d = 0; d < 3; d++) L.e.push_back(e[i][d]);
  } else {  // d3q27_cumulant/Dynamics.R:1-13: f<a><b><c>, a,b,c in {0,1,2} -> {0,+1,-1}
    const int m[3] = {0, 1, -1};
    L.Q = 27; L.D = 3;
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++)
        for (int a = 0; a < 3; a++) { L.e.push_back(m[a]); L.e.push_back(m[b]); L.e.push_back(m[c]); }
  }
  L.opp.assign(L.Q, -1);
  for (int i = 0; i < L.Q; i++)
    for (int j = 0; j < L.Q; j++)
      if (L.e[j * 3] == -L.e[i * 3] && L.e[j * 3 + 1] == -L.e[i * 3 + 1] && L.e[j * 3 + 2] == -L.e[i * 3 + 2]) L.opp[i] = j;
  return L;
}

// d'Humieres D3Q19 matrix: lib/d3q19.R:1-21 (R fills column-major, so each
// printed row there is one moment, i.e. one column of MRTMAT[direction,moment]).
static const int MRT19[19][19] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
    {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, -4, 4, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
    {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    {0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, -1, -1, 1, 1}};

// ---------------------------------------------------------------------------
// Per-model precomputed operators
// ---------------------------------------------------------------------------
template <class R>
struct Ops {
  int model;
  Lattice_desc L;
  ModelInfo info;
  std::vector<PolyR<R>> feq;  // equilibrium distribution (monomial construction)
  // d2q9 MRT (d2q9/Dynamics.c.Rt:8-23, 202-268)
  std::vector<R> B, Binv;      // B[i*Q+k]; Binv[k*Q+i]
  std::vector<int> Border;     // order of each B column
  std::vector<PolyR<R>> ReqB;  // equilibrium moments in B
  // d3q19 (d3q19/Dynamics.c.Rt:223-290)
  std::vector<PolyR<R>> Req19;
  R Mw[19];
  // Zou-He: odd part of the equilibrium: feq_i - feq_opp(i) = sum_d zh[i][d] J_d
  std::vector<R> zh;  // Q*3
  // d3q27 cumulant recursion terms
  struct Term { int n, k, m; R coef; };
  std::vector<Term> cum_fwd;  // kappa(n) -= coef*kappa(k)*m(m)
  std::vector<Term> cum_bwd;  // m(n) += coef*kappa(k)*m(m)

  void build(int model_) {
    model = model_;
    L = make_lattice(model);
    info = model_info(model);
    int Q = L.Q;
    std::vector<int> P, order;
    std::vector<double> M;
    // monomial basis: sorted as MRT_polyMatrix does for d2q9/d3q27; the d3q19
    // construction (d3q19.R:44-45) keeps direction order -- equivalent feq.
    poly_matrix(L, model != M_D3Q19, P, order, M);
    std::vector<double> Minv = mat_inverse(M, Q);
    std::vector<Poly2> feqd = feq_from_moments(L, P, Minv);
    feq.resize(Q);
    for (int i = 0; i < Q; i++) feq[i].set(feqd[i]);
    // Zou-He odd part (lib/boundary.R:80-84, 163-170)
    zh.assign(Q * 3, 0);
    for (int i = 0; i < Q; i++)
      for (int d = 0; d < 3; d++) zh[i * 3 + d] = (R)(feqd[i].b[d] - feqd[L.opp[i]].b[d]);
    if (model == M_D2Q9) build_d2q9(M, Minv, order, feqd);
    if (model == M_D3Q19) build_d3q19(feqd);
    if (model == M_D3Q27C) build_cumulant();
  }

  // d2q9/Dynamics.c.Rt:8-23: B = M * t(H), H from the Cholesky factor of the
  // reversed metric M^-1 diag(1/w) M^-T, rows scaled by fixed constants.
  void build_d2q9(const std::vector<double>& M, const std::vector<double>& Minv, const std::vector<int>& order,
                  const std::vector<Poly2>& feqd) {
    int Q = 9;
    std::vector<double> w(Q);
    for (int i = 0; i < Q; i++) w[i] = feqd[i].a;  // feq at rho=1, J=0
    std::vector<double> Dinv(Q * Q, 0.0);
    for (int i = 0; i < Q; i++) Dinv[i * Q + i] = 1.0 / w[i];
    std::vector<double> MinvT = transpose(Minv, Q, Q);
    std::vector<double> W = mat_mul(mat_mul(Minv, Dinv, Q, Q, Q), MinvT, Q, Q, Q);
    std::vector<double> Wr(Q * Q);
    for (int i = 0; i < Q; i++)
      for (int j = 0; j < Q; j++) Wr[i * Q + j] = W[(Q - 1 - i) * Q + (Q - 1 - j)];
    std::vector<double> U = chol_upper(Wr, Q);
    std::vector<double> H(Q * Q);
    for (int i = 0; i < Q; i++)
      for (int j = 0; j < Q; j++) H[i * Q + j] = U[(Q - 1 - i) * Q + (Q - 1 - j)];
    const double sc[9] = {1, std::sqrt(3.0) / 3, std::sqrt(3.0) / 3, std::sqrt(2.0), std::sqrt(2.0), 1,
                          std::sqrt(6.0) / 3, std::sqrt(6.0) / 3, 2};
    for (int i = 0; i < Q; i++)
      for (int j = 0; j < Q; j++) H[i * Q + j] *= sc[i];
    std::vector<double> Bd = mat_mul(M, transpose(H, Q, Q), Q, Q, Q);
    for (auto& v : Bd) v = std::round(v * 1e9) / 1e9;  // entries are small integers
    std::vector<double> Bdinv = mat_inverse(Bd, Q);
    // column orders (feq.R:70): max order of monomials present
    std::vector<double> T = mat_mul(Minv, Bd, Q, Q, Q);
    Border.assign(Q, 0);
    for (int k = 0; k < Q; k++)
      for (int j = 0; j < Q; j++)
        if (std::fabs(T[j * Q + k]) > 1e-10) Border[k] = std::max(Border[k], order[j]);
    B.resize(Q * Q); Binv.resize(Q * Q);
    for (int i = 0; i < Q * Q; i++) { B[i] = (R)Bd[i]; Binv[i] = (R)Bdinv[i]; }
    ReqB.resize(Q);
    for (int k = 0; k < Q; k++) {
      Poly2 p;
      for (int i = 0; i < Q; i++) p.add(feqd[i], Bd[i * Q + k]);
      ReqB[k].set(p);
    }
  }

  void build_d3q19(const std::vector<Poly2>& feqd) {
    Req19.resize(19);
    for (int k = 0; k < 19; k++) {
      Poly2 p;
      for (int i = 0; i < 19; i++) p.add(feqd[i], MRT19[k][i]);
      Req19[k].set(p);
      int s = 0;
      for (int i = 0; i < 19; i++) s += MRT19[k][i] * MRT19[k][i];
      Mw[k] = (R)s;
    }
  }

  // Moment <-> cumulant recursion (lib/cumulant.R:7-42): for multi-index n,
  // pick an axis j with n_j>0 (fewest product terms, ties to the lowest axis),
  // n' = n - e_j, and use m(n) = sum_{k<=n'} C(n',k) kappa(k+e_j) m(n'-k).
  void build_cumulant() {
    auto idx = [](int a, int b, int c) { return a + 3 * b + 9 * c; };
    auto binom = [](int n, int k) { return (n == 2 && k == 1) ? 2 : 1; };
    for (int n = 1; n < 27; n++) {
      int na[3] = {n % 3, (n / 3) % 3, n / 9};
      int best = -1, bestc = 1 << 30;
      for (int j = 0; j < 3; j++) {
        if (na[j] == 0) continue;
        int cnt = 1;
        for (int d = 0; d < 3; d++) cnt *= (na[d] - (d == j ? 1 : 0)) + 1;
        if (cnt < bestc) { bestc = cnt; best = j; }
      }
      int np[3] = {na[0], na[1], na[2]};
      np[best] -= 1;
      for (int k0 = 0; k0 <= np[0]; k0++)
        for (int k1 = 0; k1 <= np[1]; k1++)
          for (int k2 = 0; k2 <= np[2]; k2++) {
            int kk[3] = {k0, k1, k2};
            int kp[3] = {k0, k1, k2};
            kp[best] += 1;
            int ki = idx(kp[0], kp[1], kp[2]);
            int mi = idx(np[0] - k0, np[1] - k1, np[2] - k2);
            R coef = (R)(binom(np[0], kk[0]) * binom(np[1], kk[1]) * binom(np[2], kk[2]));
            if (ki == n) continue;  // the kappa(n)*m000 term
            cum_fwd.push_back({n, ki, mi, coef});
            cum_bwd.push_back({n, ki, mi, coef});
          }
    }
  }
};

// ---------------------------------------------------------------------------
// Lattice
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Storage emulation: the checker for the CUDA library's 16-bit storage
// formats. A population is stored as g = float(f - w_i) (TCLB's half-shift,
// src/LatticeAccess.inc.cpp.Rt:29-35) rounded to the format, and read back as
// decode(g) + w_i. The conversions are written here from the IEEE 754
// binary16 and bfloat16 definitions with integer bit operations; "stochastic"
// rounding rounds the magnitude up with probability equal to the discarded
// fraction, using 32 random bits per value from the integer hash below.
// ---------------------------------------------------------------------------
enum StorageEmu { EMU_NONE = 0, EMU_F16_RN = 1, EMU_F16_SR = 2, EMU_BF16_RN = 3, EMU_BF16_SR = 4, EMU_MANT = 5,
                  EMU_FIXED = 6, EMU_EXM = 7 };

// 32-bit integer hash "lowbias32" (C. Wellons, "Prospecting for Hash Functions", 2018).
static inline uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}
static inline uint32_t f2u(float v) { uint32_t b; std::memcpy(&b, &v, 4); return b; }
static inline float u2f(uint32_t b) { float v; std::memcpy(&v, &b, 4); return v; }

// float -> binary16 bits; sr: round up the magnitude when discarded + (rnd & mask) carries.
static uint16_t f32_to_f16(float v, bool sr, uint32_t rnd) {
  const uint32_t b = f2u(v), s = (b >> 16) & 0x8000u, a = b & 0x7fffffffu;
  if (a >= 0x7f800000u) return (uint16_t)(s | 0x7c00u | (a > 0x7f800000u ? 0x200u : 0));
  const int e = (int)(a >> 23) - 127;
  if (e >= -14) {  // binary16 normal range: drop 13 mantissa bits
    uint32_t val = ((uint32_t)(e + 15) << 10) | ((a & 0x7fffffu) >> 13);
    const uint32_t rem = a & 0x1fffu;
    if (sr) val += (rem + (rnd & 0x1fffu)) >> 13;
    else if (rem > 0x1000u || (rem == 0x1000u && (val & 1u))) val++;
    if (val >= 0x7c00u) val = 0x7c00u;  // overflow: infinity
    return (uint16_t)(s | val);
  }
  // subnormal: units of 2^-24; the 24-bit significand times 2^(e+1)
  const int shift = -e - 1;
  if (shift > 31) return (uint16_t)s;
  const uint64_t mf = (a & 0x7fffffu) | 0x800000u;
  uint64_t q = mf >> shift;
  const uint64_t rem = mf & ((1ull << shift) - 1), full = 1ull << shift;
  if (sr) q += (rem + ((uint64_t)rnd & (full - 1))) >> shift;
  else if (rem > full / 2 || (rem == full / 2 && (q & 1))) q++;
  return (uint16_t)(s | (uint32_t)q);
}
static float f16_to_f32(uint16_t h) {
  const uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1f, m = h & 0x3ffu;
  if (e == 0x1f) return u2f(s | 0x7f800000u | (m << 13));
  if (e == 0) return (s ? -1.0f : 1.0f) * (float)m * 5.9604644775390625e-8f;  // m * 2^-24
  return u2f(s | ((e + 112) << 23) | (m << 13));
}
static uint16_t f32_to_bf16(float v, bool sr, uint32_t rnd) {
  const uint32_t b = f2u(v);
  if ((b & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((b >> 16) | 0x40u);
  if (sr) return (uint16_t)((b + (rnd & 0xffffu)) >> 16);  // magnitude bits carry on sign-magnitude
  return (uint16_t)((b + 0x7fffu + ((b >> 16) & 1u)) >> 16);
}
static float bf16_to_f32(uint16_t h) { return u2f((uint32_t)h << 16); }

// Random bits of population i of node n written by iteration it.
static inline uint32_t storage_bits(uint32_t seed, long it, size_t n, int i) {
  return hash32(hash32((uint32_t)n ^ seed) + hash32((uint32_t)(it * 27 + i)));
}

// g rounded to nearest with k explicit mantissa bits (FP32 exponent range)
static inline float round_mantissa(float g, int k) {
  const uint32_t b = f2u(g), drop = 23 - k, half = 1u << (drop - 1), rem = b & ((1u << drop) - 1);
  uint32_t r = b - rem;
  if (rem > half || (rem == half && ((b >> drop) & 1u))) r += 1u << drop;
  return u2f(r);
}
// g stored as a signed 16-bit integer count of w * scale / 32768
static inline float round_fixed(float g, double w, double scale) {
  const double unit = w * scale / 32768.0;
  double q = std::nearbyint((double)g / unit);
  q = std::min(32767.0, std::max(-32768.0, q));
  return (float)(q * unit);
}

// h = g / w in a 16-bit float with E exponent bits, 15 - E mantissa bits and top S (param = E * 16 + log2(1/S)):
// binades [S 2^-k-1, S 2^-k) for k < 2^E - 1, then a subnormal range of spacing S 2^-(2^E - 1) 2^-(15-E).
static inline double round_exm_d(double g, double w, double param) {
  const int E = (int)param / 16, L = (int)param % 16, M = 15 - E;
  const double S = std::ldexp(1.0, -L), h = (double)g / w, a = std::fabs(h);
  const int nb = (1 << E) - 1;  // normal binades
  int k = 0;                    // binade below the top
  double unit;
  if (a >= S) return std::copysign(S - std::ldexp(S, -1 - M), h) * w;  // saturate
  if (E == 0) unit = std::ldexp(S, -M);
  else {
    while (k < nb && a < std::ldexp(S, -1 - k)) k++;
    unit = k < nb ? std::ldexp(S, -1 - k - M) : std::ldexp(S, -nb - M);
  }
  const double q = std::nearbyint(a / unit) * unit;
  return std::copysign(std::min(q, S - std::ldexp(S, -1 - M)), h) * w;
}

template <class R>
static inline R storage_roundtrip(int mode, R f, double w, uint32_t rnd, double param = 0) {
  // the deviation in the oracle's arithmetic, then rounded to the format
  const R wr = (R)w;
  const float g = (float)(f - wr);
  float d;
  switch (mode) {
    case EMU_MANT: d = round_mantissa(g, (int)param); break;
    case EMU_FIXED: d = round_fixed(g, w, param); break;
    case EMU_EXM: return (R)round_exm_d((double)(f - wr), w, param) + wr;
    case EMU_F16_RN: d = f16_to_f32(f32_to_f16(g, false, 0)); break;
    case EMU_F16_SR: d = f16_to_f32(f32_to_f16(g, true, rnd)); break;
    case EMU_BF16_RN: d = bf16_to_f32(f32_to_bf16(g, false, 0)); break;
    case EMU_BF16_SR: d = bf16_to_f32(f32_to_bf16(g, true, rnd)); break;
    default: return f;
  }
  return (R)d + wr;
}

struct GlobAcc {
  std::vector<double> v;
};

template <class R>
struct Lattice {
  int model, nx, ny, nz;
  size_t N;
  Ops<R> ops;
  std::vector<R> buf[2];
  int cur = 0;
  std::vector<flag_t> flags;
  std::vector<double> settings;
  std::vector<double> zone;  // zones * nzs
  int nzones;
  // Globals are kept as 2*nglob values: the sums, then the sums of absolute
  // contributions (the scale the tests measure summation and rounding
  // differences against).
  std::vector<double> dev_globals;  // per-iteration integrated globals (device side in TCLB)
  std::vector<double> globals;      // host accumulators (Lattice::globals)
  long iter = 0;
  int storage_mode = EMU_NONE;  // storage emulation of the iteration's stores
  uint32_t storage_seed = 0;
  double storage_param = 0;     // EMU_MANT: mantissa bits; EMU_FIXED: range of (f - w) / w
  std::vector<double> wts;      // lattice weights: the storage shift

  Lattice(int m, int nx_, int ny_, int nz_) : model(m), nx(nx_), ny(ny_), nz(nz_) {
    ops.build(m);
    N = (size_t)nx * ny * nz;
    int Q = ops.L.Q;
    buf[0].assign(Q * N, (R)0);
    buf[1].assign(Q * N, (R)0);
    flags.assign(N, 0);
    const ModelInfo& I = ops.info;
    settings.assign(I.nset, 0.0);
    for (int s = 0; s < I.nset; s++)
      if (I.st[s].has_default) settings[s] = I.st[s].def;
    nzones = 1 << (16 - I.zone_shift);
    zone.assign((size_t)nzones * I.nzs, 0.0);
    for (int z = 0; z < nzones; z++)
      for (int s = 0; s < I.nzs; s++) zone[(size_t)z * I.nzs + s] = I.zs_default[s];
    dev_globals.assign(2 * I.nglob, 0.0);
    globals.assign(2 * I.nglob, 0.0);
    wts.resize(Q);
    for (int i = 0; i < Q; i++) wts[i] = ops.feq[i].a;  // feq at rho = 1, J = 0
  }

  void set_setting(int i, double v) {  // Lattice::SetSetting (src/Lattice.cu.Rt:1350-1358)
    settings[i] = v;
    int t = derived_target(model, i);
    if (t >= 0) set_setting(t, derive(model, i, v));
  }

  R S(int i) const { return (R)settings[i]; }
  R Z(int s, flag_t fl) const { return (R)zone[(size_t)(fl >> ops.info.zone_shift) * ops.info.nzs + s]; }

  // AddTo<G>(x): value plus the Objective quirk (src/cuda.cu.Rt:114-119).
  inline void add(std::vector<double>& g, int gi, R x, flag_t fl) const {
    const int ng = ops.info.nglob;
    g[gi] += (double)x;
    g[ng + gi] += std::fabs((double)x);
    if (gi < ops.info.nsum) {
      const double w = (double)Z(gi + ops.info.in_obj_offset, fl);
      g[ops.info.obj_idx] += w;
      g[ng + ops.info.obj_idx] += std::fabs(w);
    }
  }
  inline void maxg(std::vector<double>& g, int gi, R x) const {
    g[gi] = std::max(g[gi], (double)x);
    g[ops.info.nglob + gi] = std::max(g[ops.info.nglob + gi], std::fabs((double)x));
  }

  // ---------------- d2q9 (models/flow/d2q9/Dynamics.c.Rt) ----------------
  void feq_fill(R* f, R rho, const R* J) const {
    for (int i = 0; i < ops.L.Q; i++) f[i] = ops.feq[i].eval(rho, J, ops.L.D);
  }

  // ZouHeRewrite (lib/boundary.R:143-198): normal n along axis 'ax' with sign
  // 'sg'; unknown populations are those with e.n < 0.
  void zouhe_rewrite(R* f, int ax, int sg, bool velocity, const R* V, R rho0) const {
    const int Q = ops.L.Q, D = ops.L.D;
    const int* e = ops.L.e.data();
    bool sel[27];
    for (int i = 0; i < Q; i++) sel[i] = (e[i * 3 + ax] * sg) < 0;
    // fs(R) = f_known, or f_opp + zh.R for unknowns; represented as affine
    // functions: fs_i = c0_i + sum_d c_i[d] R_d
    R c0[27], c[27][3];
    for (int i = 0; i < Q; i++) {
      for (int d = 0; d < 3; d++) c[i][d] = 0;
      if (sel[i]) {
        c0[i] = f[ops.L.opp[i]];
        for (int d = 0; d < D; d++) c[i][d] = ops.zh[i * 3 + d];
      } else c0[i] = f[i];
    }
    // equations eqn_k(R) = e0[k] + sum_d ec[k][d] R_d
    R e0[3] = {0, 0, 0}, ec[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    R s0 = 0, sc[3] = {0, 0, 0};
    for (int i = 0; i < Q; i++) { s0 += c0[i]; for (int d = 0; d < D; d++) sc[d] += c[i][d]; }
    for (int k = 0; k < D; k++) {
      R m0 = 0, mc[3] = {0, 0, 0};
      for (int i = 0; i < Q; i++) {
        m0 += c0[i] * (R)e[i * 3 + k];
        for (int d = 0; d < D; d++) mc[d] += c[i][d] * (R)e[i * 3 + k];
      }
      if (velocity) {  // sum fs U_k - V_k sum fs
        e0[k] = m0 - V[k] * s0;
        for (int d = 0; d < D; d++) ec[k][d] = mc[d] - V[k] * sc[d];
      } else if (k == ax) {  // sum fs - rho0
        e0[k] = s0 - rho0;
        for (int d = 0; d < D; d++) ec[k][d] = sc[d];
      } else {  // sum fs U_k
        e0[k] = m0;
        for (int d = 0; d < D; d++) ec[k][d] = mc[d];
      }
    }
    R Rv[3] = {0, 0, 0};
    Rv[ax] = -e0[ax] / ec[ax][ax];
    for (int k = 0; k < D; k++) {
      if (k == ax) continue;
      Rv[k] = -(e0[k] + ec[k][ax] * Rv[ax]) / ec[k][k];
    }
    for (int i = 0; i < Q; i++)
      if (sel[i]) {
        R v = c0[i];
        for (int d = 0; d < D; d++) v += c[i][d] * Rv[d];
        f[i] = v;
      }
  }

  // Symmetry (lib/boundary.R:37-53): populations whose component on 'ax' has
  // the sign 'sg' are replaced by their mirror images.
  void symmetry(R* f, int ax, int sg) const {
    const int Q = ops.L.Q;
    const int* e = ops.L.e.data();
    R g[27];
    for (int i = 0; i < Q; i++) g[i] = f[i];
    for (int i = 0; i < Q; i++) {
      if (e[i * 3 + ax] * sg <= 0) continue;
      for (int j = 0; j < Q; j++) {
        bool m = true;
        for (int d = 0; d < 3; d++) m = m && (e[j * 3 + d] == (d == ax ? -e[i * 3 + d] : e[i * 3 + d]));
        if (m) { f[i] = g[j]; break; }
      }
    }
  }

  void bounce(R* f) const {
    R g[27];
    for (int i = 0; i < ops.L.Q; i++) g[i] = f[i];
    for (int i = 0; i < ops.L.Q; i++) f[i] = g[ops.L.opp[i]];
  }

  void d2q9_mrt(R* f, flag_t fl, std::vector<double>* G) const {
    const int Q = 9;
    R Rm[9];
    for (int k = 0; k < Q; k++) {
      R s = 0;
      for (int i = 0; i < Q; i++) s += f[i] * ops.B[i * Q + k];
      Rm[k] = s;
    }
    R rho = Rm[0], J[3] = {Rm[1], Rm[2], 0};
    if (G) {  // d2q9/Dynamics.c.Rt:228-246
      R Usq = (J[0] * J[0] + J[1] * J[1]) / (rho * rho);
      int obj = fl & 0x60;
      if (obj == 0x40) {  // Outlet
        add(*G, 1, J[0] / rho / rho, fl);
        add(*G, 0, -(J[0] / rho) / rho * ((rho - (R)1) / (R)3 + Usq / rho / (R)2), fl);
      } else if (obj == 0x20) {  // Inlet
        add(*G, 2, J[0] / rho / rho, fl);
        add(*G, 0, (J[0] / rho) / rho * ((rho - (R)1) / (R)3 + Usq / rho / (R)2), fl);
      }
    }
    R Sv[5] = {0, 0, S(4), S(5), S(6)};
    for (int k = 0; k < Q; k++)
      if (ops.Border[k] > 1) Rm[k] = (Rm[k] - ops.ReqB[k].eval(rho, J, 2)) * Sv[ops.Border[k]];
    J[0] = J[0] + S(2) * rho;
    J[1] = J[1] + S(3) * rho;
    Rm[1] = J[0]; Rm[2] = J[1];
    for (int k = 0; k < Q; k++)
      if (ops.Border[k] > 1) Rm[k] = Rm[k] + ops.ReqB[k].eval(rho, J, 2);
    for (int i = 0; i < Q; i++) {
      R s = 0;
      for (int k = 0; k < Q; k++) s += Rm[k] * ops.Binv[k * Q + i];
      f[i] = s;
    }
  }

  void d2q9_run(R* f, flag_t fl, std::vector<double>* G) const {
    R V[3] = {Z(0, fl), Z(1, fl), 0};
    R rho0 = Z(2, fl) * (R)3 + (R)1;
    switch (fl & 0xF) {  // d2q9/Dynamics.c.Rt:108-143
      case 9: case 10: bounce(f); break;
      case 6: zouhe_rewrite(f, 0, 1, true, V, rho0); break;    // EVelocity
      case 2: zouhe_rewrite(f, 0, -1, false, V, rho0); break;  // WPressure
      case 5: zouhe_rewrite(f, 0, -1, true, V, rho0); break;   // WVelocity
      case 1: zouhe_rewrite(f, 0, 1, false, V, rho0); break;   // EPressure
      case 3: zouhe_rewrite(f, 1, 1, true, V, rho0); break;    // NVelocity
      case 4: zouhe_rewrite(f, 1, -1, true, V, rho0); break;   // SVelocity
      case 7: symmetry(f, 1, -1); break;                       // NSymmetry
      case 8: symmetry(f, 1, 1); break;                        // SSymmetry
      default: break;
    }
    if (fl & 0x10) d2q9_mrt(f, fl, G);
  }

  void d2q9_init(R* f, flag_t fl) const {  // d2q9/Dynamics.c.Rt:91-106
    R rho = (R)1 + Z(2, fl) * (R)3, ux = Z(0, fl), uy = Z(1, fl);
    if ((fl & 0xF) == 10) { rho = 1; ux = 0; uy = 0; }
    R J[3] = {ux * rho, uy * rho, 0};
    // SetEquilibrum: f = Req %*% solve(B) (the Req of the conserved moments are rho, J)
    R Rm[9];
    for (int k = 0; k < 9; k++) Rm[k] = ops.ReqB[k].eval(rho, J, 2);
    for (int i = 0; i < 9; i++) {
      R s = 0;
      for (int k = 0; k < 9; k++) s += Rm[k] * ops.Binv[k * 9 + i];
      f[i] = s;
    }
  }

  // ---------------- d3q19 (models/flow/d3q19/Dynamics.c.Rt) ----------------
  R d3q19_sum_where(const R* f, int ax, int sign_) const {  // sum f[X <,==,> 0]
    R s = 0;
    const int* e = ops.L.e.data();
    for (int i = 0; i < 19; i++) {
      int v = e[i * 3 + ax];
      if ((sign_ < 0 && v < 0) || (sign_ == 0 && v == 0) || (sign_ > 0 && v > 0)) s += f[i];
    }
    return s;
  }
  void d3q19_N(const R* f, R& Nxy, R& Nxz) const {  // Dynamics.c.Rt:99-100,169-170
    const int* e = ops.L.e.data();
    R a = 0, b = 0;
    for (int i = 0; i < 19; i++) {
      if (e[i * 3] != 0) continue;
      if (e[i * 3 + 1] > 0) a += f[i];
      if (e[i * 3 + 1] < 0) a -= f[i];
      if (e[i * 3 + 2] > 0) b += f[i];
      if (e[i * 3 + 2] < 0) b -= f[i];
    }
    Nxy = a / (R)2;
    Nxz = b / (R)2;
  }
  void d3q19_inlet(R* f, R rho, R ux) const {  // Dynamics.c.Rt:98-108
    R Nxy, Nxz;
    d3q19_N(f, Nxy, Nxz);
    f[1] = f[2] + rho * ux / (R)3;
    f[9] = f[8] + rho * ux / (R)6 + Nxy;
    f[7] = f[10] + rho * ux / (R)6 - Nxy;
    f[11] = f[14] + rho * ux / (R)6 - Nxz;
    f[13] = f[12] + rho * ux / (R)6 + Nxz;
  }
  void d3q19_run(R* f, flag_t fl, std::vector<double>* G) const {
    switch (fl & 0x1C) {  // Dynamics.c.Rt:181-210
      case 0x14: {  // WPressureLimited :138-153
        R SF = d3q19_sum_where(f, 0, -1);
        SF = d3q19_sum_where(f, 0, 0) + (R)2 * SF;
        R rho = S(4), ux = (R)1 - SF / rho;
        if (ux > S(2)) { ux = S(2); rho = SF / ((R)1 - ux); }
        d3q19_inlet(f, rho, ux);
        break;
      }
      case 0x10: {  // WPressure :124-136
        R rho = S(4);
        R ux = d3q19_sum_where(f, 0, -1);
        ux = d3q19_sum_where(f, 0, 0) + (R)2 * ux;
        ux = (R)1 - ux / rho;
        d3q19_inlet(f, rho, ux);
        break;
      }
      case 0x18: {  // WVelocity :110-122
        R ux = S(2);
        R rho = d3q19_sum_where(f, 0, -1);
        rho = d3q19_sum_where(f, 0, 0) + (R)2 * rho;
        rho = rho / ((R)1 - ux);
        d3q19_inlet(f, rho, ux);
        break;
      }
      case 0x04: {  // EPressure :157-179
        R rho = 1, Nxy, Nxz;
        R ux = d3q19_sum_where(f, 0, 1);
        ux = d3q19_sum_where(f, 0, 0) + (R)2 * ux;
        ux = (R)-1 + ux / rho;
        d3q19_N(f, Nxy, Nxz);
        f[2] = f[1] - rho * ux / (R)3;
        f[8] = f[9] - rho * ux / (R)6 - Nxy;
        f[10] = f[7] - rho * ux / (R)6 + Nxy;
        f[14] = f[11] - rho * ux / (R)6 + Nxz;
        f[12] = f[13] - rho * ux / (R)6 - Nxz;
        break;
      }
      case 0x0C: case 0x08: bounce(f); break;
      default: break;
    }
    if ((fl & 0x20) == 0x20) d3q19_mrt(f, fl, G);
  }
  void d3q19_mrt(R* f, flag_t fl, std::vector<double>* G) const {  // :223-290
    R Rm[19];
    for (int k = 0; k < 19; k++) {
      R s = 0;
      for (int i = 0; i < 19; i++) s += (R)MRT19[k][i] * f[i];
      Rm[k] = s;
    }
    R omega = S(0);
    R gamma1 = (R)1 - omega;
    R gamma2 = (R)1 - (R)8 * ((R)2 - omega) / ((R)8 - omega);
    R rho = Rm[0], J[3] = {Rm[3], Rm[5], Rm[7]};
    auto Sk = [&](int k) -> R {  // 0-based moment index
      if (k == 0 || k == 3 || k == 5 || k == 7) return 0;
      if (k == 1 || k == 2 || (k >= 9 && k <= 15)) return gamma1;
      return gamma2;
    };
    for (int k = 0; k < 19; k++)
      if (!(k == 0 || k == 3 || k == 5 || k == 7)) Rm[k] = Sk(k) * (Rm[k] - ops.Req19[k].eval(rho, J, 3));
    J[0] += rho * S(5);
    J[1] += rho * S(6);
    J[2] += rho * S(7);
    Rm[3] = J[0]; Rm[5] = J[1]; Rm[7] = J[2];
    for (int k = 0; k < 19; k++)
      if (!(k == 0 || k == 3 || k == 5 || k == 7)) Rm[k] = Rm[k] + ops.Req19[k].eval(rho, J, 3);
    for (int k = 0; k < 19; k++) Rm[k] /= ops.Mw[k];  // also rescales rho and J (C(R, Mw, eq="/="))
    for (int i = 0; i < 19; i++) {
      R s = 0;
      for (int k = 0; k < 19; k++) s += Rm[k] * (R)MRT19[k][i];
      f[i] = s;
    }
    if (G) {  // globals use the rescaled rho and J, as the generated code does
      R rs = Rm[0], ux = Rm[3] / rs, uy = Rm[5] / rs, uz = Rm[7] / rs;
      int pl = fl & 3;
      if (pl) {
        int base = 1 + 5 * (pl - 1);  // XY: 1.., XZ: 6.., YZ: 11..
        add(*G, base + 0, ux, fl);
        add(*G, base + 1, uy, fl);
        add(*G, base + 2, uz, fl);
        add(*G, base + 3, rs, fl);
        add(*G, base + 4, (R)1, fl);
      }
      add(*G, 16, ux, fl);
      add(*G, 17, uy, fl);
      add(*G, 18, uz, fl);
      add(*G, 19, Rm[3], fl);
      add(*G, 20, Rm[5], fl);
      add(*G, 21, Rm[7], fl);
      add(*G, 22, rs, fl);
      add(*G, 23, (R)1, fl);
      maxg(*G, 25, std::sqrt(ux * ux + uy * uy + uz * uz));
    }
  }
  void d3q19_init(R* f, flag_t) const {  // :212-221: SetEquilibrum(1, InletVelocity, 0, 0)
    R rho = 1, J[3] = {S(2), 0, 0};
    R Rm[19];
    for (int k = 0; k < 19; k++) Rm[k] = ops.Req19[k].eval(rho, J, 3) / ops.Mw[k];
    for (int i = 0; i < 19; i++) {
      R s = 0;
      for (int k = 0; k < 19; k++) s += Rm[k] * (R)MRT19[k][i];
      f[i] = s;
    }
  }

  // ---------------- d3q27_cumulant ----------------
  // ZouHe (lib/boundary.R:67-108): direction axis 'ax', 'sg' selects the
  // unknown populations (sg*e_ax > 0).
  void zouhe(R* f, int ax, int sg, bool velocity, R P, R V) const {
    const int Q = 27;
    const int* e = ops.L.e.data();
    bool sel[27];
    R c0[27], c[27][3];
    for (int i = 0; i < Q; i++) {
      sel[i] = sg * e[i * 3 + ax] > 0;
      for (int d = 0; d < 3; d++) c[i][d] = 0;
      if (sel[i]) {
        c0[i] = f[ops.L.opp[i]];
        for (int d = 0; d < 3; d++) c[i][d] = ops.zh[i * 3 + d];
      } else c0[i] = f[i];
    }
    // Rs[1] = sum fs - rho ; Rs[t+1] = sum fs e_t (tangential)
    R s0 = 0, sc[3] = {0, 0, 0};
    for (int i = 0; i < Q; i++) { s0 += c0[i]; for (int d = 0; d < 3; d++) sc[d] += c[i][d]; }
    R J[3] = {0, 0, 0}, rho;
    if (!velocity) {
      rho = P * (R)3 + (R)1;
      J[ax] = -(s0 - rho) / sc[ax];
    } else {
      // sum fs - rho with J_ax = rho V: s0 + sc_ax rho V - rho = 0
      rho = -s0 / (sc[ax] * V - (R)1);
      J[ax] = rho * V;
    }
    for (int t = 0; t < 3; t++) {
      if (t == ax) continue;
      R m0 = 0, mt = 0, ma = 0;
      for (int i = 0; i < Q; i++) {
        m0 += c0[i] * (R)e[i * 3 + t];
        mt += c[i][t] * (R)e[i * 3 + t];
        ma += c[i][ax] * (R)e[i * 3 + t];
      }
      J[t] = -(m0 + ma * J[ax]) / mt;
    }
    for (int i = 0; i < Q; i++)
      if (sel[i]) {
        R v = c0[i];
        for (int d = 0; d < 3; d++) v += c[i][d] * J[d];
        f[i] = v;
      }
  }

  void d3q27_bounce_drag(R* f, flag_t fl, std::vector<double>* G) const {  // Dynamics.c.Rt:112-127
    const int* e = ops.L.e.data();
    R p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0};
    for (int i = 0; i < 27; i++)
      for (int d = 0; d < 3; d++) p1[d] += f[i] * (R)e[i * 3 + d];
    bounce(f);
    for (int i = 0; i < 27; i++)
      for (int d = 0; d < 3; d++) p2[d] += f[i] * (R)e[i * 3 + d];
    if (G && (fl & 4) == 4) {
      add(*G, 2, -(p2[0] - p1[0]), fl);  // Drag
      add(*G, 4, -(p2[1] - p1[1]), fl);  // Lateral
      add(*G, 3, -(p2[2] - p1[2]), fl);  // Lift
    }
  }

  void d3q27_boundaries(R* f, flag_t fl, std::vector<double>* G) const {  // :224-272
    switch (fl & 3) {
      case 1: symmetry(f, 1, -1); break;  // NSymmetry
      case 2: symmetry(f, 1, 1); break;   // SSymmetry
    }
    R P = Z(1, fl), V = Z(0, fl);
    switch (fl & 0x78) {
      case 0x10: zouhe(f, 0, 1, true, P, V); break;  // WVelocityTurbulent with zero turbulence
      case 0x38: zouhe(f, 0, -1, false, P, V); break;  // EPressure
      case 0x58: zouhe(f, 0, 1, false, P, V); break;   // WPressure
      case 0x30: zouhe(f, 1, 1, false, P, V); break;   // SPressure
      case 0x28: zouhe(f, 1, -1, false, P, V); break;  // NPressure
      case 0x60: zouhe(f, 0, 1, true, P, V); break;    // WVelocity
      case 0x18: zouhe(f, 1, -1, true, P, V); break;   // NVelocity
      case 0x20: zouhe(f, 1, 1, true, P, V); break;    // SVelocity
      case 0x40: zouhe(f, 0, -1, true, P, V); break;   // EVelocity
      case 0x50: d3q27_bounce_drag(f, fl, G); break;   // Wall
      default: break;
    }
  }

  // 1D raw-moment transform along an axis and its inverse (:323-349, :479-505)
  static inline void raw3(R& a0, R& a1, R& a2) {
    a0 = a2 + a1 + a0;
    a1 = -a2 + a1;
    a2 = a1 + a2 * (R)2;
  }
  static inline void unraw3(R& a0, R& a1, R& a2) {
    a0 = -a2 + a0;
    a1 = (a2 + a1) / (R)2;
    a2 = a2 - a1;
  }
  static void transform(R* m, bool fwd) {
    for (int ax = 0; ax < 3; ax++) {
      int st = ax == 0 ? 1 : (ax == 1 ? 3 : 9);
      for (int r = 0; r < 27; r++) {
        int coord = (r / st) % 3;
        if (coord != 0) continue;
        if (fwd) raw3(m[r], m[r + st], m[r + 2 * st]);
        else unraw3(m[r], m[r + st], m[r + 2 * st]);
      }
    }
  }

  void d3q27_collide(R* f, flag_t fl, std::vector<double>* G) const {  // :309-519
    const int* e = ops.L.e.data();
    R Fx = S(3), Fy = S(4), Fz = S(5);
    if (G) {
      R rho = 0, u[3] = {0, 0, 0};
      for (int i = 0; i < 27; i++) {
        rho += f[i];
        for (int d = 0; d < 3; d++) u[d] += f[i] * (R)e[i * 3 + d];
      }
      if ((fl & 0x78) == 0x50) { u[0] = u[1] = u[2] = 0; }
      else { u[0] = (u[0] + Fx / (R)2) / rho; u[1] = (u[1] + Fy / (R)2) / rho; u[2] = (u[2] + Fz / (R)2) / rho; }
      add(*G, 0, rho, fl);
      add(*G, 1, u[0], fl);
      add(*G, 5, rho, fl);
      add(*G, 6, rho * u[0], fl);
      add(*G, 7, rho * u[1], fl);
      add(*G, 8, rho * u[2], fl);
    }
    R w0 = (R)1 / ((R)3 * S(0) + (R)0.5);
    const R w1 = 1;
    if ((fl & 0x78) != 0) w0 = (R)1 / ((R)3 * S(1) + (R)0.5);
    R m[27];
    for (int i = 0; i < 27; i++) m[i] = f[i];
    transform(m, true);
    R c[27];
    R m0 = m[0];
    c[0] = m0;
    {
      size_t p = 0;
      for (int n = 1; n < 27; n++) {
        c[n] = m[n];
        while (p < ops.cum_fwd.size() && ops.cum_fwd[p].n == n) {
          const auto& t = ops.cum_fwd[p++];
          c[n] -= t.coef * c[t.k] * m[t.m];
        }
        c[n] = c[n] / m0;
      }
    }
    auto C = [&](int a, int b, int cc) -> R& { return c[a + 3 * b + 9 * cc]; };
    R ux = C(1, 0, 0) + Fx / ((R)2 * m0), uy = C(0, 1, 0) + Fy / ((R)2 * m0), uz = C(0, 0, 1) + Fz / ((R)2 * m0);
    R c200 = C(2, 0, 0), c020 = C(0, 2, 0), c002 = C(0, 0, 2);
    R dxu = -w0 / (R)2 * ((R)2 * c200 - c020 - c002) - w1 / (R)2 * (c200 + c020 + c002 - (R)1);
    R dyv = dxu + (R)3 * w0 / (R)2 * (c200 - c020);
    R dzw = dxu + (R)3 * w0 / (R)2 * (c200 - c002);
    R gcor1 = (R)3 * ((R)1 - w0 / (R)2) * (ux * ux * dxu - uy * uy * dyv);
    R gcor2 = (R)3 * ((R)1 - w0 / (R)2) * (ux * ux * dxu - uz * uz * dzw);
    R gcor3 = (R)3 * ((R)1 - w1 / (R)2) * (ux * ux * dxu + uy * uy * dyv + uz * uz * dzw);
    R a = ((R)1 - w0) * (c200 - c020);
    R b = ((R)1 - w0) * (c200 - c002);
    R cc = w1 + ((R)1 - w1) * (c200 + c020 + c002);
    R Gc = S(2);
    a = a - gcor1 * Gc;
    b = b - gcor2 * Gc;
    cc = cc - gcor3 * Gc;
    C(1, 0, 0) = C(1, 0, 0) + Fx;
    C(2, 0, 0) = (a + b + cc) / (R)3;
    C(0, 2, 0) = (cc - (R)2 * a + b) / (R)3;
    C(0, 0, 2) = (cc - (R)2 * b + a) / (R)3;
    C(0, 1, 0) = C(0, 1, 0) + Fy;
    C(0, 0, 1) = C(0, 0, 1) + Fz;
    C(1, 1, 0) = C(1, 1, 0) * ((R)1 - w0);
    C(0, 1, 1) = C(0, 1, 1) * ((R)1 - w0);
    C(1, 0, 1) = C(1, 0, 1) * ((R)1 - w0);
    R Om = S(6);
    for (int n = 1; n < 27; n++) {
      int s = n % 3 + (n / 3) % 3 + n / 9;
      if (s == 3) c[n] = ((R)1 - Om) * c[n];
      if (s > 3) c[n] = 0;
    }
    // back to raw moments, index order (:451-477)
    m[0] = m0;
    {
      size_t p = 0;
      for (int n = 1; n < 27; n++) {
        R v = c[n] * m0;
        while (p < ops.cum_bwd.size() && ops.cum_bwd[p].n == n) {
          const auto& t = ops.cum_bwd[p++];
          v += t.coef * c[t.k] * m[t.m];
        }
        m[n] = v;
      }
    }
    transform(m, false);
    for (int i = 0; i < 27; i++) f[i] = m[i];
  }

  void d3q27_run(R* f, flag_t fl, std::vector<double>* G) const {
    d3q27_boundaries(f, fl, G);
    if ((fl & 0x80) == 0x80) d3q27_collide(f, fl, G);
  }
  void d3q27_init(R* f, flag_t fl) const {  // :290-299 (synthetic turbulence taken as zero)
    R J[3] = {Z(0, fl), 0, 0};
    R rho = (R)1 + Z(1, fl) * (R)3;
    if ((fl & 0x78) == 0x50) { rho = 1; J[0] = 0; }
    feq_fill(f, rho, J);
  }

  // ---------------- framework ----------------
  inline size_t nidx(int x, int y, int z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); }

  void node_pull(const std::vector<R>& src, int x, int y, int z, R* f) const {
    const int* e = ops.L.e.data();
    const size_t n = nidx(x, y, z);
    if (x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1) {  // no wrap: a fixed offset
      for (int i = 0; i < ops.L.Q; i++)
        f[i] = src[(size_t)i * N + n - ((ptrdiff_t)e[i * 3] + (ptrdiff_t)nx * (e[i * 3 + 1] + (ptrdiff_t)ny * e[i * 3 + 2]))];
      return;
    }
    for (int i = 0; i < ops.L.Q; i++) {
      int xs = (x - e[i * 3] + nx) % nx, ys = (y - e[i * 3 + 1] + ny) % ny, zs = (z - e[i * 3 + 2] + nz) % nz;
      f[i] = src[(size_t)i * N + nidx(xs, ys, zs)];
    }
  }

  void run_node(R* f, flag_t fl, std::vector<double>* G) const {
    if (model == M_D2Q9) d2q9_run(f, fl, G);
    else if (model == M_D3Q19) d3q19_run(f, fl, G);
    else d3q27_run(f, fl, G);
  }

  // One Iteration (src/Lattice.cu.Rt:458-533 with RunElement src/cuda.cu.Rt:322-327)
  void iteration(bool glob) {
    const std::vector<R>& src = buf[cur];
    std::vector<R>& dst = buf[1 - cur];
    const int Q = ops.L.Q;
    int ng = ops.info.nglob;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> part(nthreads, std::vector<double>(2 * ng, 0.0));
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        std::vector<double>* G = glob ? &part[tid] : nullptr;
        R f[27];
        for (int x = 0; x < nx; x++) {
          size_t n = nidx(x, y, z);
          node_pull(src, x, y, z, f);
          run_node(f, flags[n], G);
          if (storage_mode)
            for (int i = 0; i < Q; i++)
              dst[(size_t)i * N + n] =
                  storage_roundtrip(storage_mode, f[i], wts[i], storage_bits(storage_seed, iter, n, i), storage_param);
          else
            for (int i = 0; i < Q; i++) dst[(size_t)i * N + n] = f[i];
        }
      }
    if (glob) {
      for (int t = 0; t < nthreads; t++)
        for (int g = 0; g < 2 * ng; g++) {
          if (g % ng < ops.info.nsum) dev_globals[g] += part[t][g];
          else dev_globals[g] = std::max(dev_globals[g], part[t][g]);
        }
    }
    cur = 1 - cur;
    iter++;
  }

  void init() {  // Lattice::Init (src/Lattice.cu.Rt:799-821)
    const int Q = ops.L.Q;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          size_t n = nidx(x, y, z);
          R f[27];
          flag_t fl = flags[n];
          if (model == M_D2Q9) d2q9_init(f, fl);
          else if (model == M_D3Q19) d3q19_init(f, fl);
          else d3q27_init(f, fl);
          for (int i = 0; i < Q; i++) buf[cur][(size_t)i * N + n] = f[i];
        }
    iter = 0;
    std::fill(dev_globals.begin(), dev_globals.end(), 0.0);
    std::fill(globals.begin(), globals.end(), 0.0);
  }

  // Lattice::Iterate for ITER_NORM (src/Lattice.cu.Rt:900-989)
  void iterate(int niter, int iter_type) {
    int last_glob = iter_type & 0x080;
    if ((iter_type & 0x070) == 0x070) last_glob = 0;
    bool globs = (iter_type & 0x010) != 0;
    for (int i = 0; i < niter; i++) {
      if (last_glob && i == niter - 1) {
        std::fill(dev_globals.begin(), dev_globals.end(), 0.0);
        globs = true;
      }
      iteration(globs);
    }
    if (last_glob) {
      std::fill(globals.begin(), globals.end(), 0.0);
      calc_globals();
    } else if ((iter_type & 0x070) == 0x070) {
      calc_globals();
    }
  }
  void calc_globals() {  // :1299-1315 (the InObj weights are zonal, so obj stays 0)
    for (size_t g = 0; g < globals.size(); g++) globals[g] += dev_globals[g];
    std::fill(dev_globals.begin(), dev_globals.end(), 0.0);
  }

  // Quantities: pull from the current snapshot, then getX (LatticeContainer.inc.cpp.Rt:437-473)
  void quantity(int q, double* out) const {
    const int* e = ops.L.e.data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          size_t n = nidx(x, y, z);
          R f[27];
          node_pull(buf[cur], x, y, z, f);
          flag_t fl = flags[n];
          R rho = 0, u[3] = {0, 0, 0};
          if (model == M_D3Q27C && q == 1) {  // getU runs RunBoundaries first (:47-51)
            d3q27_boundaries(f, fl, nullptr);
          }
          for (int i = 0; i < ops.L.Q; i++) {
            rho += f[i];
            for (int d = 0; d < 3; d++) u[d] += f[i] * (R)e[i * 3 + d];
          }
          if (model == M_D2Q9) {
            if (q == 0) out[n] = (double)rho;
            else {  // d2q9/Dynamics.c.Rt:43-59
              R ux = u[0] / rho + S(2) * (R)0.5, uy = u[1] / rho + S(3) * (R)0.5;
              out[3 * n] = ux; out[3 * n + 1] = uy; out[3 * n + 2] = 0;
            }
          } else if (model == M_D3Q19) {
            if (q == 0) out[n] = (double)((rho - (R)1) / (R)3);
            else {  // d3q19/Dynamics.c.Rt:31-40
              R ux = u[0] / rho, uy = u[1] / rho, uz = u[2] / rho;
              if ((fl & 0x1C) == 0x0C) ux = uy = uz = 0;
              out[3 * n] = ux; out[3 * n + 1] = uy; out[3 * n + 2] = uz;
            }
          } else {
            if (q == 0) out[n] = (double)((rho - (R)1) / (R)3);
            else if (q == 2) out[n] = ((fl & 0x78) == 0x50) ? 1.0 : 0.0;
            else {  // getU_ (:30-45)
              R ux, uy, uz;
              if ((fl & 0x78) == 0x50) ux = uy = uz = 0;
              else { ux = (u[0] + S(3) / (R)2) / rho; uy = (u[1] + S(4) / (R)2) / rho; uz = (u[2] + S(5) / (R)2) / rho; }
              out[3 * n] = ux; out[3 * n + 1] = uy; out[3 * n + 2] = uz;
            }
          }
        }
  }
};

// ColorKernel's colour map (src/LatticeContainer.inc.cpp.Rt:378-401): the
// fraction branches in float, truncated to int; w scales the colour towards
// green; a non-finite l is magenta. Built without FP contraction.
void color_map(float l, float w, uint8_t* o) {
  int r = 0, g = 0, b = 0;
  if (std::isfinite(l)) {
    l = l * 111;
    if (l < -111) { r = 255; g = 255; b = 255; }
    if ((l >= -111) && (l < -11)) { r = 255 * (-l - 11) / 100; g = 255; b = 255; }
    if ((l >= -11) && (l < -1)) { r = 0; g = (255 * (-l - 1)) / 10; b = 255; }
    if ((l >= -1) && (l < 0)) { r = 0; g = 0; b = 255 * (-l); }
    if ((l >= 0) && (l < 1)) { r = 255 * l; g = 0; b = 0; }
    if ((l >= 1) && (l < 11)) { r = 255; g = 255 * (l - 1) / 10; b = 0; }
    if ((l >= 11) && (l < 111)) { r = 255; g = 255; b = 255 * (l - 11) / 100; }
    if (l >= 111) { r = 255; g = 255; b = 255; }
    r = r * w;
    g = g * w + (1 - w) * 255;
    b = b * w;
  } else {
    r = 255; b = 255; g = 0;
  }
  o[0] = (uint8_t)r; o[1] = (uint8_t)g; o[2] = (uint8_t)b; o[3] = 255;
}

// Color() of each model: l = |U| from getU, w = 0 on the drawn-blank nodes
// (d2q9/Dynamics.c.Rt:61-71 and d3q27_cumulant/Dynamics.c.Rt:101-111: the
// flag equal to Solid; d3q19/Dynamics.c.Rt:42-52: BOUNDARY group == Wall)
template <class R>
void color_plane(const Lattice<R>& L, int z, uint8_t* out) {
  std::vector<double> u((size_t)3 * L.nx * L.ny * L.nz);
  L.quantity(1, u.data());
  for (int y = 0; y < L.ny; y++)
    for (int x = 0; x < L.nx; x++) {
      const size_t n = L.nidx(x, y, z);
      const R ux = (R)u[3 * n], uy = (R)u[3 * n + 1], uz = (R)u[3 * n + 2];
      R s = ux * ux + uy * uy;
      if (L.model != M_D2Q9) s = s + uz * uz;
      const float l = (float)std::sqrt(s);
      const flag_t fl = L.flags[n];
      float w = 1;
      if (L.model == M_D2Q9) w = fl == 9 ? 0.f : 1.f;
      else if (L.model == M_D3Q19) w = (fl & 0x1C) == 0x0C ? 0.f : 1.f;
      else w = fl == 0x48 ? 0.f : 1.f;
      color_map(l, w, out + 4 * ((size_t)x + (size_t)L.nx * y));
    }
}

struct Handle {
  int precision;  // 0 fp32, 1 fp64
  Lattice<float>* lf = nullptr;
  Lattice<double>* ld = nullptr;
};

}  // namespace orc

using namespace orc;

#define DISPATCH(h, call) ((h)->precision ? (h)->ld->call : (h)->lf->call)

extern "C" {

void* orc_create(int model, int nx, int ny, int nz, int precision) {
  try {
    Handle* h = new Handle();
    h->precision = precision;
    if (precision) h->ld = new Lattice<double>(model, nx, ny, nz);
    else h->lf = new Lattice<float>(model, nx, ny, nz);
    return h;
  } catch (...) {
    return nullptr;
  }
}

void orc_destroy(void* p) {
  Handle* h = (Handle*)p;
  if (!h) return;
  delete h->lf;
  delete h->ld;
  delete h;
}

int orc_set_storage(void* p, int mode, unsigned seed, double param) {
  Handle* h = (Handle*)p;
  if (mode < EMU_NONE || mode > EMU_EXM) return -1;
  auto f = [&](auto* L) { L->storage_mode = mode; L->storage_seed = seed; L->storage_param = param; };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_set_flags(void* p, const uint16_t* fl) {
  Handle* h = (Handle*)p;
  if (h->precision) std::copy(fl, fl + h->ld->N, h->ld->flags.begin());
  else std::copy(fl, fl + h->lf->N, h->lf->flags.begin());
  return 0;
}

int orc_set_setting(void* p, int i, double v) {
  Handle* h = (Handle*)p;
  DISPATCH(h, set_setting(i, v));
  return 0;
}

int orc_get_setting(void* p, int i, double* v) {
  Handle* h = (Handle*)p;
  *v = h->precision ? h->ld->settings[i] : h->lf->settings[i];
  return 0;
}

int orc_set_zone_setting(void* p, int s, int zone, double v) {  // ZoneSettings::set (src/ZoneSettings.h:58-77)
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) {
    int nzs = L->ops.info.nzs;
    if (zone < 0)
      for (int z = 0; z < L->nzones; z++) L->zone[(size_t)z * nzs + s] = v;
    else L->zone[(size_t)zone * nzs + s] = v;
  };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

int orc_init(void* p) {
  Handle* h = (Handle*)p;
  DISPATCH(h, init());
  return 0;
}

int orc_iterate(void* p, int niter, int iter_type) {
  Handle* h = (Handle*)p;
  DISPATCH(h, iterate(niter, iter_type));
  return 0;
}

int orc_get_globals(void* p, double* out) {
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) { std::copy(L->globals.begin(), L->globals.begin() + L->ops.info.nglob, out); };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

// Sum of absolute contributions of each Global (its error scale), same cadence.
int orc_get_globals_scale(void* p, double* out) {
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) { std::copy(L->globals.begin() + L->ops.info.nglob, L->globals.end(), out); };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

int orc_get_quantity(void* p, int q, double* out) {
  Handle* h = (Handle*)p;
  DISPATCH(h, quantity(q, out));
  return 0;
}

// Densities of the current snapshot, SoA [q][z][y][x], as double
int orc_get_densities(void* p, double* out) {
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) {
    const auto& b = L->buf[L->cur];
    for (size_t i = 0; i < b.size(); i++) out[i] = (double)b[i];
  };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

int orc_set_densities(void* p, const double* in) {
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) {
    auto& b = L->buf[L->cur];
    using R = decltype(b[0] + 0);
    // an emulated 16-bit store rounds to nearest, as the library's host-side conversion does
    const int mode = L->storage_mode == EMU_F16_SR ? EMU_F16_RN : L->storage_mode == EMU_BF16_SR ? EMU_BF16_RN
                                                                                                  : L->storage_mode;
    for (size_t i = 0; i < b.size(); i++)
      b[i] = mode ? storage_roundtrip(mode, (R)in[i], L->wts[i / L->N], 0u, L->storage_param) : (R)in[i];
  };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

// Equilibrium distribution from the oracle's own construction (used by tests
// to cross-check the product's closed forms).
int orc_color(void* p, int z, uint8_t* out) {
  Handle* h = (Handle*)p;
  if (h->precision) color_plane(*h->ld, z, out); else color_plane(*h->lf, z, out);
  return 0;
}

int orc_color_map(const float* l, const float* w, int n, uint8_t* out) {
  for (int i = 0; i < n; i++) color_map(l[i], w[i], out + 4 * (size_t)i);
  return 0;
}

int orc_feq(int model, double rho, const double* J, double* out) {
  Ops<double> o;
  o.build(model);
  for (int i = 0; i < o.L.Q; i++) out[i] = o.feq[i].eval(rho, J, o.L.D);
  return o.L.Q;
}

// The Cholesky-weighted d2q9 basis (for tests): B[i*9+k], and column orders.
int orc_d2q9_basis(double* B, int* order) {
  Ops<double> o;
  o.build(M_D2Q9);
  for (int i = 0; i < 81; i++) B[i] = o.B[i];
  for (int k = 0; k < 9; k++) order[k] = o.Border[k];
  return 0;
}

int orc_node_type_value(int model, const char* name) {
  try {
    return nt_value(model, name);
  } catch (...) {
    return -1;
  }
}

// Apply the node update to one node's pulled populations (double), for
// unit tests of boundary closures. Globals are ignored.
int orc_node_update(void* p, const double* fin, uint16_t flag, double* fout) {
  Handle* h = (Handle*)p;
  auto f = [&](auto* L) {
    using R = typename std::remove_reference<decltype(L->buf[0][0])>::type;
    R f[27];
    for (int i = 0; i < L->ops.L.Q; i++) f[i] = (R)fin[i];
    L->run_node(f, flag, nullptr);
    for (int i = 0; i < L->ops.L.Q; i++) fout[i] = (double)f[i];
  };
  if (h->precision) f(h->ld); else f(h->lf);
  return 0;
}

}  // extern "C"
