// XML case front-end: TCLB's <CLBConfig> files driven through the C ABI.
//
// Mirrors the control flow of TCLB's handler tree for the Run path
// (src/main.cpp:173-425, src/Handlers/*): <Geometry> builds the node types
// (src/Geometry.cpp.Rt), <Model>/<Param>/<Init> set parameters and the initial
// state, <Solve Iterations=> advances the lattice while the registered
// callbacks (<Log>, <BIN>, <Failcheck>) fire on their iteration cadence
// (src/Handlers/acSolve.cpp:5-43, vHandler.h:69-87). Output names follow
// Solver::outIterFile (src/Solver.h.Rt:102-105).
#include <sys/stat.h>
#include <zlib.h>

#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/tclb_b200.h"
#include "tclb_models.h"
#include "xml.hpp"

namespace tclb {
namespace {

thread_local std::string g_case_err;

struct CaseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ------------------------------------------------------------------ units
// TCLB's unit system (src/unit.h, src/unit.cpp): a quantity is a number
// times powers of nine base units (m, s, kg, K, x, y, z, A, t). A value is a
// sum of terms ("1m+2mm"), each a number and unit tokens: letters then an
// optional power ("m2"), and one "/" after which every token divides
// ("1kgm/s2"). A letter group splits into known one- or two-letter symbols;
// where both splits are valid a leading "m" is read as milli, any other
// ambiguity is an error. <Units> gauges (<Param value="1m" gauge="100"/>:
// that much is one lattice unit's worth of it, here 100) fix a scale per base
// unit: the gauged quantities must come out as 1 in lattice units, which is a
// linear system in the logarithms of the scales; base units that no gauge
// involves keep scale 1, and the system must be square. A value's lattice
// number is its number times the scales to the powers of its units.
// Difference: an unknown unit symbol is an error here (TCLB reads it as 0).
constexpr int NBASE = 9;
const char* const BASE_UNITS[NBASE] = {"m", "s", "kg", "K", "x", "y", "z", "A", "t"};

struct UVal {
  double v = 1.0;
  double e[NBASE] = {};
  bool valid() const { return v != 0.0; }
};
UVal umul(const UVal& a, const UVal& b) {
  UVal r;
  r.v = a.v * b.v;
  for (int i = 0; i < NBASE; i++) r.e[i] = a.e[i] + b.e[i];
  return r;
}
UVal udiv(const UVal& a, const UVal& b) {
  UVal r;
  r.v = a.v / b.v;
  for (int i = 0; i < NBASE; i++) r.e[i] = a.e[i] - b.e[i];
  return r;
}
UVal upow(const UVal& a, double p) {
  UVal r;
  r.v = std::pow(a.v, p);
  for (int i = 0; i < NBASE; i++) r.e[i] = a.e[i] * p;
  return r;
}

class UnitEnv {
 public:
  UnitEnv() {
    for (int i = 0; i < NBASE; i++) {
      UVal b;
      b.e[i] = 1;
      units_[BASE_UNITS[i]] = b;
      scale_[i] = 1.0;
    }
    const std::pair<const char*, const char*> derived[] = {
        {"N", "1kgm/s2"}, {"Pa", "1N/m2"}, {"J", "1Nm"},     {"W", "1J/s"},     {"V", "1kgm2/t3/A"},
        {"C", "1tA"},     {"nm", "1e-9m"}, {"um", "1e-6m"},  {"mm", "1e-3m"},   {"cm", "1e-2m"},
        {"km", "1e+3m"},  {"h", "3600s"},  {"ns", "1e-9s"},  {"us", "1e-6s"},   {"ms", "1e-3s"},
        {"g", "1e-3kg"},  {"mg", "1e-6kg"}};
    for (const auto& d : derived) units_[d.first] = text(d.second);  // in order: later ones use earlier
    UVal c;
    c.v = std::acos(-1.0) / 180.0;
    units_["d"] = c;  // degree
    c.v = 0.01;
    units_["%"] = c;
    c.v = 6.022e23;
    units_["An"] = c;
  }

  UVal text(const std::string& s) const {  // a number, then units
    char* end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) {  // units alone ("s"): one of them
      if (s.empty() || !std::isalpha((unsigned char)s[0])) throw CaseError("cannot read value '" + s + "'");
      v = 1.0;
    }
    UVal r = unit(std::string(end), s);
    r.v *= v;
    return r;
  }

  // lattice value of a value text (sum of terms)
  double alt(const std::string& s) const {
    double ret = 0;
    size_t i = 0;
    while (i < s.size()) {
      size_t j = i + 1;
      while (j < s.size() && !((s[j] == '+' || s[j] == '-') && !(s[j - 1] == 'e' || s[j - 1] == 'E'))) j++;
      ret += alt(text(s.substr(i, j - i)));
      i = j;
    }
    return ret;
  }
  double alt(const UVal& u) const {
    double r = u.v;
    for (int i = 0; i < NBASE; i++)
      if (u.e[i] != 0) r *= std::pow(scale_[i], u.e[i]);
    return r;
  }

  void set_gauge(const std::string& name, const std::string& value, const std::string& gauge) {
    gauges_[name] = udiv(text(value), text(gauge));
  }

  // the scales: every gauged quantity equals 1 in lattice units
  void make_gauge() {
    std::vector<std::array<double, NBASE + 1>> rows;  // coefficients of log(1/scale), right-hand side
    for (const auto& g : gauges_) {
      std::array<double, NBASE + 1> r{};
      for (int j = 0; j < NBASE; j++) r[j] = g.second.e[j];
      r[NBASE] = std::log(g.second.v);
      rows.push_back(r);
    }
    for (int j = 0; j < NBASE; j++) {  // base units no gauge involves keep scale 1
      bool used = false;
      for (const auto& g : gauges_) used |= g.second.e[j] != 0;
      if (!used) {
        std::array<double, NBASE + 1> r{};
        r[j] = 1;
        rows.push_back(r);
      }
    }
    if (rows.size() > (size_t)NBASE) throw CaseError("<Units>: gauges over-determine the units");
    if (rows.size() < (size_t)NBASE) throw CaseError("<Units>: gauges under-determine the units");
    // Gaussian elimination with partial pivoting
    for (int c = 0; c < NBASE; c++) {
      int p = c;
      for (int r = c + 1; r < NBASE; r++)
        if (std::fabs(rows[r][c]) > std::fabs(rows[p][c])) p = r;
      if (std::fabs(rows[p][c]) < 1e-12) throw CaseError("<Units>: gauges are not independent");
      std::swap(rows[c], rows[p]);
      for (int r = 0; r < NBASE; r++) {
        if (r == c || rows[r][c] == 0) continue;
        const double f = rows[r][c] / rows[c][c];
        for (int k = c; k <= NBASE; k++) rows[r][k] -= f * rows[c][k];
      }
    }
    for (int j = 0; j < NBASE; j++) scale_[j] = std::exp(-rows[j][NBASE] / rows[j][j]);
  }
  double scale(int j) const { return scale_[j]; }

 private:
  UVal one(const std::string& sym) const {
    auto it = units_.find(sym);
    if (it == units_.end()) {
      UVal z;
      z.v = 0;
      return z;
    }
    return it->second;
  }
  // a letter group with power p on its last symbol
  UVal alpha(const std::string& s, double p, const std::string& whole) const {
    UVal r1 = one(s.substr(0, 1));
    if (s.size() < 2) return upow(r1, p);
    r1 = umul(r1, alpha(s.substr(1), p, whole));
    UVal r2 = one(s.substr(0, 2));
    r2 = s.size() > 2 ? umul(r2, alpha(s.substr(2), p, whole)) : upow(r2, p);
    if (!r1.valid()) return r2;
    if (!r2.valid()) return r1;
    if (s[0] == 'm') return r2;  // "ms", "mm", "mg": the milli reading
    throw CaseError("ambiguous unit '" + s + "' in '" + whole + "'");
  }
  UVal unit(const std::string& u, const std::string& whole) const {
    UVal ret;
    int w = 1;
    size_t i = 0;
    while (i < u.size()) {
      const size_t j = i;
      while (i < u.size() && std::isalpha((unsigned char)u[i])) i++;
      const size_t k = i;
      while (i < u.size() && (std::isdigit((unsigned char)u[i]) || u[i] == '.')) i++;
      const double p = i > k ? std::atof(u.substr(k, i - k).c_str()) : 1.0;
      if (k > j) {
        const UVal last = alpha(u.substr(j, k - j), p, whole);
        if (!last.valid()) throw CaseError("unknown unit '" + u.substr(j, k - j) + "' in '" + whole + "'");
        ret = w > 0 ? umul(ret, last) : udiv(ret, last);
      }
      const size_t q = i;
      while (i < u.size() && !std::isalnum((unsigned char)u[i])) i++;
      if (i - q > 1) throw CaseError("more than one separator in the units of '" + whole + "'");
      if (i - q == 1) {
        if (u[q] != '/') throw CaseError("only '/' may separate units in '" + whole + "'");
        w = -1;
      }
    }
    return ret;
  }

  std::map<std::string, UVal> units_;
  std::map<std::string, UVal> gauges_;  // by name, as given in <Units>
  double scale_[NBASE];
};

// The unit environment of the case being read (gauged by its <Units>).
thread_local UnitEnv g_units;

// <Units>: reset the environment and gauge it (before anything else is read,
// as src/main.cpp:31-62 does).
void read_units(const XmlNode* cfg) {
  g_units = UnitEnv();
  const XmlNode* u = cfg ? cfg->child("Units") : nullptr;
  if (u) {
    int k = 1;
    for (const auto& c : u->children) {
      if (c->name != "Param") continue;
      const std::string* v = c->attr("value");
      const std::string* g = c->attr("gauge");
      if (!v) throw CaseError("<Units><Param> without a value");
      if (!g) throw CaseError("<Units><Param> without a gauge");
      g_units.set_gauge(c->attr_or("name", "unnamed" + std::to_string(k)), *v, *g);
      k++;
    }
  }
  g_units.make_gauge();
}

double parse_value(const std::string& s) { return g_units.alt(s); }

// Units of the settings, zonal settings, Globals and quantities that have one
// (unit= of AddSetting / AddGlobal / AddQuantity in
// models/flow/<model>/Dynamics.R); all others are dimensionless ("1").
const char* quantity_unit(int model, const std::string& name) {
  static const std::map<std::string, const char*> d2q9 = {
      {"PressureLoss", "1mPa"}, {"OutletFlux", "1m2/s"}, {"InletFlux", "1m2/s"}, {"Rho", "kg/m3"}, {"U", "m/s"}};
  static const std::map<std::string, const char*> d3q19 = {
      {"nu", "1m2/s"},    {"InletVelocity", "1m/s"}, {"InletPressure", "1Pa"}, {"InletDensity", "1kg/m3"},
      {"Flux", "m3/s"},   {"XYvx", "m3/s"},          {"XYvy", "m3/s"},         {"XYvz", "m3/s"},
      {"XYrho", "kg/m"},  {"XYarea", "m2"},          {"XZvx", "m3/s"},         {"XZvy", "m3/s"},
      {"XZvz", "m3/s"},   {"XZrho", "kg/m"},         {"XZarea", "m2"},         {"YZvx", "m3/s"},
      {"YZvy", "m3/s"},   {"YZvz", "m3/s"},          {"YZrho", "kg/m"},        {"YZarea", "m2"},
      {"VOLvx", "m4/s"},  {"VOLvy", "m4/s"},         {"VOLvz", "m4/s"},        {"VOLpx", "mkg/s"},
      {"VOLpy", "mkg/s"}, {"VOLpz", "mkg/s"},        {"VOLrho", "kg"},         {"VOLvolume", "m3"},
      {"MaxV", "m3"},     {"P", "Pa"},               {"U", "m/s"}};
  static const std::map<std::string, const char*> d3q27c = {
      {"Density", "kg/m3"}, {"Flux", "m3/s"}, {"Drag", "N"},         {"Lift", "N"},         {"Lateral", "N"},
      {"Mass", "kg"},       {"XMomentum", "kgm/s"}, {"YMomentum", "kgm/s"}, {"ZMomentum", "kgm/s"},
      {"P", "Pa"},          {"U", "m/s"}};
  const std::map<std::string, const char*>& m = model == MODEL_D2Q9 ? d2q9 : (model == MODEL_D3Q19 ? d3q19 : d3q27c);
  const auto it = m.find(name);
  return it == m.end() ? "1" : it->second;
}

// Multiplier from a lattice value to SI for the Log's _si columns
// (LogScales, src/Solver.cpp.Rt:145-159): 1 / (lattice value of one unit).
double si_scale(int model, const std::string& name) { return 1.0 / g_units.alt(quantity_unit(model, name)); }

// Base64 (RFC 4648) of n bytes, '=' padded, no line breaks.
void put_base64(FILE* o, const void* data, size_t n) {
  static const char* A = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  const unsigned char* b = static_cast<const unsigned char*>(data);
  std::string out;
  out.reserve((n + 2) / 3 * 4);
  for (size_t i = 0; i < n; i += 3) {
    const unsigned w = (unsigned)b[i] << 16 | (i + 1 < n ? (unsigned)b[i + 1] << 8 : 0u) | (i + 2 < n ? b[i + 2] : 0u);
    out += A[w >> 18 & 63];
    out += A[w >> 12 & 63];
    out += i + 1 < n ? A[w >> 6 & 63] : '=';
    out += i + 2 < n ? A[w & 63] : '=';
  }
  std::fwrite(out.data(), 1, out.size(), o);
}

int parse_int(const std::string& s) { return (int)std::lround(parse_value(s)); }

// ------------------------------------------------------------------ geometry
const char* DEFAULT_ZONES =
    "<Geometry>"
    "<Zone name='Inlet'><Box dx='0' dy='0' dz='0' fx='0' fy='-1' fz='-1'/></Zone>"
    "<Zone name='Outlet'><Box dx='-1' dy='0' dz='0' fx='-1' fy='-1' fz='-1'/></Zone>"
    "<Zone name='Channel'><Box dx='0' dy='0' dz='0' fx='-1' fy='0' fz='-1'/>"
    "<Box dx='0' dy='-1' dz='0' fx='-1' fy='-1' fz='-1'/></Zone>"
    "<Zone name='Tunnel'><Box dx='0' dy='0' dz='0' fx='-1' fy='0' fz='-1'/>"
    "<Box dx='0' dy='-1' dz='0' fx='-1' fy='-1' fz='-1'/><Box dx='0' dy='0' dz='0' fx='-1' fy='-1' fz='0'/>"
    "<Box dx='0' dy='0' dz='-1' fx='-1' fy='-1' fz='-1'/></Zone>"
    "</Geometry>";

struct Region {
  int dx = 0, dy = 0, dz = 0, nx = 1, ny = 1, nz = 1;
};

struct Geometry {
  const ModelTable* T;
  int nx, ny, nz;
  std::vector<uint16_t> geom;
  std::map<std::string, int> zones;
  int fg = 0, mask = 0;
  enum { OVERWRITE, FILL, CHANGE } mode = OVERWRITE;
  const XmlNode* user = nullptr;     // the <Geometry> element
  const XmlNode* defaults = nullptr; // built-in zones

  Geometry(const ModelTable* t, int x, int y, int z) : T(t), nx(x), ny(y), nz(z), geom((size_t)x * y * z, 0) {
    zones["DefaultZone"] = 0;
  }

  int zone_mask() const { return (0xFFFF << T->zone_shift) & 0xFFFF; }

  int group_mask(const std::string& g) const {
    if (g == "ALL") return 0xFFFF;
    if (g == "NONE") return 0;
    if (g == "SETTINGZONE") return zone_mask();
    for (int i = 0; i < T->ngroups; i++)
      if (g == T->group_names[i]) return T->group_masks[i];
    throw CaseError("unknown mask " + g);
  }
  void set_flag(const std::string& n) {  // Geometry::setFlag (:141-152)
    if (n == "None") { fg = 0; mask = 0; mode = OVERWRITE; return; }
    for (int i = 0; i < T->n_node_types; i++)
      if (n == T->node_type_names[i]) {
        fg = T->node_type_values[i];
        mask = T->node_type_masks[i];
        mode = OVERWRITE;
        return;
      }
    throw CaseError("unknown node type " + n);
  }
  void set_zone(const std::string& n) {  // Geometry::setZone (:192-206)
    int z;
    auto it = zones.find(n);
    if (it != zones.end()) z = it->second;
    else {
      z = (int)zones.size();
      zones[n] = z;
    }
    if (z >= (1 << (16 - T->zone_shift))) throw CaseError("too many zones");
    fg = (fg & ~zone_mask()) | (z << T->zone_shift);
    mask |= zone_mask();
  }
  // Geometry::getRegion (:216-304)
  Region region_of(const XmlNode* n) const {
    if (!n || n->name == "#document") return Region();
    if (n->name == "Geometry") {
      Region r;
      r.nx = nx; r.ny = ny; r.nz = nz;
      return r;
    }
    Region r = region_of(n->parent);
    int* d[3] = {&r.dx, &r.dy, &r.dz};
    int* s[3] = {&r.nx, &r.ny, &r.nz};
    const char* dn[3] = {"dx", "dy", "dz"};
    const char* fn[3] = {"fx", "fy", "fz"};
    const char* nn[3] = {"nx", "ny", "nz"};
    for (int a = 0; a < 3; a++) {
      if (const std::string* v = n->attr(dn[a])) {
        std::string t = *v;
        char side = '+';
        if (!t.empty() && (t[0] == '<' || t[0] == '>')) { side = t[0]; t = t.substr(1); }
        int w = parse_int(t);
        if (side == '<') w = *s[a] + w;
        else if (w < 0) w = *s[a] + w;
        *d[a] += w;
        *s[a] -= w;
      }
    }
    for (int a = 0; a < 3; a++)
      if (const std::string* v = n->attr(fn[a])) {
        int w = parse_int(*v);
        if (w < 0) w = *s[a] + w + *d[a];
        *s[a] = w - *d[a] + 1;
      }
    for (int a = 0; a < 3; a++)
      if (const std::string* v = n->attr(nn[a])) *s[a] = parse_int(*v);
    return r;
  }
  void dot(int x, int y, int z) {  // Geometry::Dot (:307-319)
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return;
    uint16_t& g = geom[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)];
    if (g & mask) {
      if (mode == FILL) return;
    } else if (mode == CHANGE) {
      return;
    }
    g = (uint16_t)((g & ~mask) | fg);
  }
  static bool in_sphere(double x, double y, double z) {
    x = 2 * x - 1; y = 2 * y - 1; z = 2 * z - 1;
    return x * x + y * y + z * z < 1;
  }
  static bool in_wedge(double x, double y, double z, const std::string& t) {  // inWedge (:331-375)
    std::string type = t.empty() ? "UpperLeft" : t;
    double d;
    if (type == "UpperLeft") d = x - y;
    else if (type == "UpperRight") d = (1 - x) - y;
    else if (type == "LowerLeft") d = x - (1 - y);
    else if (type == "LowerRight") d = (1 - x) - (1 - y);
    else if (type == "UpperLeftXZ") d = x - z;
    else if (type == "UpperRightXZ") d = (1 - x) - z;
    else if (type == "LowerLeftXZ") d = x - (1 - z);
    else if (type == "LowerRightXZ") d = (1 - x) - (1 - z);
    else throw CaseError("unknown wedge direction " + type);
    return d < 1e-10;
  }
  const XmlNode* find_zone(const std::string& name) const {
    if (user)
      if (const XmlNode* z = user->child_by_attr("Zone", "name", name)) return z;
    if (defaults)
      if (const XmlNode* z = defaults->child_by_attr("Zone", "name", name)) return z;
    return nullptr;
  }
  // <STL> (Geometry::transformSTL :381-473, Geometry::loadSTL :507-687): a
  // binary STL file whose vertices (float, as stored in the file) are rotated
  // by Xrot, Yrot, Zrot in turn, scaled by `scale`, moved by x, y, z, rounded
  // to 1e-5 and moved by -0.5 plus a small per-axis offset, so node centres
  // do not fall on faces. side="in" (default) or "out": rays along ray_axis
  // (default y) from the start of the element's region; a node of the region
  // is drawn when the number of faces at or above it is odd (in) or even
  // (out). side="surface": a node is drawn when the link to any of its 26
  // neighbours crosses a face (TCLB also records the cut fractions, which only
  // interpolated bounce-back models read; a link parallel to a face is no cut).
  void draw_stl(const XmlNode* n, const Region& reg) {
    const std::string* file = n->attr("file");
    if (!file) throw CaseError("<STL> needs a file attribute");
    int inside_out = 0, axis = 1;
    if (const std::string* s = n->attr("side")) {
      if (*s == "in") inside_out = 0;
      else if (*s == "out") inside_out = 1;
      else if (*s == "surface") inside_out = 2;
      else throw CaseError("<STL> side must be in, out or surface");
    }
    if (const std::string* s = n->attr("ray_axis")) {
      if (inside_out == 2) throw CaseError("<STL> ray_axis applies to side in or out only");
      if (*s == "x") axis = 0;
      else if (*s == "y") axis = 1;
      else if (*s == "z") axis = 2;
      else throw CaseError("<STL> ray_axis must be x, y or z");
    }
    std::ifstream in(*file, std::ios::binary);
    if (!in) throw CaseError("cannot open " + *file);
    char header[80];
    uint32_t ntri = 0;
    in.read(header, 80);
    in.read(reinterpret_cast<char*>(&ntri), 4);
    if (!in) throw CaseError(*file + " is not a binary STL file");
    if (std::strncmp(header, "solid", 5) == 0) throw CaseError(*file + " is not in binary STL format");
    struct Tri { float p[3][3]; };
    std::vector<Tri> tri(ntri);
    for (uint32_t i = 0; i < ntri; i++) {
      char rec[50];  // normal, three vertices (float x 12), attribute (uint16)
      in.read(rec, 50);
      if (!in) throw CaseError(*file + " ended while reading its triangles");
      std::memcpy(tri[i].p, rec + 12, 36);
    }
    static const char* rot[3] = {"Xrot", "Yrot", "Zrot"};
    for (int d = 0; d < 3; d++) {
      const std::string* a = n->attr(rot[d]);
      if (!a) continue;
      const double v = parse_value(*a);
      const int i1 = (d + 1) % 3, i2 = (d + 2) % 3;
      for (auto& t : tri)
        for (auto& p : t.p) {
          const double y = p[i1], z = p[i2];
          p[i1] = (float)(std::cos(v) * y - std::sin(v) * z);
          p[i2] = (float)(std::sin(v) * y + std::cos(v) * z);
        }
    }
    if (const std::string* a = n->attr("scale")) {
      const double v = parse_value(*a);
      for (auto& t : tri)
        for (auto& p : t.p)
          for (float& c : p) c = (float)(v * c);
    }
    static const char* mv[3] = {"x", "y", "z"};
    for (int j = 0; j < 3; j++)
      if (const std::string* a = n->attr(mv[j])) {
        const double v = parse_value(*a);
        for (auto& t : tri)
          for (auto& p : t.p) p[j] = (float)(p[j] + v);
      }
    static const double perturb[3] = {0.1403e-4, 0.1687e-4, 0.1987e-4};
    auto round_int = [](double v) { return v > 0 ? (int)(v + 0.5) : (int)(v - 0.5); };
    for (auto& t : tri)
      for (auto& p : t.p)
        for (int j = 0; j < 3; j++) {
          p[j] = (float)(round_int(p[j] * 1e5) * 1e-5);
          p[j] = (float)(p[j] + (perturb[j] - 0.5));
        }
    const int rlo[3] = {reg.dx, reg.dy, reg.dz}, rn[3] = {reg.nx, reg.ny, reg.nz};
    std::vector<int> lev;
    if (inside_out != 2) lev.assign((size_t)reg.nx * reg.ny * reg.nz, inside_out);
    for (const Tri& t : tri) {
      int lo[3], hi[3];
      for (int j = 0; j < 3; j++) {
        lo[j] = (int)std::ceil(t.p[0][j]);
        if (t.p[1][j] < lo[j]) lo[j] = (int)std::ceil(t.p[1][j]);
        if (t.p[2][j] < lo[j]) lo[j] = (int)std::ceil(t.p[2][j]);
        hi[j] = (int)std::floor(t.p[0][j]);
        if (t.p[1][j] > hi[j]) hi[j] = (int)std::floor(t.p[1][j]);
        if (t.p[2][j] > hi[j]) hi[j] = (int)std::floor(t.p[2][j]);
        lo[j] -= 1;
        hi[j] += 1;
      }
      if (inside_out == 2) {
        for (int x = lo[0]; x <= hi[0]; x++)
          for (int z = lo[2]; z <= hi[2]; z++)
            for (int y = lo[1]; y <= hi[1]; y++) {
              if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
              for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                  for (int dx = -1; dx <= 1; dx++)
                    if ((dx || dy || dz) && link_cuts(t.p, x, y, z, dx, dy, dz)) dot(x, y, z);
            }
        continue;
      }
      const int a1 = axis, a2 = (axis + 1) % 3, a3 = (axis + 2) % 3;
      const double v1[2] = {(double)(float)(t.p[1][a2] - t.p[0][a2]), (double)(float)(t.p[1][a3] - t.p[0][a3])};
      const double v2[2] = {(double)(float)(t.p[2][a2] - t.p[0][a2]), (double)(float)(t.p[2][a3] - t.p[0][a3])};
      const double c0 = v1[0] * v2[1] - v1[1] * v2[0];
      const double dv[2] = {-0.5694552, 0.8220224};  // fixed direction resolving hits on an edge
      const double dc1 = (v1[0] * dv[1] - v1[1] * dv[0]) / c0, dc2 = (dv[0] * v2[1] - dv[1] * v2[0]) / c0;
      const double dc3 = -dc1 - dc2;
      for (int x2 = lo[a2]; x2 <= hi[a2]; x2++)
        for (int x3 = lo[a3]; x3 <= hi[a3]; x3++) {
          const double v[2] = {(double)((float)x2 - t.p[0][a2]), (double)((float)x3 - t.p[0][a3])};
          const double c1 = (v1[0] * v[1] - v1[1] * v[0]) / c0, c2 = (v[0] * v2[1] - v[1] * v2[0]) / c0;
          const double c3 = 1. - c1 - c2;
          int topo = 0;
          topo += c1 == 0 ? dc1 > 0 : c1 > 0;
          topo += c2 == 0 ? dc2 > 0 : c2 > 0;
          topo += c3 == 0 ? dc3 > 0 : c3 > 0;
          if (topo != 3) continue;
          const double h = t.p[0][a1] * c3 + t.p[1][a1] * c2 + t.p[2][a1] * c1;
          int p[3];
          p[a2] = x2, p[a3] = x3;
          if (p[a2] < rlo[a2] || p[a2] >= rlo[a2] + rn[a2] || p[a3] < rlo[a3] || p[a3] >= rlo[a3] + rn[a3]) continue;
          for (int x1 = rlo[a1]; x1 <= h && x1 < rlo[a1] + rn[a1]; x1++) {
            p[a1] = x1;
            lev[(size_t)(p[0] - reg.dx) + (size_t)reg.nx * ((size_t)(p[1] - reg.dy) + (size_t)reg.ny * (p[2] - reg.dz))]++;
          }
        }
    }
    if (inside_out == 2) return;
    for (int x = reg.dx; x < reg.dx + reg.nx; x++)
      for (int y = reg.dy; y < reg.dy + reg.ny; y++)
        for (int z = reg.dz; z < reg.dz + reg.nz; z++)
          if (lev[(size_t)(x - reg.dx) + (size_t)reg.nx * ((size_t)(y - reg.dy) + (size_t)reg.ny * (z - reg.dz))] % 2 == 1)
            dot(x, y, z);
  }
  // calcCut (:479-505): does the link from node (x, y, z) to (x+dx, y+dy, z+dz)
  // meet the triangle? Solves p1 + s (p2 - p1) + t (p3 - p1) = X + r d by
  // Cramer's rule; a cut needs s, t, 1 - s - t >= 0 and 0 <= r <= 1.
  static bool link_cuts(const float (&p)[3][3], int x, int y, int z, int dx, int dy, int dz) {
    const double X[3] = {(double)x, (double)y, (double)z}, d[3] = {(double)dx, (double)dy, (double)dz};
    double e1[3], e2[3], w[3], m[3];
    for (int j = 0; j < 3; j++) {
      e1[j] = (double)p[1][j] - p[0][j];
      e2[j] = (double)p[2][j] - p[0][j];
      w[j] = X[j] - p[0][j];
      m[j] = -d[j];
    }
    auto det = [](const double* a, const double* b, const double* c) {
      return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
    };
    const double D = det(e1, e2, m);
    if (D == 0) return false;
    const double s = det(w, e2, m) / D, t = det(e1, w, m) / D, r = det(e1, e2, w) / D;
    return s >= 0 && t >= 0 && 1 - s - t >= 0 && r >= 0 && r <= 1;
  }
  // B-spline of order k through the control values p at x in [0, 1]: de Boor's
  // recursion on clamped uniform knots (src/spline.h:9-41).
  static double bspline(double x, std::vector<double> p, int k) {
    const int n = (int)p.size();
    int i = (int)std::floor(x * (n - k)) + k;
    if (k > n - 1) k = n - 1;
    if (i > n - 1) i = n - 1;
    if (i < k) i = k;
    auto knot = [&](int j) { return j < k + 1 ? 0.0 : j < n ? 1.0 * (j - k) / (n - k) : 1.0; };
    for (int j = k; j > 0; j--)
      for (int l = 0; l < j; l++) {
        const double a = (x - knot(i - l)) / (knot(i - l + j) - knot(i - l));
        p[i - l] = a * p[i - l] + (1 - a) * p[i - l - 1];
      }
    return p[i];
  }
  // <Sweep> (Geometry::loadSweep :689-756): balls moved along the B-spline of
  // order `order` (default 1) through the <Point x y z r> children, r defaulting
  // to the element's r (default 1). The curve parameter steps by `step`
  // (default 1e-4) or 1/`steps`; a ball within 0.25 of the previous one in x, y,
  // z and r is skipped. A node of the element's region is drawn when its centre
  // lies in a ball. A step that is not positive is an error (TCLB would loop
  // for ever).
  void draw_sweep(const XmlNode* node, const Region& reg) {
    int order = 1;
    if (const std::string* a = node->attr("order")) order = std::atoi(a->c_str());
    double dl = 1e-4;
    if (const std::string* a = node->attr("step")) dl = std::atof(a->c_str());
    if (const std::string* a = node->attr("steps")) dl = 1 / parse_value(*a);
    if (!(dl > 0)) throw CaseError("<Sweep> needs a positive step");
    double def_r = 1;
    if (const std::string* a = node->attr("r")) def_r = parse_value(*a);
    std::vector<double> px, py, pz, pr;
    for (const auto& c : node->children) {
      if (c->name != "Point") continue;  // TCLB notes other elements and ignores them
      px.push_back(parse_value(c->attr_or("x", "0")));
      py.push_back(parse_value(c->attr_or("y", "0")));
      pz.push_back(parse_value(c->attr_or("z", "0")));
      pr.push_back(c->attr("r") ? parse_value(*c->attr("r")) : def_r);
    }
    const int n = (int)px.size();
    if (n == 0) return;
    if (order > n - 1) order = n - 1;
    double x0_ = -999.0, y0_ = -999.0, z0_ = -999.0, r0_ = -999.0;
    for (double l = 0; l < 1; l += dl) {
      const double x0 = bspline(l, px, order), y0 = bspline(l, py, order), z0 = bspline(l, pz, order),
                   r = bspline(l, pr, order);
      if (std::fabs(x0 - x0_) < 0.25 && std::fabs(y0 - y0_) < 0.25 && std::fabs(z0 - z0_) < 0.25 &&
          std::fabs(r - r0_) < 0.25)
        continue;
      x0_ = x0, y0_ = y0, z0_ = z0, r0_ = r;
      const int b[3] = {(int)(x0 - r - 1), (int)(y0 - r - 1), (int)(z0 - r - 1)}, bn = (int)(2 * r + 2);
      const int rd[3] = {reg.dx, reg.dy, reg.dz}, rn[3] = {reg.nx, reg.ny, reg.nz};
      int lo[3], hi[3];
      bool empty = false;
      for (int j = 0; j < 3; j++) {
        lo[j] = std::max(rd[j], b[j]);
        hi[j] = std::min(rd[j] + rn[j], b[j] + bn);
        empty = empty || hi[j] <= lo[j];
      }
      if (empty) continue;
      for (int x = lo[0]; x < hi[0]; x++)
        for (int y = lo[1]; y < hi[1]; y++)
          for (int z = lo[2]; z < hi[2]; z++)
            if ((.5 + x - x0) * (.5 + x - x0) + (.5 + y - y0) * (.5 + y - y0) + (.5 + z - z0) * (.5 + z - z0) < r * r)
              dot(x, y, z);
    }
  }
  // Geometry::Draw (:758-1124) for the supported primitives
  void draw(const XmlNode* node) {
    for (const auto& cp : node->children) {
      const XmlNode* n = cp.get();
      Region r = region_of(n);
      if (n->name == "Box") {
        for (int z = std::max(r.dz, 0); z < std::min(r.dz + r.nz, nz); z++)
          for (int y = std::max(r.dy, 0); y < std::min(r.dy + r.ny, ny); y++)
            for (int x = std::max(r.dx, 0); x < std::min(r.dx + r.nx, nx); x++) dot(x, y, z);
      } else if (n->name == "Sphere") {
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy; y < r.dy + r.ny; y++)
            for (int z = r.dz; z < r.dz + r.nz; z++)
              if (in_sphere((.5 + x - r.dx) / r.nx, (.5 + y - r.dy) / r.ny, (.5 + z - r.dz) / r.nz)) dot(x, y, z);
      } else if (n->name == "HalfSphere") {
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy; y < r.dy + r.ny; y++)
            for (int z = r.dz; z < r.dz + r.nz; z++)
              if (in_sphere((.5 + x - r.dx) / r.nx, 0.5 - (.5 + y - r.dy) / r.ny / 2., (.5 + z - r.dz) / r.nz))
                dot(x, y, z);
      } else if (n->name == "OffgridSphere") {
        const double x0 = parse_value(n->attr_or("x", "0")), y0 = parse_value(n->attr_or("y", "0")),
                     z0 = parse_value(n->attr_or("z", "0"));
        double Rx, Ry, Rz;
        if (n->attr("R")) Rx = Ry = Rz = parse_value(*n->attr("R"));
        else {
          Rx = parse_value(n->attr_or("Rx", "0"));
          Ry = parse_value(n->attr_or("Ry", "0"));
          Rz = parse_value(n->attr_or("Rz", "0"));
        }
        const int bx = (int)(x0 - Rx - 5), by = (int)(y0 - Ry - 5), bz = (int)(z0 - Rz - 5);
        const int ex = (int)(2 * Rx + 10), ey = (int)(2 * Ry + 10), ez = (int)(2 * Rz + 10);
        for (int x = bx; x < bx + ex; x++)
          for (int y = by; y < by + ey; y++)
            for (int z = bz; z < bz + ez; z++) {
              const double xx = .5 + x - x0, yy = .5 + y - y0, zz = .5 + z - z0;
              if (xx * xx / (Rx * Rx) + yy * yy / (Ry * Ry) + zz * zz / (Rz * Rz) < 1.) dot(x, y, z);
            }
      } else if (n->name == "Cylinder") {
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy - 1; y < r.dy + r.ny + 1; y++)
            for (int z = r.dz - 1; z < r.dz + r.nz + 1; z++)
              if (in_sphere((.5 + x - r.dx) / r.nx, (.5 + y - r.dy) / r.ny, 0.5)) dot(x, y, z);
      } else if (n->name == "Pipe" || n->name == "PipeY" || n->name == "PipeZ") {
        // (:1022-1052) the region outside the cylinder inscribed in the box, axis
        // along x (Pipe), y (PipeY) or z (PipeZ); one extra layer across the axis
        const int ax = n->name == "Pipe" ? 0 : n->name == "PipeY" ? 1 : 2;
        const int lo[3] = {r.dx - (ax != 0), r.dy - (ax != 1), r.dz - (ax != 2)};
        const int hi[3] = {r.dx + r.nx + (ax != 0), r.dy + r.ny + (ax != 1), r.dz + r.nz + (ax != 2)};
        for (int x = lo[0]; x < hi[0]; x++)
          for (int y = lo[1]; y < hi[1]; y++)
            for (int z = lo[2]; z < hi[2]; z++) {
              const double fx = (.5 + x - r.dx) / r.nx, fy = (.5 + y - r.dy) / r.ny, fz = (.5 + z - r.dz) / r.nz;
              const bool in = ax == 0 ? in_sphere(0.5, fy, fz) : ax == 1 ? in_sphere(0.5, fx, fz) : in_sphere(0.5, fy, fx);
              if (!in) dot(x, y, z);
            }
      } else if (n->name == "OffgridPipe" || n->name == "XPipe" || n->name == "YPipe" || n->name == "ZPipe" ||
                 n->name == "XAnnulus") {
        // (:835-1021) elliptic cylinders about an off-grid centre (x, y, z), the
        // axis z (OffgridPipe, ZPipe), x (XPipe, XAnnulus) or y (YPipe). Across
        // the axis the box spans the radii plus 5 nodes, truncated to int;
        // along it the element's region. YPipe and ZPipe measure the x offset
        // from y (.5 + x - y0), as TCLB does. XAnnulus keeps the nodes inside
        // the outer ellipse (Ro or Ry_o/Rz_o) and outside the inner one.
        const double c[3] = {parse_value(n->attr_or("x", "0")), parse_value(n->attr_or("y", "0")),
                             parse_value(n->attr_or("z", "0"))};
        const int ax = n->name == "XPipe" || n->name == "XAnnulus" ? 0 : n->name == "YPipe" ? 1 : 2;
        const int a = ax == 0 ? 1 : 0, b = ax == 2 ? 1 : 2;  // cross-section axes, a < b
        const char* nm = "xyz";
        const double ca = (n->name == "YPipe" || n->name == "ZPipe") ? c[1] : c[a], cb = c[b];
        const bool annulus = n->name == "XAnnulus";
        auto radius = [&](const std::string& k, const char* all) {
          if (n->attr(all)) return parse_value(*n->attr(all));
          return parse_value(n->attr_or(k, "0"));
        };
        double Ra, Rb, Ra_i = 0, Rb_i = 0;
        if (annulus) {
          Ra = radius("Ry_o", "Ro"), Rb = radius("Rz_o", "Ro");
          Ra_i = radius("Ry_i", "Ri"), Rb_i = radius("Rz_i", "Ri");
        } else {
          Ra = radius(std::string("R") + nm[a], "R"), Rb = radius(std::string("R") + nm[b], "R");
        }
        int lo[3] = {r.dx, r.dy, r.dz}, len[3] = {r.nx, r.ny, r.nz};
        lo[a] = (int)(c[a] - Ra - 5), len[a] = (int)(2 * Ra + 10);
        lo[b] = (int)(c[b] - Rb - 5), len[b] = (int)(2 * Rb + 10);
        for (int x = lo[0]; x < lo[0] + len[0]; x++)
          for (int y = lo[1]; y < lo[1] + len[1]; y++)
            for (int z = lo[2]; z < lo[2] + len[2]; z++) {
              const int p[3] = {x, y, z};
              const double pa = .5 + p[a] - ca, pb = .5 + p[b] - cb;
              bool in = pa * pa / (Ra * Ra) + pb * pb / (Rb * Rb) < 1.;
              if (annulus) in = in && pa * pa / (Ra_i * Ra_i) + pb * pb / (Rb_i * Rb_i) > 1.;
              if (in) dot(x, y, z);
            }
      } else if (n->name == "Wedge") {
        const std::string dir = n->attr_or("direction", "");
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy; y < r.dy + r.ny; y++)
            for (int z = r.dz; z < r.dz + r.nz; z++)
              if (in_wedge((x - r.dx) / (r.nx - 1.), (y - r.dy) / (r.ny - 1.), (z - r.dz) / (r.nz - 1.), dir))
                dot(x, y, z);
      } else if (n->name == "STL") {
        draw_stl(n, r);
      } else if (n->name == "Sweep") {
        draw_sweep(n, r);
      } else if (n->name == "Text") {  // node list, x outer, z inner (:1086-1112)
        Region crop = region_of(n->parent);
        const std::string* file = n->attr("file");
        if (!file) throw CaseError("<Text> needs a file attribute");
        std::ifstream in(*file);
        if (!in) throw CaseError("cannot open " + *file);
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy; y < r.dy + r.ny; y++)
            for (int z = r.dz; z < r.dz + r.nz; z++) {
              int v;
              if (!(in >> v)) throw CaseError("file " + *file + " ended while reading");
              if (v != 0 && x >= crop.dx && y >= crop.dy && z >= crop.dz && x < crop.dx + crop.nx &&
                  y < crop.dy + crop.ny && z < crop.dz + crop.nz)
                dot(x, y, z);
            }
      } else if (const XmlNode* zn = find_zone(n->name)) {
        draw(zn);
      } else {
        throw CaseError("unsupported geometry element <" + n->name + ">");
      }
    }
  }
  // Geometry::load (:1140-1184)
  void load(const XmlNode* g, const XmlNode* def) {
    user = g;
    defaults = def;
    for (const auto& cp : g->children) {
      const XmlNode* n = cp.get();
      if (n->name == "Zone" || n->name == "Type" || n->name == "Mask") continue;
      set_flag(n->name);
      for (const auto& a : n->attrs) {
        if (a.first == "name") set_zone(a.second);
        else if (a.first == "mask") mask = group_mask(a.second);
        else if (a.first == "mode") {
          if (a.second == "overwrite") mode = OVERWRITE;
          else if (a.second == "fill") mode = FILL;
          else if (a.second == "change") mode = CHANGE;
          else throw CaseError("unknown mode " + a.second);
        }
      }
      // zone="..." draws that <Zone> (the case's own or a default one) first
      // (Geometry::loadZone :1127-1137); an unknown name is reported and skipped,
      // as TCLB does
      if (const std::string* z = n->attr("zone")) {
        if (const XmlNode* zn = find_zone(*z)) draw(zn);
        else std::fprintf(stderr, "[tclb_run] unknown zone %s in <%s>\n", z->c_str(), n->name.c_str());
      }
      draw(n);
    }
  }
};

int pad_nx(int nx, int xsdim = 32) { return nx + xsdim - 1 - ((nx - 1) % xsdim); }

// ------------------------------------------------------------------ runner
struct Runner;
std::string read_file(const std::string& path);
void write_xml(std::ostream& o, const XmlNode* n, int depth);

// The previous value of a <Stop> criterion before its first check (cbStop's
// own sentinel, so a first Change check fails as in TCLB).
constexpr double STOP_UNSET = -12341234;

struct Callback {
  std::string kind;  // Log, BIN, Failcheck, SaveCheckpoint, Stop
  const XmlNode* node;
  double every = 0, start = 0;
  std::string file;
  // <Stop> (src/Handlers/cbStop.cpp): per criterion the Global, its kind,
  // limit and value at the previous check; consecutive passing checks
  enum { CHANGE, PERCENT_CHANGE, ABOVE, BELOW };
  std::vector<int> stop_global, stop_kind;
  std::vector<double> stop_limit, stop_old;
  int stop_times = 1, stop_score = 0;
  // <Sample> (src/Handlers/cbSample.cpp, src/Sampler.cpp): the sampled nodes,
  // quantities, and the rows (values at every point) recorded since the last
  // write, the first one labelled sample_start
  // <PID> (src/Handlers/cbPID.cpp): the Global it integrates, the zonal
  // setting (and zone, -1 for all) it drives, its constants and state
  int pid_global = -1, pid_setting = -1, pid_zone = -1;
  double pid_target = 0, pid_itime = 1, pid_dtime = 1, pid_scale = 1, pid_sval = 0, pid_integral = 0,
         pid_old_err = 0;
  // <Keep> (src/Handlers/cbKeep.cpp): the Global, its InObj zonal setting,
  // the threshold, the kind (1 Above, -1 Below, 0 Equal) and the force
  int keep_global = -1, keep_inobj = -1, keep_type = 0;
  double keep_thr = 0, keep_force = 1;
  // <Failcheck>: the checked region (x0, y0, z0, nx, ny, nz)
  int fc_region[6] = {0, 0, 0, 1, 1, 1};
  std::vector<std::array<int, 3>> sample_pts;
  std::vector<int> sample_q;
  std::vector<double> sample_rows;
  long long sample_start = 0;
  bool now(double it) const {  // vHandler::Now
    if (every <= 0) return false;
    it -= start;
    return std::floor(it / every) > std::floor((it - 1) / every);
  }
  int next(double it) const {  // vHandler::Next
    if (every <= 0) return -1;
    it -= start;
    const double k = std::floor(it / every);
    return (int)(-std::floor(-(k + 1) * every) - it);
  }
};

struct Runner {
  int model, precision, storage;
  const ModelTable* T;
  std::string outpath, outdir;
  tclb_h lat = nullptr;
  std::unique_ptr<Geometry> geo;
  std::unique_ptr<XmlNode> def_doc;
  long long iter = 0;
  std::vector<Callback> hands;
  int iter_type = TCLB_ITER_NORM;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  bool verbose = true;
  std::string config_text;
  std::vector<std::string> checkpoints, restarts;

  ~Runner() {
    if (lat) tclb_destroy(lat);
  }
  void ck(int rc, const char* what) {
    if (rc) throw CaseError(std::string(what) + ": " + tclb_last_error());
  }
  int setting_index(const std::string& n) const {
    for (int i = 0; i < T->nsettings; i++)
      if (n == T->setting_names[i]) return i;
    return -1;
  }
  int zone_setting_index(const std::string& n) const {
    for (int i = 0; i < T->nzonesettings; i++)
      if (n == T->zone_setting_names[i]) return i;
    return -1;
  }
  void need_lattice() const {
    if (!lat) throw CaseError("<Geometry> must come before this element");
  }

  void geometry(const XmlNode* n) {  // acGeometry + Solver::setSize
    if (lat) throw CaseError("a second <Geometry> is not supported");
    const int nx = pad_nx(parse_int(n->attr_or("nx", "1"))), ny = parse_int(n->attr_or("ny", "1")),
              nz = parse_int(n->attr_or("nz", "1"));
    ck(tclb_create(&lat, model, nx, ny, nz, precision, storage), "create");
    def_doc = XmlParser(DEFAULT_ZONES).parse();
    geo = std::make_unique<Geometry>(T, nx, ny, nz);
    geo->load(n, def_doc->children[0].get());
    ck(tclb_set_flags(lat, geo->geom.data(), 0, 0, 0, nx, ny, nz), "flags");
    if (verbose) std::printf("[tclb_run] lattice %dx%dx%d, %zu zones\n", nx, ny, nz, geo->zones.size());
  }
  void param(const XmlNode* n) {  // acParam (src/Handlers/acParam.cpp:5-60)
    need_lattice();
    const std::string name = n->attr_or("name", ""), zone = n->attr_or("zone", "");
    const std::string* value = n->attr("value");
    if (name.empty()) throw CaseError("<Param> without a name");
    if (!value) throw CaseError("<Param name=" + name + "> without a value");
    const double v = parse_value(*value);
    int zn = -1;
    if (!zone.empty()) {
      auto it = geo->zones.find(zone);
      if (it == geo->zones.end()) throw CaseError("unknown zone " + zone);
      zn = it->second;
    }
    const int s = setting_index(name);
    if (s >= 0) {
      ck(tclb_set_setting(lat, s, v), "setting");
      return;
    }
    const int zs = zone_setting_index(name);
    if (zs >= 0) {
      ck(tclb_set_zone_setting(lat, zs, zn, v), "zone setting");
      return;
    }
    throw CaseError("unknown setting " + name);
  }
  void init() {
    need_lattice();
    ck(tclb_init(lat), "init");
    iter = 0;
  }

  std::string iter_file(const std::string& name, const std::string& suffix) const {  // Solver::outIterFile
    char buf[64];
    std::snprintf(buf, sizeof(buf), "_P00_%08lld", iter);
    return outpath + "_" + name + buf + suffix;
  }

  // Solver::initLog / writeLog (src/Solver.cpp.Rt:120-206): each value and its
  // SI value (si_scale), then the SI sizes of the lattice units of length,
  // time and mass; Time_si is the iteration times that of time.
  void log_header(const std::string& f) {
    FILE* o = std::fopen(f.c_str(), "wt");
    if (!o) throw CaseError("cannot write " + f);
    std::fprintf(o, "\"Iteration\",\"Time_si\",\"Walltime\",\"Optimization\"");
    for (int i = 0; i < T->nsettings; i++) std::fprintf(o, ",\"%s\",\"%s_si\"", T->setting_names[i], T->setting_names[i]);
    for (int i = 0; i < T->nzonesettings; i++)
      for (const auto& z : geo->zones)
        std::fprintf(o, ",\"%s-%s\",\"%s-%s_si\"", T->zone_setting_names[i], z.first.c_str(), T->zone_setting_names[i],
                     z.first.c_str());
    for (int i = 0; i < T->nglobals; i++) std::fprintf(o, ",\"%s\",\"%s_si\"", T->global_names[i], T->global_names[i]);
    for (const char* s : {"dx", "dt", "dm"}) std::fprintf(o, ",\"%s_si\"", s);
    std::fprintf(o, "\n");
    std::fclose(o);
  }
  void log_row(const std::string& f) {
    FILE* o = std::fopen(f.c_str(), "at");
    if (!o) throw CaseError("cannot write " + f);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double dt_si = 1.0 / g_units.alt("s");
    std::fprintf(o, "%lld, %.13le, %.13le, %d", iter, dt_si * (double)iter, wall, 0);
    for (int i = 0; i < T->nsettings; i++) {
      double v = 0;
      tclb_get_setting(lat, i, &v);
      std::fprintf(o, ", %.13le, %.13le", v, v * si_scale(model, T->setting_names[i]));
    }
    for (int i = 0; i < T->nzonesettings; i++)
      for (const auto& z : geo->zones) {
        double v = 0;
        tclb_get_zone_setting(lat, i, z.second, &v);
        std::fprintf(o, ", %.13le, %.13le", v, v * si_scale(model, T->zone_setting_names[i]));
      }
    std::vector<double> g(T->nglobals);
    tclb_get_globals(lat, g.data());
    for (int i = 0; i < T->nglobals; i++)
      std::fprintf(o, ", %.13le, %.13le", g[i], g[i] * si_scale(model, T->global_names[i]));
    for (const char* u : {"m", "s", "kg"}) std::fprintf(o, ", %.13le", 1.0 / g_units.alt(u));
    std::fprintf(o, "\n");
    std::fclose(o);
  }
  // <VTK> (src/Handlers/cbVTK.cpp, src/vtkLattice.cpp:9-56, src/vtkOutput.cpp):
  // a VTK XML ImageData file <case>_<name>_P00_<iteration>.vti with cell data
  // of the region (dx..nz attributes, default the whole lattice), and the
  // parallel wrapper .pvti naming it as its one piece. Fields: "flag" (the
  // node-type word) when named in `what`; each node-type group and
  // SETTINGZONE as UInt8 (the group's bits); each quantity in SI units
  // (1 / lattice value of its unit). `what` is a comma list of names, default
  // "all" (every group and quantity). Arrays are inline base64: a 4-byte
  // length block, then the data block.
  void write_vtk(const Callback& c) {
    int tot[3];
    tclb_get_size(lat, &tot[0], &tot[1], &tot[2]);
    int reg[6] = {0, 0, 0, tot[0], tot[1], tot[2]};  // x0 y0 z0 nx ny nz
    const char* dn[3] = {"dx", "dy", "dz"};
    const char* nn[3] = {"nx", "ny", "nz"};
    for (int a = 0; a < 3; a++) {
      if (const std::string* v = c.node->attr(dn[a])) {
        reg[a] = parse_int(*v);
        if (reg[a] < 0) {  // from the far face
          reg[a] += tot[a];
          reg[3 + a] = tot[a] - reg[a];
        }
      }
      if (const std::string* v = c.node->attr(nn[a])) {
        reg[3 + a] = parse_int(*v);
        if (reg[3 + a] < 0) reg[3 + a] += tot[a] - reg[a];
      }
      const int lo = std::max(0, reg[a]), hi = std::min(tot[a], reg[a] + reg[3 + a]);
      reg[a] = lo;
      reg[3 + a] = std::max(0, hi - lo);
    }
    const size_t size = (size_t)reg[3] * reg[4] * reg[5];
    if (size == 0) throw CaseError("<VTK> region is empty");
    bool all = false;
    std::vector<std::string> what;
    {
      std::stringstream ss(c.node->attr_or("what", "all"));
      std::string w;
      while (std::getline(ss, w, ','))
        if (w == "all") all = true;
        else what.push_back(w);
    }
    auto named = [&](const std::string& n) { return std::find(what.begin(), what.end(), n) != what.end(); };
    const std::string name = c.node->attr_or("name", "VTK");
    const std::string fn = iter_file(name, ".vti"), pfn = iter_file(name, ".pvti");
    FILE* o = std::fopen(fn.c_str(), "wb");
    FILE* po = std::fopen(pfn.c_str(), "wb");
    if (!o || !po) {
      if (o) std::fclose(o);
      if (po) std::fclose(po);
      throw CaseError("cannot write " + fn);
    }
    const double spacing = 1.0 / g_units.alt("m");
    char ext[160];
    std::snprintf(ext, sizeof(ext), "%d %d %d %d %d %d", reg[0], reg[0] + reg[3], reg[1], reg[1] + reg[4], reg[2],
                  reg[2] + reg[5]);
    std::fprintf(o, "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(o, "<ImageData WholeExtent=\"%s\" Origin=\"0 0 0\" Spacing=\"%lg %lg %lg\">\n", ext, spacing, spacing,
                 spacing);
    std::fprintf(o, "<Piece Extent=\"%s\">\n<CellData Scalars=\"rho\" Vectors=\"velocity\">\n", ext);
    std::fprintf(po, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(po, "<PImageData WholeExtent=\"%s\" Origin=\"0 0 0\" Spacing=\"%lg %lg %lg\">\n", ext, spacing,
                 spacing, spacing);
    const size_t sl = fn.find_last_of('/');
    std::fprintf(po, "<Piece Extent=\"%s\" Source=\"%s\"/>\n<PCellData Scalars=\"rho\" Vectors=\"velocity\">\n", ext,
                 (sl == std::string::npos ? fn : fn.substr(sl + 1)).c_str());
    auto field = [&](const char* fname, const char* type, int comps, const void* data, size_t bytes) {
      std::fprintf(o, "<DataArray type=\"%s\" Name=\"%s\" format=\"binary\" encoding=\"base64\" NumberOfComponents=\"%d\">\n",
                   type, fname, comps);
      const int len = (int)bytes;
      put_base64(o, &len, sizeof(len));
      put_base64(o, data, bytes);
      std::fprintf(o, "\n</DataArray>\n");
      std::fprintf(po, "<PDataArray type=\"%s\" Name=\"%s\" format=\"binary\" encoding=\"base64\" NumberOfComponents=\"%d\"/>\n",
                   type, fname, comps);
    };
    // node types of the region
    std::vector<uint16_t> all_fl((size_t)tot[0] * tot[1] * tot[2]), fl(size);
    ck(tclb_get_flags(lat, all_fl.data()), "flags");
    size_t k = 0;
    for (int z = 0; z < reg[5]; z++)
      for (int y = 0; y < reg[4]; y++)
        for (int x = 0; x < reg[3]; x++)
          fl[k++] = all_fl[(size_t)(reg[0] + x) + (size_t)tot[0] * ((size_t)(reg[1] + y) + (size_t)tot[1] * (reg[2] + z))];
    if (named("flag")) field("flag", "UInt16", 1, fl.data(), size * 2);
    std::vector<unsigned char> small(size);
    for (int gi = 0; gi <= T->ngroups; gi++) {  // the model's groups, then SETTINGZONE
      const bool zone = gi == T->ngroups;
      const std::string gname = zone ? "SETTINGZONE" : T->group_names[gi];
      if (!all && !named(gname)) continue;
      const unsigned mask = zone ? (0xFFFFu << T->zone_shift) & 0xFFFFu : (unsigned)T->group_masks[gi];
      int shift = 0;
      while (shift < 16 && !(mask >> shift & 1u)) shift++;
      for (size_t i = 0; i < size; i++) small[i] = (unsigned char)((fl[i] & mask) >> shift);
      field(gname.c_str(), "UInt8", 1, small.data(), size);
    }
    const size_t rs = precision == TCLB_FP64 ? 8 : 4;
    for (int q = 0; q < T->nquantities; q++) {
      if (!all && !named(T->quantity_names[q])) continue;
      const int comp = T->quantity_vector[q] ? 3 : 1;
      std::vector<char> buf(size * comp * rs);
      ck(tclb_get_quantity(lat, q, reg, buf.data(), si_scale(model, T->quantity_names[q]), nullptr), "quantity");
      field(T->quantity_names[q], rs == 8 ? "Float64" : "Float32", comp, buf.data(), buf.size());
    }
    std::fprintf(o, "</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n");
    std::fprintf(po, "</PCellData>\n</PImageData>\n</VTKFile>\n");
    std::fclose(o);
    std::fclose(po);
  }

  // <TXT> (src/Handlers/cbTXT.cpp, txtWriteLattice src/vtkLattice.cpp:83-161):
  // <case>_<name>_P00_<iteration>_info.txt with the SI sizes of the lattice
  // units and the lattice size, and one text file per quantity (`what`,
  // default all) in SI units: %.8g (float) or %.16lg (double) values, a new
  // line after every nx nodes. Vector quantities give x y z per node (TCLB
  // reads them into a one-value-per-node buffer). gzip="true" writes each
  // quantity file gzip-compressed (zlib) as <file>.gz.
  void write_txt(const Callback& c) {
    int nx, ny, nz;
    tclb_get_size(lat, &nx, &ny, &nz);
    const size_t size = (size_t)nx * ny * nz;
    const std::string base = iter_file(c.node->attr_or("name", "TXT"), "");
    const std::string gz = c.node->attr_or("gzip", "false");
    const bool gzip = gz == "true" || gz == "1" || gz == "yes";
    bool all = false;
    std::vector<std::string> what;
    {
      std::stringstream ss(c.node->attr_or("what", "all"));
      std::string w;
      while (std::getline(ss, w, ','))
        if (w == "all") all = true;
        else what.push_back(w);
    }
    {
      FILE* f = std::fopen((base + "_info.txt").c_str(), "w");
      if (!f) throw CaseError("cannot write " + base + "_info.txt");
      std::fprintf(f, "dx: %lg\ndt: %lg\ndm: %lg\ndT: %lg\n", 1.0 / g_units.alt("m"), 1.0 / g_units.alt("s"),
                   1.0 / g_units.alt("kg"), 1.0 / g_units.alt("K"));
      std::fprintf(f, "size: %zu\nNX: %d\nNY: %d\nNZ: %d\n", size, nx, ny, nz);
      std::fclose(f);
    }
    const bool dbl = precision == TCLB_FP64;
    for (int q = 0; q < T->nquantities; q++) {
      const std::string qn = T->quantity_names[q];
      if (!all && std::find(what.begin(), what.end(), qn) == what.end()) continue;
      const int comp = T->quantity_vector[q] ? 3 : 1;
      std::vector<char> buf(size * comp * (dbl ? 8 : 4));
      ck(tclb_get_quantity(lat, q, nullptr, buf.data(), si_scale(model, qn), nullptr), "quantity");
      const std::string fn = base + "_" + qn + ".txt" + (gzip ? ".gz" : "");
      TextSink out(fn, gzip);
      char num[40];
      for (size_t i = 0; i < size; i++) {
        for (int k = 0; k < comp; k++) {
          if (k) out.put(" ", 1);
          const int len = dbl ? std::snprintf(num, sizeof(num), "%.16lg", reinterpret_cast<const double*>(buf.data())[i * comp + k])
                              : std::snprintf(num, sizeof(num), "%.8g",
                                              (double)reinterpret_cast<const float*>(buf.data())[i * comp + k]);
          out.put(num, (size_t)len);
        }
        out.put((i + 1) % nx == 0 ? "\n" : " ", 1);
      }
      out.close();
    }
  }

  // A text file written through a buffer, plain or gzip-compressed (zlib).
  struct TextSink {
    std::string name, buf;
    FILE* f = nullptr;
    gzFile z = nullptr;
    TextSink(const std::string& fn, bool gzip) : name(fn) {
      if (gzip) z = gzopen(fn.c_str(), "wb");
      else f = std::fopen(fn.c_str(), "w");
      if (!f && !z) throw CaseError("cannot write " + fn);
      buf.reserve(1 << 20);
    }
    ~TextSink() {
      if (f) std::fclose(f);
      if (z) gzclose(z);
    }
    void put(const char* p, size_t n) {
      buf.append(p, n);
      if (buf.size() >= (1u << 20)) flush();
    }
    void flush() {
      if (buf.empty()) return;
      const bool ok = f ? std::fwrite(buf.data(), 1, buf.size(), f) == buf.size()
                        : gzwrite(z, buf.data(), (unsigned)buf.size()) == (int)buf.size();
      if (!ok) throw CaseError("write failed for " + name);
      buf.clear();
    }
    void close() {
      flush();
      const bool ok = f ? std::fclose(f) == 0 : gzclose(z) == Z_OK;
      f = nullptr;
      z = nullptr;
      if (!ok) throw CaseError("write failed for " + name);
    }
  };

  // binWriteLattice (src/vtkLattice.cpp:58-81): one raw real_t file per quantity
  void write_bin(const std::string& prefix) {
    int nx, ny, nz;
    tclb_get_size(lat, &nx, &ny, &nz);
    const size_t N = (size_t)nx * ny * nz;
    const size_t rs = precision == TCLB_FP64 ? 8 : 4;
    for (int q = 0; q < T->nquantities; q++) {
      const int comp = T->quantity_vector[q] ? 3 : 1;
      std::vector<char> buf(N * comp * rs);
      ck(tclb_get_quantity(lat, q, nullptr, buf.data(), 1.0, nullptr), "quantity");
      const std::string fn = prefix + "." + T->quantity_names[q] + ".bin";
      FILE* o = std::fopen(fn.c_str(), "wb");
      if (!o) throw CaseError("cannot write " + fn);
      std::fwrite(buf.data(), 1, buf.size(), o);
      std::fclose(o);
    }
  }
  // cbFailcheck: stop when a quantity is not finite
  // cbFailcheck (src/Handlers/cbFailcheck.cpp:4-88): the `what` quantities
  // (default all) over the region dx..nz, which defaults to the one node at
  // the origin (lbRegion's default size 1 x 1 x 1; TCLB's examples give nx, ny
  // and nz), clipped to the lattice. NaN (not Inf) fails the check; the
  // element's children then run as final actions before the stop. TCLB sets a
  // re-entrancy flag at its first check and never clears it, so it checks
  // once; here every call checks.
  bool failcheck(const Callback& c) {
    int dims[3];
    tclb_get_size(lat, &dims[0], &dims[1], &dims[2]);
    int reg[6];
    for (int a = 0; a < 3; a++) {
      const int lo = std::max(c.fc_region[a], 0), hi = std::min(c.fc_region[a] + c.fc_region[3 + a], dims[a]);
      if (hi <= lo) return false;
      reg[a] = lo, reg[3 + a] = hi - lo;
    }
    const size_t N = (size_t)reg[3] * reg[4] * reg[5];
    std::vector<std::string> what;
    bool all = false;
    {
      std::stringstream ss(c.node->attr_or("what", "all"));
      std::string w;
      while (std::getline(ss, w, ','))
        if (w == "all") all = true;
        else what.push_back(w);
    }
    bool nan = false;
    for (int q = 0; q < T->nquantities && !nan; q++) {
      if (!all && std::find(what.begin(), what.end(), T->quantity_names[q]) == what.end()) continue;
      const int comp = T->quantity_vector[q] ? 3 : 1;
      if (precision == TCLB_FP64) {
        std::vector<double> b(N * comp);
        ck(tclb_get_quantity(lat, q, reg, b.data(), 1.0, nullptr), "quantity");
        for (double v : b) nan = nan || std::isnan(v);
      } else {
        std::vector<float> b(N * comp);
        ck(tclb_get_quantity(lat, q, reg, b.data(), 1.0, nullptr), "quantity");
        for (float v : b) nan = nan || std::isnan(v);
      }
    }
    if (!nan) return false;
    for (const auto& ch : c.node->children) {  // final actions
      Callback f = make_callback(ch.get());
      do_callback(f);
    }
    return true;
  }

  // <LoadBinary file=> (src/Handlers/acLoadBinary.cpp): Lattice::loadSolution
  // reads <file>_0.pri (rank 0) into the current snapshot.
  void load_binary(const XmlNode* n) {
    need_lattice();
    const std::string* f = n->attr("file");
    if (!f) f = n->attr("filename");
    if (!f) throw CaseError("<" + n->name + "> needs a file attribute");
    if (n->attr("comp")) {
      // acLoadMemoryDump reports comp= as deprecated and loads the snapshot
      if (n->name == "LoadBinary") throw CaseError("<LoadBinary comp=> (single fields) is not supported");
      std::fprintf(stderr, "[tclb_run] <LoadMemoryDump comp=> is deprecated; loading the whole snapshot\n");
    }
    const std::string fn = *f + "_0.pri";
    const std::string data = read_file(fn);
    if (data.size() != tclb_pri_bytes(lat)) throw CaseError(fn + " does not match this lattice");
    ck(tclb_load_pri(lat, data.data(), data.size()), "load .pri");
  }
  // cbKeep::Init (src/Handlers/cbKeep.cpp:5-43): What= names the Global; one
  // of Above, Below or Equal gives the threshold; Force (default 1) the gain
  void keep_init(Callback& c) {
    const XmlNode* n = c.node;
    const std::string* what = n->attr("What");
    if (!what) throw CaseError("<Keep> needs What= (a Global)");
    for (int g = 0; g < T->nglobals; g++)
      if (*what == T->global_names[g]) c.keep_global = g;
    if (c.keep_global < 0) throw CaseError("unknown Global in <Keep>: " + *what);
    c.keep_inobj = zone_setting_index(*what + "InObj");
    if (c.keep_inobj < 0) throw CaseError("<Keep>: " + *what + " has no InObj setting");
    const std::string* thr;
    if ((thr = n->attr("Above"))) c.keep_type = 1;
    else if ((thr = n->attr("Below"))) c.keep_type = -1;
    else if ((thr = n->attr("Equal"))) c.keep_type = 0;
    else throw CaseError("<Keep> needs Above, Below or Equal");
    c.keep_thr = std::atof(thr->c_str());
    if (const std::string* f = n->attr("Force")) c.keep_force = std::atof(f->c_str());
    iter_type |= TCLB_ITER_LASTGLOB;
  }
  // cbKeep::DoIt (:46-66): v = (threshold - Global) * Force; the Global's InObj
  // weight in every zone becomes v when it points the kept way (v > 0 for
  // Above, v < 0 for Below, always for Equal), else 0
  void keep_step(Callback& c) {
    std::vector<double> g(T->nglobals);
    tclb_get_globals(lat, g.data());
    const double v = (c.keep_thr - g[c.keep_global]) * c.keep_force;
    double s = 0.0;
    if (c.keep_type == 0 || (c.keep_type == 1 && v > 0) || (c.keep_type == -1 && v < 0)) s = v;
    ck(tclb_set_zone_setting(lat, c.keep_inobj, -1, s), "zone setting");
  }
  // cbPID::Init (src/Handlers/cbPID.cpp:4-92): integral= names the Global,
  // target= its goal, control= the zonal setting driven in zone= (all zones
  // when absent); IntegrationTime, DerivativeTime and scale default to 1 s.
  // The setting's value at this point (zone 0 for all zones) is the base the
  // control is added to.
  void pid_init(Callback& c) {
    const XmlNode* n = c.node;
    const std::string glob = n->attr_or("integral", "");
    const std::string* target = n->attr("target");
    if (!target) throw CaseError("<PID> needs a target");
    c.pid_target = parse_value(*target);
    if (glob.empty()) throw CaseError("<PID> needs integral= (a Global)");
    for (int g = 0; g < T->nglobals; g++)
      if (glob == T->global_names[g]) c.pid_global = g;
    if (c.pid_global < 0) throw CaseError("unknown Global in <PID>: " + glob);
    const std::string zone = n->attr_or("zone", "");
    if (!zone.empty()) {
      auto it = geo->zones.find(zone);
      if (it == geo->zones.end()) throw CaseError("unknown zone in <PID>: " + zone);
      c.pid_zone = it->second;
    }
    const std::string par = n->attr_or("control", "");
    if (par.empty()) throw CaseError("<PID> needs control= (a zonal setting)");
    c.pid_setting = zone_setting_index(par);
    if (c.pid_setting < 0) throw CaseError(par + " is not a zonal setting (in <PID>)");
    const double second = g_units.alt("1s");
    c.pid_itime = n->attr("IntegrationTime") ? parse_value(*n->attr("IntegrationTime")) : second;
    c.pid_dtime = n->attr("DerivativeTime") ? parse_value(*n->attr("DerivativeTime")) : second;
    c.pid_scale = n->attr("scale") ? parse_value(*n->attr("scale")) : second;
    ck(tclb_get_zone_setting(lat, c.pid_setting, c.pid_zone < 0 ? 0 : c.pid_zone, &c.pid_sval), "zone setting");
    iter_type |= TCLB_ITER_LASTGLOB;
  }
  // cbPID::DoIt (:93-125): error = target - Global; trapezoid integral over
  // the callback period DT; control = error + integral / IntegrationTime +
  // derivative * DerivativeTime; setting = base + control * scale
  void pid_step(Callback& c) {
    std::vector<double> g(T->nglobals);
    tclb_get_globals(lat, g.data());
    const double dt = c.every, err = c.pid_target - g[c.pid_global];
    c.pid_integral += (c.pid_old_err + err) * dt / 2.0;
    const double derivative = (err - c.pid_old_err) / dt;
    const double control = err + c.pid_integral / c.pid_itime + derivative * c.pid_dtime;
    c.pid_old_err = err;
    ck(tclb_set_zone_setting(lat, c.pid_setting, c.pid_zone, c.pid_sval + control * c.pid_scale), "zone setting");
  }
  // cbSample::Init (src/Handlers/cbSample.cpp:5-47), Sampler::initCSV
  // (src/Sampler.cpp:16-36): the <Point dx dy dz> nodes inside the lattice
  // (coordinates truncated to int), the `what` quantities (default all), and
  // <case>_Sampler_P00_<iteration>.csv with the header
  // Iteration,X,Y,Z,<quantity>[.x,.y,.z]...
  void sample_init(Callback& c) {
    if (c.every <= 0) throw CaseError("<Sample> needs Iterations > 0");
    std::vector<std::string> what;
    bool all = false;
    {
      std::stringstream ss(c.node->attr_or("what", "all"));
      std::string w;
      while (std::getline(ss, w, ','))
        if (w == "all") all = true;
        else what.push_back(w);
    }
    int nx, ny, nz;
    tclb_get_size(lat, &nx, &ny, &nz);
    for (const auto& ch : c.node->children) {
      if (ch->name != "Point") throw CaseError("unknown element <" + ch->name + "> in <Sample>");
      int p[3] = {0, 0, 0};
      const char* k[3] = {"dx", "dy", "dz"};
      for (int a = 0; a < 3; a++)
        if (const std::string* v = ch->attr(k[a])) p[a] = (int)parse_value(*v);
      if (p[0] >= 0 && p[1] >= 0 && p[2] >= 0 && p[0] < nx && p[1] < ny && p[2] < nz)
        c.sample_pts.push_back({p[0], p[1], p[2]});
    }
    c.file = iter_file("Sampler", ".csv");
    FILE* f = std::fopen(c.file.c_str(), "wt");
    if (!f) throw CaseError("cannot write " + c.file);
    std::fprintf(f, "Iteration,X,Y,Z");
    for (int q = 0; q < T->nquantities; q++) {
      const std::string qn = T->quantity_names[q];
      if (!all && std::find(what.begin(), what.end(), qn) == what.end()) continue;
      c.sample_q.push_back(q);
      if (T->quantity_vector[q]) std::fprintf(f, ",%s.x,%s.y,%s.z", qn.c_str(), qn.c_str(), qn.c_str());
      else std::fprintf(f, ",%s", qn.c_str());
    }
    std::fprintf(f, "\n");
    std::fclose(f);
    c.sample_start = iter;
  }
  // Lattice::updateAllSamples (src/Lattice.cu.Rt:1376-1390), after every
  // iteration: the quantities at the sampled nodes, in SI units
  void sample_record(Callback& c) {
    const bool dbl = precision == TCLB_FP64;
    for (const auto& p : c.sample_pts)
      for (int q : c.sample_q) {
        const int region[6] = {p[0], p[1], p[2], 1, 1, 1};
        char buf[24];
        ck(tclb_get_quantity(lat, q, region, buf, si_scale(model, T->quantity_names[q]), nullptr), "quantity");
        for (int k = 0; k < (T->quantity_vector[q] ? 3 : 1); k++)
          c.sample_rows.push_back(dbl ? reinterpret_cast<const double*>(buf)[k]
                                      : (double)reinterpret_cast<const float*>(buf)[k]);
      }
  }
  // cbSample::DoIt, Sampler::writeHistory (src/Sampler.cpp:37-62): one line per
  // iteration since the last write and sampled node: the iteration, the node's
  // X,Y,Z and its values (%g). TCLB prints only the x value of a vector
  // quantity (it copies the three into one real_t); all three are written here,
  // as its header names them.
  void sample_write(Callback& c) {
    FILE* f = std::fopen(c.file.c_str(), "at");
    if (!f) throw CaseError("cannot write " + c.file);
    size_t per_pt = 0;
    for (int q : c.sample_q) per_pt += T->quantity_vector[q] ? 3 : 1;
    const size_t per_row = per_pt * c.sample_pts.size();
    const size_t rows = per_row ? c.sample_rows.size() / per_row : 0;
    for (size_t r = 0; r < rows; r++)
      for (size_t j = 0; j < c.sample_pts.size(); j++) {
        std::fprintf(f, "%lld,%g,%g,%g", c.sample_start + (long long)r, (double)c.sample_pts[j][0],
                     (double)c.sample_pts[j][1], (double)c.sample_pts[j][2]);
        for (size_t k = 0; k < per_pt; k++) std::fprintf(f, ",%g", c.sample_rows[r * per_row + j * per_pt + k]);
        std::fprintf(f, "\n");
      }
    std::fclose(f);
    c.sample_rows.clear();
    c.sample_start = iter;
  }
  // <SaveBinary> (src/Handlers/cbSaveBinary.cpp:5-33, Lattice::saveSolution
  // src/Lattice.cu.Rt:240-249): the .pri snapshot to <name>_0.pri, the name
  // fixed when the element is read. comp= saves only "parameter" densities
  // (design variables of adjoint runs, Solver::saveComp), which the plain
  // models do not have, so nothing is written, as in TCLB.
  // <SaveMemoryDump> (cbSaveMemoryDump.cpp) is the same without comp=: TCLB
  // reports comp= there as deprecated and saves the snapshot.
  void save_binary(const Callback& c) {
    if (c.kind == "SaveMemoryDump" && c.node->attr("comp"))
      std::fprintf(stderr, "[tclb_run] <SaveMemoryDump comp=> is deprecated; saving the whole snapshot\n");
    else if (const std::string* comp = c.node->attr("comp")) {
      if (verbose) std::printf("[tclb_run] SaveBinary: no component %s; not saved\n", comp->c_str());
      return;
    }
    std::vector<char> buf(tclb_pri_bytes(lat));
    ck(tclb_save_pri(lat, buf.data(), buf.size()), "save .pri");
    const std::string pri = c.file + "_0.pri";
    FILE* o = std::fopen(pri.c_str(), "wb");
    if (!o) throw CaseError("cannot write " + pri);
    const size_t w = std::fwrite(buf.data(), 1, buf.size(), o);
    std::fclose(o);
    if (w != buf.size()) throw CaseError("cannot write " + pri);
  }
  // <SaveCheckpoint> (src/Handlers/cbSaveCheckpoint.cpp:37-104): .pri plus a
  // restart case that loads it before <Solve>; keep = number retained.
  void save_checkpoint(const Callback& c) {
    char it[32];
    std::snprintf(it, sizeof(it), "_%08lld", iter);
    const std::string base = outpath + "_checkpoint" + it;
    std::vector<char> buf(tclb_pri_bytes(lat));
    ck(tclb_save_pri(lat, buf.data(), buf.size()), "save .pri");
    const std::string pri = base + "_0.pri";
    FILE* o = std::fopen(pri.c_str(), "wb");
    if (!o) throw CaseError("cannot write " + pri);
    std::fwrite(buf.data(), 1, buf.size(), o);
    std::fclose(o);
    // restart file (writeRestartFile, cbSaveCheckpoint.cpp:80-101): the case
    // with its <LoadBinary> pointed at this checkpoint, or a new one inserted
    // before the first <Solve>
    const std::string restart = outpath + "_restart" + it + ".xml";
    auto doc = XmlParser(config_text).parse();
    XmlNode* cfg = nullptr;
    for (auto& ch : doc->children)
      if (ch->name == "CLBConfig") cfg = ch.get();
    if (cfg) {
      XmlNode* lb = nullptr;
      for (auto& ch : cfg->children)
        if (ch->name == "LoadBinary") {
          lb = ch.get();
          break;
        }
      if (lb) {
        for (size_t i = 0; i < lb->attrs.size(); i++)
          if (lb->attrs[i].first == "file") {
            lb->attrs.erase(lb->attrs.begin() + i);
            break;
          }
        lb->attrs.emplace_back("file", base);
      } else {
        for (size_t i = 0; i < cfg->children.size(); i++)
          if (cfg->children[i]->name == "Solve") {
            auto n = std::make_unique<XmlNode>();
            n->name = "LoadBinary";
            n->attrs.emplace_back("file", base);
            n->parent = cfg;
            cfg->children.insert(cfg->children.begin() + i, std::move(n));
            break;
          }
      }
      std::ofstream rf(restart);
      rf << "<?xml version=\"1.0\"?>\n";
      write_xml(rf, cfg, 0);
    }
    // keep: "all" -> every checkpoint; n >= 0 -> the newest n (default 1)
    int keep = 1;
    if (const std::string* k = c.node->attr("keep")) {
      if (*k == "all") keep = 0;
      else {
        keep = parse_int(*k);
        if (keep < 0) {
          std::fprintf(stderr, "[tclb_run] SaveCheckpoint keep < 0: keeping 1\n");
          keep = 1;
        }
      }
    }
    if (keep == 0) return;
    checkpoints.push_back(base);
    restarts.push_back(restart);
    while ((int)checkpoints.size() > keep) {
      std::remove((checkpoints.front() + "_0.pri").c_str());
      std::remove(restarts.front().c_str());
      checkpoints.erase(checkpoints.begin());
      restarts.erase(restarts.begin());
    }
  }

  // Handler of a callback element; returns true when it registered (has Iterations)
  bool callback(const XmlNode* n) {
    Callback c = make_callback(n);
    if (c.every > 0) {
      hands.push_back(c);
      return true;
    }
    do_callback(c);  // no Iterations: runs once, now (GenericAction::ExecuteInternal)
    return false;
  }
  // the handler's Init: what it reads and prepares when the element is read
  Callback make_callback(const XmlNode* n) {
    need_lattice();
    Callback c;
    c.kind = n->name;
    c.node = n;
    c.start = (double)iter;
    if (const std::string* it = n->attr("Iterations")) c.every = parse_value(*it);
    if (c.kind == "Log") {
      c.file = iter_file(n->attr_or("name", "Log"), ".csv");
      log_header(c.file);
      iter_type |= TCLB_ITER_LASTGLOB;  // cbLog::Init
    }
    if (c.kind == "Stop") {  // cbStop::Init
      const char* suffix[4] = {"Change", "PercentChange", "Above", "Below"};
      for (int g = 0; g < T->nglobals; g++)
        for (int k = 0; k < 4; k++)
          if (const std::string* v = n->attr(std::string(T->global_names[g]) + suffix[k])) {
            char* end = nullptr;
            const double lim = std::strtod(v->c_str(), &end);
            if (end == v->c_str()) throw CaseError("<Stop>: cannot read " + *v);
            c.stop_global.push_back(g);
            c.stop_kind.push_back(k);
            c.stop_limit.push_back(lim);
            c.stop_old.push_back(STOP_UNSET);
          }
      if (c.stop_global.empty()) throw CaseError("<Stop> names no <Global>Change/PercentChange/Above/Below");
      if (const std::string* t = n->attr("Times")) {
        c.stop_times = std::atoi(t->c_str());
        if (c.stop_times < 1) throw CaseError("<Stop> Times must be at least 1");
      }
      iter_type |= TCLB_ITER_LASTGLOB;  // the Globals it checks
    }
    if (c.kind == "Sample") sample_init(c);
    if (c.kind == "PID") pid_init(c);
    if (c.kind == "Keep") keep_init(c);
    if (c.kind == "SaveBinary" || c.kind == "SaveMemoryDump") {  // cbSaveBinary::Init: the name is fixed here
      if (const std::string* f = n->attr("file")) c.file = outpath + "_" + *f;
      else if (const std::string* f = n->attr("filename")) c.file = *f;
      else c.file = iter_file("Save", "");
    }
    if (c.kind == "Failcheck") {  // cbFailcheck::Init: the checked region
      const char* k[6] = {"dx", "dy", "dz", "nx", "ny", "nz"};
      for (int a = 0; a < 6; a++)
        if (const std::string* v = n->attr(k[a])) c.fc_region[a] = (int)parse_value(*v);
    }
    return c;
  }
  // cbStop::DoIt: true when every criterion has held on Times consecutive checks
  bool stop_check(Callback& c) {
    std::vector<double> g(T->nglobals);
    tclb_get_globals(lat, g.data());
    bool miss = false;
    for (size_t i = 0; i < c.stop_global.size(); i++) {
      const double v = g[c.stop_global[i]], old = c.stop_old[i], lim = c.stop_limit[i];
      switch (c.stop_kind[i]) {
        case Callback::CHANGE: miss |= std::fabs(old - v) > lim; break;
        case Callback::PERCENT_CHANGE: miss |= std::fabs((old - v) / v) > lim; break;
        case Callback::ABOVE: miss |= v < lim; break;
        case Callback::BELOW: miss |= v > lim; break;
      }
      c.stop_old[i] = v;
    }
    c.stop_score = miss ? 0 : c.stop_score + 1;
    if (c.stop_score < c.stop_times) return false;
    std::fill(c.stop_old.begin(), c.stop_old.end(), STOP_UNSET);
    c.stop_score = 0;
    if (verbose) std::printf("[tclb_run] Stop at iteration %lld\n", iter);
    return true;
  }

  // returns true to stop the solve
  bool do_callback(Callback& c) {
    if (c.kind == "Stop") return stop_check(c);
    if (c.kind == "Sample") sample_write(c);
    if (c.kind == "PID") pid_step(c);
    if (c.kind == "Keep") keep_step(c);
    if (c.kind == "VTK") write_vtk(c);
    if (c.kind == "TXT") write_txt(c);
    if (c.kind == "Log") log_row(c.file);
    else if (c.kind == "BIN") write_bin(iter_file(c.node->attr_or("name", "BIN"), ""));
    else if (c.kind == "SaveCheckpoint") save_checkpoint(c);
    else if (c.kind == "SaveBinary" || c.kind == "SaveMemoryDump") save_binary(c);
    else if (c.kind == "Failcheck") {
      if (failcheck(c)) {
        std::printf("[tclb_run] Failcheck: NaN at iteration %lld, stopping\n", iter);
        return true;
      }
    }
    return false;
  }

  // acSolve::Init (src/Handlers/acSolve.cpp:5-43)
  void solve(const XmlNode* n) {
    need_lattice();
    Callback self;
    self.kind = "Solve";
    self.start = (double)iter;
    self.every = parse_value(n->attr_or("Iterations", "0"));
    if (self.every <= 0) throw CaseError("<Solve> needs Iterations > 0");
    const size_t stacked = hands.size();
    const int saved_type = iter_type;
    for (const auto& c : n->children) element(c.get());  // ExecuteInternal: actions now, callbacks stacked
    bool stop = false;
    do {
      const int my_next = self.next((double)iter);
      int next = my_next;
      for (const auto& h : hands) {
        const int it = h.next((double)iter);
        if (it > 0 && it < next) next = it;
      }
      bool sampling = false;  // <Sample> records every iteration
      for (const auto& h : hands) sampling = sampling || h.kind == "Sample";
      if (sampling) next = 1;
      int type = iter_type;
      if (next == my_next) type |= TCLB_ITER_LASTGLOB;
      ck(tclb_iterate(lat, next, type, nullptr), "iterate");
      if (sampling)
        for (auto& h : hands)
          if (h.kind == "Sample") sample_record(h);
      iter += next;
      for (auto& h : hands)
        if (h.now((double)iter) && do_callback(h)) stop = true;
      if (stop) break;
    } while (!self.now((double)iter));
    hands.resize(stacked);
    iter_type = saved_type;
    if (verbose) std::printf("[tclb_run] %lld iterations\n", iter);
  }

  void run(const XmlNode* cfg) {
    for (const auto& cp : cfg->children) element(cp.get());
  }
  // one element of <CLBConfig> or of a <Container> / <Repeat> (the handler
  // factory's dispatch, src/HandlerFactory.h, src/Handlers/GenericAction.cpp)
  void element(const XmlNode* n) {
    {
      if (n->name == "Container") {  // acContainer: the children, then unstack
        const size_t stacked = hands.size();
        for (const auto& c : n->children) element(c.get());
        hands.resize(stacked);
      } else if (n->name == "Repeat") {  // acRepeat: the children Times times; no unstack
        const std::string* t = n->attr("Times");
        if (!t) throw CaseError("<Repeat> needs Times");
        const int times = std::atoi(t->c_str());
        for (int i = 0; i < times; i++)
          for (const auto& c : n->children) element(c.get());
      } else if (n->name == "EvalIf") {
        // IfContainer (src/Handlers/IfContainer.cpp:5-39): the children when the
        // model option is present (opt_present) or absent (opt_missing). The
        // plain variants built here have every option of their model off
        // (conf.mk OPT=). TCLB's opt_missing branch reads the option name from
        // the absent opt_present attribute and always fails; here it does
        // what its name says.
        const std::string* pres = n->attr("opt_present");
        const std::string* miss = n->attr("opt_missing");
        if ((pres != nullptr) == (miss != nullptr))
          throw CaseError("<EvalIf> needs one of opt_present and opt_missing");
        const std::string opt = pres ? *pres : *miss;
        static const std::vector<std::string> options[3] = {{"bc", "autosym"}, {}, {"AVG", "IB", "SMAG"}};
        const auto& known = options[model];
        if (std::find(known.begin(), known.end(), opt) == known.end())
          throw CaseError("unknown option in <EvalIf>: " + opt);
        const bool active = false;
        if (active == (pres != nullptr))
          for (const auto& c : n->children) element(c.get());
      } else if (n->name == "Geometry") geometry(n);
      else if (n->name == "Model") {  // acModel: params, then Init
        for (const auto& c : n->children) {
          if (c->name == "Param") param(c.get());
          else throw CaseError("unsupported element <" + c->name + "> in <Model>");
        }
        init();
      } else if (n->name == "Param") param(n);
      else if (n->name == "Init") init();
      else if (n->name == "Solve") solve(n);
      else if (n->name == "Log" || n->name == "BIN" || n->name == "Failcheck" || n->name == "SaveCheckpoint" ||
               n->name == "Stop" || n->name == "VTK" || n->name == "TXT" || n->name == "SaveBinary" ||
               n->name == "Sample" || n->name == "SaveMemoryDump" || n->name == "PID" ||
               n->name == "Keep")
        callback(n);
      else if (n->name == "LoadBinary" || n->name == "LoadMemoryDump") load_binary(n);
      else if (n->name == "Units") {  // read before the run (read_units)
      } else if (n->name == "Average") {
        // cbAveraging (src/Handlers/cbAveraging.cpp:5-16) zeroes the densities a
        // model declares average=TRUE and restarts the averaging count. Only the
        // AVG option of d3q27_cumulant (models/flow/d3q27_cumulant/Dynamics.R:66-90)
        // declares any; the plain d2q9, d3q19 and d3q27_cumulant have none, so
        // there is nothing to reset.
      } else {
        throw CaseError("unsupported element <" + n->name + ">");
      }
    }
  }
};

std::string xml_escape(const std::string& v) {
  std::string o;
  for (char c : v) {
    if (c == '&') o += "&amp;";
    else if (c == '<') o += "&lt;";
    else if (c == '>') o += "&gt;";
    else if (c == '"') o += "&quot;";
    else o += c;
  }
  return o;
}

void write_xml(std::ostream& o, const XmlNode* n, int depth) {
  const std::string ind(depth, '\t');
  o << ind << "<" << n->name;
  for (const auto& a : n->attrs) o << " " << a.first << "=\"" << xml_escape(a.second) << "\"";
  if (n->children.empty()) {
    o << "/>\n";
    return;
  }
  o << ">\n";
  for (const auto& c : n->children) write_xml(o, c.get(), depth + 1);
  o << ind << "</" << n->name << ">\n";
}

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw CaseError("cannot read " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

void mkpath(const std::string& file) {
  for (size_t i = 1; i < file.size(); i++)
    if (file[i] == '/') mkdir(file.substr(0, i).c_str(), 0755);
}

}  // namespace
}  // namespace tclb

using namespace tclb;

extern "C" {

const char* tclb_case_last_error(void) { return g_case_err.c_str(); }

// Node types of the <Geometry> of a case text, rasterised as TCLB does
// (nx padded to a multiple of 32). dims receives (nx, ny, nz); flags may be
// NULL to query the size; capacity is its length in elements.
int tclb_case_geometry(const char* xml_text, int model, int dims[3], uint16_t* flags, size_t capacity) {
  try {
    const ModelTable* T = model_table(model);
    if (!T) throw CaseError("unknown model");
    auto doc = XmlParser(xml_text).parse();
    const XmlNode* cfg = doc->child("CLBConfig");
    read_units(cfg);
    const XmlNode* g = cfg ? cfg->child("Geometry") : doc->child("Geometry");
    if (!g) throw CaseError("no <Geometry> element");
    const int nx = pad_nx(parse_int(g->attr_or("nx", "1"))), ny = parse_int(g->attr_or("ny", "1")),
              nz = parse_int(g->attr_or("nz", "1"));
    dims[0] = nx; dims[1] = ny; dims[2] = nz;
    if (!flags) return TCLB_OK;
    if (capacity < (size_t)nx * ny * nz) throw CaseError("flag buffer too small");
    auto def = XmlParser(DEFAULT_ZONES).parse();
    Geometry geo(T, nx, ny, nz);
    geo.load(g, def->children[0].get());
    std::copy(geo.geom.begin(), geo.geom.end(), flags);
    return TCLB_OK;
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return TCLB_ERR_ARG;
  }
}

// Run a <CLBConfig> case file (the Run path of TCLB's main, src/main.cpp:173-425)
// for one model; outputs go to <output dir><case name>_<name>_P00_<iteration>.
// out_dir overrides the case's output attribute when not NULL.
int tclb_case_run(const char* xml_path, int model, int precision, int storage, const char* out_dir, int verbose) {
  try {
    Runner R;
    R.model = model;
    R.precision = precision;
    R.storage = storage;
    R.verbose = verbose != 0;
    R.T = model_table(model);
    if (!R.T) throw CaseError("unknown model");
    const std::string text = read_file(xml_path);
    R.config_text = text;
    auto doc = XmlParser(text).parse();
    const XmlNode* cfg = doc->child("CLBConfig");
    if (!cfg) throw CaseError("no <CLBConfig> element");
    read_units(cfg);
    std::string base = xml_path;
    const size_t sl = base.find_last_of('/');
    if (sl != std::string::npos) base = base.substr(sl + 1);
    const size_t dot = base.find_last_of('.');
    if (dot != std::string::npos) base = base.substr(0, dot);
    R.outdir = out_dir ? out_dir : cfg->attr_or("output", "output/");
    R.outpath = R.outdir + base;
    mkpath(R.outpath);
    R.run(cfg);
    return TCLB_OK;
  } catch (const std::exception& e) {
    g_case_err = e.what();
    return TCLB_ERR_ARG;
  }
}

}  // extern "C"
