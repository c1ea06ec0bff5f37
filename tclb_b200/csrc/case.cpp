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
// Values are numbers with an optional unit expression ("0.01", "1m/s",
// "5mm", "1e-3m2/s"); sums of terms ("1m+2mm") are added (UnitEnv::alt,
// src/unit.h:160-194). Without <Units> gauges every base unit has scale 1, so
// a value is its number times the factors of prefixed units.
double unit_factor(const std::string& u) {
  static const std::map<std::string, double> pref = {
      {"nm", 1e-9}, {"um", 1e-6}, {"mm", 1e-3}, {"cm", 1e-2}, {"km", 1e3}, {"h", 3600}, {"ns", 1e-9},
      {"us", 1e-6}, {"ms", 1e-3}, {"N", 1}, {"Pa", 1}, {"J", 1}, {"W", 1}, {"V", 1}, {"C", 1}};
  double f = 1.0;
  size_t i = 0;
  int sign = 1;
  while (i < u.size()) {
    if (u[i] == '/') { sign = -1; i++; continue; }
    size_t j = i;
    while (j < u.size() && isalpha((unsigned char)u[j])) j++;
    size_t k = j;
    while (k < u.size() && (isdigit((unsigned char)u[k]) || u[k] == '.')) k++;
    const std::string sym = u.substr(i, j - i);
    const double p = k > j ? std::atof(u.substr(j, k - j).c_str()) : 1.0;
    // longest known prefixed unit first, else base units (scale 1)
    size_t q = 0;
    double ff = 1.0;
    while (q < sym.size()) {
      if (q + 2 <= sym.size() && pref.count(sym.substr(q, 2))) { ff *= pref.at(sym.substr(q, 2)); q += 2; }
      else if (pref.count(sym.substr(q, 1))) { ff *= pref.at(sym.substr(q, 1)); q += 1; }
      else q += 1;
    }
    f *= std::pow(ff, sign * p);
    if (k == i) k++;
    i = k;
  }
  return f;
}

double parse_value(const std::string& s) {
  double ret = 0;
  size_t i = 0;
  while (i < s.size()) {
    size_t j = i + 1;
    while (j < s.size() && !((s[j] == '+' || s[j] == '-') && !(s[j - 1] == 'e' || s[j - 1] == 'E'))) j++;
    const std::string term = s.substr(i, j - i);
    char* end = nullptr;
    const double v = std::strtod(term.c_str(), &end);
    if (end == term.c_str()) throw CaseError("cannot read value '" + s + "'");
    ret += v * unit_factor(std::string(end));
    i = j;
  }
  return ret;
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
      } else if (n->name == "Wedge") {
        const std::string dir = n->attr_or("direction", "");
        for (int x = r.dx; x < r.dx + r.nx; x++)
          for (int y = r.dy; y < r.dy + r.ny; y++)
            for (int z = r.dz; z < r.dz + r.nz; z++)
              if (in_wedge((x - r.dx) / (r.nx - 1.), (y - r.dy) / (r.ny - 1.), (z - r.dz) / (r.nz - 1.), dir))
                dot(x, y, z);
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
      draw(n);
    }
  }
};

int pad_nx(int nx, int xsdim = 32) { return nx + xsdim - 1 - ((nx - 1) % xsdim); }

// ------------------------------------------------------------------ runner
struct Runner;
std::string read_file(const std::string& path);
void write_xml(std::ostream& o, const XmlNode* n, int depth);

struct Callback {
  std::string kind;  // Log, BIN, Failcheck
  const XmlNode* node;
  double every = 0, start = 0;
  std::string file;
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

  // Solver::initLog / writeLog (src/Solver.cpp.Rt:120-206); no <Units>: every scale is 1
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
    std::fprintf(o, "%lld, %.13le, %.13le, %d", iter, (double)iter, wall, 0);
    for (int i = 0; i < T->nsettings; i++) {
      double v = 0;
      tclb_get_setting(lat, i, &v);
      std::fprintf(o, ", %.13le, %.13le", v, v);
    }
    for (int i = 0; i < T->nzonesettings; i++)
      for (const auto& z : geo->zones) {
        double v = 0;
        tclb_get_zone_setting(lat, i, z.second, &v);
        std::fprintf(o, ", %.13le, %.13le", v, v);
      }
    std::vector<double> g(T->nglobals);
    tclb_get_globals(lat, g.data());
    for (double v : g) std::fprintf(o, ", %.13le, %.13le", v, v);
    for (int i = 0; i < 3; i++) std::fprintf(o, ", %.13le", 1.0);
    std::fprintf(o, "\n");
    std::fclose(o);
  }
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
  bool failcheck() {
    int nx, ny, nz;
    tclb_get_size(lat, &nx, &ny, &nz);
    const size_t N = (size_t)nx * ny * nz;
    for (int q = 0; q < T->nquantities; q++) {
      const int comp = T->quantity_vector[q] ? 3 : 1;
      if (precision == TCLB_FP64) {
        std::vector<double> b(N * comp);
        ck(tclb_get_quantity(lat, q, nullptr, b.data(), 1.0, nullptr), "quantity");
        for (double v : b)
          if (!std::isfinite(v)) return true;
      } else {
        std::vector<float> b(N * comp);
        ck(tclb_get_quantity(lat, q, nullptr, b.data(), 1.0, nullptr), "quantity");
        for (float v : b)
          if (!std::isfinite(v)) return true;
      }
    }
    return false;
  }

  // <LoadBinary file=> (src/Handlers/acLoadBinary.cpp): Lattice::loadSolution
  // reads <file>_0.pri (rank 0) into the current snapshot.
  void load_binary(const XmlNode* n) {
    need_lattice();
    const std::string* f = n->attr("file");
    if (!f) f = n->attr("filename");
    if (!f) throw CaseError("<LoadBinary> needs a file attribute");
    if (n->attr("comp")) throw CaseError("<LoadBinary comp=> (single fields) is not supported");
    const std::string fn = *f + "_0.pri";
    const std::string data = read_file(fn);
    if (data.size() != tclb_pri_bytes(lat)) throw CaseError(fn + " does not match this lattice");
    ck(tclb_load_pri(lat, data.data(), data.size()), "load .pri");
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
    if (c.every > 0) {
      hands.push_back(c);
      return true;
    }
    do_callback(c);  // no Iterations: runs once, now (GenericAction::ExecuteInternal)
    return false;
  }
  // returns true to stop the solve
  bool do_callback(const Callback& c) {
    if (c.kind == "Log") log_row(c.file);
    else if (c.kind == "BIN") write_bin(iter_file(c.node->attr_or("name", "BIN"), ""));
    else if (c.kind == "SaveCheckpoint") save_checkpoint(c);
    else if (c.kind == "Failcheck") {
      if (failcheck()) {
        std::printf("[tclb_run] Failcheck: non-finite values at iteration %lld, stopping\n", iter);
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
    for (const auto& c : n->children) callback(c.get());
    bool stop = false;
    do {
      const int my_next = self.next((double)iter);
      int next = my_next;
      for (const auto& h : hands) {
        const int it = h.next((double)iter);
        if (it > 0 && it < next) next = it;
      }
      int type = iter_type;
      if (next == my_next) type |= TCLB_ITER_LASTGLOB;
      ck(tclb_iterate(lat, next, type, nullptr), "iterate");
      iter += next;
      for (const auto& h : hands)
        if (h.now((double)iter) && do_callback(h)) stop = true;
      if (stop) break;
    } while (!self.now((double)iter));
    hands.resize(stacked);
    iter_type = saved_type;
    if (verbose) std::printf("[tclb_run] %lld iterations\n", iter);
  }

  void run(const XmlNode* cfg) {
    for (const auto& cp : cfg->children) {
      const XmlNode* n = cp.get();
      if (n->name == "Geometry") geometry(n);
      else if (n->name == "Model") {  // acModel: params, then Init
        for (const auto& c : n->children) {
          if (c->name == "Param") param(c.get());
          else throw CaseError("unsupported element <" + c->name + "> in <Model>");
        }
        init();
      } else if (n->name == "Param") param(n);
      else if (n->name == "Init") init();
      else if (n->name == "Solve") solve(n);
      else if (n->name == "Log" || n->name == "BIN" || n->name == "Failcheck" || n->name == "SaveCheckpoint")
        callback(n);
      else if (n->name == "LoadBinary") load_binary(n);
      else if (n->name == "Units") {
        if (!n->children.empty()) throw CaseError("<Units> gauges are not supported: give values in lattice units");
      } else if (n->name == "VTK" || n->name == "TXT" || n->name == "Stop" || n->name == "Average") {
        if (verbose) std::printf("[tclb_run] <%s> is not supported; skipped\n", n->name.c_str());
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
