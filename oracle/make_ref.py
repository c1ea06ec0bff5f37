"""Build oracle/_ref: TCLB's own per-node model code, compiled for the CPU.

TEST INFRASTRUCTURE ONLY. The library this script builds is a second checker
beside the restated oracle; the product library never loads it, and nothing
it writes is committed (oracle/_ref/ is git-ignored).

TCLB's model sources are R templates (`.c.Rt`) that its build expands with R
and polyAlgebra, which this machine does not have. Several of the regions that
matter, however, are literal C with only a handful of small R blocks:

* models/flow/d3q27_cumulant/Dynamics.c.Rt -- `getRho` / `getU_` (:23-45) and
  the whole cumulant collision `CollisionMRT` (:309-519). Its R blocks are the
  `real_t c...` declarations, the third-order `(1-Omega)` scaling and the
  zeroing above third order, each a loop over the cumulant names `cABC`
  selected by the digit sum A+B+C (Dynamics.R:2 `P = expand.grid(...)`), plus
  the density sums `C(sum(f))` and `C(u, f %*% U)`.
* models/flow/d3q19/Dynamics.c.Rt -- the Zou-He closures `WVelocity`,
  `WPressure`, `WPressureLimited`, `EPressure` and their `Inlet` template
  (:86-179): literal C apart from sums of densities selected by direction
  (`sum(f[X == 0 & Y > 0])`) and the index renumbering `I[]` (:92-94).
* models/flow/d2q9_SRT/Dynamics.c -- plain C: equilibrium, BGK collision,
  bounce-back and the four Zou-He closures (:34-176).

This script reads those files where they lie, expands exactly those R
constructs (from the direction tables it parses out of the same tree: the
`expand.grid` of d3q27_cumulant/Dynamics.R and `d3q19_MRTMAT` of
src/lib/d3q19.R), refuses any R block it does not recognise, wraps the result
in a small C++ harness and compiles it twice: with `real_t = double` and with
`real_t = float` after TCLB's single-precision literal rewrite
(src/makefile.main.Rt:294-296). The expanded sums list their terms in density
order; polyAlgebra's own term order and literal spelling are not known here,
so results may differ from a TCLB build in the last bits (tests compare with
rounding-level tolerances).

    python oracle/make_ref.py [--reference DIR] [--force]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libtclb_ref.so")
GEN = os.path.join(OUT, "tclb_ref_gen.cpp")
DEFAULT_REF = os.environ.get("TCLB_REFERENCE", "/root/reference")

SOURCES = {
    "d3q27c": "models/flow/d3q27_cumulant/Dynamics.c.Rt",
    "d3q27c_R": "models/flow/d3q27_cumulant/Dynamics.R",
    "d3q19": "models/flow/d3q19/Dynamics.c.Rt",
    "d3q19_lib": "src/lib/d3q19.R",
    "d2q9srt": "models/flow/d2q9_SRT/Dynamics.c",
    "makefile": "src/makefile.main.Rt",
}


class TemplateError(RuntimeError):
    pass


# ---------------------------------------------------------------------------
# Template text -> segments
# ---------------------------------------------------------------------------
def segments(text: str):
    """Split template text into ('c', text) and ('r', code) / ('fmt', fmt, expr) pieces."""
    out, pos = [], 0
    for m in re.finditer(r"<\?(R|%[sd])(.*?)\?>", text, re.S):
        if m.start() > pos:
            out.append(("c", text[pos:m.start()]))
        if m.group(1) == "R":
            out.append(("r", m.group(2).strip()))
        else:
            out.append(("fmt", m.group(1), m.group(2).strip()))
        pos = m.end()
    if pos < len(text):
        out.append(("c", text[pos:]))
    return out


def extract_function(text: str, name: str, ret: str = r"[A-Za-z_0-9]+") -> str:
    """The template text of `CudaDeviceFunction <ret> name(...) { ... }`, braces matched outside R blocks."""
    m = re.search(r"CudaDeviceFunction\s+" + ret + r"\s+" + re.escape(name) + r"\s*\([^)]*\)\s*\{", text)
    if not m:
        raise TemplateError(f"function {name} not found")
    start, i, depth = m.start(), m.end(), 1
    while depth:
        if text.startswith("<?", i):
            j = text.find("?>", i)
            if j < 0:
                raise TemplateError("unterminated template block")
            i = j + 2
            continue
        if i >= len(text):
            raise TemplateError(f"unbalanced braces in {name}")
        ch = text[i]
        depth += ch == "{"
        depth -= ch == "}"
        i += 1
    return text[start:i]


# ---------------------------------------------------------------------------
# A tiny evaluator for the R expressions these regions use
# ---------------------------------------------------------------------------
class Model:
    """Density names and directions of one model, and the R environment of its template."""

    def __init__(self, names, dirs):
        self.names = list(names)
        self.dirs = [tuple(d) for d in dirs]
        self.env = {}
        self.templates = {}

    def sel(self, cond: str):
        """Indices of the densities meeting an R condition like `X == 0 & Y > 0` (X, Y, Z: directions)."""
        idx = list(range(len(self.names)))
        for part in cond.split("&"):
            m = re.fullmatch(r"\s*([XYZ])\s*(==|<|>|<=|>=|!=)\s*(-?\d+)\s*", part)
            if not m:
                raise TemplateError(f"unsupported density selection: {cond!r}")
            ax, op, v = "XYZ".index(m.group(1)), m.group(2), int(m.group(3))
            ok = {"==": lambda a: a == v, "<": lambda a: a < v, ">": lambda a: a > v,
                  "<=": lambda a: a <= v, ">=": lambda a: a >= v, "!=": lambda a: a != v}[op]
            idx = [i for i in idx if ok(self.dirs[i][ax])]
        return idx

    def expr(self, e: str) -> str:
        """C text of a sum/difference of `sum(f)`, `sum(f[cond])`, `k * name` and names."""
        e = e.strip()
        terms, depth, cur, sign = [], 0, "", "+"
        for ch in e:
            if ch in "([":
                depth += 1
            elif ch in ")]":
                depth -= 1
            if depth == 0 and ch in "+-" and cur.strip():
                terms.append((sign, cur.strip()))
                sign, cur = ch, ""
                continue
            if depth == 0 and ch in "+-" and not cur.strip():
                sign = "-" if (sign == "-") != (ch == "-") else "+"
                continue
            cur += ch
        terms.append((sign, cur.strip()))
        out = []
        for s, t in terms:
            if t == "sum(f)":
                c = "(" + " + ".join(self.names) + ")"
            elif (m := re.fullmatch(r"sum\(f\[(.*)\]\)", t)):
                ii = self.sel(m.group(1))
                c = "(" + " + ".join(self.names[i] for i in ii) + ")" if ii else "0"
            elif (m := re.fullmatch(r"(\d+)\s*\*\s*([A-Za-z_][A-Za-z_0-9.]*)", t)):
                c = m.group(1) + "*" + self.symbol(m.group(2))
            elif re.fullmatch(r"[A-Za-z_][A-Za-z_0-9.]*", t):
                c = self.symbol(t)
            else:
                raise TemplateError(f"unsupported R expression term: {t!r}")
            out.append(("- " if s == "-" else "+ ") + c)
        txt = " ".join(out)
        return txt[2:] if txt.startswith("+ ") else txt

    def symbol(self, name: str) -> str:
        v = self.env.get(name)
        if isinstance(v, str):
            return v
        if v is None:
            raise TemplateError(f"unknown R symbol {name!r}")
        raise TemplateError(f"R symbol {name!r} is not a scalar")

    def velocity_sums(self, lhs):
        """`C(PV(c("u.x","u.y","u.z")), f %*% U)`: u.d = sum_i f_i * e_i,d."""
        lines = []
        for d, name in enumerate(lhs):
            plus = [self.names[i] for i in range(len(self.names)) if self.dirs[i][d] == 1]
            minus = [self.names[i] for i in range(len(self.names)) if self.dirs[i][d] == -1]
            rhs = " + ".join(plus) + "".join(" - " + m for m in minus)
            lines.append(f"{name} = {rhs};")
        return "\n".join(lines) + "\n"

    # -- statements -----------------------------------------------------------
    def run(self, code: str) -> str:
        """Run one `<?R ... ?>` block of statements; return the C text it emits."""
        out = []
        for st in split_statements(code):
            out.append(self.statement(st))
        return "".join(out)

    def statement(self, st: str) -> str:
        st = st.strip()
        if not st or st.startswith("#"):
            return ""
        if (m := re.fullmatch(r"([A-Za-z_][A-Za-z_0-9.]*)\s*=\s*PV\(\s*\"([^\"]+)\"\s*\)", st)):
            self.env[m.group(1)] = m.group(2)
            return ""
        if re.fullmatch(r"cumulants\s*=\s*paste\(\s*\"c\"\s*,\s*P\$x\s*,\s*P\$y\s*,\s*P\$z\s*,\s*sep\s*=\s*\"\"\s*\)", st):
            self.env["cumulants"] = ["c" + n[1:] for n in self.names]
            return ""
        if (m := re.fullmatch(r"sel\s*=\s*rowSums\(P\)\s*(==|>)\s*(\d+)", st)):
            k = int(m.group(2))
            digits = [sum(int(ch) for ch in n[1:]) for n in self.names]
            self.env["sel"] = [d == k if m.group(1) == "==" else d > k for d in digits]
            return ""
        if (m := re.fullmatch(r"([XYZ])\s*=\s*U\[\s*,\s*([123])\s*\]", st)):
            return ""  # directions are known from the model tables
        if (m := re.fullmatch(r"renum\s*=\s*c\(([-\d,\s]+)\)", st)):
            self.env["renum"] = [int(x) for x in m.group(1).split(",")]
            return ""
        if (m := re.fullmatch(r"I\s*=\s*rep\(\s*0\s*,\s*(\d+)\s*\)", st)):
            self.env["I"] = [0] * int(m.group(1))
            return ""
        if re.fullmatch(r"I\[renum\]\s*=\s*1:(\d+)", st):
            I = self.env["I"]
            for k, r in enumerate(self.env["renum"]):
                I[r - 1] = k + 1
            return ""
        if (m := re.fullmatch(r"C\((.*)\)", st, re.S)):
            args = split_args(m.group(1))
            args = [a for a in args if not re.fullmatch(r"float\s*=\s*F", a)]
            if len(args) == 1:
                return self.expr(args[0])
            if len(args) == 2:
                lhs = args[0]
                if (mv := re.fullmatch(r"PV\(c\(([^)]*)\)\)", lhs)) and args[1].replace(" ", "") == "f%*%U":
                    names = [x.strip().strip('"') for x in mv.group(1).split(",")]
                    return self.velocity_sums(names)
                return f"{self.symbol(lhs)} = {self.expr(args[1])};\n"
            raise TemplateError(f"unsupported C() call: {st!r}")
        raise TemplateError(f"unsupported R statement: {st!r}")

    def fmt(self, kind: str, e: str, loopvar=None) -> str:
        if kind == "%s" and loopvar is not None and e == "i":
            return loopvar
        if kind == "%d" and (m := re.fullmatch(r"(-?\d+)\s*\+\s*I\[\s*(\d+)\s*\]", e)):
            return str(int(m.group(1)) + self.env["I"][int(m.group(2)) - 1])
        raise TemplateError(f"unsupported inline expression <?{kind} {e} ?>")


def split_statements(code: str):
    out, depth, cur = [], 0, ""
    for ch in code:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if depth == 0 and ch in ";\n":
            out.append(cur)
            cur = ""
            continue
        cur += ch
    out.append(cur)
    return [s for s in out if s.strip()]


def split_args(s: str):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if depth == 0 and ch == ",":
            out.append(cur.strip())
            cur = ""
            continue
        cur += ch
    out.append(cur.strip())
    return out


def expand(model: Model, text: str) -> str:
    """Expand a template region: loops over vectors, template functions and statement blocks."""
    segs = segments(text)
    out, k = [], 0

    def body_until_close(k0):
        """Segments from k0 to the matching `<?R } ?>`, and the index after it."""
        depth, j = 1, k0
        while j < len(segs):
            s = segs[j]
            if s[0] == "r":
                if s[1].rstrip().endswith("{"):
                    depth += 1
                elif s[1].strip() == "}":
                    depth -= 1
                    if depth == 0:
                        return segs[k0:j], j + 1
            j += 1
        raise TemplateError("unclosed R block")

    def render(seglist, loopvar=None):
        res = []
        for s in seglist:
            if s[0] == "c":
                res.append(s[1])
            elif s[0] == "fmt":
                res.append(model.fmt(s[1], s[2], loopvar))
            else:
                raise TemplateError(f"nested R block not supported: {s[1]!r}")
        return "".join(res)

    while k < len(segs):
        s = segs[k]
        if s[0] == "c":
            out.append(s[1])
            k += 1
            continue
        if s[0] == "fmt":
            out.append(model.fmt(s[1], s[2]))
            k += 1
            continue
        code = s[1]
        if (m := re.fullmatch(r"(.*?)for\s*\(\s*i\s+in\s+([A-Za-z_.]+)(\[sel\])?\s*\)\s*\{", code, re.S)):
            model.run(m.group(1))
            vec = model.env[m.group(2)]
            if m.group(3):
                vec = [v for v, ok in zip(vec, model.env["sel"]) if ok]
            body, k = body_until_close(k + 1)
            for v in vec:
                out.append(render(body, v))
            continue
        if (m := re.fullmatch(r"([A-Za-z_][A-Za-z_0-9]*)\s*=\s*function\(\s*\)\s*\{", code)):
            body, k = body_until_close(k + 1)
            model.templates[m.group(1)] = body
            continue
        if (m := re.fullmatch(r"([A-Za-z_][A-Za-z_0-9]*)\(\s*\)\s*;?", code)) and m.group(1) in model.templates:
            out.append(expand_segments(model, model.templates[m.group(1)]))
            k += 1
            continue
        out.append(model.run(code))
        k += 1
    return "".join(out)


def expand_segments(model: Model, segs) -> str:
    res = []
    for s in segs:
        if s[0] == "c":
            res.append(s[1])
        elif s[0] == "fmt":
            res.append(model.fmt(s[1], s[2]))
        else:
            res.append(model.run(s[1]))
    return "".join(res)


# ---------------------------------------------------------------------------
# Per-model sources
# ---------------------------------------------------------------------------
def read(ref: str, key: str) -> str:
    with open(os.path.join(ref, SOURCES[key])) as fh:
        return fh.read()


def d3q27c_model(ref: str) -> Model:
    """Names f<a><b><c> over expand.grid(x=0:2, y=0:2, z=0:2) and directions over x = c(0,1,-1) (Dynamics.R:1-3)."""
    txt = read(ref, "d3q27c_R")
    if not re.search(r"x\s*=\s*c\(\s*0\s*,\s*1\s*,\s*-1\s*\)", txt) or "P = expand.grid(x=0:2,y=0:2,z=0:2)" not in txt:
        raise TemplateError("d3q27_cumulant/Dynamics.R: unexpected direction definition")
    val = {0: 0, 1: 1, 2: -1}
    names, dirs = [], []
    for c in range(3):
        for b in range(3):
            for a in range(3):
                names.append(f"f{a}{b}{c}")
                dirs.append((val[a], val[b], val[c]))
    return Model(names, dirs)


def d3q19_model(ref: str) -> Model:
    """f0..f18 with directions from columns 4, 6, 8 of d3q19_MRTMAT (src/lib/d3q19.R:1-20, :42)."""
    txt = read(ref, "d3q19_lib")
    m = re.search(r"d3q19_MRTMAT\s*=\s*matrix\(c\((.*?)\)\s*,\s*19\s*,\s*19\s*\)", txt, re.S)
    if not m or "U = MRTMAT[,c(4,6,8)]" not in txt:
        raise TemplateError("src/lib/d3q19.R: MRT matrix not found")
    nums = [int(x) for x in m.group(1).replace("\n", " ").split(",")]
    if len(nums) != 361:
        raise TemplateError("src/lib/d3q19.R: MRT matrix is not 19x19")
    col = lambda j: nums[19 * (j - 1): 19 * j]  # R fills matrix() column by column
    dirs = list(zip(col(4), col(6), col(8)))
    return Model([f"f{i}" for i in range(19)], dirs)


def sp_rewrite(text: str, makefile: str) -> str:
    """TCLB's `%_sp.c` rule: literals with an f/L suffix become float literals (makefile.main.Rt:294-296)."""
    if "s/([^a-zA-Z0-9][0-9]+\\.[0-9]*([eE][-+]?[0-9]+)?)[fL]+/\\1f/g" not in makefile:
        raise TemplateError("src/makefile.main.Rt: single-precision rewrite rule not found")
    return re.sub(r"([^a-zA-Z0-9][0-9]+\.[0-9]*([eE][-+]?[0-9]+)?)[fL]+", r"\1f", text)


def generate(ref: str) -> str:
    d27 = read(ref, "d3q27c")
    m27 = d3q27c_model(ref)
    parts27 = [expand(m27, extract_function(d27, n)) for n in ("getRho", "getU_", "CollisionMRT")]

    d19 = read(ref, "d3q19")
    m19 = d3q19_model(ref)
    # the template head binds rho to the symbol "rho": Flow = d3q19_MRT("rho", ...), rho = Flow$rho (:11-16),
    # and d3q19_MRT turns a character rho into PV(rho) (src/lib/d3q19.R)
    if not (re.search(r'Flow\s*=\s*d3q19_MRT\(\s*"rho"', d19) and re.search(r"rho\s*=\s*Flow\$rho", d19)):
        raise TemplateError("d3q19/Dynamics.c.Rt: unexpected template head")
    m19.env["rho"] = "rho"
    # the block defining X, Y, Z, renum and I, and the Inlet template (:86-108)
    i0 = d19.rindex("<?R", 0, d19.index("renum = c("))
    i1 = d19.index("CudaDeviceFunction void WVelocity()")
    expand(m19, d19[i0:i1])
    parts19 = [expand(m19, extract_function(d19, n)) for n in ("WVelocity", "WPressure", "WPressureLimited", "EPressure")]

    d9 = read(ref, "d2q9srt")
    if "<?" in d9:
        raise TemplateError("d2q9_SRT/Dynamics.c is expected to be plain C")
    parts9 = [extract_function(d9, n) for n in ("CollisionBGK", "BounceBack", "getRho", "getU", "SetEquilibrium",
                                                 "EVelocity", "WPressure", "WVelocity", "EPressure")]
    for p in parts27 + parts19 + parts9:
        if "<?" in p:
            raise TemplateError("unexpanded template block left in generated code")

    mk = read(ref, "makefile")
    body = {}
    for prec in ("64", "32"):
        conv = (lambda t: t) if prec == "64" else (lambda t: sp_rewrite(t, mk))
        body[prec] = (
            "struct D3Q27C {\n" + D3Q27C_HEAD + "\n".join(conv(p) for p in parts27) + "\n};\n"
            "struct D3Q19 {\n" + D3Q19_HEAD + "\n".join(conv(p) for p in parts19) + "\n};\n"
            "struct D2Q9SRT {\n" + D2Q9_HEAD + "\n".join(conv(p) for p in parts9) + "\n};\n"
        )
    return (HEADER + "namespace ref64 {\ntypedef double real_t;\n" + COMMON + body["64"] + "}\n"
            "namespace ref32 {\ntypedef float real_t;\n" + COMMON + body["32"] + "}\n" + HARNESS)


HEADER = """// Generated by oracle/make_ref.py from TCLB's model sources. Test infrastructure only; not committed.
#include <cmath>
#include <cstddef>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif
#define CudaDeviceFunction
using std::sqrt;
"""

COMMON = """struct vector_t { real_t x, y, z; };
struct float2 { float x, y; };
"""

# Node-type values of the plain d3q27_cumulant and d3q19 builds (TCLB's conf.R packing).
D3Q27C_HEAD = """
  static const int NODE_BOUNDARY = 0x0078, NODE_Wall = 0x0050;
  real_t f000, f100, f200, f010, f110, f210, f020, f120, f220,
         f001, f101, f201, f011, f111, f211, f021, f121, f221,
         f002, f102, f202, f012, f112, f212, f022, f122, f222;
  real_t nu, nubuffer, GalileanCorrection, ForceX, ForceY, ForceZ, Omega;
  int NodeType;
  real_t G[6];  // Density, Flux, Mass, XMomentum, YMomentum, ZMomentum
  void AddToDensity(real_t v) { G[0] += v; }
  void AddToFlux(real_t v) { G[1] += v; }
  void AddToMass(real_t v) { G[2] += v; }
  void AddToXMomentum(real_t v) { G[3] += v; }
  void AddToYMomentum(real_t v) { G[4] += v; }
  void AddToZMomentum(real_t v) { G[5] += v; }
  real_t* fp(int i) {
    real_t* t[27] = {&f000, &f100, &f200, &f010, &f110, &f210, &f020, &f120, &f220,
                     &f001, &f101, &f201, &f011, &f111, &f211, &f021, &f121, &f221,
                     &f002, &f102, &f202, &f012, &f112, &f212, &f022, &f122, &f222};
    return t[i];
  }
"""

D3Q19_HEAD = """
  real_t f0, f1, f2, f3, f4, f5, f6, f7, f8, f9, f10, f11, f12, f13, f14, f15, f16, f17, f18;
  real_t InletVelocity, InletDensity;
  real_t* fp(int i) {
    real_t* t[19] = {&f0, &f1, &f2, &f3, &f4, &f5, &f6, &f7, &f8, &f9, &f10, &f11, &f12, &f13, &f14, &f15, &f16, &f17, &f18};
    return t[i];
  }
"""

D2Q9_HEAD = """
  real_t f[9];
  real_t omega, Velocity_x, Velocity_y, Density, GravitationX, GravitationY;
"""

HARNESS = r"""
namespace {
template <class R>
void d3q27c_collide(int n, double* f, const double* s, const int* boundary, double* glob) {
  for (int k = 0; k < n; k++) {
    R m;
    for (int i = 0; i < 27; i++) *m.fp(i) = f[27 * k + i];
    m.nu = s[0]; m.nubuffer = s[1]; m.GalileanCorrection = s[2];
    m.ForceX = s[3]; m.ForceY = s[4]; m.ForceZ = s[5]; m.Omega = s[6];
    m.NodeType = boundary[k] ? 0x0008 : 0;
    for (int g = 0; g < 6; g++) m.G[g] = 0;
    m.CollisionMRT();
    for (int i = 0; i < 27; i++) f[27 * k + i] = *m.fp(i);
    if (glob) for (int g = 0; g < 6; g++) glob[6 * k + g] = m.G[g];
  }
}
template <class R>
void d3q27c_rho_u(int n, const double* f, const double* s, double* out) {
  for (int k = 0; k < n; k++) {
    R m;
    for (int i = 0; i < 27; i++) *m.fp(i) = f[27 * k + i];
    m.ForceX = s[3]; m.ForceY = s[4]; m.ForceZ = s[5];
    m.NodeType = 0;
    auto u = m.getU_();
    out[4 * k] = m.getRho(); out[4 * k + 1] = u.x; out[4 * k + 2] = u.y; out[4 * k + 3] = u.z;
  }
}
template <class R>
void d3q19_boundary(int kind, int n, double* f, const double* s) {
  for (int k = 0; k < n; k++) {
    R m;
    for (int i = 0; i < 19; i++) *m.fp(i) = f[19 * k + i];
    m.InletVelocity = s[0]; m.InletDensity = s[1];
    switch (kind) {
      case 0: m.WVelocity(); break;
      case 1: m.WPressure(); break;
      case 2: m.WPressureLimited(); break;
      case 3: m.EPressure(); break;
    }
    for (int i = 0; i < 19; i++) f[19 * k + i] = *m.fp(i);
  }
}
template <class R, class real_t>
void d2q9srt(int op, int n, double* f, const double* s) {
  for (int k = 0; k < n; k++) {
    R m;
    for (int i = 0; i < 9; i++) m.f[i] = f[9 * k + i];
    m.omega = s[0]; m.Velocity_x = s[1]; m.Velocity_y = s[2]; m.Density = s[3];
    m.GravitationX = s[4]; m.GravitationY = s[5];
    switch (op) {
      case 0: m.CollisionBGK(); break;
      case 1: m.BounceBack(); break;
      case 2: m.EVelocity(); break;
      case 3: m.WPressure(); break;
      case 4: m.WVelocity(); break;
      case 5: m.EPressure(); break;
      case 6: {  // equilibrium at (rho, ux, uy) = f[0..2] of the input
        decltype(m.getU()) u; u.x = m.f[1]; u.y = m.f[2]; u.z = 0;
        real_t d = m.f[0];
        m.SetEquilibrium(m.f, d, u);
        break;
      }
      case 7: {  // getRho, getU -> f[0..2]
        real_t d = m.getRho(); auto u = m.getU();
        m.f[0] = d; m.f[1] = u.x; m.f[2] = u.y;
        break;
      }
    }
    for (int i = 0; i < 9; i++) f[9 * k + i] = m.f[i];
  }
}
// One iteration of a periodic lattice of all-MRT, untyped-boundary nodes: node
// x takes f_i from x - e_i (index i = a + 3b + 9c over digits 0, +1, -1), then
// TCLB's CollisionMRT. The loop is this harness's; the node code is TCLB's.
template <class R, class real>
void d3q27c_iterate(int nx, int ny, int nz, const real* src, real* dst, const double* s) {
  const size_t N = (size_t)nx * ny * nz;
  static const int dg[3] = {0, 1, -1};
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++) {
      const real* row[27];  // the source row of each population (y and z wrapped once per row)
      int ex[27];
      for (int i = 0; i < 27; i++) {
        const int ey = dg[(i / 3) % 3], ez = dg[i / 9];
        const int ys = (y - ey + ny) % ny, zs = (z - ez + nz) % nz;
        row[i] = src + (size_t)i * N + (size_t)nx * (ys + (size_t)ny * zs);
        ex[i] = dg[i % 3];
      }
      for (int x = 0; x < nx; x++) {
        R m;
        for (int i = 0; i < 27; i++) {
          int xs = x - ex[i];
          xs = xs < 0 ? xs + nx : (xs >= nx ? xs - nx : xs);
          *m.fp(i) = row[i][xs];
        }
        m.nu = s[0]; m.nubuffer = s[1]; m.GalileanCorrection = s[2];
        m.ForceX = s[3]; m.ForceY = s[4]; m.ForceZ = s[5]; m.Omega = s[6];
        m.NodeType = 0;
        for (int g = 0; g < 6; g++) m.G[g] = 0;
        m.CollisionMRT();
        const size_t n = x + (size_t)nx * (y + (size_t)ny * z);
        for (int i = 0; i < 27; i++) dst[(size_t)i * N + n] = *m.fp(i);
      }
    }
}
}  // namespace

extern "C" {
int ref_version() { return 2; }
int ref_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  return 1;
#endif
}
int ref_d3q27c_iterate(int fp64, int nx, int ny, int nz, const void* src, void* dst, const double* s) {
  if (fp64) d3q27c_iterate<ref64::D3Q27C, double>(nx, ny, nz, (const double*)src, (double*)dst, s);
  else d3q27c_iterate<ref32::D3Q27C, float>(nx, ny, nz, (const float*)src, (float*)dst, s);
  return 0;
}
int ref_d3q27c_collide(int fp64, int n, double* f, const double* s, const int* boundary, double* glob) {
  if (fp64) d3q27c_collide<ref64::D3Q27C>(n, f, s, boundary, glob); else d3q27c_collide<ref32::D3Q27C>(n, f, s, boundary, glob);
  return 0;
}
int ref_d3q27c_rho_u(int fp64, int n, const double* f, const double* s, double* out) {
  if (fp64) d3q27c_rho_u<ref64::D3Q27C>(n, f, s, out); else d3q27c_rho_u<ref32::D3Q27C>(n, f, s, out);
  return 0;
}
int ref_d3q19_boundary(int fp64, int kind, int n, double* f, const double* s) {
  if (kind < 0 || kind > 3) return -1;
  if (fp64) d3q19_boundary<ref64::D3Q19>(kind, n, f, s); else d3q19_boundary<ref32::D3Q19>(kind, n, f, s);
  return 0;
}
int ref_d2q9srt(int fp64, int op, int n, double* f, const double* s) {
  if (op < 0 || op > 7) return -1;
  if (fp64) d2q9srt<ref64::D2Q9SRT, double>(op, n, f, s); else d2q9srt<ref32::D2Q9SRT, float>(op, n, f, s);
  return 0;
}
}
"""


def build(ref: str = DEFAULT_REF, force: bool = False, verbose: bool = False) -> str:
    """Generate and compile oracle/_ref/libtclb_ref.so from the TCLB tree at `ref`."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(__file__):
        return LIB
    if not os.path.isdir(ref):
        raise FileNotFoundError(f"TCLB source tree not found at {ref}")
    os.makedirs(OUT, exist_ok=True)
    src = generate(ref)
    with open(GEN, "w") as fh:
        fh.write(src)
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-Wno-narrowing", "-w",
           "-o", LIB, GEN]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--reference", default=DEFAULT_REF)
    p.add_argument("--force", action="store_true")
    a = p.parse_args(argv)
    print(build(a.reference, a.force, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
