// Kernel generation for the Local, Focal, Zonal, Radiating and Spreading
// skeletons (see codegen.hpp); the scan skeletons run through codegen_scan.cpp.
#include "codegen.hpp"
#include "rewrite.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <sstream>

namespace mapb {


Variant reference_literal_value(const Variant &v) {
  if (v.dtype == F32) {
    std::string s = std::to_string(v.u.f32);
    Variant r = v;
    r.u.f32 = (float)std::strtod(s.c_str(), nullptr);
    return r;
  }
  if (v.dtype == F64) {
    std::string s = std::to_string(v.u.f64);
    Variant r = v;
    r.u.f64 = std::strtod(s.c_str(), nullptr);
    return r;
  }
  return v;
}

namespace {

const char *scalar_field(int dt) {
  switch (dt) {
    case F32: return "f32"; case F64: return "f64"; case B8: return "b8"; case U8: return "vu8";
    case U16: return "vu16"; case U32: return "vu32"; case U64: return "vu64"; case S8: return "vs8";
    case S16: return "vs16"; case S32: return "vs32"; case S64: return "vs64";
    default: throw MapError("invalid data type");
  }
}

std::string float_fn(int dt, const char *base) {
  // float variants carry the 'f' suffix, double ones do not
  return dt == F32 ? std::string(base) + "f" : std::string(base);
}

// C-level name of a unary function as used in device code
const char *unary_fn(int op) {
  switch (op) {
    case SIN: return "sin"; case COS: return "cos"; case TAN: return "tan"; case ASIN: return "asin";
    case ACOS: return "acos"; case ATAN: return "atan"; case SINH: return "sinh"; case COSH: return "cosh";
    case TANH: return "tanh"; case ASINH: return "asinh"; case ACOSH: return "acosh"; case ATANH: return "atanh";
    case EXP: return "exp"; case EXP2: return "exp2"; case EXP10: return "exp10"; case LOG: return "log";
    case LOG2: return "log2"; case LOG10: return "log10"; case SQRT: return "sqrt"; case CBRT: return "cbrt";
    case ABS: return "fabs"; case CEIL: return "ceil"; case FLOOR: return "floor"; case TRUNC: return "trunc";
    case ROUND: return "round";
    default: return nullptr;
  }
}

// Device function computing unary op on a float type: the engine's own sine
// and cosine for float32 (skeleton/common.cuh), the CUDA library otherwise.
std::string float_fn_own(int dt, int op) {
  if (dt == F32 && op == SIN) return "map_sinf";
  if (dt == F32 && op == COS) return "map_cosf";
  return float_fn(dt, unary_fn(op));
}

const char *binary_sym(int op) {
  switch (op) {
    case ADD: return "+"; case SUB: return "-"; case MUL: return "*"; case DIV: return "/"; case MOD: return "%";
    case EQ: return "=="; case NE: return "!="; case LT: return "<"; case GT: return ">"; case LE: return "<=";
    case GE: return ">="; case AND: return "&&"; case OR: return "||"; case bAND: return "&"; case bOR: return "|";
    case bXOR: return "^"; case SHL: return "<<"; case SHR: return ">>";
    default: return nullptr;
  }
}

struct Layout {
  size_t off = 0;
  std::ostringstream decl;
  // Appends a field; `count` > 0 declares an array of that many elements, 0 a scalar.
  size_t add(const std::string &type, const std::string &name, size_t size, size_t align, int count) {
    off = (off + align - 1) / align * align;
    size_t at = off;
    decl << "  " << type << " " << name;
    if (count > 0) decl << "[" << count << "]";
    decl << ";  // offset " << at << "\n";
    off += size * (count > 0 ? count : 1);
    return at;
  }
  std::string finish(const std::string &sname, size_t &total) {
    total = (off + 63) / 64 * 64;
    std::ostringstream s;
    s << "struct __align__(64) " << sname << " {\n" << decl.str() << "};\n";
    s << "static_assert(sizeof(" << sname << ") == " << total << ", \"argument layout\");\n";
    return s.str();
  }
};

struct Gen {
  const Group &g;
  KernelPlan &plan;
  std::map<Node *, int> member;   // node -> local index
  std::map<Node *, int> rin;      // raster input -> a.in[k]
  std::map<Node *, int> sca;      // scalar input -> a.s[k]
  std::map<Node *, int> staged;   // focal-read raster input -> staging slot
  std::map<Node *, int> outk;     // output raster -> a.out[k]
  std::set<Node *> center_read;   // raster inputs read at the centre cell
  std::map<Node *, std::string> literal;   // scalar constants written into the source
  std::set<Node *> sincos_first;  // float sin/cos pairs on one argument: emitted once with sincosf
  std::map<Node *, Node *> sincos_mate;
  // hillshade compositions computed through the shading identity (rewrite.hpp)
  std::vector<ShadeMatch> shades;
  std::map<Node *, int> shade_at;    // rewritten node -> index in `shades`
  std::set<Node *> replaced;         // nodes only the rewritten values needed: not emitted
  // Fast form of a composition whose derivatives are private, exactly weighted
  // correlations of one staged input: x = s * xc, y = s * yc (s a power of two),
  // every mask weight 0 or +-2^k (exact products), same mask extent.
  struct ShadeFast {
    bool on = false;
    Node *xc = nullptr, *yc = nullptr, *in = nullptr;
    double s = 1;
    bool arith = false;                                   // exact arithmetic choice of S / C
    float szks = 0, kks = 0, S0 = 0, dS = 0, nC0 = 0, dnC = 0, SH = 0, dSx = 0;
    float S1 = 0, S3 = 0, nC1 = 0;                        // for the selecting form
  };
  std::vector<ShadeFast> fast;
  // fast shading statements record non-finite cells in `bad` instead of branching
  mutable bool fast_flag = false;
  // where the second cell of a pair lies: (x, y + 1) for row pairs, (x + 1, y)
  // for column pairs
  int pdx = 0, pdy = 1;
  std::string x2() const { return pdx ? "x + 1" : "x"; }
  std::string y2() const { return pdy ? "y + 1" : "y"; }
  std::string lx2() const { return pdx ? "lx + 1" : "lx"; }
  std::string ly2() const { return pdy ? "ly + 1" : "ly"; }

  Gen(const Group &g, KernelPlan &p) : g(g), plan(p) {}

  std::string T(Node *n) const { return dt_ctype(n->meta.dtype); }

  // Nodes whose value is always 0 or 1: relational and logical results.
  static bool zero_one(const Node *p) {
    if (p->kind == K_BINARY) return p->op >= EQ && p->op <= OR;
    if (p->kind == K_UNARY) return p->op == NOT;
    return false;
  }
  std::string val(Node *p) const {
    auto m = member.find(p);
    if (m != member.end()) return "v" + std::to_string(m->second);
    auto l = literal.find(p);
    if (l != literal.end()) return l->second;
    auto s = sca.find(p);
    if (s != sca.end()) return "a.s[" + std::to_string(s->second) + "]." + scalar_field(p->meta.dtype);
    auto r = rin.find(p);
    if (r != rin.end()) return "i" + std::to_string(r->second);
    throw MapError(std::string("codegen: value of node ") + kind_name(p->kind) + " is not available in its group");
  }

  std::string tap(Node *in, int dx, int dy) const {
    auto s = staged.find(in);
    if (s == staged.end()) throw MapError("codegen: focal read of a raster that is not staged");
    return "f" + std::to_string(s->second) + ".tap(x, y, lx, ly, " + std::to_string(dx) + ", " + std::to_string(dy) + ")";
  }
  // the same tap of the cell pair (x, y), (x, y + 1)
  std::string tap2(Node *in, int dx, int dy) const {
    auto s = staged.find(in);
    if (s == staged.end()) throw MapError("codegen: focal read of a raster that is not staged");
    return "f" + std::to_string(s->second) + (pdx ? ".tap2c" : ".tap2") + "(x, y, lx, ly, " + std::to_string(dx) + ", " +
           std::to_string(dy) + ")";
  }

  // One term acc = acc + tap * w of a float convolution. A zero weight gives an
  // exact signed-zero product, so fma(tap, w, acc) equals the multiply and add;
  // weights 1 and -1 give exact products tap and -tap. Other weights and types
  // keep the multiply and add.
  static std::string conv_term(const std::string &acc, const std::string &ct, const std::string &tp, int tap_dt,
                               int acc_dt, const Variant &w, bool pair) {
    const std::string lit = var_literal(reference_literal_value(w));
    if (acc_dt == F32 && tap_dt == F32 && (dt_is_float(w.dtype) ? w.dtype == F32 : dt_size(w.dtype) <= 4)) {
      const double wv = var_as_f64(w);
      if (wv == 0.0)
        return acc + " = " + (pair ? "pr_fmaf(" : "fmaf(") + tp + ", " + (dt_is_float(w.dtype) ? lit : std::string("0.0f")) +
               ", " + acc + ");";
      if (wv == 1.0) return acc + " = " + ct + "(" + acc + " + " + tp + ");";
      if (wv == -1.0) return acc + " = " + ct + "(" + acc + " - " + tp + ");";
      // a packed product is added lane by lane (see pr_add_lanes)
      if (pair) return acc + " = pr_add_lanes(" + acc + ", " + tp + " * " + lit + ");";
    }
    return acc + " = " + ct + "(" + acc + " + " + tp + " * " + lit + ");";
  }

  // ---- paired cells (two rows per thread step, skeleton/common.cuh PR<T>)

  // Whether every node of the group has a pair form (float functions on F32 only).
  bool pairable() const {
    for (Node *n : g.nodes) {
      switch (n->kind) {
        case K_CONSTANT: case K_INDEX: case K_CAST: case K_BARRIER: case K_CONDITIONAL: case K_NEIGHBOR:
        case K_CONVOLUTION: case K_FOCALFUNC:
          break;
        case K_UNARY: {
          if (n->op == POS || n->op == NEG || n->op == NOT || n->op == bNOT) break;
          const int pdt = n->prev[0]->meta.dtype;
          if (!unary_fn(n->op)) return false;
          if (dt_is_float(pdt)) {
            if (pdt != F32) return false;
            break;
          }
          if (n->op == ABS || n->op == CEIL || n->op == FLOOR || n->op == TRUNC || n->op == ROUND) break;
          return false;
        }
        case K_BINARY: {
          if (binary_sym(n->op)) break;
          const int pt = dt_promote(n->prev[0]->meta.dtype, n->prev[1]->meta.dtype);
          if (n->op == MAX2 || n->op == MIN2) break;
          if ((n->op == ATAN2 || n->op == POW || n->op == HYPOT || n->op == FMOD) && pt == F32) break;
          return false;
        }
        default:
          return false;
      }
    }
    return true;
  }

  bool is_literal_one(Node *c) const { return literal.count(c) && var_as_f64(c->cnst) == 1.0; }

  // Whether the pair form of n is a packed float multiply whose product may be
  // inexact (a sum with it is then added lane by lane, see pr_add_lanes):
  // products with a 0/1 mask or with +-1 are exact.
  bool inexact_product(Node *n) const {
    if (!member.count(n) || n->kind != K_BINARY || n->meta.dtype != F32) return false;
    double rc = 0;
    if (n->op == DIV) return pow2_reciprocal(n->prev[1], rc);
    if (n->op != MUL) return false;
    for (Node *p : n->prev) {
      if (!dt_is_float(p->meta.dtype) && zero_one(p)) return false;
      if (literal.count(p) && std::fabs(var_as_f64(p->cnst)) == 1.0) return false;
    }
    return true;
  }

  // 1/c for a scalar literal c = +-2^k whose reciprocal is a normal float
  bool pow2_reciprocal(Node *c, double &rc) const {
    if (!literal.count(c)) return false;
    const double v = var_as_f64(c->cnst);
    if (!(v != 0) || !std::isfinite(v)) return false;
    int e = 0;
    const double m = std::frexp(std::fabs(v), &e);
    if (m != 0.5) return false;
    rc = 1.0 / v;
    return std::fabs(rc) >= 0x1p-126 && std::fabs(rc) <= 0x1p+127;
  }

  // Statement of node n in the pair form: the value of the cells (x, y) and
  // (x, y + 1) as PR<T>, every conversion written as PR<T>(...).
  std::string stmt2(Node *n) const {
    std::ostringstream s;
    const std::string t = T(n);
    const std::string pt_ = "PR<" + t + ">";
    const std::string v = "v" + std::to_string(member.at(n));
    const std::string decl = "const " + pt_ + " " + v + " = ";
    switch (n->kind) {
      case K_CONSTANT:
        s << decl << pt_ << "(" << var_literal(reference_literal_value(n->cnst)) << ");";
        break;
      case K_INDEX:
        if (n->op == D1) s << decl << pt_ << "((" << t << ")(x), (" << t << ")(" << x2() << "));";
        else s << decl << pt_ << "((" << t << ")(y), (" << t << ")(" << y2() << "));";
        break;
      case K_CAST: case K_BARRIER:
        s << decl << pt_ << "(" << val(n->prev[0]) << ");";
        break;
      case K_UNARY: {
        std::string p = val(n->prev[0]);
        int pdt = n->prev[0]->meta.dtype;
        switch (n->op) {
          case POS: s << decl << pt_ << "(+" << p << ");"; break;
          case NEG: s << decl << pt_ << "(-" << p << ");"; break;
          case NOT: s << decl << pt_ << "(!" << p << ");"; break;
          case bNOT: s << decl << pt_ << "(~" << p << ");"; break;
          default: {
            auto mate = sincos_mate.find(n);
            if (mate != sincos_mate.end()) {
              if (sincos_first.count(n)) {
                Node *sn = n->op == SIN ? n : mate->second, *cn = n->op == COS ? n : mate->second;
                s << "PR<float> v" << member.at(sn) << ", v" << member.at(cn) << "; map_sincosf(PR<float>(" << p
                  << "), &v" << member.at(sn) << ", &v" << member.at(cn) << ");";
              }
              break;
            }
            if (dt_is_float(pdt)) {
              const std::string f = float_fn_own(pdt, n->op);   // own functions overload PR; library ones are pr_*
              s << decl << pt_ << "(" << (f.compare(0, 4, "map_") == 0 ? f : "pr_" + f) << "(PR<float>(" << p << ")));";
            } else if (n->op == ABS) {
              s << decl << pt_ << "(psel(" << p << " < 0, -" << p << ", " << p << "));";
            } else {
              s << decl << pt_ << "(" << p << ");";   // CEIL / FLOOR / TRUNC / ROUND of an integer
            }
          }
        }
        break;
      }
      case K_BINARY: {
        std::string l = val(n->prev[0]), r = val(n->prev[1]);
        int pt = dt_promote(n->prev[0]->meta.dtype, n->prev[1]->meta.dtype);
        std::string pts = dt_ctype(pt);
        if (const char *sym = binary_sym(n->op)) {
          if (dt_is_float(pt) && (n->op == MOD || binary_is_bitwise(n->op)))
            throw MapError(std::string("binary op ") + binary_name(n->op) + " is not defined on floating types");
          if (dt_is_float(pt)) {
            if (!dt_is_float(n->prev[0]->meta.dtype) && zero_one(n->prev[0])) l = "psel(" + l + ", (" + pts + ")1, (" + pts + ")0)";
            if (!dt_is_float(n->prev[1]->meta.dtype) && zero_one(n->prev[1])) r = "psel(" + r + ", (" + pts + ")1, (" + pts + ")0)";
          }
          double rc = 0;
          Node *one = nullptr;   // 1 * x and x * 1 of a float x are x (exactly, signs and NaN included)
          if (n->op == MUL && pt == F32) {
            if (is_literal_one(n->prev[0]) && n->prev[1]->meta.dtype == F32) one = n->prev[1];
            else if (is_literal_one(n->prev[1]) && n->prev[0]->meta.dtype == F32) one = n->prev[0];
          }
          if (one) {
            s << decl << pt_ << "(" << val(one) << ");";
          } else if (n->op == ADD && pt == F32 && (inexact_product(n->prev[0]) || inexact_product(n->prev[1]))) {
            s << decl << "pr_add_lanes(" << l << ", " << r << ");";
          } else if (n->op == DIV && pt == F32 && pow2_reciprocal(n->prev[1], rc)) {
            // division by a literal power of two: the multiply by its (exact)
            // reciprocal rounds the same real value, and packs
            char b[48];
            std::snprintf(b, sizeof b, "%af", rc);
            s << decl << pt_ << "(" << l << " * " << b << ");";
          } else {
            s << decl << pt_ << "(" << l << " " << sym << " " << r << ");";
          }
        } else {
          std::string L = "PR<" + pts + ">(" + l + ")", R = "PR<" + pts + ">(" + r + ")";
          switch (n->op) {
            case MAX2: s << decl << pt_ << "(red_max(" << L << ", " << R << "));"; break;
            case MIN2: s << decl << pt_ << "(red_min(" << L << ", " << R << "));"; break;
            case ATAN2: s << decl << pt_ << "(map_atan2f(" << L << ", " << R << "));"; break;
            case POW: s << decl << pt_ << "(pr_powf(" << L << ", " << R << "));"; break;
            case HYPOT: s << decl << pt_ << "(pr_hypotf(" << L << ", " << R << "));"; break;
            case FMOD: s << decl << pt_ << "(pr_fmodf(" << L << ", " << R << "));"; break;
            default: throw MapError("codegen: invalid binary op");
          }
        }
        break;
      }
      case K_CONDITIONAL:
        s << decl << "psel(" << val(n->prev[0]) << ", " << pt_ << "(" << val(n->prev[1]) << "), " << pt_ << "("
          << val(n->prev[2]) << "));";
        break;
      case K_NEIGHBOR:
        s << decl << pt_ << "(" << tap2(n->prev[0], n->coord.arr[0], n->coord.arr[1]) << ");";
        break;
      case K_CONVOLUTION: {
        int hx = n->halo_x(), hy = n->halo_y(), mw = n->mask_ds.arr[0];
        s << pt_ << " " << v << " = " << pt_ << "((" << t << ")0);";
        for (int i1 = -hy; i1 <= hy; i1++)
          for (int i0 = -hx; i0 <= hx; i0++)
            s << "\n    " << conv_term(v, pt_, tap2(n->prev[0], i0, i1), n->prev[0]->meta.dtype, n->meta.dtype,
                                       n->mask[(i1 + hy) * mw + (i0 + hx)], true);
        break;
      }
      case K_FOCALFUNC: {
        int hx = n->halo_x(), hy = n->halo_y();
        s << pt_ << " " << v << " = " << pt_ << "(" << var_literal(reduction_neutral(n->op, n->meta.dtype)) << ");";
        for (int i1 = -hy; i1 <= hy; i1++)
          for (int i0 = -hx; i0 <= hx; i0++)
            s << "\n    " << v << " = RedOp<" << n->op << ", " << pt_ << ">::f(" << v << ", " << pt_ << "("
              << tap2(n->prev[0], i0, i1) << "));";
        break;
      }
      default:
        throw MapError(std::string("codegen: node kind ") + kind_name(n->kind) + " has no pair form");
    }
    return s.str();
  }

  std::string stores2() const {
    std::ostringstream s;
    for (auto &kv : outk) {
      Node *o = kv.first;
      if (pdx)
        s << "    str_out2x<" << T(o) << ">(a.out[" << kv.second << "], x, y, lane0(" << val(o) << "), lane1(" << val(o)
          << "));\n";
      else
        s << "    str_out<" << T(o) << ">(a.out[" << kv.second << "], x, y, lane0(" << val(o) << "));\n"
          << "    str_out<" << T(o) << ">(a.out[" << kv.second << "], x, y + 1, lane1(" << val(o) << "));\n";
    }
    return s.str();
  }

  // the group's outputs as reference parameters (deferred stores): ", T &r0, ..."
  std::string out_params(bool pair) const {
    std::ostringstream s;
    int k = 0;
    for (auto &kv : outk) s << ", " << (pair ? "PR<" + T(kv.first) + ">" : T(kv.first)) << " &r" << k++;
    return s.str();
  }
  std::string out_assigns() const {
    std::ostringstream s;
    int k = 0;
    for (auto &kv : outk) s << "    r" << k++ << " = " << val(kv.first) << ";\n";
    return s.str();
  }

  std::string center_loads2() const {
    std::ostringstream s;
    for (Node *p : plan.in_rasters) {
      if (!center_read.count(p)) continue;
      int k = rin.at(p);
      std::string t = T(p);
      if (staged.count(p)) s << "    const PR<" << t << "> i" << k << " = " << tap2(p, 0, 0) << ";\n";
      else
        s << "    const PR<" << t << "> i" << k << "(ldr<" << t << ">(a.in[" << k << "], x, y), ldr<" << t << ">(a.in[" << k
          << "], " << x2() << ", " << y2() << "));\n";
    }
    return s.str();
  }

  std::string body2() const {
    std::ostringstream s;
    for (Node *n : g.nodes) {
      if (replaced.count(n)) continue;
      s << "    " << (shade_at.count(n) ? shade_stmt(n, true) : stmt2(n)) << "\n";
    }
    return s.str();
  }

  void classify() {
    for (size_t i = 0; i < g.nodes.size(); i++) member[g.nodes[i]] = (int)i;
    for (Node *in : g.inputs) {
      if (in->meta.numdim == D0 && in->kind == K_CONSTANT && !in->as_param) {
        // Scalar constants are part of the kernel's signature (as constant values
        // are part of the reference's Version signature, runtime/dag/Constant.cpp),
        // so the device compiler folds them (x / 8 becomes an exact multiply).
        literal[in] = "((" + std::string(dt_ctype(in->meta.dtype)) + ")" + var_literal(in->cnst) + ")";
      } else if (in->meta.numdim == D0) {
        sca[in] = (int)plan.scalars.size();
        plan.scalars.push_back(in);
      } else {
        rin[in] = (int)plan.in_rasters.size();
        plan.in_rasters.push_back(in);
      }
    }
    for (Node *n : g.nodes) {
      bool focal = n->kind == K_NEIGHBOR || n->kind == K_CONVOLUTION || n->kind == K_FOCALFUNC || n->kind == K_FOCALFLOW ||
                   n->kind == K_FOCALPERCENT;
      for (size_t j = 0; j < n->prev.size(); j++) {
        Node *p = n->prev[j];
        if (!rin.count(p)) continue;
        if (focal && j == 0) {
          if (!staged.count(p)) {
            int k = (int)staged.size();
            staged[p] = k;
          }
          plan.halo_x = std::max(plan.halo_x, n->halo_x());
          plan.halo_y = std::max(plan.halo_y, n->halo_y());
        } else {
          center_read.insert(p);
        }
      }
    }
    for (Node *o : g.outputs) {
      if (o->meta.numdim == D0) continue;
      outk[o] = (int)plan.out_rasters.size();
      plan.out_rasters.push_back(o);
    }
    // sin(x) and cos(x) of the same float argument share one sincosf call
    for (Node *n : g.nodes) {
      if (n->kind != K_UNARY || (n->op != SIN && n->op != COS) || n->meta.dtype != F32) continue;
      if (sincos_mate.count(n)) continue;
      for (Node *m : g.nodes) {
        if (m == n || m->kind != K_UNARY || m->prev[0] != n->prev[0] || sincos_mate.count(m)) continue;
        if ((n->op == SIN && m->op == COS) || (n->op == COS && m->op == SIN)) {
          sincos_mate[n] = m;
          sincos_mate[m] = n;
          sincos_first.insert(n->id < m->id ? n : m);
          break;
        }
      }
    }
    if (Runtime::get().algebraic_rewrite && (g.skeleton == SK_LOCAL || g.skeleton == SK_FOCAL)) find_shades();
  }

  // Finds the hillshade compositions of the group and the nodes that only they need.
  void find_shades() {
    auto lit = [this](Node *n, double &v) {
      if (literal.count(n)) { v = var_as_f64(n->cnst); return true; }
      if (member.count(n) && n->kind == K_CONSTANT) { v = var_as_f64(reference_literal_value(n->cnst)); return true; }
      return false;
    };
    auto mem = [this](Node *n) { return member.count(n) > 0 && n->kind != K_CONSTANT; };
    std::set<Node *> in_pattern;
    for (Node *n : g.nodes) {
      if (in_pattern.count(n)) continue;
      ShadeMatch m;
      if (!match_shade(n, lit, mem, m)) continue;
      shade_at[n] = (int)shades.size();
      for (Node *p : m.pattern) in_pattern.insert(p);
      shades.push_back(m);
    }
    if (shades.empty()) return;
    std::set<Node *> outs(g.outputs.begin(), g.outputs.end());
    // a pattern node is dropped when every consumer inside the group is a
    // rewritten node or itself dropped (sin/cos mates only together)
    for (bool changed = true; changed;) {
      changed = false;
      for (auto it = g.nodes.rbegin(); it != g.nodes.rend(); ++it) {
        Node *p = *it;
        if (!in_pattern.count(p) || shade_at.count(p) || replaced.count(p) || outs.count(p)) continue;
        bool all = true;
        for (Node *c : p->next)
          if (member.count(c) && !shade_at.count(c) && !replaced.count(c)) all = false;
        if (all) {
          replaced.insert(p);
          changed = true;
        }
      }
      for (auto &kv : sincos_mate)
        if (replaced.count(kv.first) != replaced.count(kv.second)) {
          replaced.erase(kv.first);
          replaced.erase(kv.second);
        }
    }
    fast.assign(shades.size(), ShadeFast());
    if (g.skeleton == SK_FOCAL && Runtime::get().algebraic_rewrite == 1)
      for (size_t i = 0; i < shades.size(); i++) find_fast((int)i, outs);
  }

  // x (or y) = scale * conv: DIV by / MUL with a literal power of two
  bool scaled_conv(Node *x, Node *&c, double &s) const {
    if (x->kind != K_BINARY || x->meta.dtype != F32) return false;
    double rc = 0;
    if (x->op == DIV && pow2_reciprocal(x->prev[1], rc)) { c = x->prev[0]; s = rc; }
    else if (x->op == MUL && literal.count(x->prev[1]) && pow2_reciprocal(x->prev[1], rc)) { c = x->prev[0]; s = 1.0 / rc; }
    else if (x->op == MUL && literal.count(x->prev[0]) && pow2_reciprocal(x->prev[0], rc)) { c = x->prev[1]; s = 1.0 / rc; }
    else return false;
    if (c->kind != K_CONVOLUTION || c->meta.dtype != F32 || c->prev[0]->meta.dtype != F32) return false;
    if (!rin.count(c->prev[0]) || !staged.count(c->prev[0])) return false;
    for (const Variant &w : c->mask) {
      const double v = var_as_f64(w);
      if (v == 0.0) continue;
      int e = 0;
      const double mnt = std::frexp(std::fabs(v), &e);
      if (mnt != 0.5 || e < -20 || e > 20) return false;   // +-2^k: every product is exact
    }
    return true;
  }
  // a node computed only for the rewritten values (every consumer in the group replaced)
  bool private_to_rewrite(Node *n, const std::set<Node *> &outs) const {
    if (outs.count(n) || !member.count(n)) return false;
    for (Node *c : n->next)
      if (member.count(c) && !shade_at.count(c) && !replaced.count(c)) return false;
    return true;
  }
  void find_fast(int i, const std::set<Node *> &outs) {
    const ShadeMatch &m = shades[i];
    ShadeFast f;
    double sx = 0, sy = 0;
    if (!scaled_conv(m.x, f.xc, sx) || !scaled_conv(m.y, f.yc, sy) || sx != sy) return;
    if (f.xc->prev[0] != f.yc->prev[0] || f.xc->mask_ds.arr[0] != f.yc->mask_ds.arr[0] ||
        f.xc->mask_ds.arr[1] != f.yc->mask_ds.arr[1] || f.xc == f.yc)
      return;
    if (!private_to_rewrite(m.x, outs) || !private_to_rewrite(m.y, outs)) return;
    replaced.insert(m.x);
    replaced.insert(m.y);
    if (!private_to_rewrite(f.xc, outs) || !private_to_rewrite(f.yc, outs)) {
      replaced.erase(m.x);
      replaced.erase(m.y);
      return;
    }
    replaced.insert(f.xc);
    replaced.insert(f.yc);
    f.in = f.xc->prev[0];
    f.s = sx;
    f.on = true;
    f.szks = (float)((double)m.szk * f.s);
    f.kks = (float)((double)m.kk * f.s * f.s);
    f.S0 = m.S0;
    f.S1 = m.S1;
    f.SH = m.SH;
    f.S3 = m.S3;
    f.nC0 = -m.C0;
    f.nC1 = -m.C1;
    // the arithmetic choice needs S1 - S0, -C1 + C0 and S3 - SH exact in float32
    auto exact = [](float a, float b, float &d) {
      d = a - b;
      return (double)d == (double)a - (double)b;
    };
    f.arith = exact(f.S1, f.S0, f.dS) && exact(f.nC1, f.nC0, f.dnC) && exact(f.S3, f.SH, f.dSx) &&
              (double)f.szks == (double)m.szk * f.s && (double)f.kks == (double)m.kk * f.s * f.s;
    if (!f.arith) {   // keep the general form
      replaced.erase(f.xc);
      replaced.erase(f.yc);
      replaced.erase(m.x);
      replaced.erase(m.y);
      return;
    }
    fast[i] = f;
  }

  // Literal chain of shading composition i as a separate function: cells whose
  // x^2 + y^2 is not finite take it.
  // Whether the literal chain of composition i reads kernel arguments (scalar parameters).
  bool shade_reads_args(int i) const {
    for (Node *n : shades[i].pattern)
      for (Node *p : n->prev)
        if (sca.count(p)) return true;
    return false;
  }
  std::string shade_slow_decl(int i) const {
    const ShadeMatch &m = shades[i];
    std::ostringstream s;
    // without kernel arguments the function reads no memory, so the compiler
    // may keep loads of the cells around its call sites in registers
    s << "__device__ __noinline__ float shade_slow" << i << "(" << (shade_reads_args(i) ? "const Args &a, " : "")
      << "const float " << val(m.x) << ", const float " << val(m.y) << ") {\n";
    for (Node *n : m.pattern) s << "  " << stmt(n, false) << "\n";
    s << "  return " << val(m.hs) << ";\n}\n";
    return s.str();
  }
  // The fallback of fast composition i for one cell: the literal derivatives
  // (every tap in the correlation's order, as the general form computes them,
  // scaled by s) and the literal chain.
  std::string shade_cell_slow_decl(int i) const {
    const ShadeFast &f = fast[i];
    const int hx = f.xc->halo_x(), hy = f.xc->halo_y(), mw = f.xc->mask_ds.arr[0];
    const std::string fk = "f" + std::to_string(staged.at(f.in));
    std::ostringstream s;
    // the tap object by value: a reference would take its address and keep it
    // (and the row loop's loads of its pointer) in local memory
    s << "template <class F>\n__device__ __noinline__ float shade_cell_slow" << i << "("
      << (shade_reads_args(i) ? "const Args &a, " : "") << "const F " << fk << ", int x, int y, int lx, int ly) {\n";
    for (int c = 0; c < 2; c++) {
      Node *cv = c ? f.yc : f.xc;
      const std::string acc = c ? "yl" : "xl";
      s << "  float " << acc << " = 0.0f;\n";
      for (int i1 = -hy; i1 <= hy; i1++)
        for (int i0 = -hx; i0 <= hx; i0++)
          s << "  " << conv_term(acc, "(float)", tap(f.in, i0, i1), F32, F32, cv->mask[(i1 + hy) * mw + (i0 + hx)], false)
            << "\n";
    }
    s << "  return shade_slow" << i << "(" << (shade_reads_args(i) ? "a, " : "") << "__fmul_rn(xl, " << fl((float)f.s)
      << "), __fmul_rn(yl, " << fl((float)f.s) << "));\n}\n";
    return s.str();
  }
  std::string shade_decls() const {
    std::string s;
    for (size_t i = 0; i < shades.size(); i++) {
      s += shade_slow_decl((int)i);
      if (fast[i].on) s += shade_cell_slow_decl((int)i);
    }
    return s;
  }
  static std::string fl(float f) {
    char b[48];
    std::snprintf(b, sizeof b, "%af", (double)f);
    return b;
  }
  std::string shade_args(const ShadeMatch &m) const {
    return fl(m.cz) + ", " + fl(m.szk) + ", " + fl(m.kk) + ", " + fl(m.S0) + ", " + fl(m.C0) + ", " + fl(m.S1) + ", " +
           fl(m.C1) + ", " + fl(m.SH) + ", " + fl(m.S3);
  }
  // Fast statement of composition i (see ShadeFast / map_shade_fast): the two
  // correlations as fused multiply-adds over their non-zero weights (exact
  // products, so each term rounds like the literal add of the product), zero
  // weights dropped; cells where a tap that neither reads, or x^2 + y^2, is not
  // finite recompute the literal derivatives (the dropped terms added back as
  // fma(tap, 0, acc)) and take the literal chain.
  std::string shade_fast_stmt(Node *n, bool pair) const {
    const int i = shade_at.at(n);
    const ShadeFast &f = fast[i];
    const std::string v = "v" + std::to_string(member.at(n)), si = std::to_string(i);
    const std::string T = pair ? "PR<float>" : "float", fma = pair ? "pr_fmaf(" : "__fmaf_rn(";
    const int hx = f.xc->halo_x(), hy = f.xc->halo_y(), mw = f.xc->mask_ds.arr[0];
    auto tapv = [&](int dx, int dy) { return pair ? tap2(f.in, dx, dy) : tap(f.in, dx, dy); };
    std::ostringstream s;
    // z: the taps both correlations weight by zero, as fma(tap, 0, z) (zero for
    // finite taps, NaN otherwise); the x sum starts from it, so a non-finite
    // such tap makes x, hence x^2 + y^2, NaN (the sign of a zero x does not
    // change the result)
    // The terms of each sum in order: (tap, weight), the zero-weight taps
    // first (x sum only).
    std::vector<std::pair<std::string, double>> terms[2];
    for (int i1 = -hy; i1 <= hy; i1++)
      for (int i0 = -hx; i0 <= hx; i0++) {
        const int k = (i1 + hy) * mw + (i0 + hx);
        if (var_as_f64(f.xc->mask[k]) == 0.0 && var_as_f64(f.yc->mask[k]) == 0.0) terms[0].push_back({tapv(i0, i1), 0.0});
      }
    for (int c = 0; c < 2; c++) {
      Node *cv = c ? f.yc : f.xc;
      for (int i1 = -hy; i1 <= hy; i1++)
        for (int i0 = -hx; i0 <= hx; i0++) {
          const double w = var_as_f64(cv->mask[(i1 + hy) * mw + (i0 + hx)]);
          if (w != 0.0) terms[c].push_back({tapv(i0, i1), w});
        }
    }
    for (int c = 0; c < 2; c++) {
      const std::string acc = v + (c ? "_yc" : "_xc");
      std::vector<std::pair<std::string, double>> &t = terms[c];
      // A sum from +0 whose first non-zero term has weight +-1: that term is
      // exact, so it becomes the addend of the fused multiply-add before it (a
      // zero-weight tap) or after it (the next term), one instruction fewer.
      // Only the sign of a zero partial sum can differ, which changes neither
      // x^2 + y^2, nor the tests x != 0 and y < 0, nor the result.
      size_t nz = 0;
      while (nz < t.size() && t[nz].second == 0.0) nz++;
      if (!pair && focal_tune().fmerge && nz < t.size() && std::fabs(t[nz].second) == 1.0 && t.size() >= 2) {
        const std::string lead = (t[nz].second < 0 ? "-" : "") + t[nz].first;
        const size_t with = nz > 0 ? 0 : 1;   // the term that takes it as its addend
        s << " " << T << " " << acc << " = " << fma << t[with].first << ", " << fl((float)t[with].second) << ", " << lead
          << ");";
        for (size_t j = 0; j < t.size(); j++)
          if (j != with && j != nz)
            s << " " << acc << " = " << fma << t[j].first << ", " << fl((float)t[j].second) << ", " << acc << ");";
        continue;
      }
      s << " " << T << " " << acc << " = " << T << "(0.0f);";
      for (const auto &e : t)
        s << " " << acc << " = " << fma << e.first << ", " << fl((float)e.second) << ", " << acc << ");";
    }
    s << " " << T << " " << v << "_q; " << T << " " << v << " = map_shade_fast(" << v << "_xc, " << v << "_yc, "
      << fl(shades[i].cz) << ", " << fl(f.szks) << ", " << fl(f.kks) << ", " << fl(f.S0) << ", " << fl(f.dS) << ", "
      << fl(f.nC0) << ", " << fl(f.dnC) << ", " << fl(f.SH) << ", " << fl(f.dSx) << ", " << v << "_q);";
    // Cells whose x^2 + y^2 is not finite take the literal derivatives and chain
    // (shade_cell_slow, a function of its own: no code in the unrolled row loop).
    // In the flag form the row loop only records that some cell needs it, and
    // recomputes the thread's cells with the checks when one did.
    // (flag form: `bad` reaches 0x7f800000 when some cell's q is not finite;
    // either by a comparison per cell, or, as q is +0 or more, +inf or NaN, by
    // an unsigned maximum of its bits, measured 2.5% slower on the hillshade)
    if (fast_flag) {
      if (focal_tune().fflag) {
        if (!pair) s << " bad = max(bad, __float_as_uint(" << v << "_q));";
        else s << " bad = max(bad, max(__float_as_uint(" << v << "_q.a), __float_as_uint(" << v << "_q.b)));";
      } else {
        if (!pair) s << " bad |= !(" << v << "_q < MAP_INF_F) ? 0x7f800000u : 0u;";
        else s << " bad |= (!(" << v << "_q.a < MAP_INF_F) | !(" << v << "_q.b < MAP_INF_F)) ? 0x7f800000u : 0u;";
      }
      return s.str();
    }
    const std::string fk = "f" + std::to_string(staged.at(f.in));
    auto slow_lane = [&](const std::string &lane, int second) {
      const std::string sel = lane.empty() ? "" : "." + lane;
      return " " + v + sel + " = shade_cell_slow" + si + "(" + (shade_reads_args(i) ? "a, " : "") + fk + ", " +
             (second ? x2() + ", " + y2() + ", " + lx2() + ", " + ly2() : std::string("x, y, lx, ly")) + ");";
    };
    if (!pair) {
      s << " if (!(" << v << "_q < MAP_INF_F)) {" << slow_lane("", 0) << " }";
    } else {
      s << " if (!(" << v << "_q.a < MAP_INF_F) || !(" << v << "_q.b < MAP_INF_F)) {";
      s << " if (!(" << v << "_q.a < MAP_INF_F)) {" << slow_lane("a", 0) << " }";
      s << " if (!(" << v << "_q.b < MAP_INF_F)) {" << slow_lane("b", 1) << " } }";
    }
    return s.str();
  }
  bool any_fast() const {
    for (auto &f : fast)
      if (f.on) return true;
    return false;
  }

  // statement of a rewritten node (scalar or pair form)
  std::string shade_stmt(Node *n, bool pair) const {
    const int i = shade_at.at(n);
    if (fast[i].on) return shade_fast_stmt(n, pair);
    const ShadeMatch &m = shades[i];
    const std::string v = "v" + std::to_string(member.at(n)), q = v + "_q", si = std::to_string(i);
    const std::string tmpl = m.k_one ? "<true>" : "<false>";
    const std::string aa = shade_reads_args(i) ? "a, " : "";
    std::ostringstream s;
    if (!pair) {
      s << "float " << q << "; float " << v << " = map_shade" << tmpl << "(" << val(m.x) << ", " << val(m.y) << ", "
        << shade_args(m) << ", " << q << "); if (!(" << q << " < MAP_INF_F)) " << v << " = shade_slow" << si << "(" << aa
        << val(m.x) << ", " << val(m.y) << ");";
    } else {
      s << "PR<float> " << q << "; PR<float> " << v << " = map_shade" << tmpl << "(PR<float>(" << val(m.x)
        << "), PR<float>(" << val(m.y) << "), " << shade_args(m) << ", " << q << "); if (!(" << q << ".a < MAP_INF_F)) "
        << v << ".a = shade_slow" << si << "(" << aa << "lane0(" << val(m.x) << "), lane0(" << val(m.y) << ")); if (!("
        << q << ".b < MAP_INF_F)) " << v << ".b = shade_slow" << si << "(" << aa << "lane1(" << val(m.x) << "), lane1("
        << val(m.y) << "));";
    }
    return s.str();
  }

  // ---- packed byte cells (Q4 in skeleton/common.cuh): four cells of a row per step

  // Value range of a node of the packed form; `wrap`: its type reduces the
  // computed value mod 256 (the lanes are masked after the operation).
  struct QRange {
    long long lo = 0, hi = 0;
    bool wrap = false;
  };
  std::map<Node *, QRange> qr;

  // Conversion to type dt of a value in r (0 <= lo, hi <= 0xFFFF); false when the
  // converted value could leave [0, 0x7FFF] or the type is not an integer.
  static bool q_type(int dt, QRange &r) {
    r.wrap = false;
    switch (dt) {
      case U8:
        if (r.hi > 255) { r.lo = 0; r.hi = 255; r.wrap = true; }
        return true;
      case B8: return r.hi <= 1;
      case S8: return r.hi <= 127;
      case U16: case S16: case U32: case S32: case U64: case S64: return r.hi <= 0x7FFF;
      default: return false;
    }
  }
  bool q_literal(Node *p, long long &c) const {
    double v = 0;
    if (literal.count(p)) v = var_as_f64(p->cnst);
    else if (member.count(p) && p->kind == K_CONSTANT) v = var_as_f64(reference_literal_value(p->cnst));
    else return false;
    if (dt_is_float(p->meta.dtype) || !(v >= 0 && v <= 0x7FFF) || v != std::floor(v)) return false;
    c = (long long)v;
    return true;
  }
  bool q_range(Node *p, QRange &r) const {
    long long c = 0;
    if (q_literal(p, c)) { r.lo = r.hi = c; r.wrap = false; return true; }
    auto it = qr.find(p);
    if (it == qr.end()) return false;
    r = it->second;
    return true;
  }
  static bool zero_one_range(const QRange &r) { return r.lo >= 0 && r.hi <= 1; }

  // Whether every node of the group has a packed form whose lanes provably stay
  // in range: integer arithmetic on byte rasters staged in shared memory
  // (correlations with non-negative integer weights, sums, differences that stay
  // non-negative, products, relations, logical and bitwise operations, selects,
  // minimum and maximum), every value in [0, 0x7FFF] after its type's conversion,
  // every output an 8-bit cell. Fills qr.
  bool quadable() {
    qr.clear();
    if (!shades.empty() || outk.empty()) return false;
    for (Node *in : g.inputs) {
      long long c = 0;
      if (sca.count(in)) return false;
      if (literal.count(in)) {
        if (!q_literal(in, c)) return false;
        continue;
      }
      if (rin.count(in)) {
        if (in->meta.dtype != U8) return false;
        qr[in] = QRange{0, 255, false};
      }
    }
    for (auto &kv : outk)
      if (kv.first->meta.dtype != U8 && kv.first->meta.dtype != B8) return false;
    for (Node *n : g.nodes) {
      if (replaced.count(n)) return false;
      QRange r, a, b;
      switch (n->kind) {
        case K_CONSTANT: {
          long long c = 0;
          if (!q_literal(n, c)) return false;
          r.lo = r.hi = c;
          break;
        }
        case K_CAST: case K_BARRIER:
          if (!q_range(n->prev[0], r)) return false;
          break;
        case K_NEIGHBOR:
          if (n->prev[0]->meta.dtype != U8 || !staged.count(n->prev[0])) return false;
          r = QRange{0, 255, false};
          break;
        case K_CONVOLUTION: {
          if (n->prev[0]->meta.dtype != U8 || !staged.count(n->prev[0]) || dt_is_float(n->meta.dtype)) return false;
          for (const Variant &w : n->mask) {
            const double v = var_as_f64(w);
            if (!(v >= 0 && v <= 0xFFFF) || v != std::floor(v)) return false;
            r.hi += (long long)v * 255;
          }
          if (r.hi > 0xFFFF) return false;
          break;
        }
        case K_UNARY:
          if (n->op == POS) {
            if (!q_range(n->prev[0], r)) return false;
          } else if (n->op == NOT) {
            if (!q_range(n->prev[0], a)) return false;
            r = QRange{0, 1, false};
          } else {
            return false;
          }
          break;
        case K_BINARY: {
          if (!q_range(n->prev[0], a) || !q_range(n->prev[1], b)) return false;
          switch (n->op) {
            case ADD: r.lo = a.lo + b.lo; r.hi = a.hi + b.hi; break;
            case SUB: r.lo = a.lo - b.hi; r.hi = a.hi - b.lo; if (r.lo < 0) return false; break;
            case MUL:
              r.lo = a.lo * b.lo;
              r.hi = a.hi * b.hi;
              break;
            case EQ: case NE: case LT: case GT: case LE: case GE: case AND: case OR: r = QRange{0, 1, false}; break;
            case bAND: r = QRange{0, std::min(a.hi, b.hi), false}; break;
            case bOR: case bXOR: {
              long long m = 1;
              while (m <= std::max(a.hi, b.hi)) m <<= 1;
              r = QRange{0, m - 1, false};
              break;
            }
            case MAX2: r = QRange{std::max(a.lo, b.lo), std::max(a.hi, b.hi), false}; break;
            case MIN2: r = QRange{std::min(a.lo, b.lo), std::min(a.hi, b.hi), false}; break;
            default: return false;
          }
          if (r.hi > 0xFFFF) return false;
          break;
        }
        case K_CONDITIONAL: {
          QRange c;
          if (!q_range(n->prev[0], c) || !q_range(n->prev[1], a) || !q_range(n->prev[2], b)) return false;
          r = QRange{std::min(a.lo, b.lo), std::max(a.hi, b.hi), false};
          break;
        }
        default:
          return false;
      }
      if (!q_type(n->meta.dtype, r) || r.lo < 0 || r.hi > 0x7FFF) return false;
      qr[n] = r;
    }
    return true;
  }

  std::string val4(Node *p) const {
    long long c = 0;
    if (q_literal(p, c) && !member.count(p)) return "q4_splat(" + std::to_string(c) + "u)";
    auto m = member.find(p);
    if (m != member.end()) return "v" + std::to_string(m->second);
    auto r = rin.find(p);
    if (r != rin.end()) return "i" + std::to_string(r->second);
    throw MapError("codegen: packed value of a node that is not available");
  }
  std::string tap4(Node *in, int dx, int dy) const {
    return "f" + std::to_string(staged.at(in)) + ".tap4(lx, ly, " + std::to_string(dx) + ", " + std::to_string(dy) + ")";
  }
  // a value as lanes 0 / 1 (a relation's result already is)
  std::string bool4(Node *p) const {
    QRange r;
    if (q_range(p, r) && zero_one_range(r)) return val4(p);
    return "q4_ne0(" + val4(p) + ")";
  }
  std::string stmt4(Node *n) const {
    const QRange &R = qr.at(n);
    const std::string v = "v" + std::to_string(member.at(n));
    std::string e;
    switch (n->kind) {
      case K_CONSTANT: {
        long long c = 0;
        q_literal(n, c);
        e = "q4_splat(" + std::to_string(c) + "u)";
        break;
      }
      case K_CAST: case K_BARRIER: e = val4(n->prev[0]); break;
      case K_NEIGHBOR: e = tap4(n->prev[0], n->coord.arr[0], n->coord.arr[1]); break;
      case K_CONVOLUTION: {
        // Sums of lanes are exact in any order (no lane leaves its range), so the
        // correlation is summed mask row by mask row: the sum of one mask row
        // over one tap row is the same expression for every output row that
        // uses it, and the compiler computes it once for the unrolled rows.
        int hx = n->halo_x(), hy = n->halo_y(), mw = n->mask_ds.arr[0];
        std::vector<std::string> rows;
        for (int i1 = -hy; i1 <= hy; i1++) {
          std::string r;
          for (int i0 = -hx; i0 <= hx; i0++) {
            const long long w = (long long)var_as_f64(n->mask[(i1 + hy) * mw + (i0 + hx)]);
            if (w == 0) continue;
            const std::string t = tap4(n->prev[0], i0, i1);
            const std::string term = w == 1 ? t : "q4_mulc(" + t + ", " + std::to_string(w) + "u)";
            r = r.empty() ? term : "q4_add(" + r + ", " + term + ")";
          }
          if (!r.empty()) rows.push_back(r);
        }
        e = rows.empty() ? "q4_splat(0u)" : rows[0];
        for (size_t k = 1; k < rows.size(); k++) e = "q4_add(" + e + ", " + rows[k] + ")";
        break;
      }
      case K_UNARY: e = n->op == NOT ? "q4_eq0(" + val4(n->prev[0]) + ")" : val4(n->prev[0]); break;
      case K_BINARY: {
        Node *p0 = n->prev[0], *p1 = n->prev[1];
        const std::string l = val4(p0), r = val4(p1);
        QRange a, b;
        q_range(p0, a);
        q_range(p1, b);
        long long c = 0;
        switch (n->op) {
          case ADD: e = "q4_add(" + l + ", " + r + ")"; break;
          case SUB: e = "q4_sub(" + l + ", " + r + ")"; break;
          case MUL:
            if (q_literal(p1, c)) e = "q4_mulc(" + l + ", " + std::to_string(c) + "u)";
            else if (q_literal(p0, c)) e = "q4_mulc(" + r + ", " + std::to_string(c) + "u)";
            else if (zero_one_range(a)) e = "q4_mul01(" + l + ", " + r + ")";
            else if (zero_one_range(b)) e = "q4_mul01(" + r + ", " + l + ")";
            else e = "q4_mul(" + l + ", " + r + ")";
            break;
          case EQ: e = "q4_eq(" + l + ", " + r + ")"; break;
          case NE: e = "q4_ne(" + l + ", " + r + ")"; break;
          case LT: e = "q4_lt(" + l + ", " + r + ")"; break;
          case GT: e = "q4_gt(" + l + ", " + r + ")"; break;
          case LE: e = "q4_le(" + l + ", " + r + ")"; break;
          case GE: e = "q4_ge(" + l + ", " + r + ")"; break;
          case AND: e = "q4_and(" + bool4(p0) + ", " + bool4(p1) + ")"; break;
          case OR: e = "q4_or(" + bool4(p0) + ", " + bool4(p1) + ")"; break;
          case bAND: e = "q4_and(" + l + ", " + r + ")"; break;
          case bOR: e = "q4_or(" + l + ", " + r + ")"; break;
          case bXOR: e = "q4_xor(" + l + ", " + r + ")"; break;
          case MAX2: e = "q4_max(" + l + ", " + r + ")"; break;
          case MIN2: e = "q4_min(" + l + ", " + r + ")"; break;
          default: throw MapError("codegen: binary op without a packed form");
        }
        break;
      }
      case K_CONDITIONAL:
        e = "q4_sel(" + bool4(n->prev[0]) + ", " + val4(n->prev[1]) + ", " + val4(n->prev[2]) + ")";
        break;
      default:
        throw MapError(std::string("codegen: node kind ") + kind_name(n->kind) + " has no packed form");
    }
    if (R.wrap) e = "q4_wrap8(" + e + ")";
    return "const Q4 " + v + " = " + e + ";";
  }
  // inputs read at the centre cell only come from global memory as one word
  // (4-byte aligned rows, checked by quad_aligned)
  std::string center_loads4() const {
    std::ostringstream s;
    for (Node *p : plan.in_rasters) {
      if (!center_read.count(p)) continue;
      const int k = rin.at(p);
      if (staged.count(p)) s << "    const Q4 i" << k << " = " << tap4(p, 0, 0) << ";\n";
      else s << "    const Q4 i" << k << " = q4_bytes(ldr_q4_u8(a.in[" << k << "], x, y));\n";
    }
    return s.str();
  }
  std::string body4() const {
    std::ostringstream s;
    for (Node *n : g.nodes) s << "    " << stmt4(n) << "\n";
    return s.str();
  }
  // each output's address of the thread's first quad (ob<k>, pitch op<k>) is a
  // parameter; the quad of row kr below it takes one multiply-add
  std::string stores4() const {
    std::ostringstream s;
    int k = 0;
    for (auto &kv : outk)
      s << "    str_out_row<u32>(ob" << k << ", op" << k << ", kr, q4_pack_u8(" << val4(kv.first) << "));\n", k++;
    return s.str();
  }
  std::string out_params4() const {
    std::string s;
    for (size_t k = 0; k < outk.size(); k++) s += ", u64 ob" + std::to_string(k) + ", u32 op" + std::to_string(k);
    return s + ", int kr";
  }
  std::string out_bases4(const std::string &indent) const {
    std::ostringstream s;
    int k = 0;
    for (auto &kv : outk) {
      s << indent << "const u64 ob" << k << " = out_addr<u8>(a.out[" << kv.second << "], x, t.y0 + ly0);\n"
        << indent << "const u32 op" << k << " = (u32)a.out[" << kv.second << "].pitch;\n";
      k++;
    }
    return s.str();
  }
  std::string out_args4() const {
    std::string s;
    for (size_t k = 0; k < outk.size(); k++) s += ", ob" + std::to_string(k) + ", op" + std::to_string(k);
    return s;
  }
  // every output row, and every row of an input read from global memory, starts
  // on a 4-byte boundary (base and pitch)
  std::string quad_aligned() const {
    std::ostringstream s;
    s << "((0";
    for (auto &kv : outk) s << " | a.out[" << kv.second << "].p | (u64)a.out[" << kv.second << "].pitch";
    for (Node *p : plan.in_rasters)
      if (center_read.count(p) && !staged.count(p))
        s << " | a.in[" << rin.at(p) << "].p | (u64)a.in[" << rin.at(p) << "].pitch";
    s << ") & 3) == 0";
    return s.str();
  }

  // ---- per-node statements

  std::string stmt(Node *n, bool zonal_acc) const {
    std::ostringstream s;
    const std::string t = T(n);
    const std::string v = "v" + std::to_string(member.at(n));
    const int dt = n->meta.dtype;
    switch (n->kind) {
      case K_CONSTANT:
        s << "const " << t << " " << v << " = " << var_literal(reference_literal_value(n->cnst)) << ";";
        break;
      case K_INDEX:
        s << "const " << t << " " << v << " = (" << t << ")(" << (n->op == D1 ? "x" : "y") << ");";
        break;
      case K_RAND: {
        std::string c0 = v + "_c0", c1 = v + "_c1", k = v + "_k";
        s << "u32 " << c0 << " = (u32)(" << val(n->prev[0]) << "), " << c1 << " = 0u; ";
        s << "u32 " << k << " = (u32)(a.g.BS1 * (y / a.g.BS1) + a.g.BS0 * (x / a.g.BS0) + (y % a.g.BS1) * a.g.BS0 + (x % a.g.BS0)); ";
        s << "philox2x32_10(" << c0 << ", " << c1 << ", " << k << "); ";
        if (dt == F32) s << "const float " << v << " = (float)" << c0 << " / 4294967296.0f;";
        else if (dt_size(dt) <= 4 && dt != B8)
          s << "const " << t << " " << v << " = bit_cast8<" << t << ">(" << c0 << ");";
        else throw MapError("rand: unsupported output type");
        break;
      }
      case K_CAST:
        s << "const " << t << " " << v << " = (" << t << ")(" << val(n->prev[0]) << ");";
        break;
      case K_BARRIER:
        s << "const " << t << " " << v << " = " << val(n->prev[0]) << ";";
        break;
      case K_UNARY: {
        std::string p = val(n->prev[0]);
        int pdt = n->prev[0]->meta.dtype;
        switch (n->op) {
          case POS: s << "const " << t << " " << v << " = (" << t << ")(+" << p << ");"; break;
          case NEG: s << "const " << t << " " << v << " = (" << t << ")(-" << p << ");"; break;
          case NOT: s << "const " << t << " " << v << " = (" << t << ")(!" << p << ");"; break;
          case bNOT: s << "const " << t << " " << v << " = (" << t << ")(~" << p << ");"; break;
          default: {
            const char *fn = unary_fn(n->op);
            if (!fn) throw MapError("codegen: invalid unary op");
            auto mate = sincos_mate.find(n);
            if (mate != sincos_mate.end()) {
              if (sincos_first.count(n)) {
                Node *sn = n->op == SIN ? n : mate->second, *cn = n->op == COS ? n : mate->second;
                s << "float v" << member.at(sn) << ", v" << member.at(cn) << "; map_sincosf(" << p << ", &v" << member.at(sn)
                  << ", &v" << member.at(cn) << ");";
              }
              break;
            }
            if (dt_is_float(pdt)) {
              s << "const " << t << " " << v << " = " << float_fn_own(pdt, n->op) << "(" << p << ");";
            } else if (n->op == ABS) {
              s << "const " << t << " " << v << " = (" << t << ")(" << p << " < 0 ? -" << p << " : " << p << ");";
            } else if (n->op == CEIL || n->op == FLOOR || n->op == TRUNC || n->op == ROUND) {
              s << "const " << t << " " << v << " = " << p << ";";
            } else {
              s << "const " << t << " " << v << " = (" << t << ")" << fn << "((double)(" << p << "));";
            }
          }
        }
        break;
      }
      case K_BINARY: {
        std::string l = val(n->prev[0]), r = val(n->prev[1]);
        int pt = dt_promote(n->prev[0]->meta.dtype, n->prev[1]->meta.dtype);
        std::string pts = dt_ctype(pt);
        if (const char *sym = binary_sym(n->op)) {
          if (dt_is_float(pt) && (n->op == MOD || binary_is_bitwise(n->op)))
            throw MapError(std::string("binary op ") + binary_name(n->op) + " is not defined on floating types");
          // a 0 / 1 mask entering float arithmetic: a select gives the value the
          // integer-to-float conversion would, without the conversion
          if (dt_is_float(pt)) {
            if (!dt_is_float(n->prev[0]->meta.dtype) && zero_one(n->prev[0])) l = "(" + l + " ? (" + pts + ")1 : (" + pts + ")0)";
            if (!dt_is_float(n->prev[1]->meta.dtype) && zero_one(n->prev[1])) r = "(" + r + " ? (" + pts + ")1 : (" + pts + ")0)";
          }
          s << "const " << t << " " << v << " = (" << t << ")(" << l << " " << sym << " " << r << ");";
        } else {
          std::string L = "(" + pts + ")(" + l + ")", R = "(" + pts + ")(" + r + ")";
          switch (n->op) {
            case MAX2: s << "const " << t << " " << v << " = red_max<" << pts << ">(" << L << ", " << R << ");"; break;
            case MIN2: s << "const " << t << " " << v << " = red_min<" << pts << ">(" << L << ", " << R << ");"; break;
            case ATAN2: case POW: case HYPOT: case FMOD: {
              const char *fn = n->op == ATAN2 ? "atan2" : n->op == POW ? "pow" : n->op == HYPOT ? "hypot" : "fmod";
              if (n->op == ATAN2 && pt == F32)   // map_common.cuh's atan2 (<= 1.5 ulp, about half the instructions)
                s << "const " << t << " " << v << " = map_atan2f(" << L << ", " << R << ");";
              else if (dt_is_float(pt)) s << "const " << t << " " << v << " = " << float_fn(pt, fn) << "(" << L << ", " << R << ");";
              else s << "const " << t << " " << v << " = (" << t << ")" << fn << "((double)" << L << ", (double)" << R << ");";
              break;
            }
            default: throw MapError("codegen: invalid binary op");
          }
        }
        break;
      }
      case K_CONDITIONAL:
        s << "const " << t << " " << v << " = (" << val(n->prev[0]) << ") ? (" << t << ")(" << val(n->prev[1]) << ") : ("
          << t << ")(" << val(n->prev[2]) << ");";
        break;
      case K_NEIGHBOR:
        s << "const " << t << " " << v << " = " << tap(n->prev[0], n->coord.arr[0], n->coord.arr[1]) << ";";
        break;
      case K_CONVOLUTION: {
        // runtime/skeleton/FocalSkeleton.cpp:300-336: var = 0; var += in(y+i1, x+i0) * mask[i1+h1][i0+h0],
        // i1 outer, i0 inner; the mask is a correlation kernel (no flip).
        int hx = n->halo_x(), hy = n->halo_y(), mw = n->mask_ds.arr[0];
        s << t << " " << v << " = (" << t << ")0;";
        for (int i1 = -hy; i1 <= hy; i1++)
          for (int i0 = -hx; i0 <= hx; i0++)
            s << "\n    " << conv_term(v, "(" + t + ")", tap(n->prev[0], i0, i1), n->prev[0]->meta.dtype, n->meta.dtype,
                                       n->mask[(i1 + hy) * mw + (i0 + hx)], false);
        break;
      }
      case K_FOCALFUNC: {
        // FocalSkeleton.cpp:338-373: var = neutral; var = var OP in(y+i1, x+i0) over the window
        int hx = n->halo_x(), hy = n->halo_y();
        s << t << " " << v << " = " << var_literal(reduction_neutral(n->op, dt)) << ";";
        for (int i1 = -hy; i1 <= hy; i1++)
          for (int i0 = -hx; i0 <= hx; i0++)
            s << "\n    " << v << " = RedOp<" << n->op << ", " << t << ">::f(" << v << ", (" << t << ")"
              << tap(n->prev[0], i0, i1) << ");";
        break;
      }
      case K_FOCALPERCENT: {
        // FocalSkeleton.cpp:375-403: var = 0; var += (centre OP cell) over the
        // window; var /= window size, in the argument's type (OP: == for AGE,
        // > for ILE, util/PercentType.cpp). The window is centred on the cell and
        // the divisor is (2 hx + 1)(2 hy + 1): the reference's loop starts at the
        // centre (i = 0 .. 2h) and its divisor lacks parentheses, both defects.
        int hx = n->halo_x(), hy = n->halo_y();
        const char *cmp = n->op == 1 ? "==" : ">";
        s << t << " " << v << "_c = " << tap(n->prev[0], 0, 0) << "; " << t << " " << v << " = (" << t << ")0;";
        for (int i1 = -hy; i1 <= hy; i1++)
          for (int i0 = -hx; i0 <= hx; i0++)
            s << "\n    " << v << " = (" << t << ")(" << v << " + (" << t << ")(" << v << "_c " << cmp << " "
              << tap(n->prev[0], i0, i1) << "));";
        s << "\n    " << v << " = (" << t << ")(" << v << " / (" << t << ")" << (2 * hx + 1) * (2 * hy + 1) << ");";
        break;
      }
      case K_FOCALFLOW: {
        // FocalSkeleton.cpp:405-443: steepest descent among the 8 neighbours in the order
        // E, SE, S, SW, W, NW, N, NE; drop = (self - nbh) / dist with dist 1 or 1.414213f;
        // strictly greater than the running max (initially 0); code 1 << dir, 0 for none.
        static const int ox[8] = {1, 1, 0, -1, -1, -1, 0, 1}, oy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
        std::string it = T(n->prev[0]);
        s << it << " " << v << "_m = (" << it << ")0; int " << v << "_p = -1; const " << it << " " << v << "_s = "
          << tap(n->prev[0], 0, 0) << ";";
        for (int d = 0; d < 8; d++) {
          s << "\n    { const " << it << " zd = (" << it << ")(" << v << "_s - " << tap(n->prev[0], ox[d], oy[d]) << "); ";
          s << "const " << it << " ds = " << (d % 2 == 0 ? "(" + it + ")1" : "(" + it + ")1.414213f") << "; ";
          s << "const " << it << " dr = (" << it << ")(zd / ds); ";
          s << "if (dr > " << v << "_m) { " << v << "_m = dr; " << v << "_p = " << d << "; } }";
        }
        s << "\n    const u8 " << v << " = (" << v << "_p == -1) ? (u8)0 : (u8)(1 << " << v << "_p);";
        break;
      }
      case K_ZONALREDUC: {
        if (!zonal_acc) throw MapError("codegen: zonal reduction outside a zonal group");
        int z = -1;
        for (size_t i = 0; i < plan.zonal.size(); i++)
          if (plan.zonal[i] == n) z = (int)i;
        s << "acc" << z << " = RedOp<" << n->op << ", " << t << ">::f(acc" << z << ", (" << t << ")(" << val(n->prev[0])
          << "));";
        break;
      }
      default:
        throw MapError(std::string("codegen: node kind ") + kind_name(n->kind) + " cannot be computed per cell");
    }
    return s.str();
  }

  // `unordered`: Local / Focal cells, whose kernels never read their outputs (str_out)
  std::string stores(bool unordered = false) const {
    std::ostringstream s;
    for (auto &kv : outk) {
      Node *o = kv.first;
      s << "    " << (unordered ? "str_out<" : "str<") << T(o) << ">(a.out[" << kv.second << "], x, y, " << val(o) << ");\n";
    }
    return s.str();
  }

  std::string center_loads(bool from_struct) const {
    std::ostringstream s;
    for (Node *p : plan.in_rasters) {
      if (!center_read.count(p)) continue;
      int k = rin.at(p);
      std::string t = T(p);
      if (from_struct) s << "    const " << t << " i" << k << " = in.i" << k << ";\n";
      else if (staged.count(p)) s << "    const " << t << " i" << k << " = " << tap(p, 0, 0) << ";\n";
      else s << "    const " << t << " i" << k << " = ldr<" << t << ">(a.in[" << k << "], x, y);\n";
    }
    return s.str();
  }

  std::string body(bool zonal_acc) const {
    std::ostringstream s;
    for (Node *n : g.nodes) {
      if (replaced.count(n)) continue;
      s << "    " << (shade_at.count(n) ? shade_stmt(n, false) : stmt(n, zonal_acc)) << "\n";
    }
    return s.str();
  }

  std::string args_struct(int ntma, bool with_part) {
    // Every field is naturally aligned in declaration order, so these offsets
    // are the ones the device compiler assigns (checked by the size assertion).
    Layout L;
    plan.off_tm = ntma > 0 ? L.add("TmaDesc", "tm", 128, 64, ntma) : 0;
    if (!plan.in_rasters.empty()) plan.off_in = L.add("RasterArg", "in", 16, 8, (int)plan.in_rasters.size());
    if (!plan.out_rasters.empty()) plan.off_out = L.add("RasterArg", "out", 16, 8, (int)plan.out_rasters.size());
    if (!plan.scalars.empty()) plan.off_s = L.add("Scalar8", "s", 8, 8, (int)plan.scalars.size());
    plan.off_geom = L.add("Geom", "g", 48, 8, 0);
    plan.off_err = L.add("u32*", "err", 8, 8, 0);
    plan.off_aux = L.add("u64", "aux", 8, 8, 4);
    plan.aux_count = 4;
    (void)with_part;
    return L.finish("Args", plan.args_size);
  }
};

std::string fnv_hex(const std::string &s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) { h ^= c; h *= 1099511628211ull; }
  char b[17];
  snprintf(b, sizeof b, "%016llx", (unsigned long long)h);
  return b;
}

}  // namespace

// Local skeleton (runtime/skeleton/LocalSkeleton.cpp:31-180): a tile of TW x TH
// cells per CTA of NT threads; each thread owns TH*TW/NT cells of one column,
// issues all of its input loads first (memory-level parallelism), then
// evaluates the fused expression and stores the outputs.
// run_tile by linear tile index (the batched dispatcher's work items): the tile's
// coordinates from the index, then the tile's code
static std::string run_tile_by_index(int TW, int TH) {
  std::ostringstream s;
  s << "__device__ __forceinline__ bool run_tile(const Args &a, int tile, unsigned char *smem, u64 *bar, u32 &phase,\n"
    << "                                         bool gdesc) {\n"
    << "  return run_tile_t(a, tile_of<" << TW << ", " << TH << ">(a.g, tile), smem, bar, phase, gdesc);\n"
    << "}\n";
  return s.str();
}

static void gen_local(Gen &G, std::ostringstream &body, std::ostringstream &wrap) {
  KernelPlan &P = G.plan;
  const int TW = P.tile_w, TH = P.tile_h, NT = P.threads, R = TH * TW / NT;
  body << G.args_struct(0, false) << G.shade_decls();
  body << "struct In {\n";
  for (Node *p : P.in_rasters) body << "  " << G.T(p) << " i" << G.rin.at(p) << ";\n";
  body << "  int dummy;\n};\n";
  body << "__device__ __forceinline__ void load_cell(const Args &a, In &in, int x, int y) {\n";
  for (Node *p : P.in_rasters) {
    int k = G.rin.at(p);
    body << "  in.i" << k << " = ldr<" << G.T(p) << ">(a.in[" << k << "], x, y);\n";
  }
  body << "}\n";
  body << "__device__ __forceinline__ void compute_cell(const Args &a, const In &in, int x, int y) {\n";
  body << G.center_loads(true) << G.body(false) << G.stores(true) << "}\n";
  // 16-byte vector form: every raster of the group has one element size es,
  // V = 16 / es consecutive cells of a row per vector; full tiles whose rows start
  // on 16-byte boundaries load and store whole vectors and evaluate the cells
  // from their lanes (the same per-cell code), other tiles take the scalar path
  int es = 0;
  bool vec = !P.out_rasters.empty();
  for (Node *p : P.in_rasters) {
    const int s = (int)dt_size(p->meta.dtype);
    if (es && s != es) vec = false;
    es = s;
  }
  for (Node *p : P.out_rasters) {
    const int s = (int)dt_size(p->meta.dtype);
    if (es && s != es) vec = false;
    es = s;
  }
  const int V = es ? 16 / es : 0;
  const int TV = V ? TW / V : 0;                // threads per tile row
  if (!V || TW % V || TV == 0 || NT % TV || TH % (NT / TV)) vec = false;
  const int RV = vec ? TH / (NT / TV) : 0;      // vectors per thread
  if (vec) {
    body << "__device__ __forceinline__ void compute_cellr(const Args &a, const In &in, int x, int y" << G.out_params(false)
         << ") {\n" << G.center_loads(true) << G.body(false) << G.out_assigns() << "}\n";
  }
  body << "__device__ __forceinline__ bool run_tile_t(const Args &a, const Tile t, unsigned char *smem, u64 *bar,\n"
       << "                                           u32 &phase, bool gdesc) {\n";
  if (vec) {
    std::ostringstream align;
    align << "(t.x0 * " << es << ")";
    for (size_t k = 0; k < P.in_rasters.size(); k++) align << " | a.in[" << k << "].p | a.in[" << k << "].pitch";
    for (size_t k = 0; k < P.out_rasters.size(); k++) align << " | a.out[" << k << "].p | a.out[" << k << "].pitch";
    body << "  if (t.xe - t.x0 == " << TW << " && t.ye - t.y0 == " << TH << " && ((" << align.str() << ") & 15) == 0) {\n"
         << "    const int x = t.x0 + (threadIdx.x % " << TV << ") * " << V << ", ly0 = threadIdx.x / " << TV << ";\n";
    for (Node *p : P.in_rasters) body << "    uint4 w" << G.rin.at(p) << "[" << RV << "];\n";
    body << "#pragma unroll\n"
         << "    for (int r = 0; r < " << RV << "; ++r) {\n"
         << "      const int y = t.y0 + ly0 + r * " << NT / TV << ";\n";
    for (Node *p : P.in_rasters) {
      const int k = G.rin.at(p);
      body << "      w" << k << "[r] = __ldg((const uint4 *)(row_ptr<" << G.T(p) << ">(a.in[" << k << "], y) + x));\n";
    }
    body << "    }\n"
         << "#pragma unroll\n"
         << "    for (int r = 0; r < " << RV << "; ++r) {\n"
         << "      const int y = t.y0 + ly0 + r * " << NT / TV << ";\n";
    int o = 0;
    for (size_t k = 0; k < G.outk.size(); k++) body << "      uint4 q" << k << ";\n";
    body << "#pragma unroll\n"
         << "      for (int j = 0; j < " << V << "; ++j) {\n"
         << "        In in;\n";
    for (Node *p : P.in_rasters) {
      const int k = G.rin.at(p);
      body << "        in.i" << k << " = vlane<" << G.T(p) << ">(w" << k << "[r], j);\n";
    }
    o = 0;
    std::ostringstream rargs;
    for (auto &kv : G.outk) {
      body << "        " << G.T(kv.first) << " r" << o << ";\n";
      rargs << ", r" << o;
      o++;
    }
    body << "        compute_cellr(a, in, x + j, y" << rargs.str() << ");\n";
    o = 0;
    for (auto &kv : G.outk) {
      body << "        vset<" << G.T(kv.first) << ">(q" << o << ", j, r" << o << ");\n";
      o++;
    }
    body << "      }\n";
    o = 0;
    for (auto &kv : G.outk) {
      body << "      *(uint4 *)((" << G.T(kv.first) << " *)(a.out[" << kv.second << "].p + (u64)(s64)y * (u64)a.out[" << kv.second
           << "].pitch) + x) = q" << o << ";\n";
      o++;
    }
    body << "    }\n"
         << "    return true;\n"
         << "  }\n";
  }
  body << "  const int lx = threadIdx.x % " << TW << ", ly0 = threadIdx.x / " << TW << ";\n"
       << "  const int x = t.x0 + lx;\n"
       << "  In in[" << R << "];\n"
       << "#pragma unroll\n"
       << "  for (int k = 0; k < " << R << "; ++k) {\n"
       << "    const int y = t.y0 + ly0 + k * " << NT / TW << ";\n"
       << "    if (x < t.xe && y < t.ye) load_cell(a, in[k], x, y);\n"
       << "  }\n"
       << "#pragma unroll\n"
       << "  for (int k = 0; k < " << R << "; ++k) {\n"
       << "    const int y = t.y0 + ly0 + k * " << NT / TW << ";\n"
       << "    if (x < t.xe && y < t.ye) compute_cell(a, in[k], x, y);\n"
       << "  }\n"
       << "  return true;\n"
       << "}\n";
  body << run_tile_by_index(TW, TH);
  // launched as a dependent launch over the region's tiles in two dimensions:
  // no global access before griddep_wait
  wrap << "extern \"C\" __global__ void __launch_bounds__(" << NT << ") KNAME(const __grid_constant__ Args a) {\n"
       << "  u32 phase = 0;\n"
       << "  griddep_launch();\n"
       << "  griddep_wait();\n"
       << "  run_tile_t(a, tile_at<" << TW << ", " << TH << ">(a.g, blockIdx.x, blockIdx.y), nullptr, nullptr, phase, false);\n"
       << "}\n";
}

// Focal skeleton (runtime/skeleton/FocalSkeleton.cpp:37-274). A tile whose halo
// lies inside the raster is staged into shared memory by one 2-D TMA load per
// focal input (box TW + 2*pad_x by TH + 2*halo, x start rounded down to a
// 16-byte boundary), completion tracked by an mbarrier with a bounded wait; the
// taps then read shared memory. Tiles that touch the raster edge read their taps
// straight from global memory through the border rule (GatherTap), which also
// carries the reference's block-relative mirror.
static void gen_focal(Gen &G, std::ostringstream &body, std::ostringstream &wrap) {
  KernelPlan &P = G.plan;
  const int TW = P.tile_w, TH = P.tile_h, NT = P.threads;
  const int hx = P.halo_x, hy = P.halo_y;
  const int nst = (int)G.staged.size();
  std::vector<Node *> staged_nodes(nst);
  for (auto &kv : G.staged) staged_nodes[kv.second] = kv.first;
  size_t off = 0;
  for (int k = 0; k < nst; k++) {
    Node *in = staged_nodes[k];
    TmaSpec t;
    t.in_index = G.rin.at(in);
    t.dtype = in->meta.dtype;
    int es = (int)dt_size(t.dtype);
    int align_e = 16 / es;
    t.pad_x = ((hx + align_e - 1) / align_e) * align_e;
    t.box_w = TW + 2 * t.pad_x;
    t.box_h = TH + 2 * hy;
    off = (off + 127) / 128 * 128;
    t.smem_off = off;
    off += (size_t)t.box_w * t.box_h * es;
    t.halo_y = hy;
    P.tma.push_back(t);
  }
  // output tile store: the single output's TW x TH tile staged after the inputs
  // (by default for the fast hillshade form, whose interior tiles keep their
  // results in registers one cell per thread step, the form the store serves)
  const FocalTune &ft0 = focal_tune();
  if (P.tile_store && nst > 0 && G.outk.size() == 1 &&
      (ft0.tstore >= 2 || (ft0.tstore == 1 && G.any_fast() && !ft0.fpair && !ft0.cpair))) {
    Node *o = G.outk.begin()->first;
    const int es = (int)dt_size(o->meta.dtype);
    if ((TW * es) % 16 == 0) {
      TmaSpec t;
      t.in_index = G.outk.begin()->second;
      t.dtype = o->meta.dtype;
      t.box_w = TW;
      t.box_h = TH;
      off = (off + 127) / 128 * 128;
      t.smem_off = off;
      off += (size_t)TW * TH * es;
      P.tma_out.push_back(t);
    }
  }
  off = (off + 15) / 16 * 16;
  const size_t bar_off = off;
  bool use_tma = nst > 0 && hx <= 16 && hy <= 16;
  for (auto &t : P.tma)
    if (t.box_w > 256 || t.box_h > 256) use_tma = false;
  if (use_tma && off + 16 > 200 * 1024) use_tma = false;
  if (!use_tma) P.tma_out.clear();
  P.smem_bytes = use_tma ? off + 16 : 0;
  P.bar_off = bar_off;
  body << G.args_struct(use_tma ? nst + (int)P.tma_out.size() : 0, false) << G.shade_decls();
  body << "template <";
  for (int k = 0; k < nst; k++) body << (k ? ", " : "") << "class F" << k;
  body << ">\n__device__ __forceinline__ void focal_cell(const Args &a";
  for (int k = 0; k < nst; k++) body << ", const F" << k << " &f" << k;
  body << ", int x, int y, int lx, int ly) {\n";
  body << G.center_loads(false) << G.body(false) << G.stores(true) << "}\n";
  std::ostringstream call, call2;
  call << "focal_cell(a";
  call2 << "focal_cell2(a";
  for (int k = 0; k < nst; k++) call << ", f" << k;
  for (int k = 0; k < nst; k++) call2 << ", f" << k;
  call << ", x, y, lx, ly)";
  call2 << ", x, y, lx, ly)";
  // Each thread computes `rows` consecutive rows of one column, so the taps of
  // neighbouring cells in the column are the same shared-memory words (loaded
  // once when the loop is unrolled); a warp still covers 32 consecutive columns.
  const int rows = TH * TW / NT;
  bool heavy = false;   // bodies with library math functions unroll by 2 only (code size)
  for (Node *n : G.g.nodes)
    if (!G.replaced.count(n) && ((n->kind == K_UNARY && n->op >= SIN && n->op <= CBRT) ||
                                 (n->kind == K_BINARY && (n->op == ATAN2 || n->op == POW || n->op == HYPOT || n->op == FMOD))))
      heavy = true;
  // Float-heavy bodies, and bodies with a rewritten shading composition, compute
  // the cells of two consecutive rows together (PR<T> pairs: packed f32x2
  // arithmetic, one issue slot for both cells).
  // (the fast shading form runs one cell at a time: paired it measured no faster,
  // 434 against 437 Gcells/s on the 16384^2 hillshade)
  const bool pair = (heavy || (!G.shades.empty() && (!G.any_fast() || focal_tune().fpair))) && rows % 2 == 0 &&
                    Runtime::get().paired_cells && G.pairable();
  // Column pairs: the two cells of a pair are (x, y) and (x + 1, y) of one row,
  // so one 8-byte shared-memory load serves both cells' taps (tap2c) and their
  // results leave in one 8-byte store; each thread then covers two columns and
  // R = TH * TW / (2 NT) rows. For staged float inputs.
  bool all_f32 = nst > 0;
  for (Node *in : staged_nodes) all_f32 = all_f32 && in->meta.dtype == F32;
  const int cw = TW / 2;
  const bool cpair = pair && focal_tune().cpair && all_f32 && TW % 2 == 0 && cw <= NT && NT % cw == 0 && (TH * cw) % NT == 0;
  if (cpair) {
    G.pdx = 1;
    G.pdy = 0;
  }
  const int R = cpair ? TH * cw / NT : rows;   // rows per thread
  const std::string tmap = cpair ? "    const int lx = 2 * (threadIdx.x % " + std::to_string(cw) + "), ly0 = (threadIdx.x / " +
                                       std::to_string(cw) + ") * " + std::to_string(R) + ";\n"
                                 : "    const int lx = threadIdx.x % " + std::to_string(TW) + ", ly0 = (threadIdx.x / " +
                                       std::to_string(TW) + ") * " + std::to_string(rows) + ";\n";
  if (pair) {
    body << "template <";
    for (int k = 0; k < nst; k++) body << (k ? ", " : "") << "class F" << k;
    body << ">\n__device__ __forceinline__ void focal_cell2(const Args &a";
    for (int k = 0; k < nst; k++) body << ", const F" << k << " &f" << k;
    body << ", int x, int y, int lx, int ly) {\n";
    body << G.center_loads2() << G.body2() << G.stores2() << "}\n";
  }
  const FocalTune &tune = focal_tune();
  // Integer bodies on byte rasters compute four cells of a row per thread step as
  // 16-bit lanes (Q4) on interior tiles: one shared-memory word holds the taps of
  // four cells and one operation serves two cells.
  const int qw = TW / 4;
  const bool quad = !pair && use_tma && Runtime::get().paired_cells && TW % 4 == 0 && qw <= NT && NT % qw == 0 &&
                    (TH * qw) % NT == 0 && G.quadable();
  const int qrows = quad ? TH * qw / NT : 0;
  if (quad) {
    body << "template <";
    for (int k = 0; k < nst; k++) body << (k ? ", " : "") << "class F" << k;
    body << ">\n__device__ __forceinline__ void focal_cell4(const Args &a";
    for (int k = 0; k < nst; k++) body << ", const F" << k << " &f" << k;
    body << ", int x, int y, int lx, int ly" << G.out_params4() << ") {\n";
    body << G.center_loads4() << G.body4() << G.stores4() << "}\n";
  }
  const bool full_unroll = tune.unroll ? tune.unroll >= R : !heavy;
  const std::string unroll = tune.unroll ? "#pragma unroll " + std::to_string(tune.unroll) + "\n"
                                         : heavy ? (pair ? "#pragma unroll 1\n" : "#pragma unroll 2\n") : "#pragma unroll\n";
  const int step = pair && !cpair ? 2 : 1;
  // Interior tiles of a fully unrolled row loop keep the thread's results in
  // registers and store them after the last cell: no store then lies between
  // two loads of the same staged tap, which therefore load once per thread.
  const int nout = (int)G.outk.size();
  const bool defer = tune.defer && full_unroll && nout > 0 && R * nout <= 32;
  // with fast shading compositions, interior tiles first compute their cells
  // recording only whether one needs the literal chain (flag form), and redo
  // the thread's cells with the per-cell checks when one did
  const bool flagged = defer && G.any_fast();
  if (defer) {
    for (int nc = 0; nc < (flagged ? 2 : 1); nc++)
      for (int pf = 0; pf < (pair ? 2 : 1); pf++) {
        body << "template <";
        for (int k = 0; k < nst; k++) body << (k ? ", " : "") << "class F" << k;
        body << ">\n__device__ __forceinline__ void " << (pf ? "focal_cell2r" : "focal_cellr") << (nc ? "_nc" : "")
             << "(const Args &a";
        for (int k = 0; k < nst; k++) body << ", const F" << k << " &f" << k;
        body << ", int x, int y, int lx, int ly" << G.out_params(pf) << (nc ? ", u32 &bad" : "") << ") {\n";
        G.fast_flag = nc == 1;
        body << (pf ? G.center_loads2() + G.body2() : G.center_loads(false) + G.body(false)) << G.out_assigns() << "}\n";
        G.fast_flag = false;
      }
  }
  std::ostringstream loop, loop_full;
  loop << tmap
       << "    const int x = t.x0 + lx;\n"
       << unroll
       << "    for (int k = 0; k < " << R << "; k += " << step << ") {\n"
       << "      const int ly = ly0 + k, y = t.y0 + ly;\n";
  if (cpair)
    loop << "      if (y < t.ye) {\n"
         << "        if (x + 1 < t.xe) " << call2.str() << ";\n"
         << "        else if (x < t.xe) " << call.str() << ";\n"
         << "      }\n";
  else if (pair)
    loop << "      if (x < t.xe) {\n"
         << "        if (y + 1 < t.ye) " << call2.str() << ";\n"
         << "        else if (y < t.ye) " << call.str() << ";\n"
         << "      }\n";
  else
    loop << "      if (x < t.xe && y < t.ye) " << call.str() << ";\n";
  loop << "    }\n";
  // interior tiles are full: every cell of the tile is inside the raster
  loop_full << tmap << "    const int x = t.x0 + lx;\n";
  if (defer) {
    std::ostringstream callr, outs;
    callr << (pair ? "focal_cell2r(a" : "focal_cellr(a");
    for (int k = 0; k < nst; k++) callr << ", f" << k;
    callr << ", x, y, lx, ly";
    int k = 0;
    std::ostringstream bases;   // each output's address of the thread's first cell
    for (auto &kv : G.outk) {
      const std::string ty = G.T(kv.first);
      loop_full << "    " << (pair ? "PR<" + ty + ">" : ty) << " r" << k << "[" << R / step << "];\n";
      callr << ", r" << k << "[k / " << step << "]";
      const std::string o = std::to_string(kv.second);
      if (cpair)
        outs << "      str_out2x<" << ty << ">(a.out[" << o << "], x, y, lane0(r" << k << "[k]), lane1(r" << k
             << "[k]));\n";
      else if (pair) {
        bases << "    const u64 ob" << k << " = out_addr<" << ty << ">(a.out[" << o << "], x, t.y0 + ly0);\n"
              << "    const u32 op" << k << " = (u32)a.out[" << o << "].pitch;\n";
        outs << "      str_out_row<" << ty << ">(ob" << k << ", op" << k << ", k, lane0(r" << k << "[k / 2]));\n"
             << "      str_out_row<" << ty << ">(ob" << k << ", op" << k << ", k + 1, lane1(r" << k << "[k / 2]));\n";
      } else {
        bases << "    const u64 ob" << k << " = out_addr<" << ty << ">(a.out[" << o << "], x, t.y0 + ly0);\n"
              << "    const u32 op" << k << " = (u32)a.out[" << o << "].pitch;\n";
        outs << "      str_out_row<" << ty << ">(ob" << k << ", op" << k << ", k, r" << k << "[k]);\n";
      }
      k++;
    }
    callr << ")";
    if (flagged) {
      std::string cnc = callr.str();
      cnc.insert(cnc.find('('), "_nc");
      cnc.insert(cnc.size() - 1, ", bad");
      loop_full << "    u32 bad = 0u;\n"
                << "#pragma unroll\n"
                << "    for (int k = 0; k < " << R << "; k += " << step << ") {\n"
                << "      const int ly = ly0 + k, y = t.y0 + ly;\n"
                << "      " << cnc << ";\n"
                << "    }\n"
                << "    if (bad >= 0x7f800000u) {\n";
    }
    loop_full << "#pragma unroll\n"
              << "    for (int k = 0; k < " << R << "; k += " << step << ") {\n"
              << "      const int ly = ly0 + k, y = t.y0 + ly;\n"
              << "      " << callr.str() << ";\n"
              << "    }\n";
    if (flagged) loop_full << "    }\n";
    // output tile store (opt-in; whole-raster outputs, full tiles): the results
    // go to the staging tile, then one thread stores it with one TMA copy
    const bool tstore = !P.tma_out.empty() && !pair && !cpair;
    if (tstore) {
      const TmaSpec &to = P.tma_out[0];
      const std::string ty = G.T(G.outk.begin()->first);
      loop_full << "    if (a.aux[2] != 0 && t.xe == t.x0 + " << TW << " && t.ye == t.y0 + " << TH << ") {\n"
                << "      " << ty << " *os = (" << ty << " *)(smem + " << to.smem_off << ");\n"
                << "#pragma unroll\n"
                << "      for (int k = 0; k < " << R << "; k++) os[(ly0 + k) * " << TW << " + lx] = r0[k];\n"
                << "      fence_proxy_async();\n"
                << "      __syncthreads();\n"
                << "      if (threadIdx.x == 0) {\n"
                << "        tma_store_2d(&a.tm[" << nst << "], os, t.x0, t.y0 - a.g.oy);\n"
                << "        bulk_commit_group();\n"
                << "        bulk_wait_group_read0();\n"
                << "      }\n"
                << "    } else {\n";
    }
    loop_full << bases.str()
              << "#pragma unroll\n"
              << "    for (int k = 0; k < " << R << "; k += " << step << ") {\n"
              << "      const int y = t.y0 + ly0 + k;\n"
              << outs.str()
              << "    }\n";
    if (tstore) loop_full << "    }\n";
  } else {
    loop_full << unroll
              << "    for (int k = 0; k < " << R << "; k += " << step << ") {\n"
              << "      const int ly = ly0 + k, y = t.y0 + ly;\n"
              << "      " << (pair ? call2.str() : call.str()) << ";\n"
              << "    }\n";
  }
  std::string loop_edge;   // staged edge tiles (default: the one-cell loop)
  if (quad) {
    // thread t: cells 4 (t % qw) .. + 3 of rows (t / qw) * qrows .. + qrows - 1;
    // outputs whose rows are not 4-byte aligned take the one-cell form
    std::ostringstream q;
    q << "    const int lx = 4 * (threadIdx.x % " << qw << "), ly0 = (threadIdx.x / " << qw << ") * " << qrows << ";\n"
      << "    const int x = t.x0 + lx;\n"
      << "    if (" << G.quad_aligned() << ") {\n"
      << G.out_bases4("      ")
      << "#pragma unroll\n"
      << "      for (int k = 0; k < " << qrows << "; k++) {\n"
      << "        const int ly = ly0 + k, y = t.y0 + ly;\n"
      << "        focal_cell4(a";
    for (int k = 0; k < nst; k++) q << ", f" << k;
    q << ", x, y, lx, ly" << G.out_args4() << ", k);\n"
      << "      }\n"
      << "    } else {\n"
      << "      for (int k = 0; k < " << qrows << "; k++)\n"
      << "        for (int c = 0; c < 4; c++) {\n"
      << "          const int ly = ly0 + k, y = t.y0 + ly;\n"
      << "          focal_cell(a";
    for (int k = 0; k < nst; k++) q << ", f" << k;
    q << ", x + c, y, lx + c, ly);\n"
      << "        }\n"
      << "    }\n";
    loop_full.str(q.str());
    // staged edge tiles: whole quads inside the region in the packed form, the
    // cells of a quad that crosses the region's end one at a time
    std::ostringstream e;
    e << "    const int lx = 4 * (threadIdx.x % " << qw << "), ly0 = (threadIdx.x / " << qw << ") * " << qrows << ";\n"
      << "    const int x = t.x0 + lx;\n"
      << "    const bool al = " << G.quad_aligned() << ";\n"
      << G.out_bases4("    ")
      << "#pragma unroll\n"
      << "    for (int k = 0; k < " << qrows << "; k++) {\n"
      << "      const int ly = ly0 + k, y = t.y0 + ly;\n"
      << "      if (y >= t.ye) continue;\n"
      << "      if (al && x + 3 < t.xe) {\n"
      << "        focal_cell4(a";
    for (int k = 0; k < nst; k++) e << ", f" << k;
    e << ", x, y, lx, ly" << G.out_args4() << ", k);\n"
      << "      } else {\n"
      << "        for (int c = 0; c < 4; c++)\n"
      << "          if (x + c < t.xe) focal_cell(a";
    for (int k = 0; k < nst; k++) e << ", f" << k;
    e << ", x + c, y, lx + c, ly);\n"
      << "      }\n"
      << "    }\n";
    loop_edge = e.str();
  }
  // gdesc: the Args (and their tensor maps) live in global memory (batched dispatch)
  body << "__device__ __forceinline__ bool run_tile_t(const Args &a, const Tile t, unsigned char *smem, u64 *bar,\n"
       << "                                           u32 &phase, bool gdesc) {\n";
  if (use_tma) {
    size_t total = 0;
    for (auto &t : P.tma) total += (size_t)t.box_w * t.box_h * dt_size(t.dtype);
    // interior and edge tiles are staged by TMA (zero fill outside the map, then
    // the border rule: dead, raster mirror, or the raster mirror plus the
    // block-mirror exceptions recomputed afterwards); a tiled TMA copy must start
    // on a 16-byte boundary in x: tiles whose origin is not a multiple of the
    // staged types' alignment (plain-mode blocks of odd widths) take the gather path
    int align_e = 1;
    for (auto &t : P.tma) align_e = std::max(align_e, 16 / (int)dt_size(t.dtype));
    body << "  const bool inner = tile_interior<" << TW << ", " << TH << ">(a.g, t, " << hx << ", " << hy << ");\n"
         << "  if (t.x0 % " << align_e << " == 0) {\n"
         << "    if (gdesc) __syncthreads();   // a persistent CTA: earlier readers of the staging buffer are done\n"
         << "    if (threadIdx.x == 0) {\n"
         << "      fence_proxy_async();\n";
    for (int k = 0; k < nst; k++) body << "      if (gdesc) tensormap_acquire(&a.tm[" << k << "]);\n";
    body << "      mbar_arrive_expect_tx(bar, " << total << "u);\n";
    for (int k = 0; k < nst; k++) {
      auto &t = P.tma[k];
      body << "      tma_load_2d(smem + " << t.smem_off << ", &a.tm[" << k << "], bar, t.x0 - " << t.pad_x << ", t.y0 - " << hy
           << " - a.g.oy);\n";
    }
    body << "    }\n"
         << "    if (!mbar_wait_bounded(bar, phase, 1u << 14)) {\n"
         << "      skel_fail(a.err, ERR_TMA_TIMEOUT);\n"
         << "      mbar_wait_bounded(bar, phase, 1u << 14);\n"
         << "      return false;\n"
         << "    }\n"
         << "    phase ^= 1u;\n"
         << "    if (!inner) {\n";
    for (int k = 0; k < nst; k++) {
      auto &t = P.tma[k];
      std::string ty = dt_ctype(t.dtype);
      body << "      stage_fix_border<" << ty << ", " << t.box_w << ", " << t.box_h << ">((" << ty << " *)(smem + " << t.smem_off
           << "), a.g, t.x0 - " << t.pad_x << ", t.y0 - " << hy << ", " << hx << ", " << hy << ");\n";
    }
    body << "      __syncthreads();\n"
         << "    }\n";
    for (int k = 0; k < nst; k++) {
      auto &t = P.tma[k];
      std::string ty = dt_ctype(t.dtype);
      body << "    const SmemTap<" << ty << ", " << t.box_w << ", " << t.pad_x << ", " << hy << "> f" << k << "{(const " << ty
           << " *)(smem + " << t.smem_off << ")};\n";
    }
    if (loop_edge.empty()) loop_edge = loop.str();
    // block-mirror exceptions of staged edge tiles, recomputed by the same
    // threads (after their own stores of the same cells) from global memory
    {
      std::ostringstream fx;
      fx << "      if (block_fixup(a.g)) {\n";
      for (int k = 0; k < nst; k++) {
        std::string ty = G.T(staged_nodes[k]);
        fx << "        const GatherTap<" << ty << "> g" << k << "{a.in[" << G.rin.at(staged_nodes[k]) << "], &a.g};\n";
      }
      std::string call1 = "focal_cell(a";
      for (int k = 0; k < nst; k++) call1 += ", g" + std::to_string(k);
      if (quad) {
        fx << "        const int lx = 4 * (threadIdx.x % " << qw << "), ly0 = (threadIdx.x / " << qw << ") * " << qrows << ";\n"
           << "        for (int k = 0; k < " << qrows << "; k++)\n"
           << "          for (int c = 0; c < 4; c++) {\n"
           << "            const int x = t.x0 + lx + c, y = t.y0 + ly0 + k;\n"
           << "            if (x < t.xe && y < t.ye && block_exception(a.g, x, y, " << hx << ", " << hy << "))\n"
           << "              " << call1 << ", x, y, lx + c, ly0 + k);\n"
           << "          }\n";
      } else if (cpair) {
        fx << tmap
           << "        for (int k = 0; k < " << R << "; k++)\n"
           << "          for (int c = 0; c < 2; c++) {\n"
           << "            const int x = t.x0 + lx + c, y = t.y0 + ly0 + k;\n"
           << "            if (x < t.xe && y < t.ye && block_exception(a.g, x, y, " << hx << ", " << hy << "))\n"
           << "              " << call1 << ", x, y, lx + c, ly0 + k);\n"
           << "          }\n";
      } else {
        fx << tmap
           << "        const int x = t.x0 + lx;\n"
           << "        for (int k = 0; k < " << rows << "; k++) {\n"
           << "          const int y = t.y0 + ly0 + k;\n"
           << "          if (x < t.xe && y < t.ye && block_exception(a.g, x, y, " << hx << ", " << hy << "))\n"
           << "            " << call1 << ", x, y, lx, ly0 + k);\n"
           << "        }\n";
      }
      fx << "      }\n";
      loop_edge += fx.str();
    }
    body << "    if (inner) {\n" << loop_full.str() << "    } else {\n" << loop_edge << "    }\n"
         << "    return true;\n  }\n";
  }
  body << "  {\n";
  for (int k = 0; k < nst; k++) {
    std::string ty = G.T(staged_nodes[k]);
    body << "    const GatherTap<" << ty << "> f" << k << "{a.in[" << G.rin.at(staged_nodes[k]) << "], &a.g};\n";
  }
  body << loop.str() << "  }\n  return true;\n}\n";
  body << run_tile_by_index(TW, TH);
  wrap << "extern \"C\" __global__ void __launch_bounds__(" << NT;
  const int minb = tune.minb > 0 ? tune.minb : G.plan.min_blocks;
  if (minb > 0) wrap << ", " << minb;
  wrap << ") KNAME(const __grid_constant__ Args a) {\n"
       << "  extern __shared__ __align__(128) unsigned char smem[];\n"
       << "  u32 phase = 0;\n";
  // launched as a dependent launch: the barrier set-up overlaps the previous
  // kernel's last CTAs, and no global access comes before griddep_wait
  if (use_tma)
    wrap << "  u64 *bar = (u64 *)(smem + " << bar_off << ");\n"
         << "  if (threadIdx.x == 0) { mbar_init(bar, 1); fence_mbar_init(); }\n"
         << "  griddep_launch();\n"
         << "  __syncthreads();\n"
         << "  griddep_wait();\n"
         << "  run_tile_t(a, tile_at<" << TW << ", " << TH << ">(a.g, blockIdx.x, blockIdx.y), smem, bar, phase, false);\n";
  else
    wrap << "  griddep_launch();\n"
         << "  griddep_wait();\n"
         << "  run_tile_t(a, tile_at<" << TW << ", " << TH << ">(a.g, blockIdx.x, blockIdx.y), smem, nullptr, phase, false);\n";
  wrap << "}\n";
  if (!use_tma) {
    P.tma.clear();
    P.tma_out.clear();
  }
}

static std::string gen_zonal(Gen &G) {
  KernelPlan &P = G.plan;
  const int TW = P.tile_w, TH = P.tile_h, NT = P.threads;
  std::ostringstream s;
  s << "#include \"map_common.cuh\"\n";
  s << G.args_struct(0, true);
  for (Node *n : G.g.nodes)
    if (n->kind == K_ZONALREDUC) P.zonal.push_back(n);
  const int nz = (int)P.zonal.size();
  // cell: updates the accumulators
  s << "__device__ __forceinline__ void zonal_cell(const Args &a, int x, int y";
  for (int z = 0; z < nz; z++) s << ", " << G.T(P.zonal[z]) << " &acc" << z;
  s << ") {\n" << G.center_loads(false) << G.body(true) << G.stores() << "}\n";
  // main kernel: tiles strided over the grid, per-thread accumulation, CTA reduction, one partial per CTA.
  // aux[0] = partials (Scalar8[slot * nz + z]), aux[1] = first slot of this launch
  s << "extern \"C\" __global__ void __launch_bounds__(" << NT << ") KNAME(const __grid_constant__ Args a) {\n"
    << "  __shared__ Scalar8 scratch[" << NT / 32 << "];\n";
  for (int z = 0; z < nz; z++) {
    Node *n = P.zonal[z];
    s << "  " << G.T(n) << " acc" << z << " = " << var_literal(reduction_neutral(n->op, n->meta.dtype)) << ";\n";
  }
  s << "  const int lx = threadIdx.x % " << TW << ", ly0 = threadIdx.x / " << TW << ";\n"
    << "  for (int ti = blockIdx.x; ti < a.g.tiles; ti += gridDim.x) {\n"
    << "    const Tile t = tile_of<" << TW << ", " << TH << ">(a.g, ti);\n"
    << "    const int x = t.x0 + lx;\n"
    << "#pragma unroll 4\n"
    << "    for (int k = 0; k < " << TH * TW / NT << "; ++k) {\n"
    << "      const int y = t.y0 + ly0 + k * " << NT / TW << ";\n"
    << "      if (x < t.xe && y < t.ye) zonal_cell(a, x, y";
  for (int z = 0; z < nz; z++) s << ", acc" << z;
  s << ");\n    }\n  }\n"
    << "  Scalar8 *part = (Scalar8 *)a.aux[0];\n"
    << "  const u64 slot = a.aux[1] + blockIdx.x;\n";
  for (int z = 0; z < nz; z++) {
    Node *n = P.zonal[z];
    s << "  { const " << G.T(n) << " r = block_reduce<" << n->op << ", " << G.T(n) << ">(acc" << z << ", scratch);\n"
      << "    if (threadIdx.x == 0) put_scalar<" << G.T(n) << ">(&part[slot * " << nz << " + " << z << "], r); }\n";
  }
  s << "}\n";
  // finalisation: one CTA folds every partial in slot order, deterministically
  s << "struct FinalArgs { u64 part; s64 nslots; u64 res; u64 pad; };\n";
  P.final_args_size = 32;
  s << "extern \"C\" __global__ void __launch_bounds__(" << NT << ") KNAME_final(const __grid_constant__ FinalArgs f) {\n"
    << "  __shared__ Scalar8 scratch[" << NT / 32 << "];\n"
    << "  const Scalar8 *part = (const Scalar8 *)f.part;\n"
    << "  Scalar8 *res = (Scalar8 *)f.res;\n";
  for (int z = 0; z < nz; z++) {
    Node *n = P.zonal[z];
    std::string t = G.T(n);
    s << "  { " << t << " acc = " << var_literal(reduction_neutral(n->op, n->meta.dtype)) << ";\n"
      << "    for (s64 i = threadIdx.x; i < f.nslots; i += blockDim.x) acc = RedOp<" << n->op << ", " << t
      << ">::f(acc, get_scalar<" << t << ">(part[i * " << nz << " + " << z << "]));\n"
      << "    const " << t << " r = block_reduce<" << n->op << ", " << t << ">(acc, scratch);\n"
      << "    if (threadIdx.x == 0) put_scalar<" << t << ">(&res[" << z << "], r); }\n";
  }
  s << "}\n";
  return s.str();
}

// Radiating skeleton (runtime/skeleton/RadiatingSkeleton.cpp:32-323): one CTA per
// octant sweeps the fronts d0 = 1, 2, ... in order; a front's cells are spread over
// the CTA's threads. A cell's scan value is op(LIT(front d0-1 at d1, at d1-1), in)
// when `in` is finite; the start cell holds the neutral value. The previous front
// is read back (L1-bypassing loads) from the scan's own output raster, written by
// this CTA one step earlier; cells on an octant boundary are written by both
// adjacent octants with identical values. Local nodes before the scan produce
// `in` per cell; those after it run right after the cell's scan value.
static std::string gen_radial(Gen &G) {
  KernelPlan &P = G.plan;
  Node *scan = P.core;
  const std::string T = G.T(scan);
  const std::string v = G.val(scan);
  const std::string nt = var_literal(reduction_neutral(scan->op, scan->meta.dtype));
  std::ostringstream s;
  s << "#include \"map_scan.cuh\"\n" << G.args_struct(0, false);
  // the centre inputs of one cell, loaded ahead of its computation
  s << "struct In {\n";
  for (Node *p : P.in_rasters)
    if (G.center_read.count(p)) s << "  " << G.T(p) << " i" << G.rin.at(p) << ";\n";
  s << "  int dummy;\n};\n";
  s << "__device__ __forceinline__ void radial_load(const Args &a, In &in, int x, int y) {\n";
  for (Node *p : P.in_rasters)
    if (G.center_read.count(p)) {
      const int k = G.rin.at(p);
      s << "  in.i" << k << " = ldr<" << G.T(p) << ">(a.in[" << k << "], x, y);\n";
    }
  s << "}\n";
  s << "__device__ __forceinline__ " << T << " radial_cell(const Args &a, const In &in, int x, int y, " << T
    << " lit, bool observer) {\n"
    << G.center_loads(true);
  for (Node *n : G.g.nodes) {
    if (n == scan) {
      s << "    " << T << " " << v << " = lit;\n"
        << "    if (observer) " << v << " = " << nt << ";\n"
        << "    else if (isfinite((double)(" << G.val(scan->prev[0]) << "))) " << v << " = RedOp<" << scan->op << ", " << T
        << ">::f(" << v << ", (" << T << ")(" << G.val(scan->prev[0]) << "));\n";
    } else {
      s << "    " << G.stmt(n, false) << "\n";
    }
  }
  s << G.stores() << "    return " << v << ";\n}\n";
  int ri = G.outk.at(scan);
  // aux[0] start x, aux[1] start y, aux[2] last front (or -1 for all).
  // The previous front lives in shared memory (two buffers of the launch's
  // dynamic size / 2) when it fits, else it is re-read from the scan's output.
  // A thread takes the cells d1 = base + threadIdx.x + k * blockDim.x of a front,
  // RADIAL_K at a time: it issues the input loads of all of them first, so one
  // memory latency is paid per chunk of a front rather than per cell.
  s << "#define RADIAL_K 8\n"
    << "__device__ __forceinline__ void radial_run(const Args &a, int octant) {\n"
    << "  extern __shared__ __align__(16) unsigned char radial_smem[];\n"
    << "  const int sx = (int)a.aux[0], sy = (int)a.aux[1];\n"
    << "  const long long lim = (long long)a.aux[2];\n"
    << "  const RasterArg R = a.out[" << ri << "];\n"
    << "  const int W = a.g.W, H = a.g.H;\n"
    << "  int p0, p1, q0, q1;\n"
    << "  octant_units(octant, p0, p1, q0, q1);\n"
    << "  const int ep = p0 > 0 ? W - 1 - sx : p0 < 0 ? sx : p1 > 0 ? H - 1 - sy : sy;\n"
    << "  const int eq = q0 > 0 ? W - 1 - sx : q0 < 0 ? sx : q1 > 0 ? H - 1 - sy : sy;\n"
    << "  const int dmax = (lim >= 0 && lim < ep) ? (int)lim : ep;\n"
    << "  u32 dyn;\n"
    << "  asm(\"mov.u32 %0, %%dynamic_smem_size;\" : \"=r\"(dyn));\n"
    << "  const int cap = (int)(dyn / (2 * sizeof(" << T << ")));\n"
    << "  " << T << " *prev = cap > eq ? (" << T << " *)radial_smem : nullptr;\n"
    << "  " << T << " *cur = prev ? prev + cap : nullptr;\n"
    << "  if (threadIdx.x == 0) {\n"
    << "    In in0;\n"
    << "    radial_load(a, in0, sx, sy);\n"
    << "    const " << T << " v0 = radial_cell(a, in0, sx, sy, (" << T << ")0, true);\n"
    << "    if (prev) prev[0] = v0;\n"
    << "  }\n"
    << "  __syncthreads();\n"
    << "  for (int d0 = 1; d0 <= dmax; ++d0) {\n"
    << "    const int d1max = d0 < eq ? d0 : eq;\n"
    << "    for (int base = 0; base <= d1max; base += RADIAL_K * (int)blockDim.x) {\n"
    << "      In in[RADIAL_K];\n"
    << "#pragma unroll\n"
    << "      for (int k = 0; k < RADIAL_K; ++k) {\n"
    << "        const int d1 = base + (int)threadIdx.x + k * (int)blockDim.x;\n"
    << "        if (d1 <= d1max) radial_load(a, in[k], sx + p0 * d0 + q0 * d1, sy + p1 * d0 + q1 * d1);\n"
    << "      }\n"
    << "#pragma unroll\n"
    << "      for (int k = 0; k < RADIAL_K; ++k) {\n"
    << "        const int d1 = base + (int)threadIdx.x + k * (int)blockDim.x;\n"
    << "        if (d1 > d1max) break;\n"
    << "        const int x = sx + p0 * d0 + q0 * d1, y = sy + p1 * d0 + q1 * d1;\n"
    << "        " << T << " va = (" << T << ")0, vb = (" << T << ")0;\n"
    << "        if (prev) {\n"
    << "          if (d1 <= d0 - 1) va = prev[d1];\n"
    << "          if (d1 >= 1) vb = prev[d1 - 1];\n"
    << "        } else {\n"
    << "          if (d1 <= d0 - 1) va = ld_coherent<" << T << ">(R, sx + p0 * (d0 - 1) + q0 * d1, sy + p1 * (d0 - 1) + q1 * d1);\n"
    << "          if (d1 >= 1) vb = ld_coherent<" << T << ">(R, sx + p0 * (d0 - 1) + q0 * (d1 - 1), sy + p1 * (d0 - 1) + q1 * (d1 - 1));\n"
    << "        }\n"
    << "        const " << T << " vv = radial_cell(a, in[k], x, y, radial_lit<" << T << ">(va, vb, d0, d1), false);\n"
    << "        if (cur) cur[d1] = vv;\n"
    << "      }\n"
    << "    }\n"
    << "    __syncthreads();\n"
    << "    " << T << " *t = prev;\n"
    << "    prev = cur;\n"
    << "    cur = t;\n"
    << "  }\n"
    << "}\n";
  // Large rasters: a cluster of CTAs per octant. CTA `rank` of a cluster of C
  // owns the cells d1 in [rank*S, rank*S + S) of every front (S = ceil((eq+1)/C)),
  // keeping its part of the previous and current fronts in its shared memory;
  // the one previous-front value left of its segment is read from the
  // neighbour's shared memory (DSMEM). One cluster barrier per front (every CTA
  // of the cluster sweeps the same fronts, none leaves early) orders the fronts:
  // reads of a front's buffer all come before the barrier, its reuse after.
  s << "__device__ __forceinline__ u32 cl_rank() { u32 r; asm volatile(\"mov.u32 %0, %%cluster_ctarank;\" : \"=r\"(r)); return r; }\n"
    << "__device__ __forceinline__ u32 cl_size() { u32 r; asm volatile(\"mov.u32 %0, %%cluster_nctarank;\" : \"=r\"(r)); return r; }\n"
    << "__device__ __forceinline__ void cl_sync() {\n"
    << "  asm volatile(\"barrier.cluster.arrive.release.aligned;\\n\\tbarrier.cluster.wait.acquire.aligned;\" ::: \"memory\");\n"
    << "}\n"
    << "template <class V> __device__ __forceinline__ V ld_peer(const V *p, u32 rank) {\n"
    << "  u32 ra;\n"
    << "  asm volatile(\"mapa.shared::cluster.u32 %0, %1, %2;\" : \"=r\"(ra) : \"r\"((u32)__cvta_generic_to_shared(p)), \"r\"(rank));\n"
    << "  if constexpr (sizeof(V) == 8) {\n"
    << "    u64 v; asm volatile(\"ld.shared::cluster.b64 %0, [%1];\" : \"=l\"(v) : \"r\"(ra) : \"memory\"); return bit_cast8<V>(v);\n"
    << "  } else if constexpr (sizeof(V) == 4) {\n"
    << "    u32 v; asm volatile(\"ld.shared::cluster.b32 %0, [%1];\" : \"=r\"(v) : \"r\"(ra) : \"memory\"); return bit_cast8<V>(v);\n"
    << "  } else if constexpr (sizeof(V) == 2) {\n"
    << "    u32 v; asm volatile(\"ld.shared::cluster.u16 %0, [%1];\" : \"=r\"(v) : \"r\"(ra) : \"memory\"); return bit_cast8<V>((u16)v);\n"
    << "  } else {\n"
    << "    u32 v; asm volatile(\"ld.shared::cluster.u8 %0, [%1];\" : \"=r\"(v) : \"r\"(ra) : \"memory\"); return bit_cast8<V>((u8)v);\n"
    << "  }\n"
    << "}\n"
    << "__device__ __forceinline__ void radial_run_cluster(const Args &a, int octant) {\n"
    << "  extern __shared__ __align__(16) unsigned char radial_smem[];\n"
    << "  const int C = (int)cl_size(), rank = (int)cl_rank();\n"
    << "  const int sx = (int)a.aux[0], sy = (int)a.aux[1];\n"
    << "  const long long lim = (long long)a.aux[2];\n"
    << "  const int W = a.g.W, H = a.g.H;\n"
    << "  int p0, p1, q0, q1;\n"
    << "  octant_units(octant, p0, p1, q0, q1);\n"
    << "  const int ep = p0 > 0 ? W - 1 - sx : p0 < 0 ? sx : p1 > 0 ? H - 1 - sy : sy;\n"
    << "  const int eq = q0 > 0 ? W - 1 - sx : q0 < 0 ? sx : q1 > 0 ? H - 1 - sy : sy;\n"
    << "  const int dmax = (lim >= 0 && lim < ep) ? (int)lim : ep;\n"
    << "  const int S = (eq + C) / C;\n"
    << "  const int lo = rank * S;\n"
    << "  " << T << " *prev = (" << T << " *)radial_smem;\n"
    << "  " << T << " *cur = prev + S;\n"
    << "  if (rank == 0 && threadIdx.x == 0) {\n"
    << "    In in0;\n"
    << "    radial_load(a, in0, sx, sy);\n"
    << "    prev[0] = radial_cell(a, in0, sx, sy, (" << T << ")0, true);\n"
    << "  }\n"
    << "  cl_sync();\n"
    << "  for (int d0 = 1; d0 <= dmax; ++d0) {\n"
    << "    const int d1max = d0 < eq ? d0 : eq;\n"
    << "    const int n = (lo + S - 1 < d1max ? lo + S - 1 : d1max) - lo + 1;   // cells of this front in the segment\n"
    << "    for (int base = 0; base < n; base += RADIAL_K * (int)blockDim.x) {\n"
    << "      In in[RADIAL_K];\n"
    << "#pragma unroll\n"
    << "      for (int k = 0; k < RADIAL_K; ++k) {\n"
    << "        const int j = base + (int)threadIdx.x + k * (int)blockDim.x, d1 = lo + j;\n"
    << "        if (j < n) radial_load(a, in[k], sx + p0 * d0 + q0 * d1, sy + p1 * d0 + q1 * d1);\n"
    << "      }\n"
    << "#pragma unroll\n"
    << "      for (int k = 0; k < RADIAL_K; ++k) {\n"
    << "        const int j = base + (int)threadIdx.x + k * (int)blockDim.x, d1 = lo + j;\n"
    << "        if (j >= n) break;\n"
    << "        const int x = sx + p0 * d0 + q0 * d1, y = sy + p1 * d0 + q1 * d1;\n"
    << "        " << T << " va = (" << T << ")0, vb = (" << T << ")0;\n"
    << "        if (d1 <= d0 - 1) va = prev[j];\n"
    << "        if (d1 >= 1) vb = j >= 1 ? prev[j - 1] : ld_peer<" << T << ">(prev + (S - 1), (u32)(rank - 1));\n"
    << "        cur[j] = radial_cell(a, in[k], x, y, radial_lit<" << T << ">(va, vb, d0, d1), false);\n"
    << "      }\n"
    << "    }\n"
    << "    cl_sync();\n"
    << "    " << T << " *t = prev;\n"
    << "    prev = cur;\n"
    << "    cur = t;\n"
    << "  }\n"
    << "}\n"
    << "extern \"C\" __global__ void __launch_bounds__(512) KNAME_cl(const __grid_constant__ Args a) {\n"
    << "  radial_run_cluster(a, (int)(blockIdx.x / cl_size()));\n"
    << "}\n";
  // one scan: 8 CTAs (one per octant); many scans: 8 CTAs per Args of a device array
  s << "extern \"C\" __global__ void __launch_bounds__(512) KNAME(const __grid_constant__ Args a) {\n"
    << "  radial_run(a, blockIdx.x);\n"
    << "}\n"
    << "struct ManyArgs { u64 args; s64 n; };\n"
    << "extern \"C\" __global__ void __launch_bounds__(512) KNAME_many(const __grid_constant__ ManyArgs m) {\n"
    << "  if ((s64)(blockIdx.x >> 3) >= m.n) return;\n"
    << "  radial_run(((const Args *)m.args)[blockIdx.x >> 3], blockIdx.x & 7);\n"
    << "}\n";
  return s.str();
}

// Spreading skeleton (runtime/skeleton/SpreadingSkeleton.cpp:288-393). The
// reference relaxes pending spread one neighbour per iteration, block by block,
// until stable; the fixed point is, for every cell, the sum of the water of all
// strictly-upstream cells. It is reached here without iterating to convergence
// (see the passes below; codegen_scan.cpp picks the form by raster size).
static std::string gen_spread(Gen &G) {
  KernelPlan &P = G.plan;
  Node *scan = P.core;
  const int dt = scan->meta.dtype;
  if (!(dt == S32 || dt == U32 || dt == F32 || dt == F64 || dt == S64 || dt == U64))
    throw MapError("spreadScan: the accumulated raster must be a 32- or 64-bit type");
  if (!G.rin.count(scan->prev[1])) throw MapError("spreadScan: the direction raster must be materialised");
  const std::string T = G.T(scan);
  std::ostringstream s;
  s << "#include \"map_scan.cuh\"\n" << G.args_struct(0, false);
  s << "__device__ __forceinline__ " << T << " water_at(const Args &a, int x, int y) {\n";
  for (Node *p : P.in_rasters) {
    if (p == scan->prev[1] || !G.center_read.count(p)) continue;
    int k = G.rin.at(p);
    s << "    const " << G.T(p) << " i" << k << " = ldr<" << G.T(p) << ">(a.in[" << k << "], x, y);\n";
  }
  for (Node *n : G.g.nodes)
    if (n != scan) s << "    " << G.stmt(n, false) << "\n";
  s << "    return (" << T << ")(" << G.val(scan->prev[0]) << ");\n}\n";
  const int kd = G.rin.at(scan->prev[1]);
  const int ko = G.outk.at(scan);
  const bool packed = dt == S32 || dt == U32;
  // aux[0] in-degree (s32[N]; u64[N] in the packed sweep); aux[3] step limit of one downstream walk.
  // Large rasters: two grid-wide passes (kernels KNAME_init then KNAME), each CTA
  // striding over the cells from `first` by `step`:
  //  * init: zero the accumulation and count each cell's upstream neighbours
  //    (cells nothing flows into are marked as sources);
  //  * walk: from every source, a thread carries (accumulation + water) down the
  //    flow path, adding it to the next cell; it goes on into that cell only if
  //    its push was the cell's last pending one (the cell is then complete),
  //    else it stops. Every cell is completed once, by exactly one thread, after
  //    all of its upstream pushes (fences order each push before its count).
  s << "#define SPREAD_SOURCE 0x40000000\n"
    << "__device__ __forceinline__ void spread_init(const Args &a, s64 first, s64 step) {\n"
    << "  const int W = a.g.W, H = a.g.H;\n"
    << "  const s64 N = (s64)W * H;\n"
    << "  s32 *indeg = (s32 *)a.aux[0];\n"
    << "  const RasterArg D = a.in[" << kd << "];\n"
    << "  const RasterArg O = a.out[" << ko << "];\n"
    << "  for (s64 c = first; c < N; c += step) {\n"
    << "    const int x = (int)(c % W), y = (int)(c / W);\n"
    << "    *cell_ptr<" << T << ">(O, x, y) = (" << T << ")0;\n"
    << "    int cnt = 0;\n"
    << "    for (int d = 0; d < 8; ++d) {\n"
    << "      const int nx = x - d8_dx(d), ny = y - d8_dy(d);\n"
    << "      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;\n"
    << "      if (d8_index(ldr<u8>(D, nx, ny)) == d) cnt++;\n"
    << "    }\n"
    << "    indeg[c] = cnt ? cnt : SPREAD_SOURCE;\n"
    << "  }\n"
    << "}\n"
    << "__device__ __forceinline__ void spread_walk(const Args &a, s64 first, s64 step) {\n"
    << "  const int W = a.g.W, H = a.g.H;\n"
    << "  const s64 N = (s64)W * H;\n"
    << "  s32 *indeg = (s32 *)a.aux[0];\n"
    << "  const long long limit = (long long)a.aux[3];\n"
    << "  const RasterArg D = a.in[" << kd << "];\n"
    << "  const RasterArg O = a.out[" << ko << "];\n"
    << "  for (s64 c = first; c < N; c += step) {\n"
    << "    if (indeg[c] != SPREAD_SOURCE) continue;\n"
    << "    int x = (int)(c % W), y = (int)(c / W);\n"
    << "    " << T << " carry = water_at(a, x, y);\n"
    << "    for (long long it = 0;; ++it) {\n"
    << "      if (it > limit) { skel_fail(a.err, ERR_ITER_LIMIT); break; }\n"
    << "      const s64 dn = d8_down(D, W, H, x, y);\n"
    << "      if (dn < 0) break;\n"
    << "      const int dx = (int)(dn % W), dy = (int)(dn / W);\n"
    << "      atomic_add_any(cell_ptr<" << T << ">(O, dx, dy), carry);\n"
    << "      if (atomic_dec_acq_rel(&indeg[dn]) != 1) break;   // orders the push before the count\n"
    << "      x = dx;\n"
    << "      y = dy;\n"
    << "      carry = (" << T << ")(ld_coherent<" << T << ">(O, x, y) + water_at(a, x, y));\n"
    << "    }\n"
    << "  }\n"
    << "}\n";
  // Small rasters: one CTA runs a topological (Kahn) sweep, frontier by frontier
  // with block barriers (aux[1], aux[2]: frontier lists of N entries, 4 bytes
  // each, 8 in the packed sweep; the caller's scratch holds 24 bytes per cell).
  // Frontier entries pack a cell index (below 2^24) with its D8 code, fetched
  // by the thread that completes the cell while its in-degree atomic is in
  // flight, so a round reads no direction; the first KAHN_SMEM entries of a
  // frontier live in shared memory, the rest in the global lists.
  s << "#define KAHN_SMEM 4096\n"
    << "__device__ __forceinline__ void kahn_put(u32 *sf, u32 *gf, int i, u32 e) {\n"
    << "  if (i < KAHN_SMEM) sf[i] = e; else gf[i] = e;\n"
    << "}\n"
    // pre: the in-degrees were counted by spread_init (sources marked), by a
    // many-CTA launch before this one; the sweep then only collects the sources.
    // Round r takes its frontier size from cnt[r % 3], appends to cnt[(r + 1) % 3]
    // and clears cnt[(r + 2) % 3] (read by everyone before the previous barrier):
    // one block barrier per round.
    << "__device__ __forceinline__ void spread_kahn(const Args &a, bool pre) {\n"
    << "  const int W = a.g.W, H = a.g.H;\n"
    << "  const s64 N = (s64)W * H;\n"
    << "  s32 *indeg = (s32 *)a.aux[0];\n"
    << "  u32 *fa = (u32 *)a.aux[1], *fb = (u32 *)a.aux[2];\n"
    << "  const long long limit = (long long)a.aux[3];\n"
    << "  const RasterArg D = a.in[" << kd << "];\n"
    << "  const RasterArg O = a.out[" << ko << "];\n"
    << "  __shared__ int cnt[3];\n"
    << "  __shared__ u32 kf[2][KAHN_SMEM];\n"
    << "  if (N >= ((s64)1 << 24)) { if (threadIdx.x == 0) skel_fail(a.err, ERR_BAD_LAUNCH); return; }\n"
    << "  u32 *sa = kf[0], *sb = kf[1];\n"
    << "  if (threadIdx.x == 0) { cnt[0] = 0; cnt[1] = 0; cnt[2] = 0; }\n"
    << "  __syncthreads();\n"
    << "  if (pre) {\n"
    << "#pragma unroll 4\n"
    << "    for (s64 c = threadIdx.x; c < N; c += blockDim.x)\n"
    << "      if (indeg[c] == SPREAD_SOURCE)\n"
    << "        kahn_put(sa, fa, atomicAdd(&cnt[0], 1), (u32)(((u64)c << 8) | ldr<u8>(D, (int)(c % W), (int)(c / W))));\n"
    << "  } else {\n"
    << "    for (s64 c = threadIdx.x; c < N; c += blockDim.x) {\n"
    << "      const int x = (int)(c % W), y = (int)(c / W);\n"
    << "      *cell_ptr<" << T << ">(O, x, y) = (" << T << ")0;\n"
    << "      int k = 0;\n"
    << "      for (int d = 0; d < 8; ++d) {\n"
    << "        const int nx = x - d8_dx(d), ny = y - d8_dy(d);\n"
    << "        if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;\n"
    << "        if (d8_index(ldr<u8>(D, nx, ny)) == d) k++;\n"
    << "      }\n"
    << "      indeg[c] = k;\n"
    << "      if (k == 0) kahn_put(sa, fa, atomicAdd(&cnt[0], 1), (u32)(((u64)c << 8) | ldr<u8>(D, x, y)));\n"
    << "    }\n"
    << "  }\n"
    << "  __syncthreads();\n"
    << "  for (long long it = 0;; ++it) {\n"
    << "    const int r = (int)(it % 3);\n"
    << "    const int n = cnt[r];\n"
    << "    if (n == 0) break;\n"
    << "    if (it > limit) { if (threadIdx.x == 0) skel_fail(a.err, ERR_ITER_LIMIT); break; }\n"
    << "    int *nn = &cnt[r == 2 ? 0 : r + 1];\n"
    << "    for (int i = threadIdx.x; i < n; i += blockDim.x) {\n"
    << "      const u32 e = i < KAHN_SMEM ? sa[i] : fa[i];\n"
    << "      const int c = (int)(e >> 8);\n"
    << "      const int d = d8_index((u8)(e & 255));\n"
    << "      if (d < 0) continue;\n"
    << "      const int x = c % W, y = c / W;\n"
    << "      const int nx = x + d8_dx(d), ny = y + d8_dy(d);\n"
    << "      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;\n"
    << "      const int dn = ny * W + nx;\n"
    << "      const " << T << " v = (" << T << ")(ld_coherent<" << T << ">(O, x, y) + water_at(a, x, y));\n"
    << "      atomic_add_any(cell_ptr<" << T << ">(O, nx, ny), v);\n"
    << "      const u8 code = ldr<u8>(D, nx, ny);\n"
    << "      if (atomicSub(&indeg[dn], 1) == 1) kahn_put(sb, fb, atomicAdd(nn, 1), ((u32)dn << 8) | code);\n"
    << "    }\n"
    << "    if (threadIdx.x == 0) cnt[r == 0 ? 2 : r - 1] = 0;\n"
    << "    __syncthreads();\n"
    << "    u32 *t = fa; fa = fb; fb = t;\n"
    << "    t = sa; sa = sb; sb = t;\n"
    << "  }\n"
    << "}\n"
    ;
  // 32-bit integer accumulations: one 64-bit word per cell holds the cell's
  // accumulation (high half) and its pending upstream pushes (low half). A push
  // adds (value << 32) - 1 in one atomic: the count never borrows (it is at
  // least 1 before each push) and the sum wraps like the 32-bit type. The
  // pusher that sees the count at 1 knows the final sum from the returned old
  // word, writes the cell's output and queues the cell with the value it will
  // push (sum + water): a round is one atomic round trip, the direction code of
  // the next cell fetched beside it. Frontier entries: (value << 32) | (cell << 8) | code.
  if (packed) {
    s << "#define KAHN_SMEM_P 2048\n"
      << "#ifndef KAHN_CHAIN\n#define KAHN_CHAIN 8\n#endif\n"
      << "#define KAHN_SOURCE 0x80000000u   // pending-count half of a source's word (nothing flows in)\n"
      << "__device__ __forceinline__ void spread_init_packed(const Args &a, s64 first, s64 step) {\n"
      << "  const int W = a.g.W, H = a.g.H;\n"
      << "  const s64 N = (s64)W * H;\n"
      << "  u64 *pk = (u64 *)a.aux[0];\n"
      << "  const RasterArg D = a.in[" << kd << "];\n"
      << "  const RasterArg O = a.out[" << ko << "];\n"
      << "  for (s64 c = first; c < N; c += step) {\n"
      << "    const int x = (int)(c % W), y = (int)(c / W);\n"
      << "    *cell_ptr<" << T << ">(O, x, y) = (" << T << ")0;\n"
      << "    u32 k = 0;\n"
      << "    for (int d = 0; d < 8; ++d) {\n"
      << "      const int nx = x - d8_dx(d), ny = y - d8_dy(d);\n"
      << "      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;\n"
      << "      if (d8_index(ldr<u8>(D, nx, ny)) == d) k++;\n"
      << "    }\n"
      << "    pk[c] = k ? (u64)k : (u64)KAHN_SOURCE;\n"
      << "  }\n"
      << "}\n"
      << "__device__ __forceinline__ void kahn_put_p(u64 *sf, u64 *gf, int i, u64 e) {\n"
      << "  if (i < KAHN_SMEM_P) sf[i] = e; else gf[i] = e;\n"
      << "}\n"
      << "__device__ __forceinline__ u64 kahn_entry(int c, u8 code, " << T << " push) {\n"
      << "  return ((u64)(u32)push << 32) | ((u64)(u32)c << 8) | code;\n"
      << "}\n"
      << "__device__ __forceinline__ void spread_kahn_packed(const Args &a, bool pre) {\n"
      << "  const int W = a.g.W, H = a.g.H;\n"
      << "  const s64 N = (s64)W * H;\n"
      << "  u64 *pk = (u64 *)a.aux[0];\n"
      << "  u64 *fa = (u64 *)a.aux[1], *fb = (u64 *)a.aux[2];\n"
      << "  const long long limit = (long long)a.aux[3];\n"
      << "  const RasterArg D = a.in[" << kd << "];\n"
      << "  const RasterArg O = a.out[" << ko << "];\n"
      << "  __shared__ int cnt[3];\n"
      << "  __shared__ u64 kf[2][KAHN_SMEM_P];\n"
      << "  if (N >= ((s64)1 << 24)) { if (threadIdx.x == 0) skel_fail(a.err, ERR_BAD_LAUNCH); return; }\n"
      << "  u64 *sa = kf[0], *sb = kf[1];\n"
      << "  if (threadIdx.x == 0) { cnt[0] = 0; cnt[1] = 0; cnt[2] = 0; }\n"
      << "  if (!pre) spread_init_packed(a, threadIdx.x, blockDim.x);\n"
      << "  __syncthreads();\n"
      << "#pragma unroll 4\n"
      << "  for (s64 c = threadIdx.x; c < N; c += blockDim.x)\n"
      << "    if ((u32)pk[c] == KAHN_SOURCE) {\n"
      << "      const int x = (int)(c % W), y = (int)(c / W);\n"
      << "      kahn_put_p(sa, fa, atomicAdd(&cnt[0], 1), kahn_entry((int)c, ldr<u8>(D, x, y), water_at(a, x, y)));\n"
      << "    }\n"
      << "  __syncthreads();\n"
      << "  for (long long it = 0;; ++it) {\n"
      << "    const int r = (int)(it % 3);\n"
      << "    const int n = cnt[r];\n"
      << "    if (n == 0) break;\n"
      << "    if (it > limit) { if (threadIdx.x == 0) skel_fail(a.err, ERR_ITER_LIMIT); break; }\n"
      << "    int *nn = &cnt[r == 2 ? 0 : r + 1];\n"
      // a thread that completes a cell goes on down its chain, up to KAHN_CHAIN
      // cells per entry and round, before queueing the cell it reached
      << "    for (int i = threadIdx.x; i < n; i += blockDim.x) {\n"
      << "      const u64 e = i < KAHN_SMEM_P ? sa[i] : fa[i];\n"
      << "      int c = (int)((u32)e >> 8);\n"
      << "      u8 cc = (u8)(e & 255);\n"
      << "      u32 v = (u32)(e >> 32);\n"
      << "#pragma unroll 1\n"
      << "      for (int step = 0; step < KAHN_CHAIN; ++step) {\n"
      << "        const int d = d8_index(cc);\n"
      << "        if (d < 0) break;\n"
      << "        const int x = c % W, y = c / W;\n"
      << "        const int nx = x + d8_dx(d), ny = y + d8_dy(d);\n"
      << "        if (nx < 0 || ny < 0 || nx >= W || ny >= H) break;\n"
      << "        const int dn = ny * W + nx;\n"
      << "        const u8 code = ldr<u8>(D, nx, ny);\n"
      << "        const u64 old = atomicAdd((unsigned long long *)&pk[dn], ((u64)v << 32) - 1ull);\n"
      << "        if ((u32)old != 1u) break;\n"
      << "        const " << T << " sum = (" << T << ")((u32)(old >> 32) + v);\n"
      << "        *cell_ptr<" << T << ">(O, nx, ny) = sum;\n"
      << "        const " << T << " push = (" << T << ")(sum + water_at(a, nx, ny));\n"
      << "        if (step == KAHN_CHAIN - 1) { kahn_put_p(sb, fb, atomicAdd(nn, 1), kahn_entry(dn, code, push)); break; }\n"
      << "        c = dn;\n"
      << "        cc = code;\n"
      << "        v = (u32)push;\n"
      << "      }\n"
      << "    }\n"
      << "    if (threadIdx.x == 0) cnt[r == 0 ? 2 : r - 1] = 0;\n"
      << "    __syncthreads();\n"
      << "    u64 *t = fa; fa = fb; fb = t;\n"
      << "    t = sa; sa = sb; sb = t;\n"
      << "  }\n"
      << "}\n"
      // large rasters: the downstream walks with the packed word; the one atomic
      // per step orders nothing else (the sum travels in the word), so it is relaxed
      << "__device__ __forceinline__ void spread_walk_packed(const Args &a, s64 first, s64 step) {\n"
      << "  const int W = a.g.W, H = a.g.H;\n"
      << "  const s64 N = (s64)W * H;\n"
      << "  u64 *pk = (u64 *)a.aux[0];\n"
      << "  const long long limit = (long long)a.aux[3];\n"
      << "  const RasterArg D = a.in[" << kd << "];\n"
      << "  const RasterArg O = a.out[" << ko << "];\n"
      << "  for (s64 c = first; c < N; c += step) {\n"
      << "    if ((u32)pk[c] != KAHN_SOURCE) continue;\n"
      << "    int x = (int)(c % W), y = (int)(c / W);\n"
      << "    u32 carry = (u32)water_at(a, x, y);\n"
      << "    for (long long it = 0;; ++it) {\n"
      << "      if (it > limit) { skel_fail(a.err, ERR_ITER_LIMIT); break; }\n"
      << "      const s64 dn = d8_down(D, W, H, x, y);\n"
      << "      if (dn < 0) break;\n"
      << "      const u64 old = atomicAdd((unsigned long long *)&pk[dn], ((u64)carry << 32) - 1ull);\n"
      << "      if ((u32)old != 1u) break;\n"
      << "      x = (int)(dn % W);\n"
      << "      y = (int)(dn / W);\n"
      << "      const " << T << " sum = (" << T << ")((u32)(old >> 32) + carry);\n"
      << "      *cell_ptr<" << T << ">(O, x, y) = sum;\n"
      << "      carry = (u32)(" << T << ")(sum + water_at(a, x, y));\n"
      << "    }\n"
      << "  }\n"
      << "}\n";
  }
  // Integer accumulations: pointer jumping over the Euler tour of the D8 forest,
  // a fixed number of rounds (ceil(log2(2N)) + 1) whatever the length of the
  // longest flow path. Every non-root cell c (one whose D8 code leads to a cell
  // of the raster, its parent) owns two tour elements: D(c) = 2c, the step down
  // from its parent into c, carrying c's water, and U(c) = 2c + 1, the step back
  // up, carrying 0. The children of a cell are its neighbours whose codes point
  // at it, in direction order (E, SE, S, SW, W, NW, N, NE), so the tour's
  // successor function is local: after D(c) comes D(first child of c), or U(c)
  // for a leaf; after U(c) comes D(next sibling of c), or U(parent) unless the
  // parent is a root (end of the tour). Each round sets sum[e] += sum[next[e]]
  // and next[e] = next[next[e]] (Wyllie); afterwards sum[e] is the water from e
  // to the end of its tour, so the subtree of c holds
  // sum[D(c)] - sum[successor of U(c)], and the accumulation (strictly upstream
  // water) is that minus c's own water; a root's is sum[D(first child)].
  // Integer sums are exact modulo the type's width, so the result equals any
  // other order of additions bit for bit. A list still linked after the last
  // round lies on a cycle of codes: the error flag is set.
  // Scratch at aux[0]: next[2][2N] (s32), then sum[2][2N] (the sum type).
  const bool pj = dt == S32 || dt == U32 || dt == S64 || dt == U64;
  if (pj) {
    const std::string ST = dt_size(dt) == 4 ? "u32" : "u64";
    s << "#define PJ_END (-1)\n"
      << "struct PjArgs { u64 args; s64 n; s64 slices; s64 round; };\n"
      << "__device__ __forceinline__ s32 pj_child(const RasterArg &D, int W, int H, int x, int y, int j0) {\n"
      << "  for (int j = j0; j < 8; ++j) {\n"
      << "    const int nx = x + d8_dx(j), ny = y + d8_dy(j);\n"
      << "    if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;\n"
      << "    if (d8_index(ldr<u8>(D, nx, ny)) == ((j + 4) & 7)) return ny * W + nx;\n"
      << "  }\n"
      << "  return -1;\n"
      << "}\n"
      // successor of U(c) for a non-root cell (x, y) whose code has index d
      << "__device__ __forceinline__ s32 pj_after_up(const RasterArg &D, int W, int H, int x, int y, int d) {\n"
      << "  const int px = x + d8_dx(d), py = y + d8_dy(d);\n"
      << "  const s32 sib = pj_child(D, W, H, px, py, ((d + 4) & 7) + 1);\n"
      << "  if (sib >= 0) return 2 * sib;\n"
      << "  return d8_down(D, W, H, px, py) >= 0 ? 2 * (py * W + px) + 1 : PJ_END;\n"
      << "}\n"
      << "__device__ __forceinline__ void pj_init(const Args &a, s64 first, s64 step) {\n"
      << "  const int W = a.g.W, H = a.g.H;\n"
      << "  const s64 N = (s64)W * H;\n"
      << "  s32 *nx0 = (s32 *)a.aux[0];\n"
      << "  " << ST << " *sm0 = (" << ST << " *)(nx0 + 4 * N);\n"
      << "  const RasterArg D = a.in[" << kd << "];\n"
      << "  for (s64 c = first; c < N; c += step) {\n"
      << "    const int x = (int)(c % W), y = (int)(c / W);\n"
      << "    s32 nd = PJ_END, nu = PJ_END;\n"
      << "    " << ST << " w = 0;\n"
      << "    if (d8_down(D, W, H, x, y) >= 0) {\n"
      << "      const s32 fc = pj_child(D, W, H, x, y, 0);\n"
      << "      nd = fc >= 0 ? 2 * fc : (s32)(2 * c + 1);\n"
      << "      nu = pj_after_up(D, W, H, x, y, d8_index(ldr<u8>(D, x, y)));\n"
      << "      w = (" << ST << ")water_at(a, x, y);\n"
      << "    }\n"
      << "    nx0[2 * c] = nd;\n"
      << "    nx0[2 * c + 1] = nu;\n"
      << "    sm0[2 * c] = w;\n"
      << "    sm0[2 * c + 1] = 0;\n"
      << "  }\n"
      << "}\n"
      << "__device__ __forceinline__ void pj_step(const Args &a, s64 first, s64 step, int round) {\n"
      << "  const s64 N = (s64)a.g.W * a.g.H;\n"
      << "  s32 *nxs = (s32 *)a.aux[0] + (round & 1) * 2 * N, *nxd = (s32 *)a.aux[0] + ((round + 1) & 1) * 2 * N;\n"
      << "  " << ST << " *sm = (" << ST << " *)((s32 *)a.aux[0] + 4 * N);\n"
      << "  const " << ST << " *sms = sm + (round & 1) * 2 * N;\n"
      << "  " << ST << " *smd = sm + ((round + 1) & 1) * 2 * N;\n"
      << "  for (s64 e = first; e < 2 * N; e += step) {\n"
      << "    const s32 n = nxs[e];\n"
      << "    if (n == PJ_END) { nxd[e] = PJ_END; smd[e] = sms[e]; }\n"
      << "    else { smd[e] = sms[e] + sms[n]; nxd[e] = nxs[n]; }\n"
      << "  }\n"
      << "}\n"
      << "__device__ __forceinline__ void pj_final(const Args &a, s64 first, s64 step, int rounds) {\n"
      << "  const int W = a.g.W, H = a.g.H;\n"
      << "  const s64 N = (s64)W * H;\n"
      << "  const s32 *nx = (const s32 *)a.aux[0] + (rounds & 1) * 2 * N;\n"
      << "  const " << ST << " *sm = (const " << ST << " *)((const s32 *)a.aux[0] + 4 * N) + (rounds & 1) * 2 * N;\n"
      << "  const RasterArg D = a.in[" << kd << "];\n"
      << "  const RasterArg O = a.out[" << ko << "];\n"
      << "  for (s64 c = first; c < N; c += step) {\n"
      << "    const int x = (int)(c % W), y = (int)(c / W);\n"
      << "    " << ST << " acc;\n"
      << "    if (d8_down(D, W, H, x, y) < 0) {\n"
      << "      const s32 fc = pj_child(D, W, H, x, y, 0);\n"
      << "      acc = fc >= 0 ? sm[2 * fc] : (" << ST << ")0;\n"
      << "    } else {\n"
      << "      if (nx[2 * c] != PJ_END) skel_fail(a.err, ERR_ITER_LIMIT);   // a cycle of codes\n"
      << "      const s32 nu = pj_after_up(D, W, H, x, y, d8_index(ldr<u8>(D, x, y)));\n"
      << "      acc = sm[2 * c] - (nu == PJ_END ? (" << ST << ")0 : sm[nu]) - (" << ST << ")water_at(a, x, y);\n"
      << "    }\n"
      << "    *cell_ptr<" << T << ">(O, x, y) = (" << T << ")acc;\n"
      << "  }\n"
      << "}\n"
      // one raster (aux[1]: round of a step launch)
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_init(const __grid_constant__ Args a) {\n"
      << "  pj_init(a, (s64)blockIdx.x * blockDim.x + threadIdx.x, (s64)gridDim.x * blockDim.x);\n"
      << "}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_step(const __grid_constant__ Args a) {\n"
      << "  pj_step(a, (s64)blockIdx.x * blockDim.x + threadIdx.x, (s64)gridDim.x * blockDim.x, (int)a.aux[1]);\n"
      << "}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_final(const __grid_constant__ Args a) {\n"
      << "  pj_final(a, (s64)blockIdx.x * blockDim.x + threadIdx.x, (s64)gridDim.x * blockDim.x, (int)a.aux[1]);\n"
      << "}\n"
      // many rasters (serving windows): `slices` CTAs per raster
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_init_many(const __grid_constant__ PjArgs m) {\n"
      << "  const s64 r = blockIdx.x / m.slices;\n"
      << "  if (r >= m.n) return;\n"
      << "  pj_init(((const Args *)m.args)[r], (blockIdx.x % m.slices) * blockDim.x + threadIdx.x, m.slices * blockDim.x);\n"
      << "}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_step_many(const __grid_constant__ PjArgs m) {\n"
      << "  const s64 r = blockIdx.x / m.slices;\n"
      << "  if (r >= m.n) return;\n"
      << "  pj_step(((const Args *)m.args)[r], (blockIdx.x % m.slices) * blockDim.x + threadIdx.x, m.slices * blockDim.x,\n"
      << "          (int)m.round);\n"
      << "}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_pj_final_many(const __grid_constant__ PjArgs m) {\n"
      << "  const s64 r = blockIdx.x / m.slices;\n"
      << "  if (r >= m.n) return;\n"
      << "  pj_final(((const Args *)m.args)[r], (blockIdx.x % m.slices) * blockDim.x + threadIdx.x, m.slices * blockDim.x,\n"
      << "           (int)m.round);\n"
      << "}\n";
  }
  const std::string kahn_fn = packed ? "spread_kahn_packed" : "spread_kahn";
  const std::string init_fn = packed ? "spread_init_packed" : "spread_init";
  s
    << "extern \"C\" __global__ void __launch_bounds__(1024) KNAME_kahn(const __grid_constant__ Args a) {\n"
    << "  " << kahn_fn << "(a, false);\n"
    << "}\n"
    // many rasters in one launch (serving windows): one CTA each
    << "struct ManyArgs { u64 args; s64 n; };\n"
    << "extern \"C\" __global__ void __launch_bounds__(1024) KNAME_kahn_many(const __grid_constant__ ManyArgs m) {\n"
    << "  if ((s64)blockIdx.x >= m.n) return;\n"
    << "  " << kahn_fn << "(((const Args *)m.args)[blockIdx.x], false);\n"
    << "}\n"
    // many rasters, in-degree pass spread over PREP_SLICES CTAs per raster (prep),
    // then the one-CTA sweep of each raster from its marked sources (kahnp)
    << "#define PREP_SLICES 32\n"
    << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_prep_many(const __grid_constant__ ManyArgs m) {\n"
    << "  const s64 r = blockIdx.x / PREP_SLICES;\n"
    << "  if (r >= m.n) return;\n"
    << "  " << init_fn << "(((const Args *)m.args)[r], (s64)(blockIdx.x % PREP_SLICES) * blockDim.x + threadIdx.x,\n"
    << "              (s64)PREP_SLICES * blockDim.x);\n"
    << "}\n"
    << "extern \"C\" __global__ void __launch_bounds__(1024) KNAME_kahnp_many(const __grid_constant__ ManyArgs m) {\n"
    << "  if ((s64)blockIdx.x >= m.n) return;\n"
    << "  " << kahn_fn << "(((const Args *)m.args)[blockIdx.x], true);\n"
    << "}\n";
  s << "extern \"C\" __global__ void __launch_bounds__(256) KNAME_init(const __grid_constant__ Args a) {\n"
    << "  " << init_fn << "(a, (s64)blockIdx.x * blockDim.x + threadIdx.x, (s64)gridDim.x * blockDim.x);\n"
    << "}\n"
    << "extern \"C\" __global__ void __launch_bounds__(256) KNAME(const __grid_constant__ Args a) {\n"
    << "  " << (packed ? "spread_walk_packed" : "spread_walk") << "(a, (s64)blockIdx.x * blockDim.x + threadIdx.x, (s64)gridDim.x * blockDim.x);\n"
    << "}\n";
  return s.str();
}

const FocalTune &focal_tune() {
  static FocalTune t = [] {
    FocalTune r;
    const char *e = std::getenv("MAP_B200_FOCAL_TUNE");
    if (!e) return r;
    std::string s(e);
    size_t i = 0;
    while (i < s.size()) {
      size_t j = s.find(',', i);
      if (j == std::string::npos) j = s.size();
      std::string kv = s.substr(i, j - i);
      size_t eq = kv.find('=');
      if (eq != std::string::npos) {
        const std::string k = kv.substr(0, eq);
        const int v = std::atoi(kv.c_str() + eq + 1);
        if (k == "unroll") r.unroll = v;
        else if (k == "defer") r.defer = v;
        else if (k == "nt") r.nt = v;
        else if (k == "tw") r.tw = v;
        else if (k == "th") r.th = v;
        else if (k == "lnt") r.lnt = v;
        else if (k == "ltw") r.ltw = v;
        else if (k == "lth") r.lth = v;
        else if (k == "qnt") r.qnt = v;
        else if (k == "qtw") r.qtw = v;
        else if (k == "qth") r.qth = v;
        else if (k == "minb") r.minb = v;
        else if (k == "pdl") r.pdl = v;
        else if (k == "fpair") r.fpair = v;
        else if (k == "cpair") r.cpair = v;
        else if (k == "fflag") r.fflag = v;
        else if (k == "fmerge") r.fmerge = v;
        else if (k == "tstore") r.tstore = v;
      }
      i = j + 1;
    }
    return r;
  }();
  return t;
}

bool focal_fast_shade(const Group &g) {
  if (g.skeleton != SK_FOCAL) return false;
  KernelPlan P;
  Gen G(g, P);
  G.classify();
  return G.any_fast();
}

bool focal_quad_form(const Group &g) {
  if (g.skeleton != SK_FOCAL || !Runtime::get().paired_cells) return false;
  KernelPlan P;
  Gen G(g, P);
  G.classify();
  return G.quadable();
}

bool tile_cfg_valid(const TileCfg &c) {
  return c.tw > 0 && c.th > 0 && c.nt >= 32 && c.nt <= 1024 && c.nt % 32 == 0 && c.nt % c.tw == 0 &&
         (c.tw * c.th) % c.nt == 0 && c.tw <= c.nt && c.tw <= 224 && c.th <= 224;
}

KernelPlan generate_kernel(const Group &g, TileCfg cfg) {
  if (!tile_cfg_valid(cfg)) throw MapError("codegen: invalid tile configuration");
  KernelPlan P;
  P.skeleton = g.skeleton;
  P.threads = cfg.nt;
  P.tile_w = cfg.tw;
  P.tile_h = cfg.th;
  P.min_blocks = cfg.minb;
  P.tile_store = cfg.tile_store;
  Gen G(g, P);
  G.classify();
  std::string src;
  const char *prefix = "map_local";
  std::ostringstream body, wrap;
  switch (g.skeleton) {
    case SK_LOCAL: gen_local(G, body, wrap); prefix = "map_local"; break;
    case SK_FOCAL: gen_focal(G, body, wrap); prefix = "map_focal"; break;
    case SK_ZONAL: src = gen_zonal(G); prefix = "map_zonal"; break;
    case SK_RADIAL: case SK_SPREAD:
      for (Node *n : g.nodes)
        if (n->kind == K_RADIALSCAN || n->kind == K_SPREADSCAN) P.core = n;
      if (g.skeleton == SK_RADIAL) { src = gen_radial(G); prefix = "map_radial"; }
      else { src = gen_spread(G); prefix = "map_spread"; }
      break;
    default: throw MapError("codegen: group has no device skeleton");
  }
  if (g.skeleton == SK_LOCAL || g.skeleton == SK_FOCAL) {
    P.body = body.str();
    src = "#include \"map_common.cuh\"\n" + P.body + wrap.str();
  }
  std::string name = std::string(prefix) + "_" + fnv_hex(src).substr(0, 12);
  size_t pos;
  while ((pos = src.find("KNAME")) != std::string::npos) src.replace(pos, 5, name);
  P.kname = name;
  if (g.skeleton == SK_ZONAL) P.kname_final = name + "_final";
  P.source = src;
  return P;
}

}  // namespace mapb
