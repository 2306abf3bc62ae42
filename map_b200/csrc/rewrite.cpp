// Matcher of the hillshade composition (see rewrite.hpp for the identities).
#include "rewrite.hpp"

#include <algorithm>
#include <cmath>

namespace mapb {

namespace {

struct Matcher {
  const std::function<bool(Node *, double &)> &lit;
  const std::function<bool(Node *)> &member;
  std::vector<Node *> seen;   // pattern nodes (computed ones)

  bool f32(Node *n) const { return n->meta.dtype == F32; }

  // n is a computed node of the group (recorded as part of the pattern)
  bool take(Node *n) {
    if (!member(n)) return false;
    if (std::find(seen.begin(), seen.end(), n) == seen.end()) seen.push_back(n);
    return true;
  }
  bool unary(Node *n, int op, Node *&a) {
    if (n->kind != K_UNARY || n->op != op || !take(n)) return false;
    a = n->prev[0];
    return true;
  }
  bool binary(Node *n, int op, Node *&a, Node *&b) {
    if (n->kind != K_BINARY || n->op != op || !take(n)) return false;
    a = n->prev[0];
    b = n->prev[1];
    return true;
  }
  bool is_const(Node *n, double &v) const { return lit(n, v); }
  bool is_zero(Node *n) const {
    double v;
    return lit(n, v) && v == 0.0;
  }
  // op(n) with one operand the constant c and the other returned in `o`
  bool with_const(Node *n, int op, double &c, Node *&o) {
    Node *a, *b;
    if (!binary(n, op, a, b)) return false;
    if (is_const(a, c)) { o = b; return true; }
    if ((op == ADD || op == MUL) && is_const(b, c)) { o = a; return true; }
    return false;
  }
  // rel(v, 0) with v returned
  bool rel_zero(Node *n, int op, Node *&v) {
    Node *a, *b;
    if (!binary(n, op, a, b) || !is_zero(b)) return false;
    v = a;
    return true;
  }

  // s = atan(k * sqrt(x*x + y*y)) or atan(sqrt(x*x + y*y)); returns the two
  // squared nodes (in the order of the sum) and k
  bool slope(Node *s, Node *&x, Node *&y, double &k) {
    Node *t, *sq, *q, *xx, *yy, *a, *b;
    if (!unary(s, ATAN, t) || !f32(s)) return false;
    k = 1.0;
    if (!(t->kind == K_UNARY && t->op == SQRT)) {
      if (!with_const(t, MUL, k, sq)) return false;
      if (!(k > 0) || !std::isfinite(k)) return false;
    } else {
      sq = t;
    }
    if (!unary(sq, SQRT, q) || !binary(q, ADD, xx, yy)) return false;
    if (!binary(xx, MUL, a, b) || a != b) return false;
    x = a;
    if (!binary(yy, MUL, a, b) || a != b) return false;
    y = a;
    return x != y && f32(x) && f32(y) && f32(q);
  }

  // aspect = z1w + z0 with z1w = z1 + (z1 < 0) * pi2, z1 = (x != 0) * atan2(y, -x),
  // z0 = (x == 0) * ((y > 0) * pih + (y < 0) * pi32)   (python/hill.py:33-39)
  bool aspect(Node *asp, Node *x, Node *y, double &pi2, double &pih, double &pi32) {
    Node *l, *r;
    if (!binary(asp, ADD, l, r) || !f32(asp)) return false;
    for (int sw = 0; sw < 2; sw++) {
      std::vector<Node *> save = seen;
      Node *z1w = sw ? r : l, *z0 = sw ? l : r;
      if (wrapped(z1w, x, y, pi2) && branch0(z0, x, y, pih, pi32)) return true;
      seen = save;
    }
    return false;
  }
  bool wrapped(Node *z1w, Node *x, Node *y, double &pi2) {
    Node *a, *b;
    if (!binary(z1w, ADD, a, b)) return false;
    for (int sw = 0; sw < 2; sw++) {
      std::vector<Node *> save = seen;
      Node *z1 = sw ? b : a, *w = sw ? a : b, *lt, *v;
      if (with_const(w, MUL, pi2, lt) && rel_zero(lt, LT, v) && v == z1 && atan2_branch(z1, x, y)) return true;
      seen = save;
    }
    return false;
  }
  bool atan2_branch(Node *z1, Node *x, Node *y) {
    Node *a, *b;
    if (!binary(z1, MUL, a, b)) return false;
    for (int sw = 0; sw < 2; sw++) {
      std::vector<Node *> save = seen;
      Node *ne = sw ? b : a, *at = sw ? a : b, *v, *yy, *nx, *xx;
      if (rel_zero(ne, NE, v) && v == x && binary(at, ATAN2, yy, nx) && yy == y && unary(nx, NEG, xx) && xx == x &&
          f32(at))
        return true;
      seen = save;
    }
    return false;
  }
  bool branch0(Node *z0, Node *x, Node *y, double &pih, double &pi32) {
    Node *a, *b;
    if (!binary(z0, MUL, a, b)) return false;
    for (int sw = 0; sw < 2; sw++) {
      std::vector<Node *> save = seen;
      Node *eq = sw ? b : a, *sum = sw ? a : b, *v, *p, *q;
      if (rel_zero(eq, EQ, v) && v == x && binary(sum, ADD, p, q)) {
        for (int sw2 = 0; sw2 < 2; sw2++) {
          std::vector<Node *> save2 = seen;
          Node *gt, *lt, *g, *l;
          if (with_const(sw2 ? q : p, MUL, pih, gt) && with_const(sw2 ? p : q, MUL, pi32, lt) && rel_zero(gt, GT, g) &&
              g == y && rel_zero(lt, LT, l) && l == y)
            return true;
          seen = save2;
        }
      }
      seen = save;
    }
    return false;
  }

  // product of three factors {c, f, g} in any tree shape: (c * f) * g, c * (f * g), ...
  bool product3(Node *n, double &c, Node *&f, Node *&g) {
    Node *a, *b;
    if (!binary(n, MUL, a, b)) return false;
    for (int sw = 0; sw < 2; sw++) {
      std::vector<Node *> save = seen;
      Node *inner = sw ? b : a, *other = sw ? a : b, *o;
      if (with_const(inner, MUL, c, o)) {
        f = o;
        g = other;
        return true;
      }
      seen = save;
    }
    return false;
  }
};

bool near(double v, double target) { return std::isfinite(v) && std::fabs(v - target) < 1e-5; }

}  // namespace

bool match_shade(Node *hs, const std::function<bool(Node *, double &)> &lit,
                 const std::function<bool(Node *)> &member, ShadeMatch &m) {
  if (hs->kind != K_BINARY || hs->op != ADD || hs->meta.dtype != F32) return false;
  Matcher M{lit, member, {}};
  Node *l, *r;
  if (!M.binary(hs, ADD, l, r)) return false;
  const double PI = 3.14159265358979323846;
  for (int sw = 0; sw < 2; sw++) {
    M.seen = {hs};
    Node *t1 = sw ? r : l, *t2 = sw ? l : r;
    double cz, sz, k, ar, pi2, pih, pi32;
    Node *cs, *s, *f, *g, *x, *y;
    if (!M.with_const(t1, MUL, cz, cs) || !M.unary(cs, COS, s) || !M.f32(cs)) continue;
    if (!M.slope(s, x, y, k)) continue;
    if (!M.product3(t2, sz, f, g)) continue;
    // {f, g} = {sin(s), cos(ar - aspect)}; the sum of squares names x and y in
    // either order, the aspect tells which is which
    bool ok = false;
    for (int sw2 = 0; sw2 < 4 && !ok; sw2++) {
      if (sw2 == 2) std::swap(x, y);
      std::vector<Node *> save = M.seen;
      Node *sn = (sw2 & 1) ? g : f, *cc = (sw2 & 1) ? f : g, *ss, *d, *da, *db;
      if (!(M.unary(sn, SIN, ss) && ss == s && M.unary(cc, COS, d) && M.f32(cc) && M.binary(d, SUB, da, db))) {
        M.seen = save;
        continue;
      }
      // cos(ar - aspect), or cos(aspect - ar) (cosine is even)
      std::vector<Node *> save2 = M.seen;
      if (M.is_const(da, ar) && M.aspect(db, x, y, pi2, pih, pi32)) {
        ok = true;
      } else {
        M.seen = save2;
        if (M.is_const(db, ar) && M.aspect(da, x, y, pi2, pih, pi32)) ok = true;
        else M.seen = save;
      }
    }
    if (!ok) continue;
    if (!near(pi2, 2 * PI) || !near(pih, PI / 2) || !near(pi32, 1.5 * PI)) continue;
    if (!std::isfinite(cz) || !std::isfinite(sz) || !std::isfinite(ar)) continue;
    m.hs = hs;
    m.x = x;
    m.y = y;
    std::sort(M.seen.begin(), M.seen.end(), [](Node *a, Node *b) { return a->id < b->id; });
    m.pattern = M.seen;
    m.cz = (float)cz;
    m.k_one = k == 1.0;
    m.szk = (float)(sz * k);
    m.kk = (float)(k * k);
    const double d = pi2 - 2 * PI;
    m.S0 = (float)std::sin(ar);
    m.C0 = (float)std::cos(ar);
    m.S1 = (float)std::sin(ar - d);
    m.C1 = (float)std::cos(ar - d);
    m.SH = (float)std::cos(ar - pih);
    m.S3 = (float)-std::cos(ar - pi32);
    return true;
  }
  return false;
}

}  // namespace mapb
