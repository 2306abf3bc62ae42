// C++ builders of the reference's example programs (see programs.hpp).
#include "programs.hpp"

#include <cmath>

namespace mapb {

namespace {

const double PI = 3.141593;   // the constant the reference scripts use

Variant vs32(int v) {
  Variant r{};
  r.dtype = S32;
  r.u.s32 = v;
  return r;
}
Variant vf32(double v) {   // a Python float becomes an F32 Variant (python/map.py:115)
  Variant r{};
  r.dtype = F32;
  r.u.f32 = (float)v;
  return r;
}
Node *cint(Runtime &rt, int v) { return rt.constant(vs32(v), Arr2{{-1, -1}, 0}, S32, ROW + BLK, Arr2{{-1, -1}, 0}); }
Node *cflt(Runtime &rt, double v) { return rt.constant(vf32(v), Arr2{{-1, -1}, 0}, F32, ROW + BLK, Arr2{{-1, -1}, 0}); }

Node *conv3(Runtime &rt, Node *dem, const int m[9]) {
  Variant mv[9];
  for (int i = 0; i < 9; i++) mv[i] = vs32(m[i]);
  return rt.convolution(dem, mv, 9, Arr2{{3, 3}, 2});
}

const int HORI[9] = {-1, 0, 1, -2, 0, 2, -1, 0, 1};
const int VERT[9] = {-1, -2, -1, 0, 0, 0, 1, 2, 1};

Node *hori(Runtime &rt, Node *dem) { return rt.binary(conv3(rt, dem, HORI), cint(rt, 8 * 1), DIV); }
Node *vert(Runtime &rt, Node *dem) { return rt.binary(conv3(rt, dem, VERT), cint(rt, 8 * 1), DIV); }

}  // namespace

Node *prog_slope(Runtime &rt, Node *dem) {
  Node *x = hori(rt, dem);
  Node *y = vert(rt, dem);
  Node *xx = rt.binary(x, x, MUL);
  Node *yy = rt.binary(y, y, MUL);
  Node *s = rt.unary(rt.binary(xx, yy, ADD), SQRT);
  return rt.unary(rt.binary(cint(rt, 1), s, MUL), ATAN);
}

Node *prog_aspect(Runtime &rt, Node *dem) {
  Node *x = hori(rt, dem);
  Node *y = vert(rt, dem);
  Node *ne = rt.binary(x, cint(rt, 0), NE);
  Node *at = rt.binary(y, rt.unary(x, NEG), ATAN2);
  Node *z1 = rt.binary(ne, at, MUL);
  Node *lt = rt.binary(z1, cint(rt, 0), LT);
  z1 = rt.binary(z1, rt.binary(lt, cflt(rt, PI * 2), MUL), ADD);
  Node *eq = rt.binary(x, cint(rt, 0), EQ);
  Node *gt = rt.binary(y, cint(rt, 0), GT);
  Node *a = rt.binary(gt, cflt(rt, PI / 2), MUL);
  Node *lt2 = rt.binary(y, cint(rt, 0), LT);
  Node *b = rt.binary(lt2, cflt(rt, PI * 2 - PI / 2), MUL);
  Node *z0 = rt.binary(eq, rt.binary(a, b, ADD), MUL);
  return rt.binary(z1, z0, ADD);
}

Node *prog_hillshade(Runtime &rt, Node *dem, double zenith, double azimuth) {
  const double zr = (90 - zenith) / 180 * PI;
  double ar = 360 - azimuth + 90;
  ar = ar > 360 ? ar - 360 : ar;
  ar = ar / 180 * PI;
  Node *t1 = rt.binary(cflt(rt, std::cos(zr)), rt.unary(prog_slope(rt, dem), COS), MUL);
  Node *t2 = rt.binary(cflt(rt, std::sin(zr)), rt.unary(prog_slope(rt, dem), SIN), MUL);
  Node *t3 = rt.unary(rt.binary(cflt(rt, ar), prog_aspect(rt, dem), SUB), COS);
  return rt.binary(t1, rt.binary(t2, t3, MUL), ADD);
}

Node *prog_viewshed(Runtime &rt, Node *dem, int obs_x, int obs_y, float obs_h, double radius, Node **ox_out,
                    Node **oy_out, Node **oh_out) {
  Node *h = rt.scalar_param(vf32(obs_h));
  if (oh_out) *oh_out = h;
  Node *shift = rt.binary(dem, h, SUB);
  Node *ox = rt.scalar_param(vs32(obs_x));
  Node *oy = rt.scalar_param(vs32(obs_y));
  if (ox_out) *ox_out = ox;
  if (oy_out) *oy_out = oy;
  Node *x = rt.binary(ox, rt.index(dem, D1), SUB);
  Node *y = rt.binary(oy, rt.index(dem, D2), SUB);
  Node *dist = rt.unary(rt.binary(rt.binary(rt.binary(x, x, MUL), rt.binary(y, y, MUL), ADD), cflt(rt, 0.0), ADD), SQRT);
  Node *slope = rt.binary(shift, dist, DIV);
  Node *maxr = rt.radial_scan(slope, MAX, Arr2{{obs_x, obs_y}, 2}, radius);
  return rt.binary(rt.binary(rt.binary(maxr, dist, MUL), h, ADD), dem, SUB);
}

Node *prog_flow(Runtime &rt, Node *dem, Node **dirs_out) {
  Node *dirs = rt.focal_flow(dem);
  if (dirs_out) *dirs_out = dirs;
  Variant one = vs32(1);
  Node *water = rt.constant(one, dem->meta.ds, S32, dem->meta.memorder, dem->meta.bs);
  return rt.spread_scan(water, dirs, SUM);
}

}  // namespace mapb
