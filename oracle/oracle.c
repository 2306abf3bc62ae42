/*
 * CPU oracle for the map-algebra execution path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-cell semantics for the
 * workloads of the hot path, used by tests and by the CPU baseline leg of
 * bench.py as the checker. Nothing in the product links or calls it.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors, and
 * its OpenCL kernels cannot run here (no OpenCL platform). What is pinned on the
 * reference's own artefacts:
 *  - the per-cell operations, their order, the focal masks and loop nesting,
 *    the Philox counter / key, and the scalar constants the kernels receive,
 *    for hill.py, life.py and wsum.py: the reference's DAG, fusion compiler and
 *    kernel generators, built from its sources with stand-in OpenCL entry
 *    points (oracle/ref_codegen), print the kernels they generate, and
 *    tests/test_ref_codegen.py checks this file's restatements against them;
 *  - the host-side scalar operator tables, against the reference's util/
 *    sources compiled under oracle/ref_util (oracle/build_oracle.py).
 * Not pinned: cell VALUES computed by the reference's kernels (its OpenCL
 * implementation's transcendental functions have no fixed accuracy).
 *
 * Floating point: compiled with -ffp-contract=off and no fast-math so each
 * operation rounds once, in the order the reference's generated code writes
 * it; transcendental functions are the C library's (the reference used its
 * OpenCL implementation's builtins, so results agree to a few ulp).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ border rule */

/* invert(i,d) = i<0 ? -i-1 : i>=d ? d-(i-d+1) : i  (runtime/skeleton/util.cpp:493),
 * clamped into [0,d). */
static int reflect_idx(int i, int d) {
  int r = i < 0 ? -i - 1 : (i >= d ? d - (i - d + 1) : i);
  if (r < 0) r = 0;
  if (r >= d) r = d - 1;
  return r;
}

/* Source of focal read (x+dx, y+dy) by centre (x, y); returns 0 for a dead-border zero.
 * border 0: a read outside the raster is served from the centre cell's block with the
 *           block-local coordinates reflected at the block's valid extent
 *           (load_F in runtime/skeleton/util.cpp:498-506);
 * border 1: reflect at the raster edge;  border 2: zero outside. */
int orc_focal_src(int W, int H, int BS0, int BS1, int border, int x, int y, int dx, int dy, int *sx, int *sy) {
  int nx = x + dx, ny = y + dy;
  if (nx >= 0 && nx < W && ny >= 0 && ny < H) { *sx = nx; *sy = ny; return 1; }
  if (border == 2) return 0;
  if (border == 1) { *sx = reflect_idx(nx, W); *sy = reflect_idx(ny, H); return 1; }
  int bx0 = (x / BS0) * BS0, by0 = (y / BS1) * BS1;
  int bw = BS0 < W - bx0 ? BS0 : W - bx0, bh = BS1 < H - by0 ? BS1 : H - by0;
  *sx = bx0 + reflect_idx(nx - bx0, bw);
  *sy = by0 + reflect_idx(ny - by0, bh);
  return 1;
}

static float tapf(const float *in, int W, int H, int BS0, int BS1, int border, int x, int y, int dx, int dy) {
  int sx, sy;
  if (!orc_focal_src(W, H, BS0, BS1, border, x, y, dx, dy, &sx, &sy)) return 0.0f;
  return in[(size_t)sy * W + sx];
}
static uint8_t tapu8(const uint8_t *in, int W, int H, int BS0, int BS1, int border, int x, int y, int dx, int dy) {
  int sx, sy;
  if (!orc_focal_src(W, H, BS0, BS1, border, x, y, dx, dy, &sx, &sy)) return 0;
  return in[(size_t)sy * W + sx];
}

/* --------------------------------------------------------- focal: correlation */

/* Convolution node (runtime/skeleton/FocalSkeleton.cpp:300-336): acc = 0;
 * acc += in(y+i1, x+i0) * mask[i1+h1][i0+h0], i1 outer, i0 inner, F32. */
void orc_conv_f32(const float *in, int W, int H, int BS0, int BS1, int border, const float *mask, int mw, int mh,
                  float *out) {
  int hx = mw / 2, hy = mh / 2;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float acc = 0.0f;
      for (int i1 = -hy; i1 <= hy; i1++)
        for (int i0 = -hx; i0 <= hx; i0++) {
          float t = tapf(in, W, H, BS0, BS1, border, x, y, i0, i1);
          float p = t * mask[(i1 + hy) * mw + (i0 + hx)];
          acc = acc + p;
        }
      out[(size_t)y * W + x] = acc;
    }
}

/* ------------------------------------------------------------ hillshade */

/* hill.py (python/hill.py:15-50) with dist = 1 and zfactor = 1, zenith 45,
 * azimuth 315: Sobel derivatives / 8, slope = atan(sqrt(x^2+y^2)), aspect from
 * atan2(y,-x) with the script's PI = 3.141593, hs = cos(zr)cos(s) +
 * sin(zr)sin(s)cos(ar - aspect). Constants are folded in double precision by
 * Python and enter the kernel as F32 values (python/map.py:115). */
typedef struct {
  float cz, sz, ar, pi2, pih, pi32;
} HillConst;

static HillConst hill_const(double zenith, double azimuth) {
  const double PI = 3.141593;
  double zr = (90.0 - zenith) / 180.0 * PI;
  double ar = 360.0 - azimuth + 90.0;
  if (ar > 360.0) ar = ar - 360.0;
  ar = ar / 180.0 * PI;
  HillConst c;
  c.cz = (float)cos(zr);
  c.sz = (float)sin(zr);
  c.ar = (float)ar;
  c.pi2 = (float)(PI * 2);
  c.pih = (float)(PI / 2);
  c.pi32 = (float)(PI * 2 - PI / 2);
  return c;
}

static const int SOBEL_H[9] = {-1, 0, 1, -2, 0, 2, -1, 0, 1};
static const int SOBEL_V[9] = {-1, -2, -1, 0, 0, 0, 1, 2, 1};

/* One cell of the FP32 chain. */
static float hill_cell_f32(const float *dem, int W, int H, int BS0, int BS1, int border, const HillConst *c, int x,
                           int y, float *slope_v, float *aspect_v) {
  float ch = 0.0f, cv = 0.0f;
  for (int i1 = -1; i1 <= 1; i1++)
    for (int i0 = -1; i0 <= 1; i0++) {
      float t = tapf(dem, W, H, BS0, BS1, border, x, y, i0, i1);
      ch = ch + t * SOBEL_H[(i1 + 1) * 3 + (i0 + 1)];
      cv = cv + t * SOBEL_V[(i1 + 1) * 3 + (i0 + 1)];
    }
  float gx = ch / 8;
  float gy = cv / 8;
  float s = atanf(1 * sqrtf(gx * gx + gy * gy));
  float z1 = (float)(uint8_t)(gx != 0) * atan2f(gy, -gx);
  z1 = z1 + (float)(uint8_t)(z1 < 0) * c->pi2;
  float z0 = (float)(uint8_t)(gx == 0) * ((float)(uint8_t)(gy > 0) * c->pih + (float)(uint8_t)(gy < 0) * c->pi32);
  float asp = z1 + z0;
  *slope_v = s;
  *aspect_v = asp;
  return c->cz * cosf(s) + c->sz * sinf(s) * cosf(c->ar - asp);
}

void orc_hillshade_f32(const float *dem, int W, int H, int BS0, int BS1, int border, double zenith, double azimuth,
                       float *out, float *slope_out, float *aspect_out) {
  HillConst c = hill_const(zenith, azimuth);
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float s, asp;
      size_t i = (size_t)y * W + x;
      out[i] = hill_cell_f32(dem, W, H, BS0, BS1, border, &c, x, y, &s, &asp);
      if (slope_out) slope_out[i] = s;
      if (aspect_out) aspect_out[i] = asp;
    }
}

/* Rows [y0, y1) of the same computation over the whole raster (borders decided
 * by the whole raster), written to out[y * W + x]: the CPU baseline runs row
 * bands of one raster on several threads with this. */
void orc_hillshade_f32_rows(const float *dem, int W, int H, int BS0, int BS1, int border, double zenith,
                            double azimuth, int y0, int y1, float *out) {
  HillConst c = hill_const(zenith, azimuth);
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < W; x++) {
      float s, asp;
      out[(size_t)y * W + x] = hill_cell_f32(dem, W, H, BS0, BS1, border, &c, x, y, &s, &asp);
    }
}

/* FP64 twin: the same formula in double arithmetic (constants as the F32
 * values the kernel receives), used to state each implementation's error. */
void orc_hillshade_f64(const float *dem, int W, int H, int BS0, int BS1, int border, double zenith, double azimuth,
                       double *out) {
  HillConst c = hill_const(zenith, azimuth);
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double ch = 0.0, cv = 0.0;
      for (int i1 = -1; i1 <= 1; i1++)
        for (int i0 = -1; i0 <= 1; i0++) {
          double t = tapf(dem, W, H, BS0, BS1, border, x, y, i0, i1);
          ch += t * SOBEL_H[(i1 + 1) * 3 + (i0 + 1)];
          cv += t * SOBEL_V[(i1 + 1) * 3 + (i0 + 1)];
        }
      double gx = ch / 8, gy = cv / 8;
      double s = atan(sqrt(gx * gx + gy * gy));
      double z1 = (gx != 0) * atan2(gy, -gx);
      z1 = z1 + (z1 < 0) * (double)c.pi2;
      double z0 = (gx == 0) * ((gy > 0) * (double)c.pih + (gy < 0) * (double)c.pi32);
      double asp = z1 + z0;
      out[(size_t)y * W + x] = (double)c.cz * cos(s) + (double)c.sz * sin(s) * cos((double)c.ar - asp);
    }
}

/* Size of one float32 ulp at |v| (the spacing of floats there). */
static double ulp32(double v) {
  float f = fabsf((float)v);
  if (!(f < INFINITY)) return INFINITY;
  return (double)nextafterf(f, INFINITY) - (double)f;
}

/* First-order rounding-error scale of the FP32 hillshade chain at each cell,
 * from FP64 values: the chain evaluates cos and sin at rounded angles, so its
 * output moves by |d hs / d A| ulp(max(|aspect|, |A|)) for the azimuth
 * difference A = ar - aspect and by |d hs / d s| ulp(s) for the slope s, and
 * each of its two terms cz cos(s) and sz sin(s) cos(A) is itself rounded:
 *   bound = sz sin(s) |sin A| ulp(max(|aspect|, |A|))
 *         + (cz sin(s) + sz |cos(s) cos(A)|) ulp(s) + ulp(T1) + ulp(T2).
 * Used by the tests to state the hillshade tolerance where the two terms
 * cancel (there 4 ulp of the result is far below the chain's own error). */
void orc_hillshade_bound(const float *dem, int W, int H, int BS0, int BS1, int border, double zenith, double azimuth,
                         double *bound) {
  HillConst c = hill_const(zenith, azimuth);
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double ch = 0.0, cv = 0.0;
      for (int i1 = -1; i1 <= 1; i1++)
        for (int i0 = -1; i0 <= 1; i0++) {
          double t = tapf(dem, W, H, BS0, BS1, border, x, y, i0, i1);
          ch += t * SOBEL_H[(i1 + 1) * 3 + (i0 + 1)];
          cv += t * SOBEL_V[(i1 + 1) * 3 + (i0 + 1)];
        }
      double gx = ch / 8, gy = cv / 8;
      double s = atan(sqrt(gx * gx + gy * gy));
      double z1 = (gx != 0) * atan2(gy, -gx);
      z1 = z1 + (z1 < 0) * (double)c.pi2;
      double z0 = (gx == 0) * ((gy > 0) * (double)c.pih + (gy < 0) * (double)c.pi32);
      double asp = z1 + z0;
      double A = (double)c.ar - asp;
      double t1 = (double)c.cz * cos(s), t2 = (double)c.sz * sin(s) * cos(A);
      double amax = fabs(asp) > fabs(A) ? fabs(asp) : fabs(A);
      bound[(size_t)y * W + x] = (double)c.sz * sin(s) * fabs(sin(A)) * ulp32(amax) +
                                 ((double)c.cz * sin(s) + (double)c.sz * fabs(cos(s) * cos(A))) * ulp32(s) +
                                 ulp32(t1) + ulp32(t2);
    }
}

/* ------------------------------------------------------------ Game of Life */

/* life.py (python/life.py:24-34): nbh = convolve(state, [[1,1,1],[1,0,1],[1,1,1]])
 * (U8 x S32 mask -> S32), state = (nbh == 3) + (nbh == 2) * state, all U8. */
void orc_life(const uint8_t *in, int W, int H, int BS0, int BS1, int border, int gens, uint8_t *out) {
  size_t n = (size_t)W * H;
  uint8_t *a = (uint8_t *)malloc(n), *b = (uint8_t *)malloc(n);
  memcpy(a, in, n);
  for (int g = 0; g < gens; g++) {
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        int32_t nbh = 0;
        for (int i1 = -1; i1 <= 1; i1++)
          for (int i0 = -1; i0 <= 1; i0++) {
            int m = (i0 == 0 && i1 == 0) ? 0 : 1;
            nbh = nbh + tapu8(a, W, H, BS0, BS1, border, x, y, i0, i1) * m;
          }
        uint8_t s = a[(size_t)y * W + x];
        uint8_t e3 = (uint8_t)(nbh == 3), e2 = (uint8_t)(nbh == 2);
        b[(size_t)y * W + x] = (uint8_t)(e3 + (uint8_t)(e2 * s));
      }
    uint8_t *t = a; a = b; b = t;
  }
  memcpy(out, a, n);
  free(a);
  free(b);
}

/* One generation of life.py for rows [y0, y1) only, reading the whole raster
 * `in` (W x H) and writing out[y * W + x]: with in holding valid rows
 * [y0 - 1, y1 + 1) only, this is what one rank of a row-band split computes. */
void orc_life_rows(const uint8_t *in, int W, int H, int BS0, int BS1, int border, int y0, int y1, uint8_t *out) {
  for (int y = y0; y < y1; y++)
    for (int x = 0; x < W; x++) {
      int32_t nbh = 0;
      for (int i1 = -1; i1 <= 1; i1++)
        for (int i0 = -1; i0 <= 1; i0++) {
          int m = (i0 == 0 && i1 == 0) ? 0 : 1;
          nbh = nbh + tapu8(in, W, H, BS0, BS1, border, x, y, i0, i1) * m;
        }
      uint8_t s = in[(size_t)y * W + x];
      uint8_t e3 = (uint8_t)(nbh == 3), e2 = (uint8_t)(nbh == 2);
      out[(size_t)y * W + x] = (uint8_t)(e3 + (uint8_t)(e2 * s));
    }
}

/* FocalPercent (runtime/skeleton/FocalSkeleton.cpp:375-403, util/PercentType.cpp):
 * count, in the argument's type, the cells of the (2hx+1) x (2hy+1) window
 * around the cell for which `centre OP cell` holds (OP: == for type 1 AGE,
 * > for type 2 ILE), then divide by the window size in that type. The window
 * is centred and the divisor is the window size (the reference's kernel starts
 * its loop at the centre and drops the parentheses of its divisor). */
void orc_focal_percent_f32(const float *in, int W, int H, int BS0, int BS1, int border, int hx, int hy, int type,
                           float *out) {
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float c = in[(size_t)y * W + x], v = 0.0f;
      for (int i1 = -hy; i1 <= hy; i1++)
        for (int i0 = -hx; i0 <= hx; i0++) {
          float t = tapf(in, W, H, BS0, BS1, border, x, y, i0, i1);
          v = v + (float)(type == 1 ? (c == t) : (c > t));
        }
      out[(size_t)y * W + x] = v / (float)((2 * hx + 1) * (2 * hy + 1));
    }
}
void orc_focal_percent_u8(const uint8_t *in, int W, int H, int BS0, int BS1, int border, int hx, int hy, int type,
                          uint8_t *out) {
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      uint8_t c = in[(size_t)y * W + x], v = 0;
      for (int i1 = -hy; i1 <= hy; i1++)
        for (int i0 = -hx; i0 <= hx; i0++) {
          uint8_t t = tapu8(in, W, H, BS0, BS1, border, x, y, i0, i1);
          v = (uint8_t)(v + (uint8_t)(type == 1 ? (c == t) : (c > t)));
        }
      out[(size_t)y * W + x] = (uint8_t)(v / (uint8_t)((2 * hx + 1) * (2 * hy + 1)));
    }
}

/* ------------------------------------------------------------ weighted sum */

/* wsum.py (python/wsum.py:11) generalised to k layers:
 * out = ((((0 + w0*r0) + w1*r1) + ...) + 0) evaluated left to right in F32. */
void orc_wsum_f32(const float *const *layers, const float *w, int k, size_t n, float *out) {
  for (size_t i = 0; i < n; i++) {
    float acc = (float)0;
    for (int j = 0; j < k; j++) acc = acc + w[j] * layers[j][i];
    out[i] = acc + 0;
  }
}

/* ------------------------------------------------------------ Philox / rand */

/* Philox2x32-10 (Salmon et al., SC'11): multiplier 0xD256D193, Weyl key bump 0x9E3779B9. */
void orc_philox2x32_10(uint32_t *c0, uint32_t *c1, uint32_t key) {
  for (int r = 0; r < 10; r++) {
    uint64_t p = (uint64_t)0xD256D193u * (uint64_t)(*c0);
    uint32_t hi = (uint32_t)(p >> 32), lo = (uint32_t)p;
    uint32_t n0 = hi ^ key ^ *c1;
    *c1 = lo;
    *c0 = n0;
    key += 0x9E3779B9u;
  }
}

/* Rand node (runtime/skeleton/Skeleton.cpp:183-206): counter {seed, 0}, key
 * BS1*BC1 + BS0*BC0 + bc1*BS0 + bc0 (block coordinate BC, in-block coordinate bc);
 * a U8 result takes the low byte of the first counter word. */
void orc_rand_u8(uint32_t seed, int W, int H, int BS0, int BS1, uint8_t *out) {
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      uint32_t key = (uint32_t)(BS1 * (y / BS1) + BS0 * (x / BS0) + (y % BS1) * BS0 + (x % BS0));
      uint32_t c0 = seed, c1 = 0;
      orc_philox2x32_10(&c0, &c1, key);
      out[(size_t)y * W + x] = (uint8_t)(c0 & 0xffu);
    }
}

/* ------------------------------------------------------------ D8 flow direction */

/* FocalFlow (runtime/skeleton/FocalSkeleton.cpp:405-443): for dir in E, SE, S,
 * SW, W, NW, N, NE: drop = (self - nbh) / (dir even ? 1 : 1.414213f); keep the
 * first strictly greater than the running max (initially 0); code 1 << dir. */
void orc_d8(const float *dem, int W, int H, int BS0, int BS1, int border, uint8_t *out) {
  static const int ox[8] = {1, 1, 0, -1, -1, -1, 0, 1}, oy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float self = dem[(size_t)y * W + x], mx = 0.0f;
      int pos = -1;
      for (int d = 0; d < 8; d++) {
        float zd = self - tapf(dem, W, H, BS0, BS1, border, x, y, ox[d], oy[d]);
        float ds = (d % 2 == 0) ? 1.0f : 1.414213f;
        float dr = zd / ds;
        if (dr > mx) { mx = dr; pos = d; }
      }
      out[(size_t)y * W + x] = pos == -1 ? 0 : (uint8_t)(1u << pos);
    }
}

/* ------------------------------------------------------------ flow accumulation */

/* SpreadScan SUM over D8 directions (runtime/skeleton/SpreadingSkeleton.cpp:288-393,
 * runtime/task/SpreadingTask.cpp): the result at a cell is the sum of the water
 * of every strictly-upstream cell (cells whose D8 path passes through it); the
 * cell's own water is not included. Restated as a topological accumulation:
 * each cell passes (its accumulation + its water) to the neighbour its code
 * points at. Codes that point outside the raster drop their flow. */
int orc_flowacc_s32(const int32_t *water, const uint8_t *dir, int W, int H, int32_t *out) {
  static const int ox[8] = {1, 1, 0, -1, -1, -1, 0, 1}, oy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  size_t n = (size_t)W * H;
  int32_t *indeg = (int32_t *)calloc(n, sizeof(int32_t));
  int64_t *down = (int64_t *)malloc(n * sizeof(int64_t));
  int64_t *queue = (int64_t *)malloc(n * sizeof(int64_t));
  for (size_t i = 0; i < n; i++) out[i] = 0;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      down[i] = -1;
      uint8_t c = dir[i];
      int d = -1;
      for (int k = 0; k < 8; k++) if (c == (1u << k)) d = k;
      if (d < 0) continue;
      int nx = x + ox[d], ny = y + oy[d];
      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
      down[i] = (int64_t)ny * W + nx;
      indeg[down[i]]++;
    }
  size_t qh = 0, qt = 0;
  for (size_t i = 0; i < n; i++) if (indeg[i] == 0) queue[qt++] = (int64_t)i;
  while (qh < qt) {
    int64_t i = queue[qh++];
    if (down[i] >= 0) {
      out[down[i]] += out[i] + water[i];
      if (--indeg[down[i]] == 0) queue[qt++] = down[i];
    }
  }
  int cyclic = qt != n;   /* cells on a direction cycle never drain */
  free(indeg);
  free(down);
  free(queue);
  return cyclic;
}

/* ------------------------------------------------------------ radial scan */

/* RadialScan (runtime/skeleton/RadiatingSkeleton.cpp:297-323, util.cpp:556-616):
 * within each octant around the start cell, with d0 the distance along the
 * octant's primary axis and d1 along the secondary (0 <= d1 <= d0):
 *   out(d0,d1) = op(LIT(out(d0-1,d1), out(d0-1,d1-1)), in(d0,d1)) when in is finite,
 *   LIT(a,b) = a if d1 == 0, b if d0 == d1, else a*w + b*(1-w) with
 *   w = d1/(float)d0*(d0-1) - (d1-1); the start cell is the neutral value.
 * op: 6 MAX, 7 MIN, 1 SUM, 2 PROD (F32). */
void orc_radial_f32(const float *in, int W, int H, int sx, int sy, int op, float *out) {
  float neutral = op == 6 ? -INFINITY : op == 7 ? INFINITY : op == 1 ? 0.0f : 1.0f;
  /* octants: primary unit (p0,p1), secondary unit (q0,q1) */
  static const int P[8][4] = {{1, 0, 0, 1}, {1, 0, 0, -1}, {-1, 0, 0, 1}, {-1, 0, 0, -1},
                              {0, 1, 1, 0}, {0, 1, -1, 0}, {0, -1, 1, 0}, {0, -1, -1, 0}};
  for (size_t i = 0; i < (size_t)W * H; i++) out[i] = NAN;
  out[(size_t)sy * W + sx] = neutral;
  int maxd = W + H;
  for (int o = 0; o < 8; o++) {
    int p0 = P[o][0], p1 = P[o][1], q0 = P[o][2], q1 = P[o][3];
    for (int d0 = 1; d0 < maxd; d0++) {
      int any = 0;
      for (int d1 = 0; d1 <= d0; d1++) {
        int x = sx + p0 * d0 + q0 * d1, y = sy + p1 * d0 + q1 * d1;
        if (x < 0 || y < 0 || x >= W || y >= H) continue;
        any = 1;
        int ax = sx + p0 * (d0 - 1) + q0 * d1, ay = sy + p1 * (d0 - 1) + q1 * d1;
        int bx = sx + p0 * (d0 - 1) + q0 * (d1 - 1), by = sy + p1 * (d0 - 1) + q1 * (d1 - 1);
        float a = (d1 <= d0 - 1) ? out[(size_t)ay * W + ax] : NAN;
        float b = (d1 >= 1) ? out[(size_t)by * W + bx] : NAN;
        float lit;
        if (d1 == 0) lit = a;
        else if (d0 == d1) lit = b;
        else {
          float w = d1 / (float)d0 * (d0 - 1.0f) - (d1 - 1.0f);
          lit = a * w + b * (1.0f - w);
        }
        float v = in[(size_t)y * W + x], r = lit;
        if (isfinite(v)) {
          if (op == 6) r = fmaxf(lit, v);
          else if (op == 7) r = fminf(lit, v);
          else if (op == 1) r = lit + v;
          else r = lit * v;
        }
        out[(size_t)y * W + x] = r;
      }
      if (!any && d0 > 1) {
        /* the octant left the raster */
        int x0 = sx + p0 * d0, y0 = sy + p1 * d0;
        if ((x0 < 0 || y0 < 0 || x0 >= W || y0 >= H)) break;
      }
    }
  }
}

/* ---------------------------------------------------- per-zone statistics */

/* Per-zone count / min / max / sum of a float32 value raster over an int32
 * zone raster: a new operation with no counterpart in the reference (its zonal
 * skeleton, runtime/skeleton/ZonalSkeleton.cpp:33-292, reduces the whole raster
 * to one value); the per-cell rules are the reference's SUM / MIN / MAX
 * reductions (runtime/skeleton/util.cpp:518-540). A cell counts when
 * 0 <= zone < nzones and the value is not NaN. min / max compare floats in
 * totalOrder (-0 before +0). sum32 adds in float32 in row-major order, sum64 in
 * double; either may be NULL. Empty zones: count 0, min +inf, max -inf, sums 0. */
static uint32_t fkey32(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

void orc_zone_stats(const float *val, const int32_t *zone, long long n, int nzones, uint64_t *count, float *vmin,
                    float *vmax, float *sum32, double *sum64) {
  for (int z = 0; z < nzones; z++) {
    count[z] = 0;
    vmin[z] = INFINITY;
    vmax[z] = -INFINITY;
    if (sum32) sum32[z] = 0.0f;
    if (sum64) sum64[z] = 0.0;
  }
  for (long long i = 0; i < n; i++) {
    const int32_t z = zone[i];
    const float v = val[i];
    if (z < 0 || z >= nzones || v != v) continue;
    if (count[z] == 0 || fkey32(v) < fkey32(vmin[z])) vmin[z] = v;
    if (count[z] == 0 || fkey32(v) > fkey32(vmax[z])) vmax[z] = v;
    count[z]++;
    if (sum32) sum32[z] += v;
    if (sum64) sum64[z] += (double)v;
  }
}
