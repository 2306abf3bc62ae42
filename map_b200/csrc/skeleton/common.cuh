// Device building blocks shared by every generated map-algebra kernel.
// Compiled at run time by NVRTC (sm_100a) together with the per-group code the
// host generates; also compiled by nvcc at build time as a self-check.
//
// Contents: fixed-width types, the kernel argument pieces (raster references,
// scalar slots, geometry, TMA descriptors), cell loads/stores, the focal border
// rule, TMA tile staging with bounded mbarrier waits, warp/CTA reductions and a
// Philox2x32-10 counter-based generator.
#pragma once

typedef unsigned char u8;
typedef unsigned short u16;
typedef unsigned int u32;
typedef unsigned long long u64;
typedef signed char s8;
typedef short s16;
typedef int s32;
typedef long long s64;

// Opaque 128-byte TMA tensor map (filled on the host by cuTensorMapEncodeTiled).
struct __align__(64) TmaDesc { u64 w[16]; };

// A raster in device memory: base address and row pitch in bytes.
struct RasterArg { u64 p; s64 pitch; };

// One scalar (D0) value, stored in the member matching its data type.
union Scalar8 {
  float f32; double f64; bool b8; u8 vu8; u16 vu16; u32 vu32; u64 vu64;
  s8 vs8; s16 vs16; s32 vs32; s64 vs64; u64 raw;
};

// Shape of the raster a group computes and the region one launch covers.
struct Geom {
  s32 W, H;          // raster size in cells (x = columns, y = rows)
  s32 BS0, BS1;      // block size of the reference block grid
  s32 rx0, ry0;      // region origin (cells)
  s32 rx1, ry1;      // region end (exclusive)
  s32 tiles_x;       // tiles per region row
  s32 tiles;         // tiles in the region
  s32 border;        // 0 block mirror, 1 raster mirror, 2 dead
  s32 oy;            // raster row held by row 0 of the staged inputs' tensor maps (row bands; else 0)
};

enum { ERR_TMA_TIMEOUT = 1, ERR_BAD_LAUNCH = 2, ERR_ITER_LIMIT = 4, ERR_SPIN_LIMIT = 8 };

__device__ __forceinline__ void skel_fail(u32 *err, u32 code) {
  if (err) atomicOr(err, code);
}

// ------------------------------------------------------------------ loads / stores

template <class T> __device__ __forceinline__ const T *row_ptr(const RasterArg &r, int y) {
  return (const T *)(r.p + (u64)(s64)y * (u64)r.pitch);
}

template <class T> __device__ __forceinline__ T ldr(const RasterArg &r, int x, int y) {
  return __ldg(row_ptr<T>(r, y) + x);
}
template <> __device__ __forceinline__ bool ldr<bool>(const RasterArg &r, int x, int y) {
  return *(row_ptr<bool>(r, y) + x);
}

template <class T> __device__ __forceinline__ void str(const RasterArg &r, int x, int y, T v) {
  ((T *)(r.p + (u64)(s64)y * (u64)r.pitch))[x] = v;
}

// ------------------------------------------------------------------ atan2 (float)

// Two-argument arctangent of float32 operands, at most 1.5 ulp from the
// correctly rounded value (checked against double-precision atan2 on 80 M
// samples; the special cases follow IEEE 754 atan2). Method: reduce to
// t = min(|x|,|y|) / max(|x|,|y|) in [0, 1] (IEEE division), evaluate
// atan(t) = t + t*s*Q(s), s = t*t, with Q a degree-8 polynomial fitted to
// (atan(t)/t - 1)/s on [0, 1] by iteratively reweighted least squares (Lawson)
// for minimum relative error, then undo the reduction with pi/2 and pi split
// into two floats (one step per octant), and give the result the sign of y.
__device__ __forceinline__ float map_atan2f(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = ax > ay ? ax : ay, mn = ax > ay ? ay : ax;   // a NaN operand makes t NaN below
  float t = mn / mx;
  if (ax == 0.0f && ay == 0.0f) t = 0.0f;
  if (isinf(ax) && isinf(ay)) t = 1.0f;
  const float s = t * t;
  float q = -0x1.d62fecp-10f;
  q = fmaf(q, s, 0x1.65a65ap-7f);
  q = fmaf(q, s, -0x1.fed15ep-6f);
  q = fmaf(q, s, 0x1.dac9e2p-5f);
  q = fmaf(q, s, -0x1.583490p-4f);
  q = fmaf(q, s, 0x1.c099fep-4f);
  q = fmaf(q, s, -0x1.2421b6p-3f);
  q = fmaf(q, s, 0x1.9991fep-3f);
  q = fmaf(q, s, -0x1.55553ep-2f);
  float r = fmaf(t * s, q, t);
  // one reconstruction per octant, the constant's low part added first
  const bool neg = signbit(x);
  if (ay > ax) r = neg ? (-0x1.777a5cp-25f + r) + 0x1.921fb6p+0f    // pi/2 + r
                       : (-0x1.777a5cp-25f - r) + 0x1.921fb6p+0f;   // pi/2 - r
  else if (neg) r = (-0x1.777a5cp-24f - r) + 0x1.921fb6p+1f;       // pi - r
  return copysignf(r, y);
}

// ------------------------------------------------------------------ border rule

// Reflection used by the reference's focal loads: invert(i,d) = i<0 ? -i-1 : i>=d ? d-(i-d+1) : i
// (runtime/skeleton/util.cpp:493); clamped so a halo wider than the extent stays inside.
__device__ __forceinline__ int reflect_idx(int i, int d) {
  int r = i < 0 ? -i - 1 : (i >= d ? d - (i - d + 1) : i);
  return r < 0 ? 0 : (r >= d ? d - 1 : r);
}

// Source cell of the focal read (x+dx, y+dy) made by centre cell (x, y).
// Returns false when the read yields the dead-border zero.
//  block mirror (reference): a read outside the raster is served by the centre
//    cell's own block with each out-of-block local coordinate reflected at that
//    block's valid extent (util.cpp:498-506: `invert` on both coordinates when
//    the neighbour block does not exist).
//  raster mirror: each coordinate reflected at the raster edge.
__device__ __forceinline__ bool focal_src(const Geom &g, int x, int y, int dx, int dy, int &sx, int &sy) {
  int nx = x + dx, ny = y + dy;
  if ((unsigned)nx < (unsigned)g.W && (unsigned)ny < (unsigned)g.H) { sx = nx; sy = ny; return true; }
  if (g.border == 2) return false;
  if (g.border == 1) { sx = reflect_idx(nx, g.W); sy = reflect_idx(ny, g.H); return true; }
  int bx0 = (x / g.BS0) * g.BS0, by0 = (y / g.BS1) * g.BS1;
  int bw = min(g.BS0, g.W - bx0), bh = min(g.BS1, g.H - by0);
  sx = bx0 + reflect_idx(nx - bx0, bw);
  sy = by0 + reflect_idx(ny - by0, bh);
  return true;
}

// Whether a tile at the raster edge can be staged like an interior one: its halo
// cells outside the raster then hold the same value for every centre cell that
// reads them (dead border: zero; raster mirror: the mirrored cell; block mirror:
// only when the raster is one block, where it is the raster mirror).
__device__ __forceinline__ bool edge_staging(const Geom &g) {
  return g.border == 2 || g.border == 1 || (g.BS0 >= g.W && g.BS1 >= g.H);
}

// After a staged box of an edge tile has landed (raster cell (ox + bx, oy + by) at
// s[by * SW + bx]), overwrites its cells outside the raster that a centre cell can
// reach (within hx / hy of the edge) with the border rule's value. The sources
// are inside the raster, so no cell is both read and written.
template <class T, int SW, int SH>
__device__ __forceinline__ void stage_fix_border(T *s, const Geom &g, int ox, int oy, int hx, int hy) {
  for (int i = threadIdx.x; i < SW * SH; i += blockDim.x) {
    const int bx = i % SW, by = i / SW;
    const int rx = ox + bx, ry = oy + by;
    if ((unsigned)rx < (unsigned)g.W && (unsigned)ry < (unsigned)g.H) continue;
    if (rx < -hx || rx >= g.W + hx || ry < -hy || ry >= g.H + hy) continue;
    T v = (T)0;
    if (g.border != 2) v = s[(reflect_idx(ry, g.H) - oy) * SW + (reflect_idx(rx, g.W) - ox)];
    s[i] = v;
  }
}

// Focal tap served straight from global memory with the border rule (edge tiles).
template <class T> struct GatherTap {
  RasterArg r;
  const Geom *g;
  __device__ __forceinline__ T tap(int x, int y, int lx, int ly, int dx, int dy) const {
    int sx, sy;
    if (!focal_src(*g, x, y, dx, dy, sx, sy)) return (T)0;
    return ldr<T>(r, sx, sy);
  }
};

// Focal tap served from a tile staged in shared memory (interior tiles).
// The tile's element (0,0) is raster cell (x0 - PX, y0 - HY).
template <class T, int SW, int PX, int HY> struct SmemTap {
  const T *s;
  __device__ __forceinline__ T tap(int x, int y, int lx, int ly, int dx, int dy) const {
    return s[(ly + HY + dy) * SW + (lx + PX + dx)];
  }
};

// ------------------------------------------------------------------ TMA + mbarrier

__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(u64 *bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 parity) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may itself suspend for a
// while), so a copy that never lands ends the CTA with an error instead of a hang.
__device__ __forceinline__ bool mbar_wait_bounded(u64 *bar, u32 parity, u32 limit) {
  for (u32 i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// A tensor map that lives in global memory and was written through the generic
// proxy (e.g. an argument array copied from the host into reused memory) must be
// acquired by the tensor-map proxy before a TMA load uses it.
__device__ __forceinline__ void tensormap_acquire(const TmaDesc *tmap) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((u64)tmap) : "memory");
}

// 2-D tiled TMA load of box (x, y) of `tmap` into shared memory; completion is
// signalled on `bar` (complete_tx). x must be a multiple of 16 bytes of elements.
__device__ __forceinline__ void tma_load_2d(void *dst, const TmaDesc *tmap, u64 *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((u64)tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------------ tiles

// Tile t of the launch region: origin and the end of the computed cells.
struct Tile { int x0, y0, xe, ye; };

template <int TW, int TH> __device__ __forceinline__ Tile tile_of(const Geom &g, int t) {
  Tile r;
  int tx = t % g.tiles_x, ty = t / g.tiles_x;
  r.x0 = g.rx0 + tx * TW;
  r.y0 = g.ry0 + ty * TH;
  r.xe = min(r.x0 + TW, g.rx1);
  r.ye = min(r.y0 + TH, g.ry1);
  return r;
}

// Whether the tile plus its halo lies inside the raster (so TMA staging with no
// border handling serves every tap).
template <int TW, int TH> __device__ __forceinline__ bool tile_interior(const Geom &g, const Tile &t, int hx, int hy) {
  return t.x0 - hx >= 0 && t.x0 + TW + hx <= g.W && t.y0 - hy >= 0 && t.y0 + TH + hy <= g.H;
}

// ------------------------------------------------------------------ reductions

template <class T> __device__ __forceinline__ T red_max(T a, T b) { return a > b ? a : b; }
template <> __device__ __forceinline__ float red_max<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double red_max<double>(double a, double b) { return fmax(a, b); }
template <class T> __device__ __forceinline__ T red_min(T a, T b) { return a < b ? a : b; }
template <> __device__ __forceinline__ float red_min<float>(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ double red_min<double>(double a, double b) { return fmin(a, b); }

// op: 1 SUM, 2 PROD, 3 rAND, 4 rOR, 6 MAX, 7 MIN (ReductionEnum values)
template <int OP, class T> struct RedOp;
template <class T> struct RedOp<1, T> { __device__ static T f(T a, T b) { return (T)(a + b); } };
template <class T> struct RedOp<2, T> { __device__ static T f(T a, T b) { return (T)(a * b); } };
template <class T> struct RedOp<3, T> { __device__ static T f(T a, T b) { return (T)(a & b); } };
template <class T> struct RedOp<4, T> { __device__ static T f(T a, T b) { return (T)(a | b); } };
template <class T> struct RedOp<6, T> { __device__ static T f(T a, T b) { return red_max<T>(a, b); } };
template <class T> struct RedOp<7, T> { __device__ static T f(T a, T b) { return red_min<T>(a, b); } };

// Reinterprets the bytes of a value as another type of at most 8 bytes.
template <class To, class From> __device__ __forceinline__ To bit_cast8(From v) {
  union { From f; To t; u64 raw; } u;
  u.raw = 0;
  u.f = v;
  return u.t;
}

template <class T> __device__ __forceinline__ T shfl_xor_any(T v, int m) {
  if constexpr (sizeof(T) == 8) {
    u64 b = bit_cast8<u64>(v);
    u32 lo = (u32)b, hi = (u32)(b >> 32);
    lo = __shfl_xor_sync(0xffffffffu, lo, m);
    hi = __shfl_xor_sync(0xffffffffu, hi, m);
    return bit_cast8<T>(((u64)hi << 32) | lo);
  } else {
    u32 b = bit_cast8<u32>(v);
    b = __shfl_xor_sync(0xffffffffu, b, m);
    return bit_cast8<T>(b);
  }
}

// Deterministic CTA-wide reduction (fixed shuffle tree, then warps in order).
// `scratch` holds one Scalar8 per warp. Every thread must call it.
template <int OP, class T> __device__ __forceinline__ T block_reduce(T v, Scalar8 *scratch) {
  for (int m = 16; m > 0; m >>= 1) v = RedOp<OP, T>::f(v, shfl_xor_any<T>(v, m));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp].raw = bit_cast8<u64>(v);
  __syncthreads();
  T r = bit_cast8<T>(scratch[0].raw);
  for (int w = 1; w < nw; ++w) r = RedOp<OP, T>::f(r, bit_cast8<T>(scratch[w].raw));
  return r;
}

template <class T> __device__ __forceinline__ void put_scalar(Scalar8 *dst, T v) { dst->raw = bit_cast8<u64>(v); }
template <class T> __device__ __forceinline__ T get_scalar(const Scalar8 &s) { return bit_cast8<T>(s.raw); }

// ------------------------------------------------------------------ Philox2x32-10

// Counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): ten rounds of a 32x32->64 multiply with
// multiplier 0xD256D193, the key bumped by the Weyl constant 0x9E3779B9 between rounds.
__device__ __forceinline__ void philox2x32_10(u32 &c0, u32 &c1, u32 key) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    u32 hi = __umulhi(0xD256D193u, c0);
    u32 lo = 0xD256D193u * c0;
    u32 n0 = hi ^ key ^ c1;
    c1 = lo;
    c0 = n0;
    key += 0x9E3779B9u;
  }
}
