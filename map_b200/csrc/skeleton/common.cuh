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

// Store of a Local / Focal result cell as an explicit global store that declares
// no other memory effect, so the compiler keeps shared-memory taps (and other
// loads) of one cell in registers for the next cells of the column instead of
// reloading them after every store through a pointer that might alias them.
// Only for kernels that never read, within the launch, what they write.
template <int N> struct map_stg;
template <> struct map_stg<1> {
  static __device__ __forceinline__ void st(u64 p, u32 v) { asm volatile("st.global.u8 [%0], %1;" ::"l"(p), "r"(v)); }
};
template <> struct map_stg<2> {
  static __device__ __forceinline__ void st(u64 p, u32 v) { asm volatile("st.global.u16 [%0], %1;" ::"l"(p), "r"(v)); }
};
template <> struct map_stg<4> {
  static __device__ __forceinline__ void st(u64 p, u32 v) { asm volatile("st.global.u32 [%0], %1;" ::"l"(p), "r"(v)); }
};
template <> struct map_stg<8> {
  static __device__ __forceinline__ void st(u64 p, u64 v) { asm volatile("st.global.u64 [%0], %1;" ::"l"(p), "l"(v)); }
};
template <int N> struct map_stg_word { typedef u32 type; };
template <> struct map_stg_word<8> { typedef u64 type; };
template <class T> __device__ __forceinline__ void str_out(const RasterArg &r, int x, int y, T v) {
  const u64 p = r.p + (u64)(s64)y * (u64)r.pitch + (u64)(s64)x * sizeof(T);
  typename map_stg_word<sizeof(T)>::type b = 0;
  memcpy(&b, &v, sizeof(T));
  map_stg<sizeof(T)>::st(p, b);
}
template <> __device__ __forceinline__ void str_out<bool>(const RasterArg &r, int x, int y, bool v) {
  map_stg<1>::st(r.p + (u64)(s64)y * (u64)r.pitch + (u64)(s64)x, v ? 1u : 0u);
}
// Address of cell (x, y) of an output, computed once per thread: the rows of a
// thread's cells are then reached with one 32 x 32 -> 64-bit multiply-add each
// (str_out_row) instead of a 64-bit product per store.
template <class T> __device__ __forceinline__ u64 out_addr(const RasterArg &r, int x, int y) {
  return r.p + (u64)(s64)y * (u64)r.pitch + (u64)(s64)x * sizeof(T);
}
// the cell k rows below the one at `base` (pitch below 4 GiB)
template <class T> __device__ __forceinline__ void str_out_row(u64 base, u32 pitch, u32 k, T v) {
  typename map_stg_word<sizeof(T)>::type b = 0;
  memcpy(&b, &v, sizeof(T));
  map_stg<sizeof(T)>::st(base + (u64)k * (u64)pitch, b);
}
template <> __device__ __forceinline__ void str_out_row<bool>(u64 base, u32 pitch, u32 k, bool v) {
  map_stg<1>::st(base + (u64)k * (u64)pitch, v ? 1u : 0u);
}

// the cells (x, y) and (x + 1, y): one 8-byte store for 4-byte cells whose row
// and x allow it (x even, base and pitch 8-byte aligned), else two stores
template <class T> __device__ __forceinline__ void str_out2x(const RasterArg &r, int x, int y, T v0, T v1) {
  if constexpr (sizeof(T) == 4) {
    if (((r.p | (u64)r.pitch) & 7) == 0 && (x & 1) == 0) {
      u32 a, b;
      memcpy(&a, &v0, 4);
      memcpy(&b, &v1, 4);
      const u64 p = r.p + (u64)(s64)y * (u64)r.pitch + (u64)(s64)x * 4;
      asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"(a), "r"(b));
      return;
    }
  }
  str_out<T>(r, x, y, v0);
  str_out<T>(r, x + 1, y, v1);
}

// Lane j of a 16-byte vector of cells of type T, and its assignment.
template <class T> __device__ __forceinline__ T vlane(const uint4 &v, int j) {
  T r;
  memcpy(&r, (const char *)&v + j * sizeof(T), sizeof(T));
  return r;
}
template <class T> __device__ __forceinline__ void vset(uint4 &v, int j, T x) {
  memcpy((char *)&v + j * sizeof(T), &x, sizeof(T));
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
// The three steps are separate so that the polynomial can also run on packed
// pairs (map_atan2f on PR<float> below) with the same operations.
#define MAP_ATAN_Q0 -0x1.d62fecp-10f
#define MAP_ATAN_Q1 0x1.65a65ap-7f
#define MAP_ATAN_Q2 -0x1.fed15ep-6f
#define MAP_ATAN_Q3 0x1.dac9e2p-5f
#define MAP_ATAN_Q4 -0x1.583490p-4f
#define MAP_ATAN_Q5 0x1.c099fep-4f
#define MAP_ATAN_Q6 -0x1.2421b6p-3f
#define MAP_ATAN_Q7 0x1.9991fep-3f
#define MAP_ATAN_Q8 -0x1.55553ep-2f
__device__ __forceinline__ float map_atan2_arg(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = ax > ay ? ax : ay, mn = ax > ay ? ay : ax;   // a NaN operand makes t NaN below
  float t = mn / mx;
  if (ax == 0.0f && ay == 0.0f) t = 0.0f;
  if (isinf(ax) && isinf(ay)) t = 1.0f;
  return t;
}
__device__ __forceinline__ float map_atan_poly(float t) {
  const float s = t * t;
  float q = MAP_ATAN_Q0;
  q = fmaf(q, s, MAP_ATAN_Q1);
  q = fmaf(q, s, MAP_ATAN_Q2);
  q = fmaf(q, s, MAP_ATAN_Q3);
  q = fmaf(q, s, MAP_ATAN_Q4);
  q = fmaf(q, s, MAP_ATAN_Q5);
  q = fmaf(q, s, MAP_ATAN_Q6);
  q = fmaf(q, s, MAP_ATAN_Q7);
  q = fmaf(q, s, MAP_ATAN_Q8);
  return fmaf(t * s, q, t);
}
__device__ __forceinline__ float map_atan2_finish(float r, float y, float x) {
  // one reconstruction per octant, the constant's low part added first
  const bool neg = signbit(x);
  if (fabsf(y) > fabsf(x)) r = neg ? (-0x1.777a5cp-25f + r) + 0x1.921fb6p+0f    // pi/2 + r
                                   : (-0x1.777a5cp-25f - r) + 0x1.921fb6p+0f;   // pi/2 - r
  else if (neg) r = (-0x1.777a5cp-24f - r) + 0x1.921fb6p+1f;                   // pi - r
  return copysignf(r, y);
}
__device__ __forceinline__ float map_atan2f(float y, float x) {
  return map_atan2_finish(map_atan_poly(map_atan2_arg(y, x)), y, x);
}

// ------------------------------------------------------------------ sine / cosine (float)

// Sine and cosine of float32 arguments, at most 1.6 ulp from the correctly
// rounded value (checked against double-precision sin/cos on 100 M samples,
// including the floats nearest to multiples of pi/2). Method (Cody and Waite):
// x = j*pi/2 + r with j = rint(x*2/pi) (added to 1.5*2^23 so that the rounding
// gives the integer and its low bits the quadrant) and r = x - j*(P1 + P2 + P3),
// pi/2 split into three floats, each truncated so all three are positive (the
// first product is exact for |x| <= 65536); then sin(r) = r + r*s*S(s) and
// cos(r) = 1 + s*C(s), s = r*r, with S (degree 2) and C (degree 3) fitted on
// [0, pi/4] by iteratively reweighted least squares (Lawson) for minimum
// relative error; the quadrant swaps and negates. Larger |x| (and infinities)
// go to the CUDA library's functions, which reduce with more bits of 2/pi.
#define MAP_2OPI 0x1.45f306p-1f
#define MAP_PIO2_1 0x1.921fb4p+0f
#define MAP_PIO2_2 0x1.4442d0p-24f
#define MAP_PIO2_3 0x1.84698ap-48f
#define MAP_RINT 0x1.8p23f
#define MAP_TRIG_BOUND 65536.0f
#define MAP_SIN_1 -0x1.555546p-3f
#define MAP_SIN_2 0x1.11073ap-7f
#define MAP_SIN_3 -0x1.9943e2p-13f
#define MAP_COS_1 -0x1.0p-1f
#define MAP_COS_2 0x1.55553cp-5f
#define MAP_COS_3 -0x1.6c07f2p-10f
#define MAP_COS_4 0x1.99169cp-16f

// v = r + r*s*S(s) for |r| <= pi/4 is sin r; a zero keeps the sign of r (sin(-0) = -0)
__device__ __forceinline__ float map_sin_sign(float v, float r) {
  return __uint_as_float(__float_as_uint(v) | (__float_as_uint(r) & 0x80000000u));
}
// quadrant q: sin x = (q odd ? cos r : sin r), negated when bit 1 of q is set;
// cos x = (q odd ? sin r : cos r), negated when bit 1 of q + 1 is set
__device__ __forceinline__ float map_quadrant_sin(u32 q, float sr, float cr) {
  const float v = (q & 1u) ? cr : sr;
  return __uint_as_float(__float_as_uint(v) ^ ((q << 30) & 0x80000000u));
}
__device__ __forceinline__ float map_quadrant_cos(u32 q, float sr, float cr) {
  const float v = (q & 1u) ? sr : cr;
  return __uint_as_float(__float_as_uint(v) ^ (((q + 1u) << 30) & 0x80000000u));
}
// reduced argument and quadrant of |x| <= MAP_TRIG_BOUND; sin r and cos r
__device__ __forceinline__ void map_sincos_reduced(float x, u32 &q, float &sr, float &cr) {
  const float t = fmaf(x, MAP_2OPI, MAP_RINT);
  const float j = t - MAP_RINT;
  q = __float_as_uint(t);
  float r = fmaf(j, -MAP_PIO2_1, x);
  r = fmaf(j, -MAP_PIO2_2, r);
  r = fmaf(j, -MAP_PIO2_3, r);
  const float s = r * r;
  float p = fmaf(s, MAP_SIN_3, MAP_SIN_2);
  p = fmaf(s, p, MAP_SIN_1);
  sr = map_sin_sign(fmaf(r * s, p, r), r);
  float c = fmaf(s, MAP_COS_4, MAP_COS_3);
  c = fmaf(s, c, MAP_COS_2);
  c = fmaf(s, c, MAP_COS_1);
  cr = fmaf(s, c, 1.0f);
}
__device__ __forceinline__ void map_sincosf(float x, float *sp, float *cp) {
  if (fabsf(x) > MAP_TRIG_BOUND) { sincosf(x, sp, cp); return; }
  u32 q;
  float sr, cr;
  map_sincos_reduced(x, q, sr, cr);
  *sp = map_quadrant_sin(q, sr, cr);
  *cp = map_quadrant_cos(q, sr, cr);
}
__device__ __forceinline__ float map_sinf(float x) {
  if (fabsf(x) > MAP_TRIG_BOUND) return sinf(x);
  u32 q;
  float sr, cr;
  map_sincos_reduced(x, q, sr, cr);
  return map_quadrant_sin(q, sr, cr);
}
__device__ __forceinline__ float map_cosf(float x) {
  if (fabsf(x) > MAP_TRIG_BOUND) return cosf(x);
  u32 q;
  float sr, cr;
  map_sincos_reduced(x, q, sr, cr);
  return map_quadrant_cos(q, sr, cr);
}

// ------------------------------------------------------------------ paired cells

// PR<T>: the values of two cells of one column (rows y and y + 1) carried
// together, so that float work of both cells issues as Blackwell's packed
// f32x2 instructions (one issue slot for two IEEE operations). Every operation
// applies to each lane with exactly the scalar semantics: the C++ usual
// arithmetic conversions, then per-lane IEEE round-to-nearest (addition,
// subtraction and multiplication of floats are packed; division and the other
// operations run per lane). Generated code spells every conversion as PR<T>(...).
template <class T> struct map_scalar {};
#define MAP_SCALAR(T) template <> struct map_scalar<T> { typedef T type; };
MAP_SCALAR(bool) MAP_SCALAR(char) MAP_SCALAR(signed char) MAP_SCALAR(unsigned char) MAP_SCALAR(short)
MAP_SCALAR(unsigned short) MAP_SCALAR(int) MAP_SCALAR(unsigned) MAP_SCALAR(long) MAP_SCALAR(unsigned long)
MAP_SCALAR(long long) MAP_SCALAR(unsigned long long) MAP_SCALAR(float) MAP_SCALAR(double)
#undef MAP_SCALAR

template <class T> struct PR {
  T a, b;
  __device__ __forceinline__ PR() {}
  __device__ __forceinline__ PR(T a_, T b_) : a(a_), b(b_) {}
  template <class U> __device__ __forceinline__ explicit PR(const PR<U> &o) : a((T)o.a), b((T)o.b) {}
  template <class U, class = typename map_scalar<U>::type> __device__ __forceinline__ explicit PR(U s) : a((T)s), b((T)s) {}
};

template <class T> __device__ __forceinline__ T lane0(const PR<T> &p) { return p.a; }
template <class T> __device__ __forceinline__ T lane1(const PR<T> &p) { return p.b; }
template <class T, class = typename map_scalar<T>::type> __device__ __forceinline__ T lane0(const T &s) { return s; }
template <class T, class = typename map_scalar<T>::type> __device__ __forceinline__ T lane1(const T &s) { return s; }

__device__ __forceinline__ float2 pr_f2(const PR<float> &x) { return make_float2(x.a, x.b); }
__device__ __forceinline__ PR<float> pr_of(float2 v) { return PR<float>(v.x, v.y); }
__device__ __forceinline__ float2 f2_of(float c) { return make_float2(c, c); }

// lane-wise arithmetic on operands already converted to their common type
template <class T> __device__ __forceinline__ PR<T> pr_add(const PR<T> &x, const PR<T> &y) { return PR<T>(x.a + y.a, x.b + y.b); }
template <class T> __device__ __forceinline__ PR<T> pr_sub(const PR<T> &x, const PR<T> &y) { return PR<T>(x.a - y.a, x.b - y.b); }
template <class T> __device__ __forceinline__ PR<T> pr_mul(const PR<T> &x, const PR<T> &y) { return PR<T>(x.a * y.a, x.b * y.b); }
template <class T> __device__ __forceinline__ PR<T> pr_div(const PR<T> &x, const PR<T> &y) { return PR<T>(x.a / y.a, x.b / y.b); }
template <class T> __device__ __forceinline__ PR<T> pr_mod(const PR<T> &x, const PR<T> &y) { return PR<T>(x.a % y.a, x.b % y.b); }
// The device compiler fuses a packed multiply into a packed add that consumes
// it (also when the add is written as fma(x, 1, y)), whatever the fmad setting:
// such a sum would be rounded once instead of twice. Generated code therefore
// adds an inexact packed product with pr_add_lanes (scalar adds, which are not
// fused); x - y = fma(y, -1, x) keeps both roundings for products on either side
// (both checked on B200).
__device__ __forceinline__ PR<float> pr_add(const PR<float> &x, const PR<float> &y) {
  return pr_of(__fadd2_rn(pr_f2(x), pr_f2(y)));
}
template <class A, class B> __device__ __forceinline__ PR<float> pr_add_lanes(const A &x, const B &y) {
  return PR<float>((float)lane0(x) + (float)lane0(y), (float)lane1(x) + (float)lane1(y));
}
__device__ __forceinline__ PR<float> pr_sub(const PR<float> &x, const PR<float> &y) {
  return pr_of(__ffma2_rn(pr_f2(y), f2_of(-1.0f), pr_f2(x)));
}
__device__ __forceinline__ PR<float> pr_mul(const PR<float> &x, const PR<float> &y) {
  return pr_of(__fmul2_rn(pr_f2(x), pr_f2(y)));
}

#define MAP_PR_ARITH(OP, FN)                                                                                   \
  template <class A, class B>                                                                                  \
  __device__ __forceinline__ auto operator OP(const PR<A> &x, const PR<B> &y)->PR<decltype(x.a OP y.a)> {     \
    typedef decltype(x.a OP y.a) C;                                                                            \
    return FN(PR<C>(x), PR<C>(y));                                                                             \
  }                                                                                                            \
  template <class A, class B, class = typename map_scalar<B>::type>                                            \
  __device__ __forceinline__ auto operator OP(const PR<A> &x, const B &y)->PR<decltype(x.a OP y)> {           \
    typedef decltype(x.a OP y) C;                                                                              \
    return FN(PR<C>(x), PR<C>(y));                                                                             \
  }                                                                                                            \
  template <class A, class B, class = typename map_scalar<A>::type>                                            \
  __device__ __forceinline__ auto operator OP(const A &x, const PR<B> &y)->PR<decltype(x OP y.a)> {           \
    typedef decltype(x OP y.a) C;                                                                              \
    return FN(PR<C>(x), PR<C>(y));                                                                             \
  }
MAP_PR_ARITH(+, pr_add) MAP_PR_ARITH(-, pr_sub) MAP_PR_ARITH(*, pr_mul) MAP_PR_ARITH(/, pr_div) MAP_PR_ARITH(%, pr_mod)
#undef MAP_PR_ARITH

// comparisons, logical, bitwise and shift operators: per lane, C++ result types
#define MAP_PR_LANE(OP)                                                                                        \
  template <class A, class B>                                                                                  \
  __device__ __forceinline__ auto operator OP(const PR<A> &x, const PR<B> &y)->PR<decltype(x.a OP y.a)> {     \
    return PR<decltype(x.a OP y.a)>(x.a OP y.a, x.b OP y.b);                                                   \
  }                                                                                                            \
  template <class A, class B, class = typename map_scalar<B>::type>                                            \
  __device__ __forceinline__ auto operator OP(const PR<A> &x, const B &y)->PR<decltype(x.a OP y)> {           \
    return PR<decltype(x.a OP y)>(x.a OP y, x.b OP y);                                                         \
  }                                                                                                            \
  template <class A, class B, class = typename map_scalar<A>::type>                                            \
  __device__ __forceinline__ auto operator OP(const A &x, const PR<B> &y)->PR<decltype(x OP y.a)> {           \
    return PR<decltype(x OP y.a)>(x OP y.a, x OP y.b);                                                         \
  }
MAP_PR_LANE(==) MAP_PR_LANE(!=) MAP_PR_LANE(<) MAP_PR_LANE(>) MAP_PR_LANE(<=) MAP_PR_LANE(>=)
MAP_PR_LANE(&&) MAP_PR_LANE(||) MAP_PR_LANE(&) MAP_PR_LANE(|) MAP_PR_LANE(^) MAP_PR_LANE(<<) MAP_PR_LANE(>>)
#undef MAP_PR_LANE

template <class A> __device__ __forceinline__ auto operator+(const PR<A> &x)->PR<decltype(+x.a)> {
  return PR<decltype(+x.a)>(+x.a, +x.b);
}
template <class A> __device__ __forceinline__ auto operator-(const PR<A> &x)->PR<decltype(-x.a)> {
  return PR<decltype(-x.a)>(-x.a, -x.b);
}
// -x = x * -1 exactly (the sign flips, zeros included)
__device__ __forceinline__ PR<float> operator-(const PR<float> &x) { return pr_of(__fmul2_rn(pr_f2(x), f2_of(-1.0f))); }
template <class A> __device__ __forceinline__ PR<bool> operator!(const PR<A> &x) { return PR<bool>(!x.a, !x.b); }
template <class A> __device__ __forceinline__ auto operator~(const PR<A> &x)->PR<decltype(~x.a)> {
  return PR<decltype(~x.a)>(~x.a, ~x.b);
}

// c ? x : y per lane (the condition a pair or one scalar for both lanes)
template <class C, class A, class B>
__device__ __forceinline__ auto psel(const PR<C> &c, const A &x, const B &y)->PR<decltype(true ? lane0(x) : lane0(y))> {
  typedef decltype(true ? lane0(x) : lane0(y)) R;
  return PR<R>(c.a ? (R)lane0(x) : (R)lane0(y), c.b ? (R)lane1(x) : (R)lane1(y));
}
template <class C, class A, class B, class = typename map_scalar<C>::type>
__device__ __forceinline__ auto psel(const C &c, const A &x, const B &y)->PR<decltype(true ? lane0(x) : lane0(y))> {
  typedef decltype(true ? lane0(x) : lane0(y)) R;
  return PR<R>(c ? (R)lane0(x) : (R)lane0(y), c ? (R)lane1(x) : (R)lane1(y));
}

// a + t*w with w == 0 (the product is an exact signed zero, so this equals the
// separate multiply and add)
__device__ __forceinline__ PR<float> pr_fmaf(const PR<float> &t, float w, const PR<float> &a) {
  return pr_of(__ffma2_rn(pr_f2(t), f2_of(w), pr_f2(a)));
}

// library functions of the device math API, per lane. They take new names
// (pr_sqrtf, ...): overloading the library's own names changes which
// implementation the device compiler picks for them (sqrtf stops being the
// correctly rounded square root).
#define MAP_PR_F1(fn) \
  __device__ __forceinline__ PR<float> pr_##fn(const PR<float> &x) { return PR<float>(fn(x.a), fn(x.b)); }
MAP_PR_F1(sinf) MAP_PR_F1(cosf) MAP_PR_F1(tanf) MAP_PR_F1(asinf) MAP_PR_F1(acosf) MAP_PR_F1(atanf)
MAP_PR_F1(sinhf) MAP_PR_F1(coshf) MAP_PR_F1(tanhf) MAP_PR_F1(asinhf) MAP_PR_F1(acoshf) MAP_PR_F1(atanhf)
MAP_PR_F1(expf) MAP_PR_F1(exp2f) MAP_PR_F1(exp10f) MAP_PR_F1(logf) MAP_PR_F1(log2f) MAP_PR_F1(log10f)
MAP_PR_F1(sqrtf) MAP_PR_F1(cbrtf) MAP_PR_F1(fabsf) MAP_PR_F1(ceilf) MAP_PR_F1(floorf) MAP_PR_F1(truncf)
MAP_PR_F1(roundf)
#undef MAP_PR_F1
#define MAP_PR_F2(fn)                                                                   \
  __device__ __forceinline__ PR<float> pr_##fn(const PR<float> &x, const PR<float> &y) { \
    return PR<float>(fn(x.a, y.a), fn(x.b, y.b));                                       \
  }
MAP_PR_F2(powf) MAP_PR_F2(hypotf) MAP_PR_F2(fmodf) MAP_PR_F2(atan2f)
#undef MAP_PR_F2

// the engine's own atan2, sin and cos on pairs: the same operations as the
// scalar forms above (bit-identical lanes), the polynomials packed
__device__ __forceinline__ PR<float> map_atan_poly(const PR<float> &t) {
  const float2 T = pr_f2(t);
  const float2 s = __fmul2_rn(T, T);
  float2 q = f2_of(MAP_ATAN_Q0);
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q1));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q2));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q3));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q4));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q5));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q6));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q7));
  q = __ffma2_rn(q, s, f2_of(MAP_ATAN_Q8));
  return pr_of(__ffma2_rn(__fmul2_rn(T, s), q, T));
}
__device__ __forceinline__ PR<float> map_atan2f(const PR<float> &y, const PR<float> &x) {
  const PR<float> r = map_atan_poly(PR<float>(map_atan2_arg(y.a, x.a), map_atan2_arg(y.b, x.b)));
  return PR<float>(map_atan2_finish(r.a, y.a, x.a), map_atan2_finish(r.b, y.b, x.b));
}
__device__ __forceinline__ void map_sincos_reduced(const PR<float> &x, u32 &qa, u32 &qb, PR<float> &sr, PR<float> &cr) {
  const float2 X = pr_f2(x);
  const float2 t = __ffma2_rn(X, f2_of(MAP_2OPI), f2_of(MAP_RINT));
  const float2 j = __ffma2_rn(t, f2_of(1.0f), f2_of(-MAP_RINT));
  qa = __float_as_uint(t.x);
  qb = __float_as_uint(t.y);
  float2 r = __ffma2_rn(j, f2_of(-MAP_PIO2_1), X);
  r = __ffma2_rn(j, f2_of(-MAP_PIO2_2), r);
  r = __ffma2_rn(j, f2_of(-MAP_PIO2_3), r);
  const float2 s = __fmul2_rn(r, r);
  float2 p = __ffma2_rn(s, f2_of(MAP_SIN_3), f2_of(MAP_SIN_2));
  p = __ffma2_rn(s, p, f2_of(MAP_SIN_1));
  const float2 v = __ffma2_rn(__fmul2_rn(r, s), p, r);
  sr = PR<float>(map_sin_sign(v.x, r.x), map_sin_sign(v.y, r.y));
  float2 c = __ffma2_rn(s, f2_of(MAP_COS_4), f2_of(MAP_COS_3));
  c = __ffma2_rn(s, c, f2_of(MAP_COS_2));
  c = __ffma2_rn(s, c, f2_of(MAP_COS_1));
  cr = pr_of(__ffma2_rn(s, c, f2_of(1.0f)));
}
__device__ __forceinline__ bool map_trig_far(const PR<float> &x) {
  return fabsf(x.a) > MAP_TRIG_BOUND || fabsf(x.b) > MAP_TRIG_BOUND;
}
__device__ __forceinline__ void map_sincosf(const PR<float> &x, PR<float> *sp, PR<float> *cp) {
  if (map_trig_far(x)) {
    map_sincosf(x.a, &sp->a, &cp->a);
    map_sincosf(x.b, &sp->b, &cp->b);
    return;
  }
  u32 qa, qb;
  PR<float> sr, cr;
  map_sincos_reduced(x, qa, qb, sr, cr);
  *sp = PR<float>(map_quadrant_sin(qa, sr.a, cr.a), map_quadrant_sin(qb, sr.b, cr.b));
  *cp = PR<float>(map_quadrant_cos(qa, sr.a, cr.a), map_quadrant_cos(qb, sr.b, cr.b));
}
__device__ __forceinline__ PR<float> map_sinf(const PR<float> &x) {
  if (map_trig_far(x)) return PR<float>(map_sinf(x.a), map_sinf(x.b));
  u32 qa, qb;
  PR<float> sr, cr;
  map_sincos_reduced(x, qa, qb, sr, cr);
  return PR<float>(map_quadrant_sin(qa, sr.a, cr.a), map_quadrant_sin(qb, sr.b, cr.b));
}
__device__ __forceinline__ PR<float> map_cosf(const PR<float> &x) {
  if (map_trig_far(x)) return PR<float>(map_cosf(x.a), map_cosf(x.b));
  u32 qa, qb;
  PR<float> sr, cr;
  map_sincos_reduced(x, qa, qb, sr, cr);
  return PR<float>(map_quadrant_cos(qa, sr.a, cr.a), map_quadrant_cos(qb, sr.b, cr.b));
}

// ------------------------------------------------------------------ shading identity

#define MAP_INF_F __int_as_float(0x7f800000)

// 1 / sqrt(v) for finite v >= 1: the hardware estimate (rsqrt.approx.f32) and one
// Newton-Raphson step r' = r + (r / 2)(1 - v r^2), every operation rounded once.
__device__ __forceinline__ float map_rsqrt_est(float v) {
  float r;
  asm("rsqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ float map_rsqrt(float v) {
  const float r = map_rsqrt_est(v);
  const float e = __fmaf_rn(-__fmul_rn(v, r), r, 1.0f);
  return __fmaf_rn(__fmul_rn(r, 0.5f), e, r);
}
__device__ __forceinline__ PR<float> map_rsqrt(const PR<float> &v) {
  const float2 r = make_float2(map_rsqrt_est(v.a), map_rsqrt_est(v.b));
  const float2 e = __ffma2_rn(__fmul2_rn(pr_f2(v), make_float2(-r.x, -r.y)), r, f2_of(1.0f));
  return pr_of(__ffma2_rn(__fmul2_rn(r, f2_of(0.5f)), e, r));
}

// Hillshade through the shading identity (the host's rewrite of
//   cz cos(s) + sz sin(s) cos(ar - aspect),  s = atan(k sqrt(x^2 + y^2)),
//   aspect = atan2(y, -x) wrapped into [0, 2 PI'), x == 0 by its own branch):
//   hs = (cz + szk (y S - x C)) / sqrt(1 + kk (x^2 + y^2)),  szk = sz k, kk = k^2.
// (S, C) is the unit vector of the light direction the reference chain uses for
// the cell: (S0, C0) where its atan2 is not negative, (S1, C1) where the atan2 is
// negative and the wrap adds the script's 2 PI' (not 2 pi), SH / S3 for x == 0
// (aspect PI'/2 or 3 PI'/2). atan2(y, -x) < 0 exactly when y < 0, or y is -0 and
// -x < 0. Returns hs and q = x^2 + y^2; the caller takes the literal chain where
// q is not finite. The pair form performs the same operations lane by lane
// (packed where both lanes do the same), so its lanes equal the scalar form.
template <bool K1>
__device__ __forceinline__ float map_shade(float x, float y, float cz, float szk, float kk, float S0, float C0,
                                           float S1, float C1, float SH, float S3, float &q) {
  q = __fmaf_rn(x, x, __fmul_rn(y, y));
  const bool nz = x != 0.0f;
  const bool neg = y < 0.0f || ((__float_as_uint(y) >> 31) && x > 0.0f);
  const float S = nz ? (neg ? S1 : S0) : (y > 0.0f ? SH : S3);
  const float C = nz ? (neg ? C1 : C0) : 0.0f;
  const float num = __fmaf_rn(y, S, __fmul_rn(x, -C));
  const float v = K1 ? __fadd_rn(1.0f, q) : __fmaf_rn(kk, q, 1.0f);
  return __fmul_rn(__fmaf_rn(szk, num, cz), map_rsqrt(v));
}
template <bool K1>
__device__ __forceinline__ PR<float> map_shade(const PR<float> &x, const PR<float> &y, float cz, float szk, float kk,
                                               float S0, float C0, float S1, float C1, float SH, float S3,
                                               PR<float> &q) {
  const float2 X = pr_f2(x), Y = pr_f2(y);
  q = pr_of(__ffma2_rn(X, X, __fmul2_rn(Y, Y)));
  const bool nza = x.a != 0.0f, nzb = x.b != 0.0f;
  const bool nga = y.a < 0.0f || ((__float_as_uint(y.a) >> 31) && x.a > 0.0f);
  const bool ngb = y.b < 0.0f || ((__float_as_uint(y.b) >> 31) && x.b > 0.0f);
  const float2 S = make_float2(nza ? (nga ? S1 : S0) : (y.a > 0.0f ? SH : S3),
                               nzb ? (ngb ? S1 : S0) : (y.b > 0.0f ? SH : S3));
  const float2 nC = make_float2(nza ? (nga ? -C1 : -C0) : -0.0f, nzb ? (ngb ? -C1 : -C0) : -0.0f);
  const float2 num = __ffma2_rn(Y, S, __fmul2_rn(X, nC));
  const float2 v = K1 ? __fadd2_rn(f2_of(1.0f), pr_f2(q)) : __ffma2_rn(f2_of(kk), pr_f2(q), f2_of(1.0f));
  return pr_of(__fmul2_rn(__ffma2_rn(f2_of(szk), num, f2_of(cz)), pr_f2(map_rsqrt(pr_of(v)))));
}

// The same identity on unscaled derivatives: x = s xc, y = s yc for a power of
// two s folded into the constants (szks = sz k s, kks = k^2 s^2), y never -0
// (the derivatives are sums that start from +0), and the light direction chosen
// arithmetically: with negf = (yc < 0), S = S0 + negf (S1 - S0) and -C = -C0 +
// negf (C0 - C1) for xc != 0, S = SH + negf (S3 - SH) for xc == 0, where the
// differences are exact in float32 (the host checks this before choosing this
// form), so S and -C are exactly S0 / S1 / SH / S3 and -C0 / -C1. The caller's
// xc starts from the taps neither derivative weights (fma(tap, 0, .): +-0, or
// NaN when such a tap is not finite); q = xc^2 + yc^2, and the caller takes the
// literal chain where q is not finite. Every operation rounds once; the pair
// form performs the same operations lane by lane.
__device__ __forceinline__ float map_shade_fast(float xc, float yc, float cz, float szks, float kks, float S0,
                                                float dS, float nC0, float dnC, float SH, float dSx, float &q) {
  q = __fmaf_rn(xc, xc, __fmul_rn(yc, yc));
  // the same values chosen by selects (S0 + dS etc. are exact, folded on the host)
  const bool neg = yc < 0.0f;
  const float S = xc != 0.0f ? (neg ? S0 + dS : S0) : (neg ? SH + dSx : SH);
  const float nC = neg ? nC0 + dnC : nC0;
  const float num = __fmaf_rn(yc, S, __fmul_rn(xc, nC));
  return __fmul_rn(__fmaf_rn(szks, num, cz), map_rsqrt(__fmaf_rn(kks, q, 1.0f)));
}
__device__ __forceinline__ PR<float> map_shade_fast(const PR<float> &xc, const PR<float> &yc, float cz,
                                                    float szks, float kks, float S0, float dS, float nC0, float dnC,
                                                    float SH, float dSx, PR<float> &q) {
  const float2 X = pr_f2(xc), Y = pr_f2(yc);
  q = pr_of(__ffma2_rn(X, X, __fmul2_rn(Y, Y)));
  const float2 negf = make_float2(yc.a < 0.0f ? 1.0f : 0.0f, yc.b < 0.0f ? 1.0f : 0.0f);
  const float2 Sn = __ffma2_rn(negf, f2_of(dS), f2_of(S0)), nC = __ffma2_rn(negf, f2_of(dnC), f2_of(nC0));
  const float2 Sx = __ffma2_rn(negf, f2_of(dSx), f2_of(SH));
  const float2 S = make_float2(xc.a != 0.0f ? Sn.x : Sx.x, xc.b != 0.0f ? Sn.y : Sx.y);
  const float2 num = __ffma2_rn(Y, S, __fmul2_rn(X, nC));
  const PR<float> r = map_rsqrt(pr_of(__ffma2_rn(f2_of(kks), pr_f2(q), f2_of(1.0f))));
  return pr_of(__fmul2_rn(__ffma2_rn(f2_of(szks), num, f2_of(cz)), pr_f2(r)));
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

// Block mirror on a raster of several blocks: an out-of-raster tap takes the
// raster mirror's value (what stage_fix_border writes) except where the
// reference's reflection inside the reading cell's block differs from it: the
// tap's other coordinate crosses the reading cell's block boundary, or the tap
// leaves the raster past the right / bottom edge from a block that is not the
// last one, or from a last block narrower than the halo (the reflection inside
// it is clamped). Only cells within the halo of a raster edge qualify; staged
// edge tiles recompute them from global memory afterwards.
__device__ __forceinline__ bool block_fixup(const Geom &g) {
  return g.border == 0 && !(g.BS0 >= g.W && g.BS1 >= g.H);
}
__device__ __forceinline__ bool block_exception(const Geom &g, int x, int y, int hx, int hy) {
  const int bx = x % g.BS0, by = y % g.BS1;
  const bool near_bx = bx < hx || bx >= g.BS0 - hx || x >= g.W - hx;
  const bool near_by = by < hy || by >= g.BS1 - hy || y >= g.H - hy;
  const bool edge_y = y < hy || y >= g.H - hy, edge_x = x < hx || x >= g.W - hx;
  const int lastx = (g.W - 1) / g.BS0, lasty = (g.H - 1) / g.BS1;
  const bool inner_last_x = x >= g.W - hx && (x / g.BS0 != lastx || g.W - lastx * g.BS0 < hx);
  const bool inner_last_y = y >= g.H - hy && (y / g.BS1 != lasty || g.H - lasty * g.BS1 < hy);
  return (edge_y && near_bx) || (edge_x && near_by) || inner_last_x || inner_last_y;
}

// After a staged box of an edge tile has landed (raster cell (ox + bx, oy + by) at
// s[by * SW + bx]), overwrites its cells outside the raster that a centre cell can
// reach (within hx / hy of the edge) with the border rule's value: zero (dead) or
// the cell mirrored at the raster edge (raster mirror; block mirror, whose
// exceptions block_exception names). The sources are inside the raster, so no
// cell is both read and written.
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
  // the same tap of the cells (x, y) and (x, y + 1)
  __device__ __forceinline__ PR<T> tap2(int x, int y, int lx, int ly, int dx, int dy) const {
    return PR<T>(tap(x, y, lx, ly, dx, dy), tap(x, y + 1, lx, ly + 1, dx, dy));
  }
  // the same tap of the cells (x, y) and (x + 1, y)
  __device__ __forceinline__ PR<T> tap2c(int x, int y, int lx, int ly, int dx, int dy) const {
    return PR<T>(tap(x, y, lx, ly, dx, dy), tap(x + 1, y, lx + 1, ly, dx, dy));
  }
};

// Focal tap served from a tile staged in shared memory (interior tiles).
// The tile's element (0,0) is raster cell (x0 - PX, y0 - HY).
// ------------------------------------------------------------------ packed byte cells

// Four consecutive cells of a row (x .. x + 3) of an integer expression whose
// every value lies in [0, 0x7FFF], as 16-bit lanes of two words, interleaved:
// lo holds the cells x (bits 0-15) and x + 2 (bits 16-31), hi the cells x + 1
// and x + 3. With this layout the taps of neighbouring offsets share words
// (the lanes of offset +1 are hi and the even lanes of offset +2), so a row of
// byte cells costs one byte permute per word of taps (see SmemTap::tap4).
// Sums, differences and products by non-negative constants of such lanes are
// plain 32-bit operations as long as no lane leaves [0, 0xFFFF], which the code
// generator proves by interval arithmetic before it uses this form; results of
// an 8-bit unsigned type are reduced mod 256 lane by lane (q4_wrap8).
struct Q4 { u32 lo, hi; };
__device__ __forceinline__ Q4 q4_splat(u32 c) { return Q4{c * 0x00010001u, c * 0x00010001u}; }
// four bytes (cells x .. x + 3) as lanes
__device__ __forceinline__ u32 q4_even(u32 w) { return __byte_perm(w, 0u, 0x4240); }   // bytes 0, 2
__device__ __forceinline__ u32 q4_odd(u32 w) { return __byte_perm(w, 0u, 0x4341); }    // bytes 1, 3
__device__ __forceinline__ Q4 q4_bytes(u32 w) { return Q4{q4_even(w), q4_odd(w)}; }
// the four lanes (each < 256) as the bytes of one word, cell x in the low byte
__device__ __forceinline__ u32 q4_pack_u8(Q4 v) { return __byte_perm(v.lo, v.hi, 0x6240); }
__device__ __forceinline__ Q4 q4_add(Q4 a, Q4 b) { return Q4{a.lo + b.lo, a.hi + b.hi}; }
__device__ __forceinline__ Q4 q4_sub(Q4 a, Q4 b) { return Q4{a.lo - b.lo, a.hi - b.hi}; }
__device__ __forceinline__ Q4 q4_mulc(Q4 a, u32 c) { return Q4{a.lo * c, a.hi * c}; }
__device__ __forceinline__ Q4 q4_and(Q4 a, Q4 b) { return Q4{a.lo & b.lo, a.hi & b.hi}; }
__device__ __forceinline__ Q4 q4_or(Q4 a, Q4 b) { return Q4{a.lo | b.lo, a.hi | b.hi}; }
__device__ __forceinline__ Q4 q4_xor(Q4 a, Q4 b) { return Q4{a.lo ^ b.lo, a.hi ^ b.hi}; }
__device__ __forceinline__ Q4 q4_wrap8(Q4 a) { return Q4{a.lo & 0x00FF00FFu, a.hi & 0x00FF00FFu}; }
// lane products: m has lanes 0 or 1 (a mask times a value)
__device__ __forceinline__ u32 q4_mul01_w(u32 m, u32 b) { return (m * 0xFFFFu) & b; }
__device__ __forceinline__ Q4 q4_mul01(Q4 m, Q4 b) { return Q4{q4_mul01_w(m.lo, b.lo), q4_mul01_w(m.hi, b.hi)}; }
// general lane products (each product below 2^16)
__device__ __forceinline__ u32 q4_mul_w(u32 a, u32 b) {
  return ((a & 0xFFFFu) * (b & 0xFFFFu)) | (((a >> 16) * (b >> 16)) << 16);
}
__device__ __forceinline__ Q4 q4_mul(Q4 a, Q4 b) { return Q4{q4_mul_w(a.lo, b.lo), q4_mul_w(a.hi, b.hi)}; }
// relations of lanes in [0, 0x7FFF], as lanes 0 / 1: a lane plus 0x7FFF sets its
// bit 15 exactly when it is not zero, and 0x8000 + a - b keeps bit 15 exactly when
// a >= b; neither carries nor borrows across lanes
__device__ __forceinline__ u32 q4_ne0_w(u32 a) { return ((a + 0x7FFF7FFFu) & 0x80008000u) >> 15; }
__device__ __forceinline__ u32 q4_ge_w(u32 a, u32 b) { return (((a | 0x80008000u) - b) & 0x80008000u) >> 15; }
__device__ __forceinline__ Q4 q4_ne(Q4 a, Q4 b) { return Q4{q4_ne0_w(a.lo ^ b.lo), q4_ne0_w(a.hi ^ b.hi)}; }
__device__ __forceinline__ Q4 q4_eq(Q4 a, Q4 b) {
  return Q4{q4_ne0_w(a.lo ^ b.lo) ^ 0x00010001u, q4_ne0_w(a.hi ^ b.hi) ^ 0x00010001u};
}
__device__ __forceinline__ Q4 q4_ge(Q4 a, Q4 b) { return Q4{q4_ge_w(a.lo, b.lo), q4_ge_w(a.hi, b.hi)}; }
__device__ __forceinline__ Q4 q4_lt(Q4 a, Q4 b) {
  return Q4{q4_ge_w(a.lo, b.lo) ^ 0x00010001u, q4_ge_w(a.hi, b.hi) ^ 0x00010001u};
}
__device__ __forceinline__ Q4 q4_gt(Q4 a, Q4 b) { return q4_lt(b, a); }
__device__ __forceinline__ Q4 q4_le(Q4 a, Q4 b) { return q4_ge(b, a); }
__device__ __forceinline__ Q4 q4_ne0(Q4 a) { return Q4{q4_ne0_w(a.lo), q4_ne0_w(a.hi)}; }
__device__ __forceinline__ Q4 q4_eq0(Q4 a) { return Q4{q4_ne0_w(a.lo) ^ 0x00010001u, q4_ne0_w(a.hi) ^ 0x00010001u}; }
// lanes of t where m (lanes 0 / 1) is 1, else of f
__device__ __forceinline__ Q4 q4_sel(Q4 m, Q4 t, Q4 f) {
  const u32 ml = m.lo * 0xFFFFu, mh = m.hi * 0xFFFFu;
  return Q4{(t.lo & ml) | (f.lo & ~ml), (t.hi & mh) | (f.hi & ~mh)};
}
__device__ __forceinline__ Q4 q4_max(Q4 a, Q4 b) { return q4_sel(q4_ge(a, b), a, b); }
__device__ __forceinline__ Q4 q4_min(Q4 a, Q4 b) { return q4_sel(q4_ge(b, a), a, b); }
// the four U8 cells x .. x + 3 of row y of a raster as one 32-bit load (the row
// address plus x must be 4-byte aligned)
__device__ __forceinline__ u32 ldr_q4_u8(const RasterArg &r, int x, int y) {
  return __ldg((const u32 *)(r.p + (u64)(s64)y * (u64)r.pitch + (u64)(s64)x));
}


// a 4-byte cell value carried in a float register, as its own type
template <class T> __device__ __forceinline__ T __float_as_raw(float f) {
  T r;
  memcpy(&r, &f, sizeof(T));
  return r;
}

template <class T, int SW, int PX, int HY> struct SmemTap {
  const T *s;
  __device__ __forceinline__ T tap(int x, int y, int lx, int ly, int dx, int dy) const {
    return s[(ly + HY + dy) * SW + (lx + PX + dx)];
  }
  __device__ __forceinline__ PR<T> tap2(int x, int y, int lx, int ly, int dx, int dy) const {
    return PR<T>(s[(ly + HY + dy) * SW + (lx + PX + dx)], s[(ly + 1 + HY + dy) * SW + (lx + PX + dx)]);
  }
  // The tap at (dx, dy) of the cells lx and lx + 1 of a row (4-byte cells, lx +
  // PX and SW even): aligned pairs of the staged row, one 8-byte load each; an
  // odd dx takes the second cell of one pair and the first of the next, so the
  // three taps of a 3-wide window come from three loads for both cells.
  __device__ __forceinline__ PR<T> tap2c(int x, int y, int lx, int ly, int dx, int dy) const {
    static_assert(sizeof(T) == 4 && SW % 2 == 0 && PX % 2 == 0, "tap2c: 4-byte cells, even row stride and pad");
    const float2 *row = (const float2 *)(s + (ly + HY + dy) * SW + lx + PX);
    const int o = dx & 1, m = (dx - o) / 2;
    const float2 p = row[m];
    if (!o) return PR<T>(__float_as_raw<T>(p.x), __float_as_raw<T>(p.y));
    const float2 q = row[m + 1];
    return PR<T>(__float_as_raw<T>(p.y), __float_as_raw<T>(q.x));
  }
  // The taps at (dx, dy) of the byte cells lx .. lx + 3 (lx a multiple of 4, the
  // row stride SW and pad PX multiples of 4, |dx| <= PX), in the interleaved
  // lane layout of Q4. With dx = 4 m + o and W_m the m-th aligned word from the
  // cell lx: the even and odd bytes of W_m (q4_even / q4_odd) are the lanes of
  // o = 0; lanes (4m + 2, 4m + 4) take byte 2 of W_m and byte 0 of W_m+1
  // beside the zero bytes of q4_even(W_m); lanes (4m + 3, 4m + 5) take byte 3 of
  // W_m and the odd lanes of W_m+1. Each piece is one byte permute of loaded
  // words, and the pieces of neighbouring offsets are the same expressions.
  __device__ __forceinline__ u32 word(int lx, int ly, int dy, int m) const {
    return ((const u32 *)(s + (ly + HY + dy) * SW + lx + PX))[m];
  }
  __device__ __forceinline__ u32 tap4_e(int lx, int ly, int dy, int m) const {   // lanes 4m + 2, 4m + 4
    return __byte_perm(q4_even(word(lx, ly, dy, m)), word(lx, ly, dy, m + 1), 0x1412);
  }
  __device__ __forceinline__ u32 tap4_o(int lx, int ly, int dy, int m) const {   // lanes 4m + 3, 4m + 5
    return __byte_perm(word(lx, ly, dy, m), q4_odd(word(lx, ly, dy, m + 1)), 0x5453);
  }
  __device__ __forceinline__ Q4 tap4(int lx, int ly, int dx, int dy) const {
    static_assert(sizeof(T) == 1 && SW % 4 == 0 && PX % 4 == 0, "tap4: byte cells, word-aligned rows");
    const int o = dx & 3, m = (dx - o) / 4;
    switch (o) {
      case 0: return q4_bytes(word(lx, ly, dy, m));
      case 1: return Q4{q4_odd(word(lx, ly, dy, m)), tap4_e(lx, ly, dy, m)};
      case 2: return Q4{tap4_e(lx, ly, dy, m), tap4_o(lx, ly, dy, m)};
      default: return Q4{tap4_o(lx, ly, dy, m), q4_even(word(lx, ly, dy, m + 1))};
    }
  }
};

// ------------------------------------------------------------------ dependent launches

// Programmatic dependent launch: a kernel launched with it may start before the
// previous kernel of its stream has finished. griddep_launch lets the next
// kernel's CTAs start as this grid's CTAs leave; griddep_wait blocks until the
// previous grid has completed and its memory is visible (immediately when the
// launch had no such dependency). Every global access comes after the wait.
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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
// The same test with a suspend-time hint: a thread whose phase has not completed
// sleeps until it completes or `ns` nanoseconds pass, instead of returning at
// once, so waiting warps take no issue slots from the warps that compute.
__device__ __forceinline__ bool mbar_try_wait_sleep(u64 *bar, u32 parity, u32 ns) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls of at most about 0.26 ms each
// (about 4 s for the skeletons' 2^14), so a copy that never lands ends the CTA
// with an error instead of a hang.
__device__ __forceinline__ bool mbar_wait_bounded(u64 *bar, u32 parity, u32 limit) {
  for (u32 i = 0; i < limit; ++i)
    if (mbar_try_wait_sleep(bar, parity, 1u << 18)) return true;
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

// Tile store from shared memory to the tensor the map describes, at element
// (x, y): x times the element size a multiple of 16 bytes, y >= 0; cells outside
// the tensor's extent are not written. Threads fence their shared-memory
// writes (fence_proxy_async) and synchronise before one thread issues it, and
// that thread waits until the copy has read shared memory before the CTA ends.
__device__ __forceinline__ void tma_store_2d(const TmaDesc *tmap, const void *src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"((u64)tmap),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit_group() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_group_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

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

// Tile (tx, ty) of the region, for launches whose grid is the region's tiles in
// two dimensions (no division to recover the tile's coordinates)
template <int TW, int TH> __device__ __forceinline__ Tile tile_at(const Geom &g, int tx, int ty) {
  Tile r;
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
// pairs: per lane (sums and products go through the pair operators)
template <class T> __device__ __forceinline__ PR<T> red_max(const PR<T> &a, const PR<T> &b) {
  return PR<T>(red_max<T>(a.a, b.a), red_max<T>(a.b, b.b));
}
template <class T> __device__ __forceinline__ PR<T> red_min(const PR<T> &a, const PR<T> &b) {
  return PR<T>(red_min<T>(a.a, b.a), red_min<T>(a.b, b.b));
}
template <class T> struct RedOp<6, PR<T>> { __device__ static PR<T> f(PR<T> a, PR<T> b) { return red_max(a, b); } };
template <class T> struct RedOp<7, PR<T>> { __device__ static PR<T> f(PR<T> a, PR<T> b) { return red_min(a, b); } };

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
