/*
 * map_b200.hpp -- C++ front end of the B200 map-algebra engine, header-only,
 * over the C ABI of map_b200.h (link with libmap_b200.so).
 *
 * Mirrors the reference's C++ front end (front/Raster.hpp:20-302,
 * front/Raster.cpp): class map::Raster wraps one IR node and holds a reference
 * on it (ma_increaseRef / ma_decreaseRef), operators and functions build new
 * nodes, eval / value / write evaluate. Names, argument order and meaning follow
 * the reference; scalar operands are map::Variant (the reference's VariantType:
 * an int literal is S32, a float F32, a double F64, a bool B8).
 *
 * Differences: errors throw map::Error with the library's message (the
 * reference asserts); operations the engine does not support (lhs access,
 * diversity, focal percentages, neighbour-direction access) throw from the
 * library's error; extensions at the end (host / device rasters, border and
 * launch switches, flow direction, zone statistics) map to the extension ABI.
 */
#ifndef MAP_B200_HPP_
#define MAP_B200_HPP_

#include "map_b200.h"

#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace map {

/* ---- enumerations (values of util/DataType.hpp:21, NumDim, MemOrder and the
 * operator orders of python/map.py:35-90; the C ABI takes them as ints) ---- */
enum DataType : int { NONE_DATATYPE = 0, F32, F64, B8, U8, U16, U32, U64, S8, S16, S32, S64 };
enum NumDim : int { NONE_NUMDIM = 0x00, TIME = 0x01, D0 = 0x02, D1 = 0x04, D2 = 0x06, D3 = 0x08 };
enum MemOrder : int { NONE_MEMORDER = 0x00, BLK = 0x01, ROW = 0x02, COL = 0x04, SFC = 0x06 };
enum DeviceType : int { DEV_DEF = 0x01, DEV_CPU = 0x02, DEV_GPU = 0x04, DEV_ACC = 0x08, DEV_CUS = 0x16 };
enum UnaryType : int {
  NONE_UNARY = 0, POS, NEG, NOT, bNOT, MARK_UNARY, SIN, COS, TAN, ASIN, ACOS, ATAN, SINH, COSH, TANH, ASINH, ACOSH,
  ATANH, EXP, EXP2, EXP10, LOG, LOG2, LOG10, SQRT, CBRT, ABS, CEIL, FLOOR, TRUNC, ROUND
};
enum BinaryType : int {
  NONE_BINARY = 0, ADD, SUB, MUL, DIV, MOD, EQ, NE, LT, GT, LE, GE, AND, OR, bAND, bOR, bXOR, SHL, SHR, MARK_BINARY,
  MAX2, MIN2, ATAN2, POW, HYPOT, FMOD
};
enum ReductionType : int { NONE_REDUCTION = 0, SUM, PROD, rAND, rOR, MARK_REDUCTION, MAX, MIN };
enum Border : int { BORDER_BLOCK_MIRROR = 0, BORDER_RASTER_MIRROR = 1, BORDER_DEAD = 2 };
enum ExecMode : int { EXEC_FUSED = 0, EXEC_PLAIN = 1 };

struct Error : std::runtime_error {
  explicit Error(const std::string &m) : std::runtime_error(m) {}
};

namespace detail {
inline void check() {
  if (ma_errorCode()) throw Error(ma_lastError());
}
inline ma_Node *checked(ma_Node *n) {
  if (!n) throw Error(ma_lastError());
  return n;
}
inline ma_Array array(std::initializer_list<int> v) {
  ma_Array a{{0, 0}, 0};
  for (int x : v) {
    if (a.n == 2) throw Error("map: arrays hold at most two values");
    a.arr[a.n++] = x;
  }
  return a;
}
}  // namespace detail

/* Two ints: data sizes, block sizes and coordinates (util/Array4.hpp). */
struct Coord {
  ma_Array a{{0, 0}, 0};
  Coord() = default;
  Coord(std::initializer_list<int> v) : a(detail::array(v)) {}
  explicit Coord(ma_Array x) : a(x) {}
  int operator[](int i) const { return a.arr[i]; }
  int size() const { return a.n; }
};
typedef Coord DataSize;
typedef Coord BlockSize;

/* Scalar value with its data type (util/VariantType.hpp). */
struct Variant {
  ma_Variant v;
  Variant() { std::memset(&v, 0, sizeof v); }
  explicit Variant(ma_Variant x) : v(x) {}
  Variant(float x) : Variant() { v.u.f32 = x; v.dtype = F32; }
  Variant(double x) : Variant() { v.u.f64 = x; v.dtype = F64; }
  Variant(bool x) : Variant() { v.u.b8 = x ? 1 : 0; v.dtype = B8; }
  Variant(int8_t x) : Variant() { v.u.s8 = x; v.dtype = S8; }
  Variant(int16_t x) : Variant() { v.u.s16 = x; v.dtype = S16; }
  Variant(int32_t x) : Variant() { v.u.s32 = x; v.dtype = S32; }
  Variant(int64_t x) : Variant() { v.u.s64 = x; v.dtype = S64; }
  Variant(uint8_t x) : Variant() { v.u.u8 = x; v.dtype = U8; }
  Variant(uint16_t x) : Variant() { v.u.u16 = x; v.dtype = U16; }
  Variant(uint32_t x) : Variant() { v.u.u32 = x; v.dtype = U32; }
  Variant(uint64_t x) : Variant() { v.u.u64 = x; v.dtype = U64; }
  DataType datatype() const { return (DataType)v.dtype; }
  /* the value as a double (any data type) */
  double get() const {
    switch (v.dtype) {
      case F32: return v.u.f32;
      case F64: return v.u.f64;
      case B8: return v.u.b8;
      case U8: return v.u.u8;
      case U16: return v.u.u16;
      case U32: return v.u.u32;
      case U64: return (double)v.u.u64;
      case S8: return v.u.s8;
      case S16: return v.u.s16;
      case S32: return v.u.s32;
      case S64: return (double)v.u.s64;
      default: return 0.0;
    }
  }
};
typedef Variant VariantType;

/* A focal mask: size {width, height} and values in row-major order (util/Mask.hpp). */
struct Mask {
  Coord size;
  std::vector<ma_Variant> values;
  Mask(Coord sz, std::initializer_list<Variant> vals) : size(sz) {
    for (const Variant &x : vals) values.push_back(x.v);
    if ((int)values.size() != sz[0] * (sz.size() > 1 ? sz[1] : 1)) throw Error("map: mask size and values differ");
  }
};

/* Front-end raster: a counted reference to one node of the DAG (front/Raster.hpp:39-131). */
class Raster {
 public:
  ma_Node *node = nullptr;

  Raster() = default;
  /* takes a reference on `n` (from a node constructor of the C ABI) */
  explicit Raster(ma_Node *n) : node(detail::checked(n)) { ma_increaseRef(node); }
  Raster(const Raster &o) : node(o.node) {
    if (node) ma_increaseRef(node);
  }
  Raster(Raster &&o) noexcept : node(o.node) { o.node = nullptr; }
  Raster &operator=(Raster o) noexcept {
    std::swap(node, o.node);
    return *this;
  }
  ~Raster() {
    if (node) ma_decreaseRef(node);
  }
  /* a D0 constant (front/Raster.cpp:114-117) */
  Raster(Variant val) : Raster(ma_constant(val.v, ma_Array{{0, 0}, 0}, val.v.dtype, ROW, ma_Array{{0, 0}, 0})) {}

  /* neighbour at relative coordinate (front/Raster.hpp:96) */
  Raster operator()(const Coord &c) const { return Raster(ma_neighbor(node, c.a)); }
  /* value carried from the neighbour the direction raster points from (front/Raster.hpp:101) */
  Raster operator()(const Raster &dir, ReductionType red) const { return Raster(ma_spreadNeighbor(node, dir.node, red)); }

  DataType datatype() const { return (DataType)ma_datatype(node); }
  NumDim numdim() const { return (NumDim)ma_numdim(node); }
  MemOrder memorder() const { return (MemOrder)ma_memorder(node); }
  DataSize datasize() const { return DataSize(ma_datasize(node)); }
  BlockSize blocksize() const { return BlockSize(ma_blocksize(node)); }
};

/* ---- other methods (front/Raster.hpp:136-150) ---- */
inline void setupDevices(const std::string &plat, DeviceType dev, const std::string &name) {
  ma_setupDevices(plat.c_str(), dev, name.c_str());
  detail::check();
}
inline void eval(std::initializer_list<Raster> list) {
  std::vector<ma_Node *> v;
  for (const Raster &r : list) v.push_back(r.node);
  ma_eval(v.data(), (int)v.size());
  detail::check();
}
inline Variant value(const Raster &r) {
  ma_Variant v = ma_value(r.node);
  detail::check();
  return Variant(v);
}
/* The truth value of a scalar (D0) raster, evaluated: the test of a loop over
 * rasters (the reference captures Python `while` loops, python/map.py:234-330,
 * but cannot run them). */
inline bool truth(const Raster &r) {
  if (r.numdim() != D0) throw Error("map: the truth value of a 2-D raster is ambiguous: reduce it first");
  eval({r});
  return value(r).get() != 0.0;
}
/* Evaluates the rasters in one evaluation and makes each hold its value
 * (ma_materialize): 2-D rasters stay in device memory the library owns, scalars
 * become constants, and the nodes no raster refers to are dropped. A loop
 * keeps its loop-carried rasters resident this way, so an iteration evaluates
 * only its own body:
 *   while (map::truth(d > 0)) { y = step(x); d = zonalSum(y - x); x = y; map::materialize({&x, &d}); } */
inline void materialize(std::initializer_list<Raster *> list) {
  std::vector<ma_Node *> in, out(list.size(), nullptr);
  for (Raster *r : list) in.push_back(r->node);
  if (ma_materialize(in.data(), (int)in.size(), out.data()) != 0) throw Error(ma_lastError());
  size_t i = 0;
  for (Raster *r : list) *r = Raster(out[i++]);
  ma_collectGarbage();
}
inline Raster read(const std::string &path) { return Raster(ma_read(path.c_str())); }
inline int write(const Raster &r, const std::string &path) {
  int e = ma_write(r.node, path.c_str());
  if (e) throw Error(ma_lastError());
  return e;
}
inline Raster stats(const Raster &r) { return Raster(ma_stats(r.node)); }
inline Raster barrier(const Raster &r) { return Raster(ma_barrier(r.node)); }

/* ---- construction (front/Raster.hpp:158-178) ---- */
inline Raster full(Variant v, DataSize ds = DataSize(), DataType dt = F32, MemOrder mo = MemOrder(ROW + BLK),
                   BlockSize bs = BlockSize()) {
  ma_Variant c = v.v;
  return Raster(ma_constant(c, ds.a, dt, mo, bs.a));
}
inline Raster zeros(DataSize ds = DataSize(), DataType dt = F32, MemOrder mo = MemOrder(ROW + BLK), BlockSize bs = BlockSize()) {
  return full(Variant((int32_t)0), ds, dt, mo, bs);
}
inline Raster ones(DataSize ds = DataSize(), DataType dt = F32, MemOrder mo = MemOrder(ROW + BLK), BlockSize bs = BlockSize()) {
  return full(Variant((int32_t)1), ds, dt, mo, bs);
}
inline Raster full_like(Variant v, const Raster &r, DataType dt = NONE_DATATYPE, MemOrder mo = NONE_MEMORDER) {
  return full(v, r.datasize(), dt == NONE_DATATYPE ? r.datatype() : dt, mo == NONE_MEMORDER ? r.memorder() : mo,
              r.blocksize());
}
inline Raster zeros_like(const Raster &r, DataType dt = NONE_DATATYPE, MemOrder mo = NONE_MEMORDER) {
  return full_like(Variant((int32_t)0), r, dt, mo);
}
inline Raster ones_like(const Raster &r, DataType dt = NONE_DATATYPE, MemOrder mo = NONE_MEMORDER) {
  return full_like(Variant((int32_t)1), r, dt, mo);
}
inline Raster rand(const Raster &seed, DataType dt = NONE_DATATYPE, MemOrder mo = NONE_MEMORDER) {
  return Raster(ma_rand(seed.node, dt, mo));
}
inline Raster rand(Variant seed, DataSize ds, DataType dt = F32, MemOrder mo = MemOrder(ROW + BLK), BlockSize bs = BlockSize()) {
  return rand(full(seed, ds, seed.datatype(), mo, bs), dt, mo);
}
inline Raster astype(const Raster &r, DataType dt) { return Raster(ma_cast(r.node, dt)); }
inline Raster index(const Raster &r, NumDim dim = D1) { return Raster(ma_index(r.node, dim)); }
inline Raster con(const Raster &c, const Raster &l, const Raster &r) { return Raster(ma_conditional(c.node, l.node, r.node)); }
inline Raster con(Variant c, const Raster &l, const Raster &r) { return con(Raster(c), l, r); }
inline Raster con(const Raster &c, Variant l, const Raster &r) { return con(c, Raster(l), r); }
inline Raster con(const Raster &c, const Raster &l, Variant r) { return con(c, l, Raster(r)); }
inline Raster con(const Raster &c, Variant l, Variant r) { return con(c, Raster(l), Raster(r)); }

/* ---- element-wise operators and functions (front/Raster.hpp:193-277) ---- */
inline Raster unary(const Raster &r, UnaryType t) { return Raster(ma_unary(r.node, t)); }
inline Raster binary(const Raster &l, const Raster &r, BinaryType t) { return Raster(ma_binary(l.node, r.node, t)); }

inline Raster operator+(const Raster &r) { return unary(r, POS); }
inline Raster operator-(const Raster &r) { return unary(r, NEG); }
inline Raster operator!(const Raster &r) { return unary(r, NOT); }
inline Raster operator~(const Raster &r) { return unary(r, bNOT); }

#define MAPB_UNARY_FUNC(name, type) \
  inline Raster name(const Raster &r) { return unary(r, type); }
MAPB_UNARY_FUNC(sin, SIN)
MAPB_UNARY_FUNC(cos, COS)
MAPB_UNARY_FUNC(tan, TAN)
MAPB_UNARY_FUNC(asin, ASIN)
MAPB_UNARY_FUNC(acos, ACOS)
MAPB_UNARY_FUNC(atan, ATAN)
MAPB_UNARY_FUNC(sinh, SINH)
MAPB_UNARY_FUNC(cosh, COSH)
MAPB_UNARY_FUNC(tanh, TANH)
MAPB_UNARY_FUNC(asinh, ASINH)
MAPB_UNARY_FUNC(acosh, ACOSH)
MAPB_UNARY_FUNC(atanh, ATANH)
MAPB_UNARY_FUNC(exp, EXP)
MAPB_UNARY_FUNC(exp2, EXP2)
MAPB_UNARY_FUNC(exp10, EXP10)
MAPB_UNARY_FUNC(log, LOG)
MAPB_UNARY_FUNC(log2, LOG2)
MAPB_UNARY_FUNC(log10, LOG10)
MAPB_UNARY_FUNC(sqrt, SQRT)
MAPB_UNARY_FUNC(cbrt, CBRT)
MAPB_UNARY_FUNC(abs, ABS)
MAPB_UNARY_FUNC(ceil, CEIL)
MAPB_UNARY_FUNC(floor, FLOOR)
MAPB_UNARY_FUNC(trunc, TRUNC)
MAPB_UNARY_FUNC(round, ROUND)
#undef MAPB_UNARY_FUNC

#define MAPB_BINARY(sig, type)                                                                              \
  inline Raster sig(const Raster &l, const Raster &r) { return binary(l, r, type); }                        \
  inline Raster sig(const Raster &l, Variant r) { return binary(l, Raster(r), type); }                      \
  inline Raster sig(Variant l, const Raster &r) { return binary(Raster(l), r, type); }
MAPB_BINARY(operator+, ADD)
MAPB_BINARY(operator-, SUB)
MAPB_BINARY(operator*, MUL)
MAPB_BINARY(operator/, DIV)
MAPB_BINARY(operator%, MOD)
MAPB_BINARY(operator==, EQ)
MAPB_BINARY(operator!=, NE)
MAPB_BINARY(operator<, LT)
MAPB_BINARY(operator>, GT)
MAPB_BINARY(operator<=, LE)
MAPB_BINARY(operator>=, GE)
MAPB_BINARY(operator&&, AND)
MAPB_BINARY(operator||, OR)
MAPB_BINARY(operator&, bAND)
MAPB_BINARY(operator|, bOR)
MAPB_BINARY(operator^, bXOR)
MAPB_BINARY(operator<<, SHL)
MAPB_BINARY(operator>>, SHR)
MAPB_BINARY(max, MAX2)
MAPB_BINARY(min, MIN2)
MAPB_BINARY(atan2, ATAN2)
MAPB_BINARY(pow, POW)
MAPB_BINARY(hypot, HYPOT)
MAPB_BINARY(fmod, FMOD)
#undef MAPB_BINARY

/* ---- focal and zonal (front/Raster.hpp:279-296) ---- */
inline Raster convolve(const Raster &r, const Mask &m) {
  std::vector<ma_Variant> v = m.values;
  return Raster(ma_convolution(r.node, v.data(), (int)v.size(), m.size.a));
}
#define MAPB_FOCAL(name, red)                                                              \
  inline Raster name(const Raster &r, const Mask &m) {                                    \
    std::vector<ma_Variant> v = m.values;                                                  \
    return Raster(ma_focalFunc(r.node, v.data(), (int)v.size(), m.size.a, red));          \
  }
MAPB_FOCAL(focalSum, SUM)
MAPB_FOCAL(focalProd, PROD)
MAPB_FOCAL(focalMax, MAX)
MAPB_FOCAL(focalMin, MIN)
#undef MAPB_FOCAL
#define MAPB_ZONAL(name, red) \
  inline Raster name(const Raster &r) { return Raster(ma_zonalReduc(r.node, red)); }
MAPB_ZONAL(zonalSum, SUM)
MAPB_ZONAL(zonalProd, PROD)
MAPB_ZONAL(zonalMax, MAX)
MAPB_ZONAL(zonalMin, MIN)
#undef MAPB_ZONAL
inline Raster radialScan(const Raster &r, ReductionType red, const Coord &start) {
  return Raster(ma_radialScan(r.node, red, start.a));
}
inline Raster spreadScan(const Raster &r, const Raster &dir, ReductionType red) {
  return Raster(ma_spreadScan(r.node, dir.node, red));
}

/* ---- compound methods (front/Raster.cpp:452-579) ---- */
/* vec[data] where data holds an index into vec, else 0 (front/Raster.cpp:465-472) */
inline Raster pick(const Raster &data, const std::vector<Variant> &vec) {
  if (vec.empty()) throw Error("pick: empty value list");
  Raster acu = zeros(DataSize(), vec[0].datatype());
  for (int i = 0; i < (int)vec.size(); i++) acu = con(data == Variant((int32_t)i), Raster(vec[i]), acu);
  return acu;
}
/* sqrt(x*x + y*y + 0.0f) with x = c0 - index(D1), y = c1 - index(D2) (front/Raster.cpp:473-478) */
inline Raster distance(const Raster &data, const Coord &c) {
  Raster x = Variant((int32_t)c[0]) - index(data, D1);
  Raster y = Variant((int32_t)c[1]) - index(data, D2);
  return sqrt(x * x + y * y + Variant(0.0f));
}
inline Raster square(const Raster &data) { return data * data; }
/* height above the line of sight (front/Raster.cpp:558-569) */
inline Raster viewshed(const Raster &data, const Coord &obs, float obs_h) {
  Raster shift = data - Variant(obs_h);
  Raster dist = distance(data, obs);
  Raster slope = shift / dist;
  Raster mx = radialScan(slope, MAX, obs);
  return (mx * dist + Variant(obs_h)) - data;
}
/* upstream sum of `data` along D8 directions (front/Raster.cpp:571-579) */
inline Raster flowAccumulation(const Raster &data, const Raster &dir) { return spreadScan(data, dir, SUM); }

/* ---- extensions (map_b200.h) ---- */
/* D8 steepest-descent directions, U8 codes 1 << dir in E, SE, S, SW, W, NW, N, NE order */
inline Raster flowDirection(const Raster &dem) { return Raster(ma_focalFlow(dem.node)); }
/* raster input from host memory (dense, row-major; copied unless copy is false) */
inline Raster fromHost(const void *data, DataSize ds, DataType dt, BlockSize bs = BlockSize(), bool copy = true) {
  return Raster(ma_fromHost(data, ds.a, dt, bs.a, copy ? 1 : 0));
}
/* raster input from device memory (pitch in bytes) */
inline Raster fromDevice(void *dptr, long long pitch, DataSize ds, DataType dt, BlockSize bs = BlockSize()) {
  return Raster(ma_fromDevice(dptr, pitch, ds.a, dt, bs.a));
}
/* evaluates `r` into dense row-major host memory */
inline void toHost(const Raster &r, void *dst, size_t bytes) {
  if (ma_toHost(r.node, dst, bytes)) throw Error(ma_lastError());
}
inline void toDevice(const Raster &r, void *dptr, long long pitch, bool async = false) {
  if (ma_toDevice(r.node, dptr, pitch, async ? 1 : 0)) throw Error(ma_lastError());
}
inline void setBorder(Border b) {
  ma_setBorder(b);
  detail::check();
}
inline void setExecMode(ExecMode m) {
  ma_setExecMode(m);
  detail::check();
}
inline void setStreamRows(int rows) {
  ma_setStreamRows(rows);
  detail::check();
}

}  // namespace map

#endif /* MAP_B200_HPP_ */
