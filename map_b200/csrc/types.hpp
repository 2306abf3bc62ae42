// Value types shared by the whole host runtime: the enum tables of the map-algebra
// language, the two POD structs that cross the C ABI by value, dtype promotion,
// and the host-side evaluation of one operator on scalar (D0) values.
//
// Enum numbering follows the reference's public tables so that the Python
// bindings and any caller compiled against the reference header keep working:
//   DataTypeEnum   util/DataType.hpp:21      (python/map.py:37-38)
//   NumDimEnum     util/NumDim.hpp           (python/map.py:40-41)
//   MemOrderEnum   util/MemOrder.hpp:17      (python/map.py:43-44)
//   UnaryEnum      python/map.py:49-63       (util/UnaryType.hpp)
//   BinaryEnum     python/map.py:65-79       (util/BinaryType.hpp)
//   ReductionEnum  python/map.py:81-82       (util/ReductionType.hpp)
#pragma once

#include <cstdint>
#include <cstring>
#include <string>
#include <stdexcept>

namespace mapb {

enum DataTypeEnum : int { NONE_DATATYPE = 0, F32, F64, B8, U8, U16, U32, U64, S8, S16, S32, S64, N_DATATYPE };
enum NumDimEnum : int { NONE_NUMDIM = 0x00, TIME = 0x01, D0 = 0x02, D1 = 0x04, D2 = 0x06, D3 = 0x08, N_NUMDIM = 0x0A };
enum MemOrderEnum : int { NONE_MEMORDER = 0x00, BLK = 0x01, ROW = 0x02, COL = 0x04, SFC = 0x06, N_MEMORDER = 0x08 };
enum DeviceTypeEnum : int { DEV_DEF = 0x01, DEV_CPU = 0x02, DEV_GPU = 0x04, DEV_ACC = 0x08, DEV_CUS = 0x16 };

enum UnaryEnum : int {
  NONE_UNARY = 0, POS, NEG, NOT, bNOT, MARK_UNARY,
  SIN, COS, TAN, ASIN, ACOS, ATAN,
  SINH, COSH, TANH, ASINH, ACOSH, ATANH,
  EXP, EXP2, EXP10, LOG, LOG2, LOG10,
  SQRT, CBRT, ABS,
  CEIL, FLOOR, TRUNC, ROUND, N_UNARY
};

enum BinaryEnum : int {
  NONE_BINARY = 0, ADD, SUB, MUL, DIV, MOD,
  EQ, NE, LT, GT, LE, GE, AND, OR,
  bAND, bOR, bXOR, SHL, SHR, MARK_BINARY,
  MAX2, MIN2, ATAN2, POW, HYPOT, FMOD, N_BINARY
};

enum ReductionEnum : int { NONE_REDUCTION = 0, SUM, PROD, rAND, rOR, MARK_REDUCTION, MAX, MIN, N_REDUCTION };

// Access patterns of nodes and fusion groups (bit set, as runtime/Pattern.hpp:20).
enum PatternBits : int {
  P_NONE = 0x00, P_FREE = 0x01, P_LOCAL = 0x02, P_FOCAL = 0x04, P_ZONAL = 0x08,
  P_RADIAL = 0x10, P_SPREAD = 0x20, P_SPECIAL = 0x40, P_BARRIER = 0x80
};

// How a focal read that falls outside the raster is resolved.
//  BORDER_BLOCK_MIRROR: the reference's rule (runtime/skeleton/util.cpp:493-506):
//     a neighbour outside the block grid is read from the centre cell's own
//     block with both block-local coordinates reflected (invert(i,d)).
//  BORDER_RASTER_MIRROR: reflect each coordinate at the true raster edge.
//  BORDER_DEAD: cells outside the raster read as zero.
enum BorderEnum : int { BORDER_BLOCK_MIRROR = 0, BORDER_RASTER_MIRROR = 1, BORDER_DEAD = 2 };

// How a program is launched on the device.
//  EXEC_FUSED: one launch per fusion group over the whole raster.
//  EXEC_PLAIN: one launch per fusion group per block, in the scheduler's order
//              (the reference's launch granularity, runtime/task/Task.cpp:322-389).
enum ExecModeEnum : int { EXEC_FUSED = 0, EXEC_PLAIN = 1 };

// Variant: 8-byte value + dtype tag, 16 bytes, passed by value across the ABI
// (util/VariantType.hpp:20-40, python/map.py:91-110).
union VariantUnion {
  float f32; double f64; bool b8; uint8_t u8; uint16_t u16; uint32_t u32; uint64_t u64;
  int8_t s8; int16_t s16; int32_t s32; int64_t s64;
};
struct Variant {
  VariantUnion u;
  int dtype;
};
static_assert(sizeof(Variant) == 16, "Variant must be 16 bytes");

// Array2: two ints + count, 12 bytes, passed by value (util/Array4.hpp:42-45, python/map.py:157-162).
struct Arr2 {
  int arr[2];
  int n;
};
static_assert(sizeof(Arr2) == 12, "Arr2 must be 12 bytes");

struct MapError : std::runtime_error {
  explicit MapError(const std::string &m) : std::runtime_error(m) {}
};
#define MAPB_CHECK(cond, msg) do { if (!(cond)) throw ::mapb::MapError(std::string(msg)); } while (0)

// ---- dtype helpers ----
size_t dt_size(int dt);
const char *dt_name(int dt);      // "F32", "U8", ...
const char *dt_ctype(int dt);     // device C type used in generated code
bool dt_is_float(int dt);
bool dt_is_signed(int dt);        // signed integer
bool dt_is_unsigned(int dt);      // unsigned integer (B8 counts as unsigned)
int dt_promote(int a, int b);     // util/promote.hpp table
int numdim_toint(int nd);         // D0->0, D1->1, D2->2, D3->3
int numdim_fromsize(const Arr2 &ds);
const char *unary_name(int u);
const char *binary_name(int b);
const char *reduction_name(int r);
bool unary_is_operator(int u);
bool binary_is_operator(int b);
bool binary_is_relational(int b);
bool binary_is_bitwise(int b);

// ---- Variant helpers ----
Variant var_make_f64(double v, int dt);     // value converted to dtype dt with C casts
Variant var_convert(const Variant &v, int dt);
double var_as_f64(const Variant &v);
int64_t var_as_i64(const Variant &v);
bool var_equal(const Variant &a, const Variant &b);
bool var_is_zero(const Variant &v);
std::string var_to_string(const Variant &v);  // std::to_string of the stored type
std::string var_literal(const Variant &v);    // exact literal for generated device code
size_t var_hash(const Variant &v);

// ---- Host evaluation of operators on scalars ----
// Unary ops compute in the operand's own type (util/UnaryType.tpl:66-113).
Variant host_unary(int op, const Variant &v);
// Binary ops convert both operands to promote(lt,rt) and compute in that type;
// relational ops return U8 (util/BinaryType.tpl:22-135).
Variant host_binary(int op, const Variant &l, const Variant &r);
// Reduction op on two values of the same type (util/ReductionType.cpp).
Variant host_reduce(int op, const Variant &l, const Variant &r);
Variant reduction_neutral(int op, int dt);

}  // namespace mapb
