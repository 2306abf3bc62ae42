// Dtype tables, Variant conversions and the host (scalar) operator semantics.
// Scalar results are what the reference computes on the host for D0 values
// (runtime/task/ScalarTask.cpp:69-190 through util/UnaryType.tpl and
// util/BinaryType.tpl), restated here with the same C++ numeric behaviour.
#include "types.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <limits>

namespace mapb {

size_t dt_size(int dt) {
  switch (dt) {
    case F32: return 4; case F64: return 8; case B8: return 1; case U8: return 1;
    case U16: return 2; case U32: return 4; case U64: return 8; case S8: return 1;
    case S16: return 2; case S32: return 4; case S64: return 8;
    default: throw MapError("invalid data type " + std::to_string(dt));
  }
}

const char *dt_name(int dt) {
  static const char *n[] = {"NONE_DATATYPE", "F32", "F64", "B8", "U8", "U16", "U32", "U64", "S8", "S16", "S32", "S64"};
  if (dt < 0 || dt >= N_DATATYPE) throw MapError("invalid data type");
  return n[dt];
}

const char *dt_ctype(int dt) {
  switch (dt) {
    case F32: return "float"; case F64: return "double"; case B8: return "bool";
    case U8: return "u8"; case U16: return "u16"; case U32: return "u32"; case U64: return "u64";
    case S8: return "s8"; case S16: return "s16"; case S32: return "s32"; case S64: return "s64";
    default: throw MapError("invalid data type");
  }
}

bool dt_is_float(int dt) { return dt == F32 || dt == F64; }
bool dt_is_signed(int dt) { return dt == S8 || dt == S16 || dt == S32 || dt == S64; }
bool dt_is_unsigned(int dt) { return dt == B8 || dt == U8 || dt == U16 || dt == U32 || dt == U64; }

// Promotion of a pair of operand types, in the order
// F32 F64 B8 U8 U16 U32 U64 S8 S16 S32 S64 (util/promote.hpp:17-131).
// The U64 x B8 -> B8 entry is kept as the reference defines it.
int dt_promote(int a, int b) {
  static const int T[11][11] = {
      /* F32 */ {F32, F64, F32, F32, F32, F32, F32, F32, F32, F32, F32},
      /* F64 */ {F64, F64, F64, F64, F64, F64, F64, F64, F64, F64, F64},
      /* B8  */ {F32, F64, B8, U8, U16, U32, U64, S8, S16, S32, S64},
      /* U8  */ {F32, F64, U8, U8, U16, U32, U64, S8, S16, S32, S64},
      /* U16 */ {F32, F64, U16, U16, U16, U32, U64, U16, S16, S32, S64},
      /* U32 */ {F32, F64, U32, U32, U32, U32, U64, S32, S32, S32, S64},
      /* U64 */ {F32, F64, B8, U64, U64, U64, U64, S64, S64, S64, S64},
      /* S8  */ {F32, F64, S8, S8, S16, S32, S64, S8, S16, S32, S64},
      /* S16 */ {F32, F64, S16, S16, S16, S32, S64, S16, S16, S32, S64},
      /* S32 */ {F32, F64, S32, S32, S32, S32, S64, S32, S32, S32, S64},
      /* S64 */ {F32, F64, S64, S64, S64, S64, S64, S64, S64, S64, S64},
  };
  if (a <= NONE_DATATYPE || a >= N_DATATYPE || b <= NONE_DATATYPE || b >= N_DATATYPE)
    throw MapError("promote: invalid data type");
  return T[a - 1][b - 1];
}

int numdim_toint(int nd) {
  switch (nd) {
    case D0: return 0; case D1: return 1; case D2: return 2; case D3: return 3;
    default: throw MapError("invalid numdim");
  }
}

int numdim_fromsize(const Arr2 &ds) {
  int n = 0;
  for (int i = 0; i < 2; i++) if (ds.arr[i] > 0) n++;
  if (ds.n == 0) return D0;
  return n == 0 ? D0 : n == 1 ? D1 : D2;
}

const char *unary_name(int u) {
  static const char *n[] = {"NONE_UNARY", "POS", "NEG", "NOT", "bNOT", "MARK_UNARY", "SIN", "COS", "TAN", "ASIN", "ACOS",
                            "ATAN", "SINH", "COSH", "TANH", "ASINH", "ACOSH", "ATANH", "EXP", "EXP2", "EXP10", "LOG",
                            "LOG2", "LOG10", "SQRT", "CBRT", "ABS", "CEIL", "FLOOR", "TRUNC", "ROUND"};
  if (u <= NONE_UNARY || u >= N_UNARY || u == MARK_UNARY) throw MapError("invalid unary op " + std::to_string(u));
  return n[u];
}
const char *binary_name(int b) {
  static const char *n[] = {"NONE_BINARY", "ADD", "SUB", "MUL", "DIV", "MOD", "EQ", "NE", "LT", "GT", "LE", "GE", "AND",
                            "OR", "bAND", "bOR", "bXOR", "SHL", "SHR", "MARK_BINARY", "MAX2", "MIN2", "ATAN2", "POW",
                            "HYPOT", "FMOD"};
  if (b <= NONE_BINARY || b >= N_BINARY || b == MARK_BINARY) throw MapError("invalid binary op " + std::to_string(b));
  return n[b];
}
const char *reduction_name(int r) {
  static const char *n[] = {"NONE_REDUCTION", "SUM", "PROD", "rAND", "rOR", "MARK_REDUCTION", "MAX", "MIN"};
  if (r <= NONE_REDUCTION || r >= N_REDUCTION || r == MARK_REDUCTION) throw MapError("invalid reduction " + std::to_string(r));
  return n[r];
}
bool unary_is_operator(int u) { return u < MARK_UNARY; }
bool binary_is_operator(int b) { return b < MARK_BINARY; }
bool binary_is_relational(int b) { return b >= EQ && b <= OR; }
bool binary_is_bitwise(int b) { return b >= bAND && b <= SHR; }

// ---------------------------------------------------------------- Variant

template <typename T> static T get_as(const Variant &v) {
  switch (v.dtype) {
    case F32: return (T)v.u.f32; case F64: return (T)v.u.f64; case B8: return (T)v.u.b8;
    case U8: return (T)v.u.u8; case U16: return (T)v.u.u16; case U32: return (T)v.u.u32; case U64: return (T)v.u.u64;
    case S8: return (T)v.u.s8; case S16: return (T)v.u.s16; case S32: return (T)v.u.s32; case S64: return (T)v.u.s64;
    default: throw MapError("variant with invalid data type " + std::to_string(v.dtype));
  }
}

template <typename T> static Variant set_as(T x, int dt) {
  Variant r;
  std::memset(&r, 0, sizeof(r));
  r.dtype = dt;
  switch (dt) {
    case F32: r.u.f32 = (float)x; break; case F64: r.u.f64 = (double)x; break; case B8: r.u.b8 = (bool)x; break;
    case U8: r.u.u8 = (uint8_t)x; break; case U16: r.u.u16 = (uint16_t)x; break; case U32: r.u.u32 = (uint32_t)x; break;
    case U64: r.u.u64 = (uint64_t)x; break; case S8: r.u.s8 = (int8_t)x; break; case S16: r.u.s16 = (int16_t)x; break;
    case S32: r.u.s32 = (int32_t)x; break; case S64: r.u.s64 = (int64_t)x; break;
    default: throw MapError("invalid data type");
  }
  return r;
}

Variant var_make_f64(double v, int dt) { return set_as<double>(v, dt); }

// VariantType::convert: value read in its stored type and cast to dt (util/VariantType.cpp:106-121).
Variant var_convert(const Variant &v, int dt) {
  switch (v.dtype) {
    case F32: return set_as(v.u.f32, dt); case F64: return set_as(v.u.f64, dt); case B8: return set_as(v.u.b8, dt);
    case U8: return set_as(v.u.u8, dt); case U16: return set_as(v.u.u16, dt); case U32: return set_as(v.u.u32, dt);
    case U64: return set_as(v.u.u64, dt); case S8: return set_as(v.u.s8, dt); case S16: return set_as(v.u.s16, dt);
    case S32: return set_as(v.u.s32, dt); case S64: return set_as(v.u.s64, dt);
    default: throw MapError("variant with invalid data type");
  }
}

double var_as_f64(const Variant &v) { return get_as<double>(v); }
int64_t var_as_i64(const Variant &v) { return get_as<int64_t>(v); }

bool var_equal(const Variant &a, const Variant &b) {
  if (a.dtype != b.dtype) return false;
  return std::memcmp(&a.u, &b.u, dt_size(a.dtype)) == 0;
}

bool var_is_zero(const Variant &v) { return dt_is_float(v.dtype) ? var_as_f64(v) == 0.0 : var_as_i64(v) == 0; }

std::string var_to_string(const Variant &v) {
  switch (v.dtype) {
    case F32: return std::to_string(v.u.f32); case F64: return std::to_string(v.u.f64);
    case B8: return std::to_string(v.u.b8); case U8: return std::to_string(v.u.u8);
    case U16: return std::to_string(v.u.u16); case U32: return std::to_string(v.u.u32);
    case U64: return std::to_string(v.u.u64); case S8: return std::to_string(v.u.s8);
    case S16: return std::to_string(v.u.s16); case S32: return std::to_string(v.u.s32);
    case S64: return std::to_string(v.u.s64);
    default: throw MapError("variant with invalid data type");
  }
}

std::string var_literal(const Variant &v) {
  char buf[64];
  switch (v.dtype) {
    case F32: {
      float f = v.u.f32;
      if (std::isnan(f)) return "__int_as_float(0x7fc00000)";
      if (std::isinf(f)) return f > 0 ? "__int_as_float(0x7f800000)" : "__int_as_float(0xff800000)";
      std::snprintf(buf, sizeof buf, "%af", (double)f);
      return buf;
    }
    case F64: {
      double d = v.u.f64;
      if (std::isnan(d)) return "__longlong_as_double(0x7ff8000000000000ULL)";
      if (std::isinf(d)) return d > 0 ? "__longlong_as_double(0x7ff0000000000000ULL)" : "__longlong_as_double(0xfff0000000000000ULL)";
      std::snprintf(buf, sizeof buf, "%a", d);
      return buf;
    }
    case B8: return v.u.b8 ? "true" : "false";
    case U8: return "((u8)" + std::to_string(v.u.u8) + "u)";
    case U16: return "((u16)" + std::to_string(v.u.u16) + "u)";
    case U32: return std::to_string(v.u.u32) + "u";
    case U64: return std::to_string(v.u.u64) + "ull";
    case S8: return "((s8)" + std::to_string(v.u.s8) + ")";
    case S16: return "((s16)" + std::to_string(v.u.s16) + ")";
    case S32: return v.u.s32 == std::numeric_limits<int32_t>::min() ? "(-2147483647-1)" : std::to_string(v.u.s32);
    case S64: return v.u.s64 == std::numeric_limits<int64_t>::min() ? "(-9223372036854775807ll-1)" : std::to_string(v.u.s64) + "ll";
    default: throw MapError("variant with invalid data type");
  }
}

size_t var_hash(const Variant &v) {
  uint64_t bits = 0;
  std::memcpy(&bits, &v.u, dt_size(v.dtype));
  return std::hash<uint64_t>()(bits) ^ (std::hash<int>()(v.dtype) << 1);
}

// ------------------------------------------------------- host operators

template <typename T> static T unary_fn(int op, T x) {
  if constexpr (std::is_floating_point<T>::value) {
    switch (op) {
      case POS: return +x; case NEG: return -x; case NOT: return (T)(!x);
      case SIN: return std::sin(x); case COS: return std::cos(x); case TAN: return std::tan(x);
      case ASIN: return std::asin(x); case ACOS: return std::acos(x); case ATAN: return std::atan(x);
      case SINH: return std::sinh(x); case COSH: return std::cosh(x); case TANH: return std::tanh(x);
      case ASINH: return std::asinh(x); case ACOSH: return std::acosh(x); case ATANH: return std::atanh(x);
      case EXP: return std::exp(x); case EXP2: return std::exp2(x); case EXP10: return (T)std::pow(10, x);
      case LOG: return std::log(x); case LOG2: return std::log2(x); case LOG10: return std::log10(x);
      case SQRT: return std::sqrt(x); case CBRT: return std::cbrt(x); case ABS: return std::abs(x);
      case CEIL: return std::ceil(x); case FLOOR: return std::floor(x); case TRUNC: return std::trunc(x);
      case ROUND: return std::round(x);
      case bNOT: throw MapError("bitwise not on a floating type");
      default: throw MapError("invalid unary op");
    }
  } else {
    double d = (double)x;
    switch (op) {
      case POS: return (T)(+x); case NEG: return (T)(-x); case NOT: return (T)(!x);
      case bNOT:
        if (!std::is_unsigned<T>::value) throw MapError("bitwise not on a signed type");
        return (T)(~x);
      case SIN: return (T)std::sin(d); case COS: return (T)std::cos(d); case TAN: return (T)std::tan(d);
      case ASIN: return (T)std::asin(d); case ACOS: return (T)std::acos(d); case ATAN: return (T)std::atan(d);
      case SINH: return (T)std::sinh(d); case COSH: return (T)std::cosh(d); case TANH: return (T)std::tanh(d);
      case ASINH: return (T)std::asinh(d); case ACOSH: return (T)std::acosh(d); case ATANH: return (T)std::atanh(d);
      case EXP: return (T)std::exp(d); case EXP2: return (T)std::exp2(d); case EXP10: return (T)std::pow(10.0, d);
      case LOG: return (T)std::log(d); case LOG2: return (T)std::log2(d); case LOG10: return (T)std::log10(d);
      case SQRT: return (T)std::sqrt(d); case CBRT: return (T)std::cbrt(d);
      case ABS: return std::is_signed<T>::value ? (T)(x < 0 ? -x : x) : x;
      case CEIL: case FLOOR: case TRUNC: case ROUND: return x;
      default: throw MapError("invalid unary op");
    }
  }
}

template <typename T> static Variant unary_typed(int op, const Variant &v, int dt) {
  return set_as<T>(unary_fn<T>(op, get_as<T>(v)), dt);
}

Variant host_unary(int op, const Variant &v) {
  switch (v.dtype) {
    case F32: return unary_typed<float>(op, v, F32); case F64: return unary_typed<double>(op, v, F64);
    case B8: return unary_typed<uint8_t>(op, v, B8); case U8: return unary_typed<uint8_t>(op, v, U8);
    case U16: return unary_typed<uint16_t>(op, v, U16); case U32: return unary_typed<uint32_t>(op, v, U32);
    case U64: return unary_typed<uint64_t>(op, v, U64); case S8: return unary_typed<int8_t>(op, v, S8);
    case S16: return unary_typed<int16_t>(op, v, S16); case S32: return unary_typed<int32_t>(op, v, S32);
    case S64: return unary_typed<int64_t>(op, v, S64);
    default: throw MapError("unary on invalid data type");
  }
}

template <typename T> static Variant binary_typed(int op, T a, T b, int dt) {
  if (binary_is_relational(op)) {
    uint8_t r;
    switch (op) {
      case EQ: r = a == b; break; case NE: r = a != b; break; case LT: r = a < b; break;
      case GT: r = a > b; break; case LE: r = a <= b; break; case GE: r = a >= b; break;
      case AND: r = a && b; break; case OR: r = a || b; break;
      default: throw MapError("invalid relational op");
    }
    return set_as<uint8_t>(r, U8);
  }
  if constexpr (std::is_floating_point<T>::value) {
    switch (op) {
      case ADD: return set_as<T>(a + b, dt); case SUB: return set_as<T>(a - b, dt);
      case MUL: return set_as<T>(a * b, dt); case DIV: return set_as<T>(a / b, dt);
      case MAX2: return set_as<T>(std::max(a, b), dt); case MIN2: return set_as<T>(std::min(a, b), dt);
      case ATAN2: return set_as<T>(std::atan2(a, b), dt); case POW: return set_as<T>(std::pow(a, b), dt);
      case HYPOT: return set_as<T>(std::hypot(a, b), dt); case FMOD: return set_as<T>(std::fmod(a, b), dt);
      default: throw MapError(std::string("binary op ") + binary_name(op) + " is not defined on floating types");
    }
  } else {
    switch (op) {
      case ADD: return set_as<T>((T)(a + b), dt); case SUB: return set_as<T>((T)(a - b), dt);
      case MUL: return set_as<T>((T)(a * b), dt);
      case DIV: if (b == 0) throw MapError("integer division by zero"); return set_as<T>((T)(a / b), dt);
      case MOD: if (b == 0) throw MapError("integer modulo by zero"); return set_as<T>((T)(a % b), dt);
      case bAND: return set_as<T>((T)(a & b), dt); case bOR: return set_as<T>((T)(a | b), dt);
      case bXOR: return set_as<T>((T)(a ^ b), dt); case SHL: return set_as<T>((T)(a << b), dt);
      case SHR: return set_as<T>((T)(a >> b), dt);
      case MAX2: return set_as<T>(std::max(a, b), dt); case MIN2: return set_as<T>(std::min(a, b), dt);
      case ATAN2: return set_as<T>((T)std::atan2((double)a, (double)b), dt);
      case POW: return set_as<T>((T)std::pow((double)a, (double)b), dt);
      case HYPOT: return set_as<T>((T)std::hypot((double)a, (double)b), dt);
      case FMOD: return set_as<T>((T)std::fmod((double)a, (double)b), dt);
      default: throw MapError("invalid binary op");
    }
  }
}

Variant host_binary(int op, const Variant &l, const Variant &r) {
  int pt = dt_promote(l.dtype, r.dtype);
  switch (pt) {
    case F32: return binary_typed<float>(op, get_as<float>(l), get_as<float>(r), F32);
    case F64: return binary_typed<double>(op, get_as<double>(l), get_as<double>(r), F64);
    case B8: return binary_typed<uint8_t>(op, get_as<bool>(l), get_as<bool>(r), B8);
    case U8: return binary_typed<uint8_t>(op, get_as<uint8_t>(l), get_as<uint8_t>(r), U8);
    case U16: return binary_typed<uint16_t>(op, get_as<uint16_t>(l), get_as<uint16_t>(r), U16);
    case U32: return binary_typed<uint32_t>(op, get_as<uint32_t>(l), get_as<uint32_t>(r), U32);
    case U64: return binary_typed<uint64_t>(op, get_as<uint64_t>(l), get_as<uint64_t>(r), U64);
    case S8: return binary_typed<int8_t>(op, get_as<int8_t>(l), get_as<int8_t>(r), S8);
    case S16: return binary_typed<int16_t>(op, get_as<int16_t>(l), get_as<int16_t>(r), S16);
    case S32: return binary_typed<int32_t>(op, get_as<int32_t>(l), get_as<int32_t>(r), S32);
    case S64: return binary_typed<int64_t>(op, get_as<int64_t>(l), get_as<int64_t>(r), S64);
    default: throw MapError("binary on invalid data type");
  }
}

template <typename T> static Variant reduce_typed(int op, T a, T b, int dt) {
  switch (op) {
    case SUM: return set_as<T>((T)(a + b), dt);
    case PROD: return set_as<T>((T)(a * b), dt);
    case MAX: return set_as<T>(std::max(a, b), dt);
    case MIN: return set_as<T>(std::min(a, b), dt);
    case rAND: case rOR:
      if constexpr (std::is_floating_point<T>::value) {
        throw MapError("bitwise reduction on a floating type");
      } else {
        return set_as<T>((T)(op == rAND ? (a & b) : (a | b)), dt);
      }
    default: throw MapError("invalid reduction");
  }
}

Variant host_reduce(int op, const Variant &l, const Variant &r) {
  MAPB_CHECK(l.dtype == r.dtype, "reduction operands must share a type");
  switch (l.dtype) {
    case F32: return reduce_typed<float>(op, l.u.f32, r.u.f32, F32);
    case F64: return reduce_typed<double>(op, l.u.f64, r.u.f64, F64);
    case B8: return reduce_typed<uint8_t>(op, l.u.b8, r.u.b8, B8);
    case U8: return reduce_typed<uint8_t>(op, l.u.u8, r.u.u8, U8);
    case U16: return reduce_typed<uint16_t>(op, l.u.u16, r.u.u16, U16);
    case U32: return reduce_typed<uint32_t>(op, l.u.u32, r.u.u32, U32);
    case U64: return reduce_typed<uint64_t>(op, l.u.u64, r.u.u64, U64);
    case S8: return reduce_typed<int8_t>(op, l.u.s8, r.u.s8, S8);
    case S16: return reduce_typed<int16_t>(op, l.u.s16, r.u.s16, S16);
    case S32: return reduce_typed<int32_t>(op, l.u.s32, r.u.s32, S32);
    case S64: return reduce_typed<int64_t>(op, l.u.s64, r.u.s64, S64);
    default: throw MapError("reduction on invalid data type");
  }
}

// Neutral elements (util/ReductionType.cpp neutralString / ReductionType.tpl):
// SUM 0, PROD 1, MAX the type's lowest (-inf for floats), MIN the type's highest
// (+inf for floats), rAND all-ones, rOR zero.
Variant reduction_neutral(int op, int dt) {
  auto lowest = [&]() -> Variant {
    switch (dt) {
      case F32: return set_as<float>(-std::numeric_limits<float>::infinity(), dt);
      case F64: return set_as<double>(-std::numeric_limits<double>::infinity(), dt);
      case S8: return set_as<int64_t>(INT8_MIN, dt); case S16: return set_as<int64_t>(INT16_MIN, dt);
      case S32: return set_as<int64_t>(INT32_MIN, dt); case S64: return set_as<int64_t>(INT64_MIN, dt);
      default: return set_as<int>(0, dt);
    }
  };
  auto highest = [&]() -> Variant {
    switch (dt) {
      case F32: return set_as<float>(std::numeric_limits<float>::infinity(), dt);
      case F64: return set_as<double>(std::numeric_limits<double>::infinity(), dt);
      case B8: return set_as<int>(1, dt);
      case U8: return set_as<uint64_t>(UINT8_MAX, dt); case U16: return set_as<uint64_t>(UINT16_MAX, dt);
      case U32: return set_as<uint64_t>(UINT32_MAX, dt); case U64: return set_as<uint64_t>(UINT64_MAX, dt);
      case S8: return set_as<int64_t>(INT8_MAX, dt); case S16: return set_as<int64_t>(INT16_MAX, dt);
      case S32: return set_as<int64_t>(INT32_MAX, dt); case S64: return set_as<int64_t>(INT64_MAX, dt);
      default: throw MapError("invalid data type");
    }
  };
  switch (op) {
    case SUM: return set_as<int>(0, dt);
    case PROD: return set_as<int>(1, dt);
    case rAND: return highest();
    case rOR: return lowest();
    case MAX: return lowest();
    case MIN: return highest();
    default: throw MapError("invalid reduction");
  }
}

}  // namespace mapb
