// Test-only C shim over the reference's own host-side operator tables
// (util/BinaryType.tpl, util/UnaryType.tpl, util/ReductionType.*, util/promote.hpp),
// compiled from the reference sources by oracle/build_oracle.py into
// oracle/_ref/libref_util.so. The tests use it to pin the engine's scalar (D0)
// semantics against the reference implementation itself.
#include "util/BinaryType.hpp"
#include "util/ReductionType.hpp"
#include "util/UnaryType.hpp"
#include "util/VariantType.hpp"
#include "util/promote.hpp"

#include <cstring>

using namespace map::detail;

namespace {
VariantType make(const void *bits, int dt) {
  VariantUnion u;
  std::memset(&u, 0, sizeof u);
  std::memcpy(&u, bits, DataType((DataTypeEnum)dt).sizeOf());
  return VariantType(u, DataType((DataTypeEnum)dt));
}
void put(const VariantType &v, void *out, int *odt) {
  std::memset(out, 0, 8);
  std::memcpy(out, &v.get(), v.datatype().sizeOf());
  *odt = v.datatype().get();
}
}  // namespace

extern "C" {
int ref_promote(int a, int b) { return promote(DataType((DataTypeEnum)a), DataType((DataTypeEnum)b)).get(); }
void ref_binary(int op, const void *l, int ldt, const void *r, int rdt, void *out, int *odt) {
  put(BinaryType((BinaryEnum)op).apply(make(l, ldt), make(r, rdt)), out, odt);
}
void ref_unary(int op, const void *v, int dt, void *out, int *odt) {
  put(UnaryType((UnaryEnum)op).apply(make(v, dt)), out, odt);
}
void ref_neutral(int op, int dt, void *out, int *odt) {
  put(ReductionType((ReductionEnum)op).neutral(DataType((DataTypeEnum)dt)), out, odt);
}
void ref_reduce(int op, const void *l, const void *r, int dt, void *out, int *odt) {
  put(ReductionType((ReductionEnum)op).apply(make(l, dt), make(r, dt)), out, odt);
}
}
