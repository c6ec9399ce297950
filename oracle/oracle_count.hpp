// ORACLE — test infrastructure only (see oracle_tables.hpp header).
//
// A single-precision number type that counts the floating-point operations
// done on it, so that the oracle's restatement, instantiated with it, gives
// the operation counts of the reference's algorithm per sea point and per
// spectral bin: additions (and subtractions), multiplications, divisions,
// square roots, transcendental functions (EXP, LOG, LOG10, **, TANH, COS,
// SIN, ATAN2, SINH, COSH, ACOS; each counted as 1) and comparisons (MAX,
// MIN and IF tests).  Values are those of the float restatement.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <limits>

namespace wamo {

struct OpCounts {
  uint64_t add = 0, mul = 0, div = 0, sqrt = 0, trans = 0, cmp = 0;
};
inline thread_local OpCounts g_ops;

struct CF {
  float v;
  constexpr CF() : v(0) {}
  constexpr CF(double x) : v((float)x) {}
  explicit constexpr operator double() const { return v; }
  explicit constexpr operator float() const { return v; }
  explicit constexpr operator int() const { return (int)v; }
};

#define WAMO_CF_BIN(OP, CNT)                                                         \
  constexpr CF operator OP(CF a, CF b) {                                             \
    if (!__builtin_is_constant_evaluated()) ++g_ops.CNT;                             \
    return CF(a.v OP b.v);                                                           \
  }
WAMO_CF_BIN(+, add)
WAMO_CF_BIN(-, add)
WAMO_CF_BIN(*, mul)
WAMO_CF_BIN(/, div)
#undef WAMO_CF_BIN
constexpr CF operator-(CF a) { return CF(-a.v); }
#define WAMO_CF_CMP(OP)                                \
  constexpr bool operator OP(CF a, CF b) {             \
    if (!__builtin_is_constant_evaluated()) ++g_ops.cmp; \
    return a.v OP b.v;                                 \
  }
WAMO_CF_CMP(<) WAMO_CF_CMP(>) WAMO_CF_CMP(<=) WAMO_CF_CMP(>=) WAMO_CF_CMP(==) WAMO_CF_CMP(!=)
#undef WAMO_CF_CMP

inline int JAFU(double CL, int J, int IAN);  // oracle_tables.hpp
inline int JAFU(CF CL, int J, int IAN) { return JAFU((double)CL.v, J, IAN); }
inline int int_f(CF x) { return (int)std::trunc((double)x.v); }
inline int nint_f(CF x) { return (int)std::lround((double)x.v); }
inline CF crlog10(CF x) { ++g_ops.trans; return CF(std::log10((double)x.v)); }
inline CF crlog(CF x) { ++g_ops.trans; return CF(std::log((double)x.v)); }
inline CF crexp(CF x) { ++g_ops.trans; return CF(std::exp((double)x.v)); }
inline CF crcos(CF x) { ++g_ops.trans; return CF(std::cos((double)x.v)); }
inline CF crsin(CF x) { ++g_ops.trans; return CF(std::sin((double)x.v)); }
inline CF crtanh(CF x) { ++g_ops.trans; return CF(std::tanh((double)x.v)); }
inline CF crcosh(CF x) { ++g_ops.trans; return CF(std::cosh((double)x.v)); }
inline CF crsinh(CF x) { ++g_ops.trans; return CF(std::sinh((double)x.v)); }

}  // namespace wamo

namespace std {
// the restatement calls the <cmath> functions qualified
inline wamo::CF sqrt(wamo::CF x) { ++wamo::g_ops.sqrt; return wamo::CF(std::sqrt(x.v)); }
inline wamo::CF fabs(wamo::CF x) { return wamo::CF(std::fabs(x.v)); }
#define WAMO_CF_T1(F)                                                               \
  inline wamo::CF F(wamo::CF x) { ++wamo::g_ops.trans; return wamo::CF(std::F(x.v)); }
WAMO_CF_T1(exp) WAMO_CF_T1(log) WAMO_CF_T1(log10) WAMO_CF_T1(tanh) WAMO_CF_T1(cos) WAMO_CF_T1(sin)
WAMO_CF_T1(sinh) WAMO_CF_T1(cosh) WAMO_CF_T1(acos)
#undef WAMO_CF_T1
inline wamo::CF floor(wamo::CF x) { return wamo::CF(std::floor(x.v)); }
inline wamo::CF ceil(wamo::CF x) { return wamo::CF(std::ceil(x.v)); }
inline wamo::CF pow(wamo::CF x, wamo::CF y) { ++wamo::g_ops.trans; return wamo::CF(std::pow(x.v, y.v)); }
inline wamo::CF atan2(wamo::CF y, wamo::CF x) { ++wamo::g_ops.trans; return wamo::CF(std::atan2(y.v, x.v)); }
template <> struct numeric_limits<wamo::CF> {
  static constexpr bool is_specialized = true;
  static constexpr wamo::CF min() { return wamo::CF(FLT_MIN); }
  static constexpr wamo::CF max() { return wamo::CF(FLT_MAX); }
};
}  // namespace std
