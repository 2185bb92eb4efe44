// scalars.hpp - extra scalar types for the oracle (test infrastructure only).
//
//  * Counted: a double that counts the floating-point operations done on it,
//    used to freeze the algorithmic FLOPs per integration step that the
//    roofline figures divide by.
//  * __float128 overloads (libquadmath) for the high-precision check of the
//    FP64 stepper, the role MPFR-256 plays in the reference's
//    tests/precision_regression_test.cpp:150-195.
#pragma once

#include <cmath>
#include <cstdint>
#include <quadmath.h>

namespace bho {

struct OpCounts {
  int64_t add = 0, mul = 0, div = 0, sqrt = 0, trig = 0, pow = 0, cmp = 0;
};
inline thread_local OpCounts g_counts;

struct Counted {
  double v = 0.0;
  Counted() = default;
  Counted(double x) : v(x) {}  // NOLINT: implicit on purpose, literals mix with Counted
  explicit operator double() const { return v; }
};
inline Counted operator+(Counted a, Counted b) { ++g_counts.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_counts.add; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_counts.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_counts.div; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }  // sign flip: free
inline Counted &operator+=(Counted &a, Counted b) { a = a + b; return a; }
inline bool operator<(Counted a, Counted b) { ++g_counts.cmp; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++g_counts.cmp; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++g_counts.cmp; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { ++g_counts.cmp; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { ++g_counts.cmp; return a.v == b.v; }
inline Counted s_sqrt(Counted x) { ++g_counts.sqrt; return Counted(std::sqrt(x.v)); }
inline Counted s_sin(Counted x) { ++g_counts.trig; return Counted(std::sin(x.v)); }
inline Counted s_cos(Counted x) { ++g_counts.trig; return Counted(std::cos(x.v)); }
inline Counted s_acos(Counted x) { ++g_counts.trig; return Counted(std::acos(x.v)); }
inline Counted s_abs(Counted x) { return Counted(std::fabs(x.v)); }
inline Counted s_cbrt(Counted x) { ++g_counts.pow; return Counted(std::cbrt(x.v)); }
inline Counted s_pow(Counted x, Counted y) { ++g_counts.pow; return Counted(std::pow(x.v, y.v)); }
// exp / log family: counted with the transcendental functions (trig), not as FLOPs
inline Counted s_log(Counted x) { ++g_counts.trig; return Counted(std::log(x.v)); }
inline Counted s_exp(Counted x) { ++g_counts.trig; return Counted(std::exp(x.v)); }
inline Counted s_expm1(Counted x) { ++g_counts.trig; return Counted(std::expm1(x.v)); }
inline Counted s_floor(Counted x) { return Counted(std::floor(x.v)); }
inline Counted s_ceil(Counted x) { return Counted(std::ceil(x.v)); }

using f128 = __float128;
inline f128 s_sqrt(f128 x) { return sqrtq(x); }
inline f128 s_sin(f128 x) { return sinq(x); }
inline f128 s_cos(f128 x) { return cosq(x); }
inline f128 s_abs(f128 x) { return fabsq(x); }
inline f128 s_acos(f128 x) { return acosq(x); }
inline f128 s_cbrt(f128 x) { return cbrtq(x); }
inline f128 s_pow(f128 x, f128 y) { return powq(x, y); }

}  // namespace bho
