// Forward-mode dual numbers for the adjoint and tangent kernels.
//
// Dual{v, d} carries a value and its derivative along one direction.  The element
// functional of adjoint.cu evaluates the FDV physics templated on the scalar type;
// with S = Dual every operation propagates the derivative by the chain rule, so the
// result is the exact directional derivative of the same floating-point program
// (branches taken on the values, as the primal takes them).
//
// The rn_* functions are the non-contracting round-to-nearest operations the primal
// physics uses for its exact-zero decisions (FDVGalerkin.h:308-379); for doubles they
// are the intrinsics, for duals the value part uses the same intrinsics.
#pragma once
#include <cmath>

#include "cfdv_types.h"

namespace cfdv {

// the double overloads stay visible beside the Dual ones declared below
using ::cos;
using ::cosh;
using ::fabs;
using ::fmax;
using ::fmin;
using ::pow;
using ::sin;
using ::sinh;
using ::sqrt;

struct Dual {
  double v, d;
  CFDV_HD CFDV_INLINE Dual() : v(0.0), d(0.0) {}
  CFDV_HD CFDV_INLINE Dual(double x) : v(x), d(0.0) {}  // NOLINT: constants promote implicitly
  CFDV_HD CFDV_INLINE Dual(double x, double dx) : v(x), d(dx) {}
  CFDV_HD CFDV_INLINE Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
  CFDV_HD CFDV_INLINE Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
  CFDV_HD CFDV_INLINE Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  CFDV_HD CFDV_INLINE Dual& operator/=(const Dual& o) { const double q = v / o.v; d = (d - q * o.d) / o.v; v = q; return *this; }
};

CFDV_HD CFDV_INLINE Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
CFDV_HD CFDV_INLINE Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
CFDV_HD CFDV_INLINE Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
CFDV_HD CFDV_INLINE Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
CFDV_HD CFDV_INLINE Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
CFDV_HD CFDV_INLINE Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
CFDV_HD CFDV_INLINE Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
CFDV_HD CFDV_INLINE Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
CFDV_HD CFDV_INLINE Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
CFDV_HD CFDV_INLINE Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
CFDV_HD CFDV_INLINE Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
CFDV_HD CFDV_INLINE Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
CFDV_HD CFDV_INLINE Dual operator/(double a, const Dual& b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
// comparisons look at values only (the branch the primal program takes)
CFDV_HD CFDV_INLINE bool operator<(const Dual& a, double b) { return a.v < b; }
CFDV_HD CFDV_INLINE bool operator<=(const Dual& a, double b) { return a.v <= b; }
CFDV_HD CFDV_INLINE bool operator>(const Dual& a, double b) { return a.v > b; }
CFDV_HD CFDV_INLINE bool operator>=(const Dual& a, double b) { return a.v >= b; }
CFDV_HD CFDV_INLINE bool operator==(const Dual& a, double b) { return a.v == b; }
CFDV_HD CFDV_INLINE bool operator!=(const Dual& a, double b) { return a.v != b; }
CFDV_HD CFDV_INLINE bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
CFDV_HD CFDV_INLINE bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }

CFDV_HD CFDV_INLINE Dual sqrt(const Dual& a) {
  const double s = ::sqrt(a.v);
  return Dual(s, a.d == 0.0 ? 0.0 : a.d / (2.0 * s));
}
CFDV_HD CFDV_INLINE Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
CFDV_HD CFDV_INLINE Dual fmin(const Dual& a, const Dual& b) { return (b.v < a.v) ? b : a; }
CFDV_HD CFDV_INLINE Dual fmax(const Dual& a, const Dual& b) { return (b.v > a.v) ? b : a; }
CFDV_HD CFDV_INLINE Dual fmin(const Dual& a, double b) { return (b < a.v) ? Dual(b) : a; }
CFDV_HD CFDV_INLINE Dual cosh(const Dual& a) { return Dual(::cosh(a.v), a.d * ::sinh(a.v)); }
CFDV_HD CFDV_INLINE Dual sinh(const Dual& a) { return Dual(::sinh(a.v), a.d * ::cosh(a.v)); }
CFDV_HD CFDV_INLINE Dual cos(const Dual& a) { return Dual(::cos(a.v), -a.d * ::sin(a.v)); }
CFDV_HD CFDV_INLINE Dual sin(const Dual& a) { return Dual(::sin(a.v), a.d * ::cos(a.v)); }
// x^p for a constant exponent; the derivative is taken as 0 where x == 0 (s2 = (1 + s1^0.2)/2
// is only reached with s1 == 0 as a constant branch value)
CFDV_HD CFDV_INLINE Dual pow(const Dual& a, double p) {
  const double r = ::pow(a.v, p);
  return Dual(r, (a.d == 0.0 || a.v == 0.0) ? 0.0 : a.d * p * r / a.v);
}

CFDV_HD CFDV_INLINE double value(double a) { return a; }
CFDV_HD CFDV_INLINE double value(const Dual& a) { return a.v; }
CFDV_HD CFDV_INLINE double deriv(double) { return 0.0; }
CFDV_HD CFDV_INLINE double deriv(const Dual& a) { return a.d; }

// ---- non-contracting round-to-nearest operations -------------------------------
#if defined(__CUDA_ARCH__)
CFDV_HD CFDV_INLINE double rn_mul(double a, double b) { return __dmul_rn(a, b); }
CFDV_HD CFDV_INLINE double rn_add(double a, double b) { return __dadd_rn(a, b); }
CFDV_HD CFDV_INLINE double rn_sub(double a, double b) { return __dsub_rn(a, b); }
CFDV_HD CFDV_INLINE double rn_div(double a, double b) { return __ddiv_rn(a, b); }
#else
// host: separate calls so that no host compiler setting can fuse them either
__attribute__((noinline)) inline double rn_mul(double a, double b) { return a * b; }
__attribute__((noinline)) inline double rn_add(double a, double b) { return a + b; }
__attribute__((noinline)) inline double rn_sub(double a, double b) { return a - b; }
__attribute__((noinline)) inline double rn_div(double a, double b) { return a / b; }
#endif
CFDV_HD CFDV_INLINE Dual rn_mul(const Dual& a, const Dual& b) { return Dual(rn_mul(a.v, b.v), a.d * b.v + a.v * b.d); }
CFDV_HD CFDV_INLINE Dual rn_add(const Dual& a, const Dual& b) { return Dual(rn_add(a.v, b.v), a.d + b.d); }
CFDV_HD CFDV_INLINE Dual rn_sub(const Dual& a, const Dual& b) { return Dual(rn_sub(a.v, b.v), a.d - b.d); }
CFDV_HD CFDV_INLINE Dual rn_div(const Dual& a, const Dual& b) {
  const double q = rn_div(a.v, b.v);
  return Dual(q, (a.d - q * b.d) / b.v);
}
CFDV_HD CFDV_INLINE Dual rn_mul(double a, const Dual& b) { return rn_mul(Dual(a), b); }
CFDV_HD CFDV_INLINE Dual rn_mul(const Dual& a, double b) { return rn_mul(a, Dual(b)); }
CFDV_HD CFDV_INLINE Dual rn_add(double a, const Dual& b) { return rn_add(Dual(a), b); }
CFDV_HD CFDV_INLINE Dual rn_add(const Dual& a, double b) { return rn_add(a, Dual(b)); }
CFDV_HD CFDV_INLINE Dual rn_sub(double a, const Dual& b) { return rn_sub(Dual(a), b); }
CFDV_HD CFDV_INLINE Dual rn_sub(const Dual& a, double b) { return rn_sub(a, Dual(b)); }
CFDV_HD CFDV_INLINE Dual rn_div(double a, const Dual& b) { return rn_div(Dual(a), b); }
CFDV_HD CFDV_INLINE Dual rn_div(const Dual& a, double b) { return rn_div(a, Dual(b)); }

}  // namespace cfdv
