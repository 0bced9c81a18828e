// Forward-mode dual numbers for the oracle's tangent-linear model (test
// infrastructure only).  The value part is computed with exactly the
// operations of the plain FP64 restatement, so a dual run follows the same
// branches (limiters, upwind choices, remap cases) as the FP64 run: the
// derivative is that of the branch-frozen algorithm, the definition the
// hand-written adjoint of the CUDA library implements.
//
// Conventions at non-differentiable points (shared with the adjoint):
// d|x|/dx = 0 at x = 0; d copysign(a, b)/da = sgn(a) * (sign of b);
// min/max pass the derivative of the argument they return.
#pragma once

#include <cmath>

struct Dual {
  double v = 0., d = 0.;
  Dual() = default;
  Dual(double x) : v(x), d(0.) {}  // NOLINT: constants and plain values promote
  Dual(double x, double dx) : v(x), d(dx) {}
};

inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) {
  double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator+(const Dual& a) { return a; }
inline Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
inline Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
inline Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
inline Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
inline Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
inline Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
inline Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
inline Dual operator/(double a, const Dual& b) {
  double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator<(const Dual& a, double b) { return a.v < b; }
inline bool operator>(const Dual& a, double b) { return a.v > b; }
inline bool operator<=(const Dual& a, double b) { return a.v <= b; }
inline bool operator>=(const Dual& a, double b) { return a.v >= b; }
inline bool operator<(double a, const Dual& b) { return a < b.v; }
inline bool operator>(double a, const Dual& b) { return a > b.v; }
inline bool operator<=(double a, const Dual& b) { return a <= b.v; }
inline bool operator>=(double a, const Dual& b) { return a >= b.v; }

inline double value_of(double x) { return x; }
inline double value_of(const Dual& x) { return x.v; }

inline double fabs_(double x) { return std::fabs(x); }
inline Dual fabs_(const Dual& x) {
  double s = x.v > 0. ? 1. : (x.v < 0. ? -1. : 0.);
  return Dual(std::fabs(x.v), s * x.d);
}
inline double copysign_(double a, double b) { return std::copysign(a, b); }
inline Dual copysign_(const Dual& a, const Dual& b) {
  double sa = a.v > 0. ? 1. : (a.v < 0. ? -1. : 0.);
  double sb = std::signbit(b.v) ? -1. : 1.;
  return Dual(std::copysign(a.v, b.v), sa * sb * a.d);
}
inline bool isfinite_(double x) { return std::isfinite(x); }
inline bool isfinite_(const Dual& x) { return std::isfinite(x.v); }
