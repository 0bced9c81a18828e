// Vector dual numbers for the local Jacobians of the adjoint kernels.
//
// DV<N> carries a value and N partial derivatives.  The value part is
// computed with exactly the operations of the plain double code (the
// translation unit is built without fused multiply-add), so evaluating one
// of the templated sweep functions (slopes, edges_pre, flux_pre,
// flux_con_pre) on DV<N> follows the same branches as the forward sweep and
// returns, next to the forward value, the derivatives with respect to the N
// seeded inputs: the local Jacobian of the branch-frozen function.
//
// Conventions at non-differentiable points: d|x|/dx = 0 at x = 0;
// d copysign(a, b)/da = sgn(a) * (sign of b); min/max pass the derivative of
// the argument they return (the forward's tie rule decides which).
#pragma once

#include "atm_common.cuh"

namespace atm {

template <int N>
struct DV {
  double v;
  double d[N];
  __device__ __forceinline__ DV() {}
  __device__ __forceinline__ DV(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.;
  }
  // x seeded as input number `seed` (0 <= seed < N)
  __device__ __forceinline__ static DV seeded(double x, int seed) {
    DV r(x);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (i == seed) ? 1. : 0.;
    return r;
  }
};

template <int N> __device__ __forceinline__ DV<N> operator+(const DV<N>& a, const DV<N>& b) {
  DV<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N> __device__ __forceinline__ DV<N> operator-(const DV<N>& a, const DV<N>& b) {
  DV<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N> __device__ __forceinline__ DV<N> operator-(const DV<N>& a) {
  DV<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N> __device__ __forceinline__ DV<N> operator+(const DV<N>& a) { return a; }
template <int N> __device__ __forceinline__ DV<N> operator*(const DV<N>& a, const DV<N>& b) {
  DV<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N> __device__ __forceinline__ DV<N> operator/(const DV<N>& a, const DV<N>& b) {
  DV<N> r;
  r.v = a.v / b.v;
  const double rb = 1. / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * rb;
  return r;
}
template <int N> __device__ __forceinline__ bool operator<(const DV<N>& a, const DV<N>& b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ bool operator>(const DV<N>& a, const DV<N>& b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<=(const DV<N>& a, const DV<N>& b) { return a.v <= b.v; }
template <int N> __device__ __forceinline__ bool operator>=(const DV<N>& a, const DV<N>& b) { return a.v >= b.v; }

template <int N> __device__ __forceinline__ DV<N> fab(const DV<N>& a) {
  const double s = a.v > 0. ? 1. : (a.v < 0. ? -1. : 0.);
  DV<N> r;
  r.v = fabs(a.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N> __device__ __forceinline__ DV<N> cpsign(const DV<N>& a, const DV<N>& b) {
  const double sa = a.v > 0. ? 1. : (a.v < 0. ? -1. : 0.);
  const double s = signbit(b.v) ? -sa : sa;
  DV<N> r;
  r.v = copysign(a.v, b.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int B, int N> __device__ __forceinline__ DV<N> div_const(const DV<N>& x) {
  DV<N> r;
  r.v = div_const<B>(x.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = x.d[i] / (double)B;
  return r;
}

}  // namespace atm
