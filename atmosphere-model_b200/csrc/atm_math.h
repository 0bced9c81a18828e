// Portable natural logarithm, exponential and power for host and device.
//
// The dynamical core evaluates plev**kappa and log(pkap ratio) millions of
// times per step (src/mod_sw_dyn.f90:91,101,282,436,459,612;
// src/mod_remap.f90:46-70).  CUDA's and the host C library's pow/log are
// different approximations, so a GPU run and a CPU run of the same FP64
// program would drift apart by an ulp here and there.  These routines use
// only IEEE-754 double additions, multiplications and correctly rounded
// fused multiply-adds, in a fixed order, so that host code compiled with
// -ffp-contract=off and device code compiled with --fmad=false return
// bit-identical results.
//
// Method: table-driven reduction after P. T. P. Tang (ACM TOMS 15(2) 1989
// for exp, 16(4) 1990 for log).  log(x) = e*ln2 + log(F) + log1p(r) with
// F = i/128 nearest the mantissa m in [sqrt2/2, sqrt2) and r = m/F - 1
// (|r| < 2^-7.4), carried as a double-double; exp(t) = 2^m * 2^(j/32) *
// exp(r) with |r| <= ln2/64.  Tables come from gen_math_tables.py.  The
// error of atm_pow is about 0.52 ulp, the same class as glibc's pow.
#pragma once

#include <stdint.h>
#include "atm_math_tables.h"

#include <cmath>
#include <cstring>
#ifdef __CUDACC__
#define ATM_HD __host__ __device__ __forceinline__
#else
#define ATM_HD inline
#endif

namespace atm_math {

#ifdef __CUDACC__
static __device__ const double d_log_invf[ATM_LOG_TAB_SIZE] = {ATM_LOG_INVF_VALUES};
static __device__ const double d_log_hi[ATM_LOG_TAB_SIZE] = {ATM_LOG_TAB_HI_VALUES};
static __device__ const double d_log_lo[ATM_LOG_TAB_SIZE] = {ATM_LOG_TAB_LO_VALUES};
static __device__ const double d_exp_hi[32] = {ATM_EXP_TAB_HI_VALUES};
static __device__ const double d_exp_lo[32] = {ATM_EXP_TAB_LO_VALUES};
#endif
static const double h_log_invf[ATM_LOG_TAB_SIZE] = {ATM_LOG_INVF_VALUES};
static const double h_log_hi[ATM_LOG_TAB_SIZE] = {ATM_LOG_TAB_HI_VALUES};
static const double h_log_lo[ATM_LOG_TAB_SIZE] = {ATM_LOG_TAB_LO_VALUES};
static const double h_exp_hi[32] = {ATM_EXP_TAB_HI_VALUES};
static const double h_exp_lo[32] = {ATM_EXP_TAB_LO_VALUES};

#ifdef __CUDA_ARCH__
#define ATM_TAB(name, i) __ldg(&d_##name[i])
#else
#define ATM_TAB(name, i) h_##name[i]
#endif

ATM_HD double fma_rn(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

ATM_HD int64_t as_bits(double x) {
#ifdef __CUDA_ARCH__
  return __double_as_longlong(x);
#else
  int64_t b;
  std::memcpy(&b, &x, sizeof b);
  return b;
#endif
}

ATM_HD double from_bits(int64_t b) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(b);
#else
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
#endif
}

ATM_HD void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

ATM_HD void fast_two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  e = b - (s - a);
}

ATM_HD void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = fma_rn(a, b, -p);
}

// log(x) = hi + lo for finite x > 0 (|lo| <= ulp(hi)/2)
ATM_HD void log_dd(double x, double& hi, double& lo) {
  int64_t bits = as_bits(x);
  int ex = (int)((bits >> 52) & 0x7ff);
  int adj = 0;
  if (ex == 0) {  // subnormal: scale into the normal range
    x = x * 0x1p54;
    bits = as_bits(x);
    ex = (int)((bits >> 52) & 0x7ff);
    adj = -54;
  }
  int e = ex - 1023 + adj;
  double m = from_bits((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
  if (m >= 0x1.6a09e667f3bcdp+0) {
    m = m * 0.5;
    e += 1;
  }
  int i = (int)(m * 128.0 + 0.5) - ATM_LOG_TAB_FIRST;
  double invf = ATM_TAB(log_invf, i);
  // r + rl = m*invf - 1 exactly (p - 1 is exact since p is within [1/2, 2])
  double pm, pe, r, rl;
  two_prod(m, invf, pm, pe);
  two_sum(pm - 1.0, pe, r, rl);
  double q = r * r *
             (ATM_LOG_C2 +
              r * (ATM_LOG_C3 +
                   r * (ATM_LOG_C4 + r * (ATM_LOG_C5 + r * (ATM_LOG_C6 + r * (ATM_LOG_C7 + r * (ATM_LOG_C8 + r * ATM_LOG_C9)))))));
  double ed = (double)e;
  double s, t, s2, t2;
  two_sum(ed * ATM_LN2_HI, ATM_TAB(log_hi, i), s, t);
  t = t + (ed * ATM_LN2_LO + ATM_TAB(log_lo, i));
  two_sum(s, r, s2, t2);
  t = t + t2;
  t = t + (rl + q);
  fast_two_sum(s2, t, hi, lo);
}

// exp(th + tl) for |th| < 700
ATM_HD double exp_dd(double th, double tl) {
  const double shift = 0x1.8p52;
  double kd = th * ATM_EXP_INV_L + shift;
  double nd = kd - shift;
  int n = (int)nd;
  int j = n & 31;
  int m = (n - j) / 32;
  double r1 = th - nd * ATM_EXP_L1;
  double r2 = tl - nd * ATM_EXP_L2;
  double r = r1 + r2;
  double p = r * r *
             (ATM_EXP_C2 +
              r * (ATM_EXP_C3 + r * (ATM_EXP_C4 + r * (ATM_EXP_C5 + r * (ATM_EXP_C6 + r * (ATM_EXP_C7 + r * ATM_EXP_C8))))));
  double u = r1 + (r2 + p);
  double thi = ATM_TAB(exp_hi, j), tlo = ATM_TAB(exp_lo, j);
  double c = thi * u + (tlo + tlo * u);
  double res = thi + c;
  // scale by 2^m in two exact steps so that |m| up to ~1040 stays finite
  int m1 = m / 2, m2 = m - m1;
  res = res * from_bits((int64_t)(m1 + 1023) << 52);
  return res * from_bits((int64_t)(m2 + 1023) << 52);
}

}  // namespace atm_math

// log(x), correctly handling 0, negative, infinite and NaN arguments
ATM_HD double atm_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -HUGE_VAL : (x - x) / (x - x);  // -inf or NaN
  if (!(x < HUGE_VAL)) return x;                                     // +inf
  double hi, lo;
  atm_math::log_dd(x, hi, lo);
  return hi;
}

// exp(x): the radiation's transmittances (src/mod_radiation.f90:214,216,
// 300); 0 below the smallest subnormal, +inf above the largest double
ATM_HD double atm_exp(double x) {
  if (x != x) return x;
  if (x > 709.78) return HUGE_VAL;
  if (x < -745.0) return 0.0;
  return atm_math::exp_dd(x, 0.0);
}

// x**y for x > 0 (the only case the dynamical core needs); x == 0 gives
// 0 (y > 0) or +inf (y < 0), negative x gives NaN
ATM_HD double atm_pow(double x, double y) {
  if (!(x > 0.0)) return x == 0.0 ? (y > 0.0 ? 0.0 : HUGE_VAL) : (x - x) / (x - x);
  if (!(x < HUGE_VAL)) return y > 0.0 ? x : 0.0;
  double lh, ll, ph, pl, th, tl;
  atm_math::log_dd(x, lh, ll);
  atm_math::two_prod(y, lh, ph, pl);
  pl = pl + y * ll;
  atm_math::fast_two_sum(ph, pl, th, tl);
  if (th > 709.0) return HUGE_VAL;
  if (th < -745.0) return 0.0;
  return atm_math::exp_dd(th, tl);
}
