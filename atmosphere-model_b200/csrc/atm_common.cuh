// Shared device definitions of the B200 dynamical core: field geometry in
// HBM, physical constants, and the one-dimensional flux-form
// semi-Lagrangian flux with its PPM reconstruction.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "atm_math.h"

namespace atm {

// Halo width of every stored field, src/mod_tiles.f90:12.
constexpr int H = 7;
// Leading pad of each row so that interior column i = 0 starts 64 bytes
// into a 256-byte-aligned row for FP64 (32 bytes for FP32).
constexpr int XOFF = 1;

// src/mod_constants.f90:8-14; R_dry is a default-real (FP32) literal.
constexpr double R_DRY = (double)287.052874f;
constexpr double CP_DRY = 1005.0;
constexpr double CV_DRY = CP_DRY - R_DRY;
constexpr double KAPPA = R_DRY / CP_DRY;
// Default-real constant expressions of src/mod_sw_dyn.f90:933-953 and
// src/mod_remap.f90:86-100,243.
constexpr double C7_12 = (double)(7.0f / 12.0f);
constexpr double C1_12 = (double)(1.0f / 12.0f);
constexpr double C9_32 = (double)(9.0f / 32.0f);
constexpr double C1_32 = (double)(1.0f / 32.0f);
constexpr double C2_3 = (double)(2.0f / 3.0f);

// Flux variants, src/mod_sw_dyn.f90:73-76.
enum { PC = 0, PPM_UNC = 1, PPM_CON = 2, PPM_NN = 3 };

// Layout of one field in HBM: nlev levels of (ny + 2H) rows of pitch P
// elements; element (i, j, k) of the reference's (is:ie, js:je, 1:K) array
// with i = isd + ii, j = jsd + jj lives at ((k-1)*NYP + jj + H)*P + ii + H + XOFF.
// ii, jj run over [-H, n + H).
struct Geom {
  int nx, ny, L;
  int P;       // row pitch, elements
  int NYP;     // rows per level = ny + 2H
  long long S; // level stride = P * NYP
  __host__ __device__ long long at(int i, int j) const { return (long long)(j + H) * P + (i + H + XOFF); }
  __host__ __device__ long long at(int i, int j, int k) const { return (long long)k * S + at(i, j); }
};

// Constants of init_sw_dyn (src/mod_sw_dyn.f90:961-1021) and the step.
struct Consts {
  double rdx, rdy, rdx2, rdy2, rdx2rdy2, rA;
  double vdx, vdy;        // vortdamp_xcoeff, vortdamp_ycoeff
  double divdamp;         // divdamp_coeff = (c_div dx dy)^2
  double coriolis, gravity;
  double ptop, pk_top;    // Ak(1) and Ak(1)**kappa
  double dt, dtdx, dtdy;  // per call: dtdx = dt*rdx, dtdy = dt*rdy
};

// Status words shared by every kernel of a context.
struct Status {
  int nonfinite_step;   // a non-finite prognostic value left the D-grid step
  int nonfinite_remap;  // ... or the vertical remap
  int nonfinite_check;  // standalone stability check
  int fallback_pairs;   // columns whose remap used the all-pairs search
  int tma_timeout;      // a TMA tile load did not complete within its wait limit
  int radiation_range;  // a radiation table lookup left its table
};

// Hybrid coordinate of the vertical remap (src/mod_remap.f90:57-71).
struct RemapArgs {
  const double* ak;  // device, nlay+1 entries (k = 1..nlay+1 at index k-1)
  const double* bk;
  double ptop, pk_top;
};

// std::min/std::max semantics (return the first argument on ties), so that
// signed zeros behave exactly as in the host restatement.
template <typename T> __device__ __forceinline__ T mn(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T mx(T a, T b) { return (a < b) ? b : a; }
template <typename T> __device__ __forceinline__ T mn3(T a, T b, T c) { return mn(mn(a, b), c); }
template <typename T> __device__ __forceinline__ T mx3(T a, T b, T c) { return mx(mx(a, b), c); }
__device__ __forceinline__ double cpsign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float cpsign(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double fab(double a) { return fabs(a); }
__device__ __forceinline__ float fab(float a) { return fabsf(a); }

// Division by the constants 3 and 12 of the PPM formulas
// (src/mod_sw_dyn.f90:878-879,899), correctly rounded like an IEEE
// division: q = x*RN(1/b) is within one ulp of x/b, the remainder
// r = x - q*b is exact in one FMA, and RN(q + r*RN(1/b)) is the correctly
// rounded quotient (P. Markstein, IBM J. Res. Dev. 34(1), 1990).  Zeros,
// infinities, NaN and magnitudes near the ends of the exponent range take
// the IEEE division.
static __device__ __noinline__ double div_ieee(double x, double b) { return x / b; }
template <int B> __device__ __forceinline__ double div_const(double x) {
  constexpr double r = 1.0 / B;  // RN(1/B)
  double a = fabs(x);
  if (!(a > 0x1p-960 && a < 0x1p1000)) return div_ieee(x, (double)B);
  double q = x * r;
  double e = __fma_rn(-q, (double)B, x);
  return __fma_rn(e, r, q);
}
// The mixed form's FP32 sweeps need no correctly rounded quotient: a
// multiplication by the rounded reciprocal.
template <int B> __device__ __forceinline__ float div_const(float x) { return x * (1.0f / B); }

// Monotone slope dqi_mono(i) and raw slope dqi(i) of src/mod_sw_dyn.f90:870-875
// from q(i-1), q(i), q(i+1).
template <typename T>
__device__ __forceinline__ void slopes(T qm, T q0, T qp, T& dqi, T& mono) {
  dqi = (qp - qm) * T(0.25);
  T dmax = mx3(qp, q0, qm) - q0;
  T dmin = q0 - mn3(qp, q0, qm);
  mono = cpsign(mn3(fab(dqi), dmin, dmax), dqi);
}

// Edge anomalies edge_L(i), edge_R(i) of cell i, src/mod_sw_dyn.f90:877-911.
// q points at cell i; s is the distance between neighbouring cells.
template <typename T, int V>
__device__ __forceinline__ void edges(const T* q, int s, T& eL, T& eR) {
  T qm2 = q[-2 * s], qm1 = q[-s], q0 = q[0], qp1 = q[s], qp2 = q[2 * s];
  T d_m, mono_m, d_0, mono_0, d_p, mono_p;
  slopes(qm2, qm1, q0, d_m, mono_m);
  slopes(qm1, q0, qp1, d_0, mono_0);
  slopes(q0, qp1, qp2, d_p, mono_p);
  eL = (qm1 - q0) * T(0.5) + div_const<3>(mono_m - mono_0);
  eR = (qp1 - q0) * T(0.5) + div_const<3>(mono_0 - mono_p);
  if (V == PPM_CON || V == PPM_NN) {
    T lim = T(2) * fab(d_0);
    eL = -cpsign(mn(lim, fab(eL)), d_0);
    eR = +cpsign(mn(lim, fab(eR)), d_0);
    if (V == PPM_NN) {
      eL = mx(eL, -q0);
      eR = mx(eR, -q0);
      T a = eR - eL;
      T b = T(-3) * (eR + eL);
      if ((fab(a) < -b) && (q0 + a * a / (T(4) * b) + div_const<12>(b) < T(0))) {
        if (eL * eR > T(0)) {
          eL = T(0);
          eR = T(0);
        } else if (eL > eR) {
          eL = T(2) * fab(eR);
        } else {
          eR = T(2) * fab(eL);
        }
      }
    }
  }
}

// Upwind flux at the interface between cells i-1 and i (src/mod_sw_dyn.f90:
// 802-838).  q points at cell i, s is the cell spacing in the array, c is the
// Courant number of the interface.  Reads q[-3s .. 2s].
template <typename T, int V>
__device__ __forceinline__ T flux(const T* q, int s, T c) {
  if (V == PC) return (c > T(0)) ? q[-s] : q[0];
  T sa = fab(c);
  T k1 = (T(1) - T(2) * sa) * (T(1) - sa);
  T k2 = sa * (sa - T(1));
  if (V == PPM_CON) {
    T eLm, eRm, eL0, eR0;
    edges<T, V>(q - s, s, eLm, eRm);
    edges<T, V>(q, s, eL0, eR0);
    if ((T(3) * fab(eL0 + eR0) > fab(eL0 - eR0)) && (T(3) * fab(eLm + eRm) > fab(eLm - eRm)))
      return (c > T(0)) ? q[-s] : q[0];
    if (c > T(0)) return q[-s] + k1 * eRm + k2 * eLm;
    return q[0] + k1 * eL0 + k2 * eR0;
  }
  T eL, eR;
  if (c > T(0)) {
    edges<T, V>(q - s, s, eL, eR);
    return q[-s] + k1 * eR + k2 * eL;
  }
  edges<T, V>(q, s, eL, eR);
  return q[0] + k1 * eL + k2 * eR;
}

// A window of a 2-D shared-memory array addressed with absolute interior
// coordinates (x, y) of the tile's region [x0, x0+w) x [y0, y0+h).
template <typename T>
struct Sm {
  T* p;
  int x0, y0, w;
  __device__ __forceinline__ T& operator()(int x, int y) const { return p[(y - y0) * w + (x - x0)]; }
  __device__ __forceinline__ T* ptr(int x, int y) const { return p + (y - y0) * w + (x - x0); }
};

}  // namespace atm
