// Kernels of the B200 dynamical core, templated on the sweep type T
// (double for the FP64 form, float for the mixed form).  Column sums,
// pkap, gz and the vertical remap always run in double.
//
// Every per-layer kernel processes one TX x TY tile of one layer: it stages
// the tile plus the stencil halo of its inputs in shared memory, runs the
// stages of the reference's layer loop on that tile, and writes its outputs.
// Index ranges, staggering shifts and evaluation order follow the
// reference line by line (cited per stage).
#pragma once

#include <type_traits>

#include "atm_common.cuh"
#include "atm_kappa_tables.h"

namespace atm {

constexpr int NT = 256;  // threads per block of the per-layer kernels

// ---------------------------------------------------------------- loads ----
// s[(y - y0) * w + (x - x0)] = field(x, y, k) for the box [x0, x0+w) x
// [y0, y0+h); points outside the stored (halo-padded) array read as zero and
// only ever feed outputs outside the kernel's output region.
template <typename T>
__device__ __forceinline__ void load_box(T* s, const T* __restrict__ f, const Geom& g, int k, int x0, int y0, int w,
                                         int h) {
  const T* base = f + (long long)k * g.S;
  for (int idx = threadIdx.x; idx < w * h; idx += blockDim.x) {
    int y = idx / w, x = idx - y * w;
    int gx = x0 + x, gy = y0 + y;
    T v = T(0);
    if (gx >= -H && gx < g.nx + H && gy >= -H && gy < g.ny + H) v = base[g.at(gx, gy)];
    s[idx] = v;
  }
}

template <typename T>
__device__ __forceinline__ Sm<T> carve(unsigned char*& p, int x0, int y0, int w, int h) {
  Sm<T> s{reinterpret_cast<T*>(p), x0, y0, w};
  p += ((size_t)w * h * sizeof(T) + 15) & ~(size_t)15;
  return s;
}
template <typename T>
__host__ __device__ constexpr size_t box_bytes(int w, int h) {
  return ((size_t)w * h * sizeof(T) + 15) & ~(size_t)15;
}

// Raise a context's non-finite flag (bad values are rare: one atomic each).
__device__ __forceinline__ void flag_nonfinite(int* flag, bool bad) {
  if (bad) atomicOr(flag, 1);
}
__device__ __forceinline__ bool finite_(double v) { return isfinite(v); }
__device__ __forceinline__ bool finite_(float v) { return isfinite(v); }

// ====================================================== column pressure ====
// plev = ptop + suffix sum of dp from the model top, pkap = plev**kappa,
// hydrostatic gz from the bottom (src/mod_sw_dyn.f90:276-292 and 606-626).
// One thread per column over [lo, n-1+hi]^2.  The downward pass writes
// pkap; the upward pass reads it back (from L2: a block's columns were just
// written), so no shared memory limits the occupancy.  Both passes load
// eight levels at a time before using them, so that a thread keeps eight
// loads in flight (the persistent ensemble kernel runs this at a quarter of
// the column kernel's occupancy) and the eight pow calls of a batch,
// independent once the running sum is formed, overlap.
// plev**kappa and the log of a pkap ratio in the column and remap kernels.
// PortablePow is atm_math.h's (bit-identical on host and device: the FP64
// form and its oracle).  DevicePow serves the mixed form, whose error is its
// FP32 sweeps': p**kappa = 2^(kappa e) F_j**kappa (1 + r)**kappa from the
// tables of atm_kappa_tables.h and a degree-7 binomial series (within 3 ulp;
// outside p in [2^-126, 2^128) the device library's exp(kappa log p)) and the
// device library's log.  Measured at 1024x1024x64: a column pass 0.63 ms
// with the portable pow, 0.45 with exp(kappa log p).
struct PortablePow {
  __device__ static double kappa(double x) { return atm_pow(x, KAPPA); }
  __device__ static double log(double x) { return atm_log(x); }
};
static_assert(KAPPA == ATM_KAP_KAPPA, "atm_kappa_tables.h was generated for another kappa");
static __device__ const double d_kap_e[] = {ATM_KAP_E_VALUES};
static __device__ const double d_kap_f[] = {ATM_KAP_F_VALUES};
static __device__ const double d_kap_invf[] = {ATM_KAP_INVF_VALUES};
struct DevicePow {
  __device__ static double kappa(double x) {
    const long long b = __double_as_longlong(x);
    const int e = (int)((b >> 52) & 0x7ff) - 1023;
    if (b < 0 || e < ATM_KAP_E_FIRST || e > ATM_KAP_E_LAST) return ::exp(KAPPA * ::log(x));
    const int j = (int)((b >> 45) & 127);
    const double m = __longlong_as_double((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    const double r = m * __ldg(d_kap_invf + j) - 1.0;
    double q = ::fma(r, ATM_KAP_C7, ATM_KAP_C6);
    q = ::fma(r, q, ATM_KAP_C5);
    q = ::fma(r, q, ATM_KAP_C4);
    q = ::fma(r, q, ATM_KAP_C3);
    q = ::fma(r, q, ATM_KAP_C2);
    q = ::fma(r, q, ATM_KAP_C1);
    const double t = __ldg(d_kap_e + (e - ATM_KAP_E_FIRST)) * __ldg(d_kap_f + j);
    return ::fma(t, q * r, t);
  }
  __device__ static double log(double x) { return ::log(x); }
};
// the one a form with sweep type T uses
template <typename T>
using FormPow = std::conditional_t<std::is_same_v<T, double>, PortablePow, DevicePow>;

template <typename T, typename PW = PortablePow>
__device__ __forceinline__ void column_at(const Geom& g, const Consts& c, const T* dpl, const T* ptl, double* pkap,
                                          double* gz, int lo, int hi, double* plev_out, int col) {
  constexpr int B = 8;  // levels whose loads are in flight together
  const int w = g.nx - lo + hi;
  const int hgt = g.ny - lo + hi;
  if (col >= w * hgt) return;
  const int x = lo + col % w, y = lo + col / w;
  const long long o = g.at(x, y);
  const long long S = g.S;
  const int L = g.L;
  double plev = c.ptop;
  if (plev_out) plev_out[o + (long long)L * S] = plev;
  for (int k0 = L - 1; k0 >= 0; k0 -= B) {
    T dv[B];
#pragma unroll
    for (int u = 0; u < B; ++u) dv[u] = k0 - u >= 0 ? dpl[o + (long long)(k0 - u) * S] : T(0);
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int k = k0 - u;
      if (k < 0) break;
      plev = plev + (double)dv[u];
      if (plev_out) plev_out[o + (long long)k * S] = plev;
      pkap[o + (long long)k * S] = PW::kappa(plev);
    }
  }
  double z = gz[o];
  double pk0 = pkap[o];
  for (int k0 = 0; k0 < L; k0 += B) {
    double pk[B];
    T pv[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int k = k0 + u;
      pk[u] = k + 1 < L ? pkap[o + (long long)(k + 1) * S] : c.pk_top;
      pv[u] = k < L ? ptl[o + (long long)k * S] : T(0);
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int k = k0 + u;
      if (k >= L) break;
      z = z + CP_DRY * (double)pv[u] * (pk0 - pk[u]);
      gz[o + (long long)(k + 1) * S] = z;
      pk0 = pk[u];
    }
  }
}

template <typename T, typename PW = PortablePow>
__global__ void __launch_bounds__(128) k_column(Geom g, Consts c, const T* __restrict__ dpl, const T* __restrict__ ptl,
                                                double* __restrict__ pkap, double* __restrict__ gz, int lo, int hi,
                                                double* __restrict__ plev_out) {
  column_at<T, PW>(g, c, dpl, ptl, pkap, gz, lo, hi, plev_out, blockIdx.x * blockDim.x + threadIdx.x);
}

// Heating rate of the layer from the radiative net flux,
// src/mod_sw_dyn.f90:89-106 (C) and 433-464 (D): pkap from dp (C step) or
// dpc (D step) over the whole padded domain, playkap, then
// heat = (nf(k+1) - nf(k)) / (cp dp / g) / playkap.
template <typename T>
__global__ void __launch_bounds__(64) k_heating(Geom g, Consts c, const T* __restrict__ dpl,
                                                const double* __restrict__ nf, double* __restrict__ heat) {
  const int w = g.nx + 2 * H;
  const int col = blockIdx.x * 64 + threadIdx.x;
  if (col >= w * g.NYP) return;
  const int x = -H + col % w, y = -H + col / w;
  const long long o = g.at(x, y);
  const int L = g.L;
  double plev = c.ptop, pk_up = c.pk_top;
  for (int k = L - 1; k >= 0; --k) {
    long long ok = o + (long long)k * g.S;
    double d = (double)dpl[ok];
    plev = plev + d;
    double pk = atm_pow(plev, KAPPA);
    double playkap = (pk_up - pk) / atm_log(pk_up / pk);
    heat[ok] = (nf[ok + g.S] - nf[ok]) / (CP_DRY * d / c.gravity) / playkap;
    pk_up = pk;
  }
}

// ============================================================= corners ====
// interpolate_to_corners (src/mod_sw_dyn.f90:921-956) of pkap (levels
// 1..L -> pkapb) and gz (levels 2..L+1 -> gzb) on [0, nx] x [0, ny]; the
// first level of gzb is done once at set-up (level0 = 0, nlev = 1).
__device__ __forceinline__ double tx_(const double* q, long long o, int P) {
  return C7_12 * (q[o] + q[o - 1]) - C1_12 * (q[o + 1] + q[o - 2]);
}
__device__ __forceinline__ double ty_(const double* q, long long o, int P) {
  return C7_12 * (q[o] + q[o - P]) - C1_12 * (q[o + P] + q[o - 2 * P]);
}
__device__ __forceinline__ double corner(const double* q, long long o, int P) {
  double out = C9_32 * (tx_(q, o, P) + tx_(q, o - P, P)) - C1_32 * (tx_(q, o + P, P) + tx_(q, o - 2 * P, P));
  out = out + C9_32 * (ty_(q, o, P) + ty_(q, o - 1, P)) - C1_32 * (ty_(q, o + 1, P) + ty_(q, o - 2, P));
  return out;
}

// B levels' loads are issued before their stores: 1 in the corner kernel
// (measured fastest there), 4 in the persistent ensemble kernel, whose
// pointers carry no no-alias promise and which runs at lower occupancy.
template <int B = 1>
__device__ __forceinline__ void corner_at(const Geom& g, const double* pkap, const double* gz, double* pkapb,
                                          double* gzb, int with_pkap, int lev0, int nlev, int idx) {
  const int w = g.nx + 1, h = g.ny + 1;
  if (idx >= w * h) return;
  const int x = idx % w, y = idx / w;
  for (int l0 = lev0; l0 < lev0 + nlev; l0 += B) {
    double pb[B], zb[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int l = l0 + u;
      if (l >= lev0 + nlev) break;
      if (with_pkap) pb[u] = corner(pkap, g.at(x, y, l), g.P);
      zb[u] = corner(gz, g.at(x, y, l + (with_pkap ? 1 : 0)), g.P);
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int l = l0 + u;
      if (l >= lev0 + nlev) break;
      if (with_pkap) pkapb[g.at(x, y, l)] = pb[u];
      gzb[g.at(x, y, l + (with_pkap ? 1 : 0))] = zb[u];
    }
  }
}

// blockIdx.y selects a chunk of `chunk` levels (8: 0.67 ms at 1024x1024x64,
// against 0.72 / 0.67 / 0.68 / 0.73 at 1 / 4 / 16 / 64), so that more threads share
// the levels' independent loads
static __global__ void k_corners(Geom g, const double* __restrict__ pkap, const double* __restrict__ gz,
                          double* __restrict__ pkapb, double* __restrict__ gzb, int with_pkap, int lev0, int nlev,
                          int chunk) {
  const int l0 = lev0 + blockIdx.y * chunk;
  const int n = min(chunk, lev0 + nlev - l0);
  if (n > 0) corner_at(g, pkap, gz, pkapb, gzb, with_pkap, l0, n, blockIdx.x * blockDim.x + threadIdx.x);
}

// =============================================================== halos ====
// Periodic fill of the 7-wide ring (the single-image halo_exchange,
// src/mod_sync.f90:67-217): every ring point takes the value of its
// periodic image in the interior.  With copy = true the ring of src is
// copied to dst instead (the ring of a new time level keeps the old ring).
// ring point idx of level k of one field f (src: the copy's source)
// Ring point idx (the halo bands of ring_at) of a level: its (x, y); false
// past the ring.
__device__ __forceinline__ bool ring_xy(const Geom& g, int idx, int& x, int& y) {
  const int wide = g.nx + 2 * H;
  const int nband = 2 * H * wide;
  const int nring = nband + 2 * H * g.ny;
  if (idx >= nring) return false;
  if (idx < nband) {
    const int r = idx / wide;
    y = r < H ? r - H : g.ny + (r - H);
    x = idx % wide - H;
  } else {
    const int q = idx - nband;
    y = q / (2 * H);
    const int cc = q % (2 * H);
    x = cc < H ? cc - H : g.nx + (cc - H);
  }
  return true;
}

template <typename T, bool COPY>
__device__ __forceinline__ void ring_at(const Geom& g, T* f, const T* s, int idx, int k) {
  int x, y;
  if (!ring_xy(g, idx, x, y)) return;
  long long o = g.at(x, y, k);
  if (COPY) {
    f[o] = s[o];
  } else {
    int xs = x < 0 ? x + g.nx : (x >= g.nx ? x - g.nx : x);
    int ys = y < 0 ? y + g.ny : (y >= g.ny ? y - g.ny : y);
    f[o] = f[g.at(xs, ys, k)];
  }
}

// R ring points idx0, idx0 + 32, ... of a level: all loads issued before the
// stores (the ring's sources are interior points, which no store of the
// pass touches)
template <typename T, bool COPY, int R>
__device__ __forceinline__ void ring_batch(const Geom& g, T* f, const T* s, int idx0, int k) {
  T v[R];
  long long od[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    int x, y;
    od[r] = -1;
    v[r] = T(0);
    if (!ring_xy(g, idx0 + 32 * r, x, y)) continue;
    od[r] = g.at(x, y, k);
    if (COPY) {
      v[r] = s[od[r]];
    } else {
      const int xs = x < 0 ? x + g.nx : (x >= g.nx ? x - g.nx : x);
      const int ys = y < 0 ? y + g.ny : (y >= g.ny ? y - g.ny : y);
      v[r] = f[g.at(xs, ys, k)];
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (od[r] >= 0) f[od[r]] = v[r];
}

template <typename T, bool COPY>
__global__ void k_ring(Geom g, T* f0, T* f1, T* f2, T* f3, const T* s0, const T* s1, const T* s2, const T* s3, int K) {
  const int k = blockIdx.y;
  if (k >= K) return;
  const int fld = blockIdx.z;
  T* f = fld == 0 ? f0 : fld == 1 ? f1 : fld == 2 ? f2 : f3;
  const T* s = fld == 0 ? s0 : fld == 1 ? s1 : fld == 2 ? s2 : s3;
  ring_at<T, COPY>(g, f, s, blockIdx.x * blockDim.x + threadIdx.x, k);
}

// ========================================================= vertical remap ==
template <int LM>
struct PPMWork {
  double gam[LM + 2], lv[LM + 2], top[LM + 2], btm[LM + 2], curv[LM + 2];
};

// vertical_ppm, src/mod_remap.f90:287-356; arrays are 1-based.  The test of
// the last interface reads gam(nlay+1), past the end of gam in the
// reference; level_var(nlay) is already clamped to the same bounds at
// :319-320, so both clamps are applied there (any branch leaves it as is).
template <int LM>
__device__ void vertical_ppm(PPMWork<LM>& w, int L, const double* var, const double* coord) {
  double* gam = w.gam;
  double* lv = w.lv;
  double alpha, beta;
  alpha = (coord[L] - coord[L - 1]) / (coord[L + 1] - coord[L]);
  beta = alpha * (.5 + alpha);
  lv[L + 1] = (2. * alpha * (1. + alpha) * var[L] + var[L - 1]) / beta;
  gam[L] = (1. + alpha * (1.5 + alpha)) / beta;
  for (int k = L; k >= 2; --k) {
    alpha = (coord[k + 1] - coord[k]) / (coord[k] - coord[k - 1]);
    beta = 2. + 2. * alpha - gam[k];
    lv[k] = (3. * (var[k] + alpha * var[k - 1]) - lv[k + 1]) / beta;
    gam[k - 1] = alpha / beta;
  }
  beta = 1. + alpha * (1.5 + alpha);
  lv[1] = (2. * alpha * (1. + alpha) * var[1] + var[2] - beta * lv[2]) / (alpha * (.5 + alpha) - beta * gam[1]);
  for (int k = 2; k <= L + 1; ++k) lv[k] = lv[k] - gam[k - 1] * lv[k - 1];
  lv[L] = mn(lv[L], mx(var[L], var[L - 1]));
  lv[L] = mx(lv[L], mn(var[L], var[L - 1]));
  lv[2] = mn(lv[2], mx(var[2], var[1]));
  lv[2] = mx(lv[2], mn(var[2], var[1]));
  for (int k = 2; k <= L - 1; ++k) {
    double lo = mn(var[k], var[k + 1]), hi = mx(var[k], var[k + 1]);
    if (k + 2 > L || gam[k + 2] * gam[k] > 0) {
      lv[k + 1] = mn(lv[k + 1], hi);
      lv[k + 1] = mx(lv[k + 1], lo);
    } else if (gam[k + 2] > 0) {
      lv[k + 1] = mx(lv[k + 1], lo);
    } else {
      lv[k + 1] = mn(lv[k + 1], hi);
    }
  }
  for (int k = 1; k <= L; ++k) {
    w.top[k] = lv[k + 1];
    w.btm[k] = lv[k];
  }
  for (int k = 2; k <= L - 1; ++k) {
    double pmp1 = var[k + 1] - 2. * gam[k];
    double lac1 = pmp1 + 1.5 * gam[k - 1];
    w.top[k + 1] = mn(mx(w.top[k + 1], mn3(var[k + 1], pmp1, lac1)), mx3(var[k + 1], pmp1, lac1));
    pmp1 = var[k + 1] + 2. * gam[k + 1];
    lac1 = pmp1 - 1.5 * gam[k];
    w.btm[k + 1] = mn(mx(w.btm[k + 1], mn3(var[k + 1], pmp1, lac1)), mx3(var[k + 1], pmp1, lac1));
  }
  for (int k = 1; k <= L; ++k) w.curv[k] = 6. * var[k] - 3. * (w.top[k] + w.btm[k]);
}

// Contribution of source layer k (edges btm, top, curvature cv, mean vk,
// coordinates sk = coord(k), sk1 = coord(k+1)) to destination layer m
// (coordinates d0 = coord(m), d1 = coord(m+1)), added to acc: the body of
// the pair loop of src/mod_remap.f90:188-280.  Returns the case tag(s).
__device__ __forceinline__ int pair_add(double& acc, double btm, double top, double cv, double vk, double sk,
                                        double sk1, double d0, double d1) {
  double dsrc = sk1 - sk;
  double s1 = (d0 - sk) / dsrc;
  double s2 = (d1 - sk) / dsrc;
  double integral_factor = dsrc / (d1 - d0);
  int which = 0;
  double tmp3 = 2. * s1 * s1;
  if (d1 <= sk1 && sk1 < d0 && d0 < sk) {
    double tmp1 = s1 - 1., tmp2 = s1 + 1.;
    acc = acc + tmp1 / 6. * (3. * (btm * tmp1 - top * tmp2) + cv * (tmp3 - tmp2)) * integral_factor;
    which = 3;
  }
  if (sk1 < d1 && d1 < sk && sk <= d0) {
    acc = acc + (s2 / 2.) * (btm * (2. - s2) + s2 * (top + cv * (1. - C2_3 * s2))) * integral_factor;
    which = which * 10 + 4;
  }
  if (d1 <= sk1 && sk <= d0) {
    acc = acc + vk * integral_factor;
    which = which * 10 + 5;
  }
  if (sk1 < d1 && d0 < sk) {
    double tmp1 = s1 + s2;
    acc = acc + (s1 - s2) / 6. * (3. * (btm * (tmp1 - 2.) - top * tmp1) + cv * (tmp3 + tmp1 * (2. * s2 - 3.))) *
                    integral_factor;
    which = which * 10 + 6;
  }
  return which;
}

template <int LM>
__device__ __forceinline__ int remap_pair(const PPMWork<LM>& w, const double* src_var, double* dst_var,
                                          const double* sc, const double* dc, int k, int m) {
  return pair_add(dst_var[m], w.btm[k], w.top[k], w.curv[k], src_var[k], sc[k], sc[k + 1], dc[m], dc[m + 1]);
}

// remap_column, src/mod_remap.f90:165-285.  When both coordinates are
// non-increasing the pairs that pass the reference's overlap test are, for
// each destination layer m, a contiguous run of source layers whose ends
// move monotonically with m; they are visited in that order (ascending k
// for each m, the order in which the reference accumulates dst_var(m)).
// Otherwise the reference's all-pairs loop runs.  trace, when non-null,
// receives {first k, last k, case of first, case of last, count} per m.
template <int LM>
__device__ void remap_column(PPMWork<LM>& w, int L, const double* src_var, double* dst_var, const double* sc,
                             const double* dc, int* trace, long long tstride, int* fallback) {
  for (int m = 1; m <= L; ++m) dst_var[m] = 0.;
  vertical_ppm<LM>(w, L, src_var, sc);
  bool mono = true;
  for (int k = 1; k <= L; ++k) mono = mono && (sc[k + 1] <= sc[k]) && (dc[k + 1] <= dc[k]);
  if (trace)
    for (int m = 1; m <= L; ++m) {
      int* t = trace + (long long)(m - 1) * 5 * tstride;
      t[0] = -1; t[tstride] = -1; t[2 * tstride] = -1; t[3 * tstride] = -1; t[4 * tstride] = 0;
    }
  if (mono) {
    int k0 = 1;
    for (int m = 1; m <= L; ++m) {
      while (k0 <= L && sc[k0 + 1] >= dc[m]) ++k0;
      for (int k = k0; k <= L && sc[k] > dc[m + 1]; ++k) {
        int which = remap_pair<LM>(w, src_var, dst_var, sc, dc, k, m);
        if (trace) {
          int* t = trace + (long long)(m - 1) * 5 * tstride;
          if (t[0] < 0) { t[0] = k; t[2 * tstride] = which; }
          t[tstride] = k;
          t[3 * tstride] = which;
          t[4 * tstride] += 1;
        }
      }
    }
  } else {
    if (fallback) atomicAdd(fallback, 1);
    for (int k = 1; k <= L; ++k)
      for (int m = 1; m <= L; ++m) {
        if (sc[k + 1] >= dc[m] || sc[k] <= dc[m + 1]) continue;
        int which = remap_pair<LM>(w, src_var, dst_var, sc, dc, k, m);
        if (trace) {
          int* t = trace + (long long)(m - 1) * 5 * tstride;
          if (t[0] < 0) { t[0] = k; t[2 * tstride] = which; }
          else if (t[tstride] != k - 1) t[4 * tstride] = -1000000;
          t[tstride] = k;
          t[3 * tstride] = which;
          if (t[4 * tstride] >= 0) t[4 * tstride] += 1;
        }
      }
  }
}

// ------------------------------------------------ streaming remap_column --
// vertical_ppm + remap_column (src/mod_remap.f90:165-356) reorganised into
// one descending and one ascending pass over the column, so that a column
// keeps three stored arrays (the source coordinate, the interface values
// before forward substitution, gam) instead of nine:
//  * descending: the elimination of vertical_ppm (:296-309), fed level by
//    level by the producer of the coordinate and of the remapped variable;
//  * ascending: forward substitution (:311-313), boundary and monotonicity
//    clamps (:316-334), the Huynh constraint (:339-352) and the curvature
//    (:354) of layer k, produced when the pair loop (:188-280, visited as a
//    monotone merge, see remap_column) first reaches layer k.
// Every value comes from the same operations in the same order as in
// vertical_ppm/remap_column above, so results and (k, m, case) sets are
// identical; columns whose coordinates are not monotone take the
// all-arrays path.

// One column array, element k at p[k * s].
// A column array of element type E read and written as doubles (k * s
// apart).  The mixed form keeps the PPM interface values and elimination
// coefficients of its wind remap in FP32 (half the local-memory traffic of
// the thread's column arrays); every other column array is FP64.
template <typename E>
struct ColArrT {
  E* p;
  int s;
  struct Ref {
    E* q;
    __device__ __forceinline__ operator double() const { return (double)*q; }
    __device__ __forceinline__ Ref& operator=(double v) {
      *q = (E)v;
      return *this;
    }
  };
  __device__ __forceinline__ Ref operator[](int k) const { return Ref{p + k * s}; }
};
template <>
struct ColArrT<double> {
  double* p;
  int s;
  __device__ __forceinline__ double& operator[](int k) const { return p[k * s]; }
};
using ColArr = ColArrT<double>;

// Elimination sweep of vertical_ppm in descending k.  cnext() yields
// coord(L+1), coord(L), ..., coord(1) and vnext() var(L), ..., var(1), one
// call each in that order.  Stores lv (before forward substitution) for
// levels 1..L+1, gam for 1..L and, with STORE_SC, the coordinate.  L >= 3.
template <bool STORE_SC, typename FC, typename FV, typename LA = ColArr>
__device__ __forceinline__ void ppm_eliminate(int L, FC&& cnext, FV&& vnext, ColArr sc, LA lv, LA gam) {
  double c2 = cnext(), c1 = cnext(), c0 = cnext();  // coord(k+1), coord(k), coord(k-1)
  if (STORE_SC) {
    sc[L + 1] = c2;
    sc[L] = c1;
    sc[L - 1] = c0;
  }
  double v1 = vnext(), v0 = vnext();  // var(k), var(k-1)
  double alpha = (c1 - c0) / (c2 - c1);
  double beta = alpha * (.5 + alpha);
  double lvk = (2. * alpha * (1. + alpha) * v1 + v0) / beta;
  lv[L + 1] = lvk;
  double g = (1. + alpha * (1.5 + alpha)) / beta;
  gam[L] = g;
  for (int k = L; k >= 2; --k) {
    alpha = (c2 - c1) / (c1 - c0);
    beta = 2. + 2. * alpha - g;
    lvk = (3. * (v1 + alpha * v0) - lvk) / beta;
    lv[k] = lvk;
    g = alpha / beta;
    gam[k - 1] = g;
    if (k > 2) {
      c2 = c1;
      c1 = c0;
      c0 = cnext();
      if (STORE_SC) sc[k - 2] = c0;
      v1 = v0;
      v0 = vnext();
    }
  }
  // v1 = var(2), v0 = var(1), lvk = lv(2), g = gam(1)
  beta = 1. + alpha * (1.5 + alpha);
  lv[1] = (2. * alpha * (1. + alpha) * v0 + v1 - beta * lvk) / (alpha * (.5 + alpha) - beta * g);
}

// Layer k's edges and curvature in ascending k from the eliminated column.
template <typename FV, typename LA = ColArr>
struct PPMLayers {
  LA lv, gam;
  int L;
  const FV& var;  // var(k), k = 1..L
  int k;
  double lvf, lvc, vk, vk1, top, btm, curv;
  __device__ __forceinline__ PPMLayers(LA lv_, LA gam_, int L_, const FV& v)
      : lv(lv_), gam(gam_), L(L_), var(v), k(0) {
    lvf = lv[1];
    lvc = lvf;
    vk1 = var(1);
  }
  __device__ __forceinline__ void next() {
    ++k;
    vk = vk1;
    if (k < L) vk1 = var(k + 1);
    const int j = k + 1;  // the level at the top of layer k
    const double f = lv[j] - gam[k] * lvf;
    double c = f;
    if (j == L) {
      c = mn(c, mx(vk1, vk));
      c = mx(c, mn(vk1, vk));
    }
    if (j == 2) {
      c = mn(c, mx(vk1, vk));
      c = mx(c, mn(vk1, vk));
    }
    if (j >= 3 && j <= L) {
      const double lo = mn(vk, vk1), hi = mx(vk, vk1);
      if (j == L || gam[j + 1] * gam[j - 1] > 0) {
        c = mn(c, hi);
        c = mx(c, lo);
      } else if (gam[j + 1] > 0) {
        c = mx(c, lo);
      } else {
        c = mn(c, hi);
      }
    }
    top = c;
    btm = lvc;
    if (k >= 3) {
      const double gk1 = gam[k - 1];
      double pmp1 = vk - 2. * gk1;
      double lac1 = pmp1 + 1.5 * gam[k - 2];
      top = mn(mx(top, mn3(vk, pmp1, lac1)), mx3(vk, pmp1, lac1));
      pmp1 = vk + 2. * gam[k];
      lac1 = pmp1 - 1.5 * gk1;
      btm = mn(mx(btm, mn3(vk, pmp1, lac1)), mx3(vk, pmp1, lac1));
    }
    curv = 6. * vk - 3. * (top + btm);
    lvf = f;
    lvc = c;
  }
};

// The pair loop as a monotone merge over the eliminated column: dst(m) for
// m = 1..L in ascending order goes to put(m, value); dc(m) gives the
// destination coordinate.  trace as in remap_column.
template <typename FV, typename FD, typename FO, typename LA = ColArr>
__device__ __forceinline__ void remap_merge(int L, ColArr sc, LA lv, LA gam, const FV& var, FD&& dc,
                                            FO&& put, int* trace, long long ts) {
  PPMLayers<FV, LA> ly(lv, gam, L, var);
  int k0 = 1;
  double d0 = dc(1);
  for (int m = 1; m <= L; ++m) {
    const double d1 = dc(m + 1);
    while (k0 <= L && sc[k0 + 1] >= d0) ++k0;
    double acc = 0.;
    int first = -1, last = -1, w0 = -1, w1 = -1, cnt = 0;
    for (int k = k0; k <= L; ++k) {
      const double sk = sc[k];
      if (!(sk > d1)) break;
      while (ly.k < k) ly.next();
      const int which = pair_add(acc, ly.btm, ly.top, ly.curv, ly.vk, sk, sc[k + 1], d0, d1);
      if (first < 0) {
        first = k;
        w0 = which;
      }
      last = k;
      w1 = which;
      ++cnt;
    }
    put(m, acc);
    if (trace) {
      int* t = trace + (long long)(m - 1) * 5 * ts;
      t[0] = first;
      t[ts] = last;
      t[2 * ts] = w0;
      t[3 * ts] = w1;
      t[4 * ts] = cnt;
    }
    d0 = d1;
  }
}

// Winds on the cell faces over [isd-1, ied+1]^2, src/mod_remap.f90:80-105.
// The D-grid winds here still carry last step's halo (the remap runs before
// the D-grid halo exchange), exactly as in the reference.  Face column
// (i, j), direction dir (0: u, columns (i, j-2..j+1); 1: v, (i-2..i+1, j)).
// The all-arrays form, for columns with non-monotone coordinates.
template <typename T, int LM>
__device__ __noinline__ void remap_winds_full(const Geom& g, const RemapArgs& ra, const T* dp,
                                              const T* f, T* r, int* tr, Status* st, int i,
                                              int j, int dir) {
  const int L = g.L;
  double sc[LM + 2], dc[LM + 2], var[LM + 2], out[LM + 2];
  PPMWork<LM> wk;
  // a, b: the face's two neighbours (weight 7/12), c, d: the outer pair (1/12)
  const long long oa = g.at(i, j);
  const long long ob = dir == 0 ? g.at(i, j - 1) : g.at(i - 1, j);
  const long long oc = dir == 0 ? g.at(i, j + 1) : g.at(i + 1, j);
  const long long od = dir == 0 ? g.at(i, j - 2) : g.at(i - 2, j);
  double psa = ra.ptop, psb = ra.ptop, psc = ra.ptop, psd = ra.ptop;
  for (int k = L - 1; k >= 0; --k) {
    const long long kk = (long long)k * g.S;
    psa = psa + (double)dp[oa + kk];
    psb = psb + (double)dp[ob + kk];
    psc = psc + (double)dp[oc + kk];
    psd = psd + (double)dp[od + kk];
  }
  double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop;
  for (int k = L + 1; k >= 1; --k) {
    if (k <= L) {
      long long kk = (long long)(k - 1) * g.S;
      pa = pa + (double)dp[oa + kk];
      pb = pb + (double)dp[ob + kk];
      pc = pc + (double)dp[oc + kk];
      pd = pd + (double)dp[od + kk];
    }
    sc[k] = C7_12 * (pa + pb) - C1_12 * (pc + pd);
    double ta, tb, tc, td;
    if (k <= L) {
      double a = ra.ak[k - 1], b = ra.bk[k - 1];
      ta = a + b * (psa - ra.ptop);
      tb = a + b * (psb - ra.ptop);
      tc = a + b * (psc - ra.ptop);
      td = a + b * (psd - ra.ptop);
    } else {
      ta = tb = tc = td = ra.ptop;
    }
    dc[k] = C7_12 * (ta + tb) - C1_12 * (tc + td);
  }
  for (int k = 1; k <= L; ++k) var[k] = (double)f[oa + (long long)(k - 1) * g.S];
  remap_column<LM>(wk, L, var, out, sc, dc, tr, 1, &st->fallback_pairs);
  for (int k = 1; k <= L; ++k) r[oa + (long long)(k - 1) * g.S] = T(out[k]);
}

// One thread per face column and direction (blockIdx.y); three column
// arrays of LM + 2 per thread: the coordinate in FP64, the eliminated
// interface values and coefficients in E (FP64, or FP32 in the mixed form).
// face column col of direction dir (0: u, 1: v)
template <typename T, int LM, typename E = double>
__device__ __forceinline__ void remap_winds_at(const Geom& g, const RemapArgs& ra, const T* dp,
                                               const T* ud, const T* vd,
                                               T* urem, T* vrem, int* trace, Status* st,
                                               int col, int dir) {
  const int w = g.nx + 2, h = g.ny + 2;
  if (col >= w * h) return;
  const int i = -1 + col % w, j = -1 + col / w;
  const int L = g.L;
  const long long S = g.S;
  const T* f = dir == 0 ? ud : vd;
  T* r = dir == 0 ? urem : vrem;
  int* tr = nullptr;
  if (trace) tr = trace + ((long long)dir * h * w + (long long)(j + 1) * w + (i + 1)) * L * 5;  // [3][ny+2][nx+2][L][5]
  double sca[LM + 2];
  E lva[LM + 2], gama[LM + 2];
  const ColArr sc{sca, 1};
  const ColArrT<E> lv{lva, 1}, gam{gama, 1};
  const long long oa = g.at(i, j);
  const long long ob = dir == 0 ? g.at(i, j - 1) : g.at(i - 1, j);
  const long long oc = dir == 0 ? g.at(i, j + 1) : g.at(i + 1, j);
  const long long od = dir == 0 ? g.at(i, j - 2) : g.at(i - 2, j);
  // source coordinate: running sums from the model top (the face
  // interpolation of src/mod_remap.f90:84-85 of the levels of :42-44)
  double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop, prev = 0.;
  int kc = L + 2, kv = L + 1;
  bool mono = true;
  auto cnext = [&]() {
    --kc;
    if (kc <= L) {
      const long long kk = (long long)(kc - 1) * S;
      pa = pa + (double)dp[oa + kk];
      pb = pb + (double)dp[ob + kk];
      pc = pc + (double)dp[oc + kk];
      pd = pd + (double)dp[od + kk];
    }
    const double c = C7_12 * (pa + pb) - C1_12 * (pc + pd);
    if (kc <= L) mono = mono && (prev <= c);
    prev = c;
    return c;
  };
  auto vnext = [&]() {
    --kv;
    return (double)f[oa + (long long)(kv - 1) * S];
  };
  ppm_eliminate<true>(L, cnext, vnext, sc, lv, gam);
  // pa..pd now hold the surface pressures of the four columns
  auto dc = [&](int k) {
    double ta, tb, tc, td;
    if (k <= L) {
      const double a = ra.ak[k - 1], b = ra.bk[k - 1];
      ta = a + b * (pa - ra.ptop);
      tb = a + b * (pb - ra.ptop);
      tc = a + b * (pc - ra.ptop);
      td = a + b * (pd - ra.ptop);
    } else {
      ta = tb = tc = td = ra.ptop;
    }
    return C7_12 * (ta + tb) - C1_12 * (tc + td);
  };
  double dprev = dc(1);
  for (int k = 2; k <= L + 1; ++k) {
    const double d = dc(k);
    mono = mono && (d <= dprev);
    dprev = d;
  }
  if (!mono) {
    remap_winds_full<T, LM>(g, ra, dp, f, r, tr, st, i, j, dir);
    return;
  }
  auto var = [&](int k) { return (double)f[oa + (long long)(k - 1) * S]; };
  remap_merge(L, sc, lv, gam, var, dc, [&](int m, double v) { r[oa + (long long)(m - 1) * S] = T(v); }, tr, 1);
}

// 16 blocks of 64 threads per SM (a 64-register budget, the column arrays in
// local memory either way): more columns in flight hide more of the local
// memory latency (measured at 1024x1024x64: 4.67 ms against 5.88 at the
// compiler's own budget, 5.34 at 24 blocks, 7.05 at 32).
template <typename T, int LM, typename E = double>
__global__ void __launch_bounds__(64, 16) k_remap_winds(Geom g, RemapArgs ra, const T* __restrict__ dp,
                                                    const T* __restrict__ ud, const T* __restrict__ vd,
                                                    T* __restrict__ urem, T* __restrict__ vrem, int* trace,
                                                    Status* st) {
  remap_winds_at<T, LM, E>(g, ra, dp, ud, vd, urem, vrem, trace, st, blockIdx.x * blockDim.x + threadIdx.x,
                           blockIdx.y);
}

// Energy remap and potential-temperature recovery on the interior,
// src/mod_remap.f90:42-78 (columns) and 111-161.  The all-arrays form, for
// columns with non-monotone coordinates.
template <typename T, int LM, typename PW = PortablePow>
__device__ __noinline__ void remap_energy_full(const Geom& g, const RemapArgs& ra, const T* dp,
                                               const T* pt, const T* ud,
                                               const T* vd, const T* urem,
                                               const T* vrem, const double* gzs,
                                               T* dpo, T* pto, T* udo,
                                               T* vdo, int* tr, Status* st, int i, int j) {
  const int L = g.L;
  const long long S = g.S;
  const long long o = g.at(i, j);
  double plev[LM + 2], pk[LM + 2], tpl[LM + 2], tpk[LM + 2], lyk[LM + 2], tlyk[LM + 2], gzv[LM + 2];
  double en[LM + 2], er[LM + 2];
  PPMWork<LM> wk;
  plev[L + 1] = ra.ptop;
  pk[L + 1] = ra.pk_top;
  for (int k = L; k >= 1; --k) {
    plev[k] = plev[k + 1] + (double)dp[o + (long long)(k - 1) * S];
    pk[k] = PW::kappa(plev[k]);
    double plog = PW::log(pk[k + 1] / pk[k]);
    lyk[k] = (pk[k + 1] - pk[k]) / plog;
  }
  tpl[L + 1] = ra.ptop;
  tpk[L + 1] = ra.pk_top;
  for (int k = L; k >= 1; --k) {
    tpl[k] = ra.ak[k - 1] + ra.bk[k - 1] * (plev[1] - ra.ptop);
    tpk[k] = PW::kappa(tpl[k]);
    double plog = PW::log(tpk[k + 1] / tpk[k]);
    tlyk[k] = (tpk[k + 1] - tpk[k]) / plog;
  }
  gzv[1] = gzs[o];
  for (int k = 1; k <= L; ++k) gzv[k + 1] = gzv[k] + CP_DRY * (double)pt[o + (long long)(k - 1) * S] * (pk[k] - pk[k + 1]);
  const int P = g.P;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    double ua = (.25 * ((double)ud[ok] + (double)ud[ok + P]) +
                 .125 * ((double)ud[ok - 1] + (double)ud[ok - 1 + P] + (double)ud[ok + 1] + (double)ud[ok + 1 + P]));
    double va = (.25 * ((double)vd[ok] + (double)vd[ok + 1]) +
                 .125 * ((double)vd[ok - P] + (double)vd[ok + 1 - P] + (double)vd[ok + P] + (double)vd[ok + 1 + P]));
    en[k] = CV_DRY * (double)pt[ok] * lyk[k] + .5 * (gzv[k + 1] + gzv[k] + ua * ua + va * va);
  }
  remap_column<LM>(wk, L, en, er, plev, tpl, tr, 1, &st->fallback_pairs);
  double gzr = gzv[1];
  bool bad = false;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    double ua = (.25 * ((double)urem[ok] + (double)urem[ok + P]) +
                 .125 * ((double)urem[ok - 1] + (double)urem[ok - 1 + P] + (double)urem[ok + 1] + (double)urem[ok + 1 + P]));
    double va = (.25 * ((double)vrem[ok] + (double)vrem[ok + 1]) +
                 .125 * ((double)vrem[ok - P] + (double)vrem[ok + 1 - P] + (double)vrem[ok + P] + (double)vrem[ok + 1 + P]));
    double ptr = (er[k] - gzr - .5 * (ua * ua + va * va)) / (CV_DRY * tlyk[k] + .5 * CP_DRY * (tpk[k] - tpk[k + 1]));
    gzr = gzr + CP_DRY * ptr * (tpk[k] - tpk[k + 1]);
    T dpn = T(tpl[k] - tpl[k + 1]);
    T un = urem[ok], vn = vrem[ok], tn = T(ptr);
    dpo[ok] = dpn;
    pto[ok] = tn;
    udo[ok] = un;
    vdo[ok] = vn;
    bad = bad || !(finite_(dpn) && finite_(tn) && finite_(un) && finite_(vn));
  }
  flag_nonfinite(&st->nonfinite_remap, bad);
}

// One thread per interior column; four column arrays of LM + 2 doubles per
// thread (levels, pkap then the eliminated interface values, energy, gam).
// interior column col
template <typename T, int LM, typename PW = PortablePow>
__device__ __forceinline__ void remap_energy_at(const Geom& g, const RemapArgs& ra, const T* dp,
                                                const T* pt, const T* ud,
                                                const T* vd, const T* urem,
                                                const T* vrem, const double* gzs,
                                                T* dpo, T* pto, T* udo,
                                                T* vdo, int* trace, Status* st, int col) {
  if (col >= g.nx * g.ny) return;
  const int i = col % g.nx, j = col / g.nx;
  const int L = g.L;
  const long long S = g.S;
  const long long o = g.at(i, j);
  const int P = g.P;
  int* tr = nullptr;
  if (trace) {
    const int w = g.nx + 2, h = g.ny + 2;
    tr = trace + ((long long)2 * h * w + (long long)(j + 1) * w + (i + 1)) * L * 5;
  }
  double arr[4 * (LM + 2)];
  const ColArr plev{arr, 1}, pk{arr + (LM + 2), 1}, en{arr + 2 * (LM + 2), 1}, gam{arr + 3 * (LM + 2), 1};
  const ColArr lv = pk;  // pkap is dead once the energy is formed
  // current levels and pkap (src/mod_remap.f90:42-54), downward
  bool mono = true;
  plev[L + 1] = ra.ptop;
  pk[L + 1] = ra.pk_top;
  double pl = ra.ptop;
  for (int k = L; k >= 1; --k) {
    const double pn = pl + (double)dp[o + (long long)(k - 1) * S];
    mono = mono && (pl <= pn);
    plev[k] = pn;
    pk[k] = PW::kappa(pn);
    pl = pn;
  }
  const double ps = pl;
  // gz (:70-75) and the total energy (:111-125), upward
  {
    double gz0 = gzs[o], pk0 = pk[1];
    for (int k = 1; k <= L; ++k) {
      const long long ok = o + (long long)(k - 1) * S;
      const double pk1 = pk[k + 1];
      const double ptk = (double)pt[ok];
      const double gz1 = gz0 + CP_DRY * ptk * (pk0 - pk1);
      const double plog = PW::log(pk1 / pk0);
      const double lyk = (pk1 - pk0) / plog;
      double ua = (.25 * ((double)ud[ok] + (double)ud[ok + P]) +
                   .125 * ((double)ud[ok - 1] + (double)ud[ok - 1 + P] + (double)ud[ok + 1] + (double)ud[ok + 1 + P]));
      double va = (.25 * ((double)vd[ok] + (double)vd[ok + 1]) +
                   .125 * ((double)vd[ok - P] + (double)vd[ok + 1 - P] + (double)vd[ok + P] + (double)vd[ok + 1 + P]));
      en[k] = CV_DRY * ptk * lyk + .5 * (gz1 + gz0 + ua * ua + va * va);
      gz0 = gz1;
      pk0 = pk1;
    }
  }
  // target levels (:57-59)
  auto tpl = [&](int k) { return k <= L ? ra.ak[k - 1] + ra.bk[k - 1] * (ps - ra.ptop) : ra.ptop; };
  {
    double tprev = tpl(1);
    for (int k = 2; k <= L + 1; ++k) {
      const double t = tpl(k);
      mono = mono && (t <= tprev);
      tprev = t;
    }
  }
  if (!mono) {
    remap_energy_full<T, LM, PW>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, tr, st, i, j);
    return;
  }
  int kc = L + 2, kv = L + 1;
  ppm_eliminate<false>(L, [&]() { return plev[--kc]; }, [&]() { return en[--kv]; }, plev, lv, gam);
  // remapped energy -> potential temperature (:127-161), upward
  double gzr = gzs[o];
  double tpl0 = tpl(1);
  double tpk0 = PW::kappa(tpl0);
  bool bad = false;
  auto put = [&](int m, double erm) {
    const long long ok = o + (long long)(m - 1) * S;
    const double tpl1 = tpl(m + 1);
    const double tpk1 = m < L ? PW::kappa(tpl1) : ra.pk_top;
    const double plog = PW::log(tpk1 / tpk0);
    const double tlyk = (tpk1 - tpk0) / plog;
    double ua = (.25 * ((double)urem[ok] + (double)urem[ok + P]) +
                 .125 * ((double)urem[ok - 1] + (double)urem[ok - 1 + P] + (double)urem[ok + 1] + (double)urem[ok + 1 + P]));
    double va = (.25 * ((double)vrem[ok] + (double)vrem[ok + 1]) +
                 .125 * ((double)vrem[ok - P] + (double)vrem[ok + 1 - P] + (double)vrem[ok + P] + (double)vrem[ok + 1 + P]));
    double ptr = (erm - gzr - .5 * (ua * ua + va * va)) / (CV_DRY * tlyk + .5 * CP_DRY * (tpk0 - tpk1));
    gzr = gzr + CP_DRY * ptr * (tpk0 - tpk1);
    T dpn = T(tpl0 - tpl1);
    T un = urem[ok], vn = vrem[ok], tn = T(ptr);
    dpo[ok] = dpn;
    pto[ok] = tn;
    udo[ok] = un;
    vdo[ok] = vn;
    bad = bad || !(finite_(dpn) && finite_(tn) && finite_(un) && finite_(vn));
    tpl0 = tpl1;
    tpk0 = tpk1;
  };
  remap_merge(L, plev, lv, gam, [&](int k) { return en[k]; }, tpl, put, tr, 1);
  flag_nonfinite(&st->nonfinite_remap, bad);
}

// 16 blocks per SM, as k_remap_winds (4.91 ms against 5.45)
template <typename T, int LM, typename PW = PortablePow>
__global__ void __launch_bounds__(64, 16) k_remap_energy(Geom g, RemapArgs ra, const T* __restrict__ dp,
                                                     const T* __restrict__ pt, const T* __restrict__ ud,
                                                     const T* __restrict__ vd, const T* __restrict__ urem,
                                                     const T* __restrict__ vrem, const double* __restrict__ gzs,
                                                     T* __restrict__ dpo, T* __restrict__ pto, T* __restrict__ udo,
                                                     T* __restrict__ vdo, int* trace, Status* st) {
  remap_energy_at<T, LM, PW>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st,
                             blockIdx.x * blockDim.x + threadIdx.x);
}

// ============================================================ reductions ===
// Finite check of the interior of four fields (src/mod_fields.f90:69-106).
template <typename T>
__global__ void k_check_finite(Geom g, const T* f0, const T* f1, const T* f2, const T* f3, int* flag) {
  const int n = g.nx * g.ny;
  bool bad = false;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * g.L; idx += gridDim.x * blockDim.x) {
    int k = idx / n, r = idx - k * n;
    long long o = g.at(r % g.nx, r / g.nx, k);
    bad = bad || !(finite_(f0[o]) && finite_(f1[o]) && finite_(f2[o]) && finite_(f3[o]));
  }
  flag_nonfinite(flag, bad);
}

// Sum of the interior pressure thickness in FP64, in a fixed order: each
// block reduces a fixed slice of the (level, row) pairs with a fixed tree,
// the host-visible result sums the block partials in index order.
template <typename T>
__global__ void k_mass_partial(Geom g, const T* dp, double* partial) {
  __shared__ double red[256];
  const int rows = g.ny * g.L;
  double acc = 0.;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    int k = r / g.ny, j = r - k * g.ny;
    const T* row = dp + g.at(0, j, k);
    for (int i = threadIdx.x; i < g.nx; i += blockDim.x) acc += (double)row[i];
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}
static __global__ void k_mass_final(const double* partial, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.;
    for (int i = 0; i < n; ++i) s += partial[i];
    *out = s;
  }
}

// Precision conversion of whole padded fields (mixed-precision uploads and
// downloads go through an FP64 staging field).
template <typename A, typename B>
__global__ void k_convert(const A* __restrict__ src, B* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = B(src[i]);
}

}  // namespace atm
