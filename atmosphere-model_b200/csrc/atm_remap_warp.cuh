// Warp-cooperative vertical remap (the mixed form's).
//
// One warp per column: the layers are spread over the lanes (LPL layers a
// lane, layer k = lane * LPL + e + 1), so a column's working set lives in
// registers instead of per-thread local arrays.  The remap's sequential
// parts become warp scans with shuffles:
//  * the cumulative masses (interface pressures from the model top,
//    src/mod_remap.f90:42-44, 84-85) and the hydrostatic geopotential
//    (:73-78) are suffix / prefix sums, in FP64;
//  * the elimination of vertical_ppm's tridiagonal system (:295-309) is a
//    suffix product of 2x2 Moebius matrices (the continued fraction of gam)
//    followed by a suffix composition of affine maps (the interface
//    values), its forward substitution (:311-313) a prefix composition;
//  * the potential-temperature recovery (:127-155) is a prefix composition
//    of affine maps of the remapped geopotential;
//  * each destination layer finds its first and last overlapping source
//    layer by binary searches over the shuffled source interfaces, and
//    sums the pair integrals of :188-280 in ascending source order.
// The limiters, the Huynh constraint and the curvature (:316-354) are per
// interface and layer.  The association of the sums differs from the
// sequential FP64 form, so this remap agrees with it to rounding, not bit
// for bit; the FP64 form keeps the sequential kernels (its pin to the
// oracle is bit-exact).  Columns whose coordinates are not monotone take
// the sequential all-pairs path (one lane).
#pragma once

#include "atm_kernels.cuh"

namespace atm {

namespace wr {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// x -> a + b x
struct Aff {
  double a, b;
};
__device__ __forceinline__ Aff compose(Aff f, Aff g) { return {f.a + f.b * g.a, f.b * g.b}; }  // f(g(x))
__device__ __forceinline__ Aff shfl_dn(Aff f, int d) {
  return {__shfl_down_sync(FULL, f.a, d), __shfl_down_sync(FULL, f.b, d)};
}
__device__ __forceinline__ Aff shfl_up(Aff f, int d) {
  return {__shfl_up_sync(FULL, f.a, d), __shfl_up_sync(FULL, f.b, d)};
}
// inclusive suffix composition over lanes: F_l o F_{l+1} o ... o F_31
__device__ __forceinline__ Aff suffix(Aff f) {
  const int l = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Aff g = shfl_dn(f, d);
    if (l + d < 32) f = compose(f, g);
  }
  return f;
}
// inclusive prefix composition over lanes: F_l o F_{l-1} o ... o F_0
__device__ __forceinline__ Aff prefix(Aff f) {
  const int l = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Aff g = shfl_up(f, d);
    if (l >= d) f = compose(f, g);
  }
  return f;
}

// 2x2 matrix [[a, b], [c, d]] of a Moebius map x -> (a x + b) / (c x + d)
struct M2 {
  double a, b, c, d;
};
__device__ __forceinline__ M2 mul(M2 x, M2 y) {
  return {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
// the same map with its entries scaled by a power of two near 1/max|entry|
__device__ __forceinline__ M2 norm(M2 x) {
  const double m = fmax(fmax(fabs(x.a), fabs(x.b)), fmax(fabs(x.c), fabs(x.d)));
  if (!(m > 0.) || !isfinite(m)) return x;
  const double s = ldexp(1., -ilogb(m));
  return {x.a * s, x.b * s, x.c * s, x.d * s};
}
__device__ __forceinline__ M2 shfl_dn(M2 m, int d) {
  return {__shfl_down_sync(FULL, m.a, d), __shfl_down_sync(FULL, m.b, d), __shfl_down_sync(FULL, m.c, d),
          __shfl_down_sync(FULL, m.d, d)};
}
// inclusive suffix product over lanes: M_l M_{l+1} ... M_31
__device__ __forceinline__ M2 suffix(M2 m) {
  const int l = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const M2 y = shfl_dn(m, d);
    if (l + d < 32) m = norm(mul(m, y));
  }
  return m;
}

__device__ __forceinline__ double suffix_sum(double x) {
  const int l = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double y = __shfl_down_sync(FULL, x, d);
    if (l + d < 32) x += y;
  }
  return x;
}
__device__ __forceinline__ double prefix_sum(double x) {
  const int l = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double y = __shfl_up_sync(FULL, x, d);
    if (l >= d) x += y;
  }
  return x;
}

// element of layer (or interface) q, 1-based, of a distributed column array
template <int LPL>
__device__ __forceinline__ double fetch(const double (&a)[LPL], int q) {
  const int src = ((q - 1) / LPL) & 31, idx = (q - 1) % LPL;
  double out = 0.;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const double v = __shfl_sync(FULL, a[e], src);
    if (e == idx) out = v;
  }
  return out;
}
// the element of the next (k+1) and previous (k-1) layer of each own layer
template <int LPL>
__device__ __forceinline__ void neighbours(const double (&a)[LPL], double (&nx)[LPL], double (&pv)[LPL]) {
  const double n0 = __shfl_down_sync(FULL, a[0], 1);
  const double pl = __shfl_up_sync(FULL, a[LPL - 1], 1);
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    nx[e] = e + 1 < LPL ? a[e + 1] : n0;
    pv[e] = e > 0 ? a[e - 1] : pl;
  }
}

// vertical_ppm (src/mod_remap.f90:287-356) of var(k) on the source
// interfaces c(k) (interface k at the bottom of layer k; ctop = c(L+1)),
// then the pair loop (:165-285) onto the destination interfaces d(m)
// (dtop = d(L+1)), as warp scans; out(m) for the own layers.  The
// coordinates decrease with k.  L >= 3.
template <int LPL>
__device__ __forceinline__ void remap_column_w(int L, const double (&var)[LPL], const double (&c)[LPL], double ctop,
                                               const double (&dd)[LPL], double dtop, double (&out)[LPL]) {
  const int lane = lane_id();
  double cn[LPL], cp[LPL], vn[LPL], vp[LPL];
  neighbours<LPL>(c, cn, cp);
  neighbours<LPL>(var, vn, vp);
  int kk[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    kk[e] = lane * LPL + e + 1;
    if (kk[e] == L) cn[e] = ctop;
  }
  // ---- the elimination's top row (:296-299), on the lane of layer L
  const int srcL = (L - 1) / LPL;
  double lvT = 0., gamL = 0.;
  {
    double alpha = 0., vL = 0., vLm = 0., c0 = 0., c1 = 0.;
#pragma unroll
    for (int e = 0; e < LPL; ++e)
      if (kk[e] == L) {
        vL = var[e];
        vLm = vp[e];
        c0 = cp[e];
        c1 = c[e];
      }
    alpha = (c1 - c0) / (ctop - c1);
    const double beta = alpha * (.5 + alpha);
    lvT = __shfl_sync(FULL, (2. * alpha * (1. + alpha) * vL + vLm) / beta, srcL);
    gamL = __shfl_sync(FULL, (1. + alpha * (1.5 + alpha)) / beta, srcL);
  }
  // ---- gam(k-1) = alpha_k / (2 + 2 alpha_k - gam(k)), k = L .. 2 (:300-309):
  // a suffix product of Moebius maps applied to gam(L)
  double alpha[LPL];
  M2 mloc[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const bool row = kk[e] >= 2 && kk[e] <= L;
    alpha[e] = row ? (cn[e] - c[e]) / (c[e] - cp[e]) : 0.;
    mloc[e] = row ? M2{0., alpha[e], -1., 2. + 2. * alpha[e]} : M2{1., 0., 0., 1.};
  }
  M2 lane_prod = mloc[LPL - 1];
#pragma unroll
  for (int e = LPL - 2; e >= 0; --e) {
    mloc[e] = norm(mul(mloc[e], mloc[e + 1]));
    lane_prod = mloc[e];
  }
  M2 after = shfl_dn(suffix(lane_prod), 1);  // product over the lanes above
  if (lane == 31) after = M2{1., 0., 0., 1.};
  double gm1[LPL];  // gam(k-1) of each own layer k >= 2
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const M2 p = mul(mloc[e], after);
    gm1[e] = (p.a * gamL + p.b) / (p.c * gamL + p.d);
  }
  // gam(k) of each own layer: gam(k-1) of the next layer, gam(L) on top
  double gk[LPL], gdummy[LPL];
  neighbours<LPL>(gm1, gk, gdummy);
#pragma unroll
  for (int e = 0; e < LPL; ++e)
    if (kk[e] == L) gk[e] = gamL;
  // ---- lv(k) = (3 (var(k) + alpha var(k-1)) - lv(k+1)) / beta: a suffix
  // composition of affine maps applied to lv(L+1)
  Aff aloc[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    if (kk[e] >= 2 && kk[e] <= L) {
      const double beta = 2. + 2. * alpha[e] - gk[e];
      aloc[e] = Aff{3. * (var[e] + alpha[e] * vp[e]) / beta, -1. / beta};
    } else {
      aloc[e] = Aff{0., 1.};
    }
  }
#pragma unroll
  for (int e = LPL - 2; e >= 0; --e) aloc[e] = compose(aloc[e], aloc[e + 1]);
  Aff aafter = shfl_dn(suffix(aloc[0]), 1);
  if (lane == 31) aafter = Aff{0., 1.};
  double lv[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const Aff f = compose(aloc[e], aafter);
    lv[e] = f.a + f.b * lvT;
  }
  // lv(1) (:310), on lane 0
  {
    const double v1 = fetch<LPL>(var, 1), v2 = fetch<LPL>(var, 2), lv2 = fetch<LPL>(lv, 2);
    const double a2 = fetch<LPL>(alpha, 2), g1 = fetch<LPL>(gm1, 2);
    const double beta = 1. + a2 * (1.5 + a2);
    const double lv1 = (2. * a2 * (1. + a2) * v1 + v2 - beta * lv2) / (a2 * (.5 + a2) - beta * g1);
    if (lane == 0) lv[0] = lv1;
  }
  // ---- forward substitution lv(k) -= gam(k-1) lv(k-1), k = 2 .. L+1 (:311-313)
  Aff bloc[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    if (kk[e] == 1) bloc[e] = Aff{lv[e], 0.};
    else if (kk[e] <= L) bloc[e] = Aff{lv[e], -gm1[e]};
    else bloc[e] = Aff{0., 1.};
  }
#pragma unroll
  for (int e = 1; e < LPL; ++e) bloc[e] = compose(bloc[e], bloc[e - 1]);
  Aff before = shfl_up(prefix(bloc[LPL - 1]), 1);
  if (lane == 0) before = Aff{0., 1.};
#pragma unroll
  for (int e = 0; e < LPL; ++e) lv[e] = compose(bloc[e], before).a;
  // the top interface L+1
  double lvtop = 0.;
  {
    double lvL = 0.;
#pragma unroll
    for (int e = 0; e < LPL; ++e)
      if (kk[e] == L) lvL = lv[e];
    lvtop = __shfl_sync(FULL, lvT - gamL * lvL, srcL);
  }
  // ---- boundary and monotonicity limiters of interfaces 2 .. L (:316-334):
  // interface m with k = m-1 of the reference's loop tests gam(m+1) gam(m-1)
  double gk1[LPL], gm2[LPL];  // gam(k+1): gam(k) of the next layer; gam(k-2): gam(k-1) of the previous one
  neighbours<LPL>(gk, gk1, gdummy);
  neighbours<LPL>(gm1, gdummy, gm2);
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int m = kk[e];
    if (m < 2 || m > L) continue;
    const double lo = mn(vp[e], var[e]), hi = mx(vp[e], var[e]);
    double x = lv[e];
    if (m == 2 || m == L) {
      x = mn(x, mx(var[e], vp[e]));
      x = mx(x, mn(var[e], vp[e]));
    } else if (gk1[e] * gm1[e] > 0) {
      x = mn(x, hi);
      x = mx(x, lo);
    } else if (gk1[e] > 0) {
      x = mx(x, lo);
    } else {
      x = mn(x, hi);
    }
    lv[e] = x;
  }
  // ---- layer edges, the Huynh constraint (:336-352) and the curvature (:354)
  double top[LPL], btm[LPL], curv[LPL];
  {
    double lvn[LPL];
    neighbours<LPL>(lv, lvn, gdummy);
#pragma unroll
    for (int e = 0; e < LPL; ++e) {
      const int m = kk[e];
      top[e] = (m == L) ? lvtop : lvn[e];
      btm[e] = lv[e];
      if (m >= 3 && m <= L) {
        double pmp1 = var[e] - 2. * gm1[e];
        double lac1 = pmp1 + 1.5 * gm2[e];
        top[e] = mn(mx(top[e], mn3(var[e], pmp1, lac1)), mx3(var[e], pmp1, lac1));
        pmp1 = var[e] + 2. * gk[e];
        lac1 = pmp1 - 1.5 * gm1[e];
        btm[e] = mn(mx(btm[e], mn3(var[e], pmp1, lac1)), mx3(var[e], pmp1, lac1));
      }
      curv[e] = 6. * var[e] - 3. * (top[e] + btm[e]);
    }
  }
  // ---- the pair loop (:188-280) as a merge: for each own destination
  // layer m, the source layers k0 .. k1 that overlap it, found by binary
  // searches over the shuffled source interfaces
  auto cat = [&](int q) {  // source interface q, 1 .. L+1
    const double v = fetch<LPL>(c, q <= L ? q : 1);
    return q <= L ? v : ctop;
  };
  double dn[LPL], ddum[LPL];
  neighbours<LPL>(dd, dn, ddum);
  int k0[LPL], cnt[LPL];
  int maxcnt = 0;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const double d0 = dd[e], d1 = (kk[e] == L) ? dtop : dn[e];
    // first k in [1, L] with c(k+1) < d0 (L+1 if none)
    int lo = 1, hi = L + 1;
    while (__any_sync(FULL, lo < hi)) {
      const int mid = (lo + hi) >> 1;
      const bool act = lo < hi;
      const double cm = cat(act ? mid + 1 : 1);
      if (act) {
        if (cm < d0) hi = mid;
        else lo = mid + 1;
      }
    }
    k0[e] = lo;
    // last k in [1, L] with c(k) > d1 (0 if none)
    int lo2 = 0, hi2 = L;
    while (__any_sync(FULL, lo2 < hi2)) {
      const int mid = (lo2 + hi2 + 1) >> 1;
      const bool act = lo2 < hi2;
      const double cm = cat(act ? mid : 1);
      if (act) {
        if (cm > d1) lo2 = mid;
        else hi2 = mid - 1;
      }
    }
    cnt[e] = (kk[e] <= L && lo2 >= k0[e]) ? lo2 - k0[e] + 1 : 0;
    maxcnt = max(maxcnt, cnt[e]);
  }
  maxcnt = __reduce_max_sync(FULL, maxcnt);
#pragma unroll
  for (int e = 0; e < LPL; ++e) out[e] = 0.;
  for (int t = 0; t < maxcnt; ++t) {
#pragma unroll
    for (int e = 0; e < LPL; ++e) {
      const bool act = t < cnt[e];
      const int k = act ? k0[e] + t : 1;
      const double bk = fetch<LPL>(btm, k), tk = fetch<LPL>(top, k), cv = fetch<LPL>(curv, k);
      const double vk = fetch<LPL>(var, k), sk = cat(k), sk1 = cat(k + 1);
      if (act) {
        const double d0 = dd[e], d1 = (kk[e] == L) ? dtop : dn[e];
        pair_add(out[e], bk, tk, cv, vk, sk, sk1, d0, d1);
      }
    }
  }
}

}  // namespace wr

// Winds on the cell faces over [isd-1, ied+1]^2 (src/mod_remap.f90:80-105):
// one warp per face column and direction.
template <int LPL>
__global__ void __launch_bounds__(128) k_remap_winds_w(Geom g, RemapArgs ra, const double* __restrict__ dp,
                                                       const double* __restrict__ ud, const double* __restrict__ vd,
                                                       double* __restrict__ urem, double* __restrict__ vrem,
                                                       Status* st) {
  constexpr int LM = 32 * LPL;
  const int lane = wr::lane_id();
  const int w = g.nx + 2, h = g.ny + 2;
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= 2LL * w * h) return;  // the whole warp
  const int dir = (int)(wid / ((long long)w * h));
  const int col = (int)(wid % ((long long)w * h));
  const int i = -1 + col % w, j = -1 + col / w;
  const int L = g.L;
  const long long S = g.S;
  const double* f = dir == 0 ? ud : vd;
  double* r = dir == 0 ? urem : vrem;
  const long long oa = g.at(i, j);
  const long long ob = dir == 0 ? g.at(i, j - 1) : g.at(i - 1, j);
  const long long oc = dir == 0 ? g.at(i, j + 1) : g.at(i + 1, j);
  const long long od = dir == 0 ? g.at(i, j - 2) : g.at(i - 2, j);
  // the face-interpolated thickness of each own layer; the interface
  // pressures are its suffix sums from the model top
  double th[LPL], var[LPL];
  bool mono = true;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    if (k <= L) {
      const long long kk = (long long)(k - 1) * S;
      th[e] = C7_12 * (dp[oa + kk] + dp[ob + kk]) - C1_12 * (dp[oc + kk] + dp[od + kk]);
      var[e] = f[oa + kk];
      mono = mono && th[e] >= 0.;
    } else {
      th[e] = 0.;
      var[e] = 0.;
    }
  }
  const double ptop = ra.ptop;
  const double ctop = C7_12 * (ptop + ptop) - C1_12 * (ptop + ptop);
  double loc[LPL];
  double acc = 0.;
#pragma unroll
  for (int e = LPL - 1; e >= 0; --e) {
    acc += th[e];
    loc[e] = acc;
  }
  const double incl = wr::suffix_sum(acc);
  const double above = incl - acc;
  const double total = __shfl_sync(wr::FULL, incl, 0);
  double c[LPL], dd[LPL];
  const double wA = (C7_12 + C7_12) - (C1_12 + C1_12);
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    c[e] = ctop + (above + loc[e]);
    dd[e] = k <= L ? wA * ra.ak[k - 1] + ra.bk[k - 1] * total : ctop;
  }
  {  // the destination interfaces decrease with k
    double dnx[LPL], dpv[LPL];
    wr::neighbours<LPL>(dd, dnx, dpv);
#pragma unroll
    for (int e = 0; e < LPL; ++e) {
      const int k = lane * LPL + e + 1;
      const double up = (k == L) ? ctop : dnx[e];
      if (k <= L) mono = mono && up <= dd[e];
    }
  }
  if (!__all_sync(wr::FULL, mono)) {
    if (lane == 0) remap_winds_full<double, LM>(g, ra, dp, f, r, nullptr, st, i, j, dir);
    return;
  }
  double out[LPL];
  wr::remap_column_w<LPL>(L, var, c, ctop, dd, ctop, out);
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    if (k <= L) r[oa + (long long)(k - 1) * S] = out[e];
  }
}

// Energy remap and potential-temperature recovery on the interior
// (src/mod_remap.f90:42-78, 111-161): one warp per column.
template <int LPL>
__global__ void __launch_bounds__(128) k_remap_energy_w(Geom g, RemapArgs ra, const double* __restrict__ dp,
                                                        const double* __restrict__ pt, const double* __restrict__ ud,
                                                        const double* __restrict__ vd, const double* __restrict__ urem,
                                                        const double* __restrict__ vrem,
                                                        const double* __restrict__ gzs, double* __restrict__ dpo,
                                                        double* __restrict__ pto, double* __restrict__ udo,
                                                        double* __restrict__ vdo, Status* st) {
  constexpr int LM = 32 * LPL;
  const int lane = wr::lane_id();
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= (long long)g.nx * g.ny) return;  // the whole warp
  const int i = (int)(wid % g.nx), j = (int)(wid / g.nx);
  const int L = g.L;
  const long long S = g.S;
  const int P = g.P;
  const long long o = g.at(i, j);
  double dpk[LPL], ptk[LPL], ke[LPL];
  bool mono = true;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    dpk[e] = 0.;
    ptk[e] = 0.;
    ke[e] = 0.;
    if (k <= L) {
      const long long ok = o + (long long)(k - 1) * S;
      dpk[e] = dp[ok];
      ptk[e] = pt[ok];
      const double ua = (.25 * (ud[ok] + ud[ok + P]) + .125 * (ud[ok - 1] + ud[ok - 1 + P] + ud[ok + 1] + ud[ok + 1 + P]));
      const double va = (.25 * (vd[ok] + vd[ok + 1]) + .125 * (vd[ok - P] + vd[ok + 1 - P] + vd[ok + P] + vd[ok + 1 + P]));
      ke[e] = ua * ua + va * va;
      mono = mono && dpk[e] >= 0.;
    }
  }
  // current interface pressures (suffix sums from the top) and pkap
  double loc[LPL];
  double acc = 0.;
#pragma unroll
  for (int e = LPL - 1; e >= 0; --e) {
    acc += dpk[e];
    loc[e] = acc;
  }
  const double incl = wr::suffix_sum(acc);
  const double above = incl - acc;
  const double total = __shfl_sync(wr::FULL, incl, 0);
  const double ptop = ra.ptop, ps = ptop + total;
  double plev[LPL], pk[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    plev[e] = ptop + (above + loc[e]);
    pk[e] = k <= L ? atm_pow(plev[e], KAPPA) : ra.pk_top;
  }
  double pkn[LPL], pkp[LPL];
  wr::neighbours<LPL>(pk, pkn, pkp);
  // gz at the interfaces (a prefix sum from the surface) and the energy
  double inc[LPL], lyk[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    if (k == L) pkn[e] = ra.pk_top;
    inc[e] = k <= L ? CP_DRY * ptk[e] * (pk[e] - pkn[e]) : 0.;
    lyk[e] = k <= L ? (pkn[e] - pk[e]) / atm_log(pkn[e] / pk[e]) : 0.;
  }
  double lpre[LPL];
  acc = 0.;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    acc += inc[e];
    lpre[e] = acc;
  }
  const double pincl = wr::prefix_sum(acc);
  const double below = pincl - acc;
  const double gz0 = gzs[o];
  double en[LPL], tpl[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    const double gzt = gz0 + (below + lpre[e]);
    const double gzb = gzt - inc[e];
    en[e] = k <= L ? CV_DRY * ptk[e] * lyk[e] + .5 * (gzt + gzb + ke[e]) : 0.;
    tpl[e] = k <= L ? ra.ak[k - 1] + ra.bk[k - 1] * (ps - ptop) : ptop;
  }
  {  // the target levels decrease with k
    double tn[LPL], tp[LPL];
    wr::neighbours<LPL>(tpl, tn, tp);
#pragma unroll
    for (int e = 0; e < LPL; ++e) {
      const int k = lane * LPL + e + 1;
      const double up = (k == L) ? ptop : tn[e];
      if (k <= L) mono = mono && up <= tpl[e];
    }
  }
  if (!__all_sync(wr::FULL, mono)) {
    if (lane == 0)
      remap_energy_full<double, LM>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, nullptr, st, i, j);
    return;
  }
  double er[LPL];
  wr::remap_column_w<LPL>(L, en, plev, ptop, tpl, ptop, er);
  // remapped energy -> potential temperature (:127-161): gzr(m+1) =
  // gzr(m) + cp ptr(m) (tpk(m) - tpk(m+1)) with ptr(m) = (er(m) - gzr(m) -
  // KE/2) / E(m), an affine recurrence of gzr composed as a prefix scan
  double tpk[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    tpk[e] = k <= L ? atm_pow(tpl[e], KAPPA) : ra.pk_top;
  }
  double tpkn[LPL], tpkp[LPL], tpln[LPL], tplp[LPL];
  wr::neighbours<LPL>(tpk, tpkn, tpkp);
  wr::neighbours<LPL>(tpl, tpln, tplp);
  double X[LPL], E[LPL], D[LPL];
  wr::Aff gl[LPL];
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    if (k == L) {
      tpkn[e] = ra.pk_top;
      tpln[e] = ptop;
    }
    if (k <= L) {
      const long long ok = o + (long long)(k - 1) * S;
      const double ua = (.25 * (urem[ok] + urem[ok + P]) +
                         .125 * (urem[ok - 1] + urem[ok - 1 + P] + urem[ok + 1] + urem[ok + 1 + P]));
      const double va = (.25 * (vrem[ok] + vrem[ok + 1]) +
                         .125 * (vrem[ok - P] + vrem[ok + 1 - P] + vrem[ok + P] + vrem[ok + 1 + P]));
      const double tlyk = (tpkn[e] - tpk[e]) / atm_log(tpkn[e] / tpk[e]);
      D[e] = CP_DRY * (tpk[e] - tpkn[e]);
      E[e] = CV_DRY * tlyk + .5 * CP_DRY * (tpk[e] - tpkn[e]);
      X[e] = er[e] - .5 * (ua * ua + va * va);
      gl[e] = wr::Aff{D[e] * X[e] / E[e], 1. - D[e] / E[e]};
    } else {
      D[e] = E[e] = 1.;
      X[e] = 0.;
      gl[e] = wr::Aff{0., 1.};
    }
  }
  // gzr at the bottom of each own layer: the composition of the maps of the
  // layers below applied to gzs
  wr::Aff pre[LPL];
  pre[0] = gl[0];
#pragma unroll
  for (int e = 1; e < LPL; ++e) pre[e] = wr::compose(gl[e], pre[e - 1]);
  wr::Aff before = wr::shfl_up(wr::prefix(pre[LPL - 1]), 1);
  if (lane == 0) before = wr::Aff{0., 1.};
  bool bad = false;
#pragma unroll
  for (int e = 0; e < LPL; ++e) {
    const int k = lane * LPL + e + 1;
    const wr::Aff below_e = e == 0 ? before : wr::compose(pre[e - 1], before);
    const double gzr = below_e.a + below_e.b * gz0;
    if (k <= L) {
      const long long ok = o + (long long)(k - 1) * S;
      const double ptr = (X[e] - gzr) / E[e];
      const double dpn = tpl[e] - tpln[e];
      const double un = urem[ok], vn = vrem[ok];
      dpo[ok] = dpn;
      pto[ok] = ptr;
      udo[ok] = un;
      vdo[ok] = vn;
      bad = bad || !(finite_(dpn) && finite_(ptr) && finite_(un) && finite_(vn));
    }
  }
  flag_nonfinite(&st->nonfinite_remap, bad);
}

}  // namespace atm
