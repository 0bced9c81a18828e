// Warp-cooperative adjoint of the wind remap (src/mod_remap.f90:80-105 with
// remap_column and vertical_ppm, :165-356) for columns of at most 64 layers.
//
// The thread-per-column adjoint (k_remap_winds_adj) keeps about fifteen
// column arrays per thread in local memory; at full occupancy they spill
// through L2 to HBM, and their traffic bounds it.  Here a warp takes a
// group of G face columns (consecutive in x, one wind direction) and keeps
// their arrays in its shared memory:
//  * phase 1, a lane per column: the forward's sequential parts exactly as
//    the forward kernel (remap_winds_at) runs them -- the running sums of the
//    four columns' interface pressures, the elimination of vertical_ppm and
//    its forward substitution -- so that every limiter, edge and pair
//    decision of the reverse pass is the forward's;
//  * phase 2, the whole warp on one column at a time with its levels spread
//    over the lanes: the limited interface values, edges and curvatures; the
//    pair integrals' adjoints, a lane per destination layer (its first
//    source layer found by binary search); the adjoints of the Huynh and
//    interface limiters, a lane per interface; the linear recurrences of the
//    back substitution and of the elimination as warp scans of affine maps;
//    and the coordinate adjoints turned into the dp adjoints of the four
//    columns by a warp prefix sum.
// The reverse pass sums in another order than the sequential one (scans,
// shared-memory atomics), so its results agree with it to rounding.
// Columns whose coordinates are not monotone take the thread-per-column
// all-pairs path on one lane.
#pragma once

#include "atm_adjoint.cuh"

namespace atm {
namespace rwa {

constexpr unsigned FULL = 0xffffffffu;
constexpr int G = 8;    // face columns per group: the lanes of phase 1
constexpr int NWB = 2;  // warps per block

// x -> a + b x
struct Af {
  double a, b;
};
// f after g: x -> f(g(x))
__device__ __forceinline__ Af after(Af f, Af g) { return {f.a + f.b * g.a, f.b * g.b}; }
__device__ __forceinline__ Af shfl_up_af(Af f, int d) {
  return {__shfl_up_sync(FULL, f.a, d), __shfl_up_sync(FULL, f.b, d)};
}

// The chain y(p) = F(idx(p))(y(p-1)), p = 0..n-1 (n <= 96), y(-1) = y0, by
// the whole warp: lane l takes positions 3l..3l+2, composes their maps,
// and an inclusive scan of the compositions over the lanes gives each lane
// the value entering its block.  out(idx(p), y(p)) receives every value,
// after every map has been read (so out may overwrite what F reads).
template <typename FI, typename FM, typename FO>
__device__ __forceinline__ void chain(int n, double y0, FI&& idx, FM&& F, FO&& out) {
  const int lane = threadIdx.x & 31;
  const int p0 = 3 * lane;
  Af m[3];
  Af agg{0., 1.};
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    m[e] = (p0 + e < n) ? F(idx(p0 + e)) : Af{0., 1.};
    agg = after(m[e], agg);
  }
  Af inc = agg;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Af o = shfl_up_af(inc, d);
    if (lane >= d) inc = after(inc, o);
  }
  Af ex = shfl_up_af(inc, 1);
  if (lane == 0) ex = Af{0., 1.};
  __syncwarp();
  double y = ex.a + ex.b * y0;
#pragma unroll
  for (int e = 0; e < 3; ++e)
    if (p0 + e < n) {
      y = m[e].a + m[e].b * y;
      out(idx(p0 + e), y);
    }
  __syncwarp();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  return v;
}

// per-warp shared memory: the group's phase-1 arrays and one column's
// phase-2 arrays (indices 0..L+1)
template <int LM>
struct Work {
  static constexpr int NA = LM + 2;
  double sc[G][NA], gam[G][NA], lvb[G][NA];
  double ps[G][4];
  int flag[G];  // bit 0: some output adjoint is non-zero; bit 1: both coordinates monotone
  double var[NA], dc[NA], lvc[NA], top[NA], btm[NA], curv[NA], Ld[NA];
  double Lsrc[NA], Ltop[NA], Lbtm[NA], Lsc[NA], Ldc[NA], LL[NA], Lgam[NA];
  double La2;
};

// face column (i, j) and direction of group member q; false past the end
__device__ __forceinline__ bool face(const Geom& g, long long q, int& i, int& j, int& dir, long long& oa,
                                     long long& ob, long long& oc, long long& od) {
  const int w = g.nx + 2, h = g.ny + 2;
  const long long ncol = (long long)w * h;
  if (q >= 2 * ncol) return false;
  dir = (int)(q / ncol);
  const int col = (int)(q - dir * ncol);
  i = -1 + col % w;
  j = -1 + col / w;
  oa = g.at(i, j);
  ob = dir == 0 ? g.at(i, j - 1) : g.at(i - 1, j);
  oc = dir == 0 ? g.at(i, j + 1) : g.at(i + 1, j);
  od = dir == 0 ? g.at(i, j - 2) : g.at(i - 2, j);
  return true;
}

// destination coordinate of interface k from the four surface pressures,
// as remap_winds_at forms it
__device__ __forceinline__ double dcoord(const RemapArgs& ra, int L, int k, double pa, double pb, double pc,
                                        double pd) {
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
}

// adjoint of r = mn(mx(x0, mn3(a, b, c)), mx3(a, b, c)) (the edge limiter of
// src/mod_remap.f90:342-352, b = a + s2 gam(j2), c = b + s15 gam(j15)) with
// the gam adjoints added atomically; returns the adjoint of x0
__device__ __forceinline__ double edge_clamp_adj_at(double x0, double a, double b, double c, double lam,
                                                   double& lvar, double* Lgam, int j2, double s2, int j15,
                                                   double s15) {
  const double lo = mn3(a, b, c), hi = mx3(a, b, c);
  const double inner = mx(x0, lo);
  int which;  // 0: x0, 1: lo, 2: hi
  if (hi < inner) which = 2;
  else if (x0 < lo) which = 1;
  else which = 0;
  if (which == 0) return lam;
  const int s = which == 1 ? sel_mn3(a, b, c) : sel_mx3(a, b, c);
  lvar += lam;
  if (s != 0) {
    atomicAdd(Lgam + j2, s2 * lam);
    if (s == 2) atomicAdd(Lgam + j15, s15 * lam);
  }
  return 0.;
}

// One column's wind remap adjoint on the thread-per-column all-pairs path
// (coordinates that are not monotone).
template <int LM>
__device__ __noinline__ void winds_adj_column_full(const Geom& g, const RemapArgs& ra, const double* __restrict__ dp,
                                                   const double* __restrict__ f, const double* __restrict__ lr,
                                                   double* lam_dp, double* lf, long long oa, long long ob,
                                                   long long oc, long long od) {
  const int L = g.L;
  const long long S = g.S;
  double sc[LM + 2], dc[LM + 2], var[LM + 2], Ld[LM + 2], Lv[LM + 2], Ls[LM + 2], Lt[LM + 2];
  double psa = ra.ptop, psb = ra.ptop, psc = ra.ptop, psd = ra.ptop;
  for (int k = L - 1; k >= 0; --k) {
    const long long kk = (long long)k * S;
    psa = psa + dp[oa + kk];
    psb = psb + dp[ob + kk];
    psc = psc + dp[oc + kk];
    psd = psd + dp[od + kk];
  }
  double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop;
  for (int k = L + 1; k >= 1; --k) {
    if (k <= L) {
      const long long kk = (long long)(k - 1) * S;
      pa = pa + dp[oa + kk];
      pb = pb + dp[ob + kk];
      pc = pc + dp[oc + kk];
      pd = pd + dp[od + kk];
    }
    sc[k] = C7_12 * (pa + pb) - C1_12 * (pc + pd);
    dc[k] = dcoord(ra, L, k, psa, psb, psc, psd);
  }
  for (int k = 1; k <= L; ++k) {
    var[k] = f[oa + (long long)(k - 1) * S];
    Ld[k] = lr[oa + (long long)(k - 1) * S];
  }
  for (int k = 0; k <= L + 1; ++k) {
    Lv[k] = 0.;
    Ls[k] = 0.;
    Lt[k] = 0.;
  }
  remap_column_adj_full<LM>(L, var, Ld, sc, dc, Lv, Ls, Lt);
  for (int k = 1; k <= L; ++k) lf[oa + (long long)(k - 1) * S] += Lv[k];
  double Z = 0.;
  for (int k = 1; k <= L; ++k) Z += ra.bk[k - 1] * Lt[k];
  double P = 0.;
  for (int m = 1; m <= L; ++m) {
    P += Ls[m];
    const double v = P + Z;
    if (v == 0.) continue;
    const long long kk = (long long)(m - 1) * S;
    atomicAdd(lam_dp + oa + kk, C7_12 * v);
    atomicAdd(lam_dp + ob + kk, C7_12 * v);
    atomicAdd(lam_dp + oc + kk, -C1_12 * v);
    atomicAdd(lam_dp + od + kk, -C1_12 * v);
  }
}

// Adjoint of k_remap_winds: the adjoints of urem, vrem in; those of ud, vd
// (the face column's own) and of dp (the four columns of its interface
// pressures) added.  One warp per group of G face columns; a grid-stride
// loop over the groups.
template <int LM>
__global__ void __launch_bounds__(32 * NWB) k_remap_winds_adj_w(Geom g, RemapArgs ra, const double* __restrict__ dp,
                                                                 const double* __restrict__ ud,
                                                                 const double* __restrict__ vd,
                                                                 const double* __restrict__ lam_ur,
                                                                 const double* __restrict__ lam_vr, double* lam_dp,
                                                                 double* lam_ud, double* lam_vd) {
  __shared__ Work<LM> wsm[NWB];
  Work<LM>& sm = wsm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int L = g.L;
  const long long S = g.S;
  const long long nq = 2LL * (g.nx + 2) * (g.ny + 2);
  const long long ngroups = (nq + G - 1) / G;
  const long long gw = (long long)blockIdx.x * NWB + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * NWB;
  for (long long grp = gw; grp < ngroups; grp += nw) {
    // ---------------- phase 1: a lane per face column
    if (lane < G) {
      int i, j, dir;
      long long oa, ob, oc, od;
      int fl = 0;
      if (face(g, grp * G + lane, i, j, dir, oa, ob, oc, od)) {
        const double* f = dir == 0 ? ud : vd;
        const double* lr = dir == 0 ? lam_ur : lam_vr;
        bool any = false;
        for (int k = 0; k < L; ++k) any = any || lr[oa + (long long)k * S] != 0.;
        if (any) {
          fl = 1;
          // the forward's coordinate sums and elimination (remap_winds_at)
          double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop, prev = 0.;
          int kc = L + 2, kv = L + 1;
          bool mono = true;
          auto cnext = [&]() {
            --kc;
            if (kc <= L) {
              const long long kk = (long long)(kc - 1) * S;
              pa = pa + dp[oa + kk];
              pb = pb + dp[ob + kk];
              pc = pc + dp[oc + kk];
              pd = pd + dp[od + kk];
            }
            const double c = C7_12 * (pa + pb) - C1_12 * (pc + pd);
            if (kc <= L) mono = mono && (prev <= c);
            prev = c;
            return c;
          };
          auto vnext = [&]() {
            --kv;
            return f[oa + (long long)(kv - 1) * S];
          };
          const ColArr csc{sm.sc[lane], 1}, clv{sm.lvb[lane], 1}, cgam{sm.gam[lane], 1};
          ppm_eliminate<true>(L, cnext, vnext, csc, clv, cgam);
          double dprev = dcoord(ra, L, 1, pa, pb, pc, pd);
          for (int k = 2; k <= L + 1; ++k) {
            const double d = dcoord(ra, L, k, pa, pb, pc, pd);
            mono = mono && (d <= dprev);
            dprev = d;
          }
          sm.ps[lane][0] = pa;
          sm.ps[lane][1] = pb;
          sm.ps[lane][2] = pc;
          sm.ps[lane][3] = pd;
          if (mono) {
            fl |= 2;
            // forward substitution in place, as PPMLayers forms it
            double* b = sm.lvb[lane];
            const double* gm = sm.gam[lane];
            double lvf = b[1];
            for (int jj = 2; jj <= L + 1; ++jj) {
              const double fv = b[jj] - gm[jj - 1] * lvf;
              b[jj] = fv;
              lvf = fv;
            }
          }
        }
      }
      sm.flag[lane] = fl;
    }
    __syncwarp();
    // ---------------- phase 2: the warp on one column at a time
    for (int c = 0; c < G; ++c) {
      const int fl = sm.flag[c];
      if (!(fl & 1)) continue;
      int i, j, dir;
      long long oa, ob, oc, od;
      face(g, grp * G + c, i, j, dir, oa, ob, oc, od);
      const double* f = dir == 0 ? ud : vd;
      const double* lr = dir == 0 ? lam_ur : lam_vr;
      double* lf = dir == 0 ? lam_ud : lam_vd;
      if (!(fl & 2)) {
        if (lane == 0) winds_adj_column_full<LM>(g, ra, dp, f, lr, lam_dp, lf, oa, ob, oc, od);
        __syncwarp();
        continue;
      }
      const double* sc = sm.sc[c];
      const double* gm = sm.gam[c];
      const double* lb = sm.lvb[c];
      const double pa = sm.ps[c][0], pb = sm.ps[c][1], pc = sm.ps[c][2], pd = sm.ps[c][3];
      for (int k = lane; k <= L + 1; k += 32) {
        const bool lay = k >= 1 && k <= L;
        sm.var[k] = lay ? f[oa + (long long)(k - 1) * S] : 0.;
        sm.Ld[k] = lay ? lr[oa + (long long)(k - 1) * S] : 0.;
        sm.dc[k] = k >= 1 ? dcoord(ra, L, k, pa, pb, pc, pd) : 0.;
        sm.Lsrc[k] = 0.;
        sm.Ltop[k] = 0.;
        sm.Lbtm[k] = 0.;
        sm.Lsc[k] = 0.;
        sm.Ldc[k] = 0.;
      }
      __syncwarp();
      // limited interface values (src/mod_remap.f90:319-339), as PPMLayers
      for (int jj = lane + 1; jj <= L + 1; jj += 32) {
        double cv = lb[jj];
        if (jj >= 2 && jj <= L) {
          const double vk = sm.var[jj - 1], vk1 = sm.var[jj];
          if (jj == L) {
            cv = mn(cv, mx(vk1, vk));
            cv = mx(cv, mn(vk1, vk));
          }
          if (jj == 2) {
            cv = mn(cv, mx(vk1, vk));
            cv = mx(cv, mn(vk1, vk));
          }
          if (jj >= 3) {
            const double lo = mn(vk, vk1), hi = mx(vk, vk1);
            if (jj == L || gm[jj + 1] * gm[jj - 1] > 0) {
              cv = mn(cv, hi);
              cv = mx(cv, lo);
            } else if (gm[jj + 1] > 0) {
              cv = mx(cv, lo);
            } else {
              cv = mn(cv, hi);
            }
          }
        }
        sm.lvc[jj] = cv;
      }
      __syncwarp();
      // edges and curvature of each layer (:340-354)
      for (int k = lane + 1; k <= L; k += 32) {
        const double vk = sm.var[k];
        double top = sm.lvc[k + 1], btm = sm.lvc[k];
        if (k >= 3) {
          const double gk1 = gm[k - 1];
          double pmp1 = vk - 2. * gk1;
          double lac1 = pmp1 + 1.5 * gm[k - 2];
          top = mn(mx(top, mn3(vk, pmp1, lac1)), mx3(vk, pmp1, lac1));
          pmp1 = vk + 2. * gm[k];
          lac1 = pmp1 - 1.5 * gk1;
          btm = mn(mx(btm, mn3(vk, pmp1, lac1)), mx3(vk, pmp1, lac1));
        }
        sm.top[k] = top;
        sm.btm[k] = btm;
        sm.curv[k] = 6. * vk - 3. * (top + btm);
      }
      __syncwarp();
      // pair integrals (:188-280), a lane per destination layer m
      for (int m = lane + 1; m <= L; m += 32) {
        const double ldst = sm.Ld[m];
        if (ldst == 0.) continue;
        const double d0 = sm.dc[m], d1 = sm.dc[m + 1];
        // the merge's first source layer: the lowest k with sc(k+1) < dc(m)
        int lo = 1, hi = L + 1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (sc[mid + 1] < d0) hi = mid;
          else lo = mid + 1;
        }
        double ldm = 0., ldm1 = 0.;
        const double ddst = d1 - d0;
        for (int k = lo; k <= L && sc[k] > d1; ++k) {
          const double sk = sc[k], sk1 = sc[k + 1];
          const double btm = sm.btm[k], top = sm.top[k], curv = sm.curv[k], vk = sm.var[k];
          const double dsrc = sk1 - sk;
          const double s1 = (d0 - sk) / dsrc;
          const double s2 = (d1 - sk) / dsrc;
          const double IF = dsrc / ddst;
          const double tmp3 = 2. * s1 * s1;
          double Ls1 = 0., Ls2 = 0., LIF = 0., Lb = 0., Lt = 0., Lcv = 0., Lv = 0.;
          if (d1 <= sk1 && sk1 < d0 && d0 < sk) {
            const double t1 = s1 - 1., t2 = s1 + 1.;
            const double A = 3. * (btm * t1 - top * t2) + curv * (tmp3 - t2);
            const double fa = t1 / 6. * IF * ldst;
            Lb += fa * 3. * t1;
            Lt -= fa * 3. * t2;
            Lcv += fa * (tmp3 - t2);
            LIF += t1 / 6. * A * ldst;
            Ls1 += (A / 6. * IF + t1 / 6. * IF * (3. * (btm - top) + curv * (4. * s1 - 1.))) * ldst;
          }
          if (sk1 < d1 && d1 < sk && sk <= d0) {
            const double B = btm * (2. - s2) + s2 * (top + curv * (1. - C2_3 * s2));
            const double fb = s2 / 2. * IF * ldst;
            Lb += fb * (2. - s2);
            Lt += fb * s2;
            Lcv += fb * s2 * (1. - C2_3 * s2);
            LIF += s2 / 2. * B * ldst;
            Ls2 += (.5 * B * IF + s2 / 2. * IF * (-btm + top + curv * (1. - 2. * C2_3 * s2))) * ldst;
          }
          if (d1 <= sk1 && sk <= d0) {
            Lv += IF * ldst;
            LIF += vk * ldst;
          }
          if (sk1 < d1 && d0 < sk) {
            const double t1 = s1 + s2;
            const double Cc = 3. * (btm * (t1 - 2.) - top * t1) + curv * (tmp3 + t1 * (2. * s2 - 3.));
            const double fc = (s1 - s2) / 6. * IF * ldst;
            Lb += fc * 3. * (t1 - 2.);
            Lt -= fc * 3. * t1;
            Lcv += fc * (tmp3 + t1 * (2. * s2 - 3.));
            LIF += (s1 - s2) / 6. * Cc * ldst;
            const double dC1 = 3. * (btm - top) + curv * (4. * s1 + 2. * s2 - 3.);
            const double dC2 = 3. * (btm - top) + curv * (2. * s2 - 3. + 2. * t1);
            Ls1 += (Cc * IF / 6. + (s1 - s2) / 6. * IF * dC1) * ldst;
            Ls2 += (-Cc * IF / 6. + (s1 - s2) / 6. * IF * dC2) * ldst;
          }
          // curvature = 6 var - 3 (top + btm)
          Lv += 6. * Lcv;
          atomicAdd(&sm.Lsrc[k], Lv);
          atomicAdd(&sm.Ltop[k], Lt - 3. * Lcv);
          atomicAdd(&sm.Lbtm[k], Lb - 3. * Lcv);
          const double Ldsrc = -(Ls1 * s1 + Ls2 * s2) / dsrc + LIF / ddst;
          ldm += Ls1 / dsrc + LIF * IF / ddst;
          ldm1 += Ls2 / dsrc - LIF * IF / ddst;
          atomicAdd(&sm.Lsc[k], -(Ls1 + Ls2) / dsrc - Ldsrc);
          atomicAdd(&sm.Lsc[k + 1], Ldsrc);
        }
        atomicAdd(&sm.Ldc[m], ldm);
        atomicAdd(&sm.Ldc[m + 1], ldm1);
      }
      __syncwarp();
      // ---- adjoint of vertical_ppm (:287-356)
      for (int k = lane; k <= L + 1; k += 32) sm.Lgam[k] = 0.;
      __syncwarp();
      // Huynh edge limiters (:340-352)
      for (int k = lane + 2; k <= L - 1; k += 32) {
        double lt = sm.Ltop[k + 1];
        const double vk1 = sm.var[k + 1];
        double lv = 0.;
        if (lt != 0.) {
          const double pmp1 = vk1 - 2. * gm[k];
          const double lac1 = pmp1 + 1.5 * gm[k - 1];
          lt = edge_clamp_adj_at(sm.lvc[k + 2], vk1, pmp1, lac1, lt, lv, sm.Lgam, k, -2., k - 1, 1.5);
        }
        double lbt = sm.Lbtm[k + 1];
        if (lbt != 0.) {
          const double pmp1 = vk1 + 2. * gm[k + 1];
          const double lac1 = pmp1 - 1.5 * gm[k];
          lbt = edge_clamp_adj_at(sm.lvc[k + 1], vk1, pmp1, lac1, lbt, lv, sm.Lgam, k + 1, 2., k, -1.5);
        }
        sm.Ltop[k + 1] = lt;
        sm.Lbtm[k + 1] = lbt;
        if (lv != 0.) atomicAdd(&sm.Lsrc[k + 1], lv);
      }
      __syncwarp();
      // the interface values' adjoint: top of layer j-1 and bottom of layer j
      for (int jj = lane; jj <= L + 1; jj += 32) {
        double v = 0.;
        if (jj >= 2) v = v + sm.Ltop[jj - 1];
        if (jj >= 1 && jj <= L) v = v + sm.Lbtm[jj];
        sm.LL[jj] = v;
      }
      __syncwarp();
      // interface-value limiters (:319-339): each interface's chain of clamps, reversed
      for (int jj = lane + 2; jj <= L; jj += 32) {
        bool is_min[6];
        double bound[6];
        int vsel[6];
        int n = 0;
        auto min_hi = [&](int p, int q) {  // x = mn(x, mx(var[p], var[q]))
          is_min[n] = true;
          const bool t = sm.var[p] < sm.var[q];
          bound[n] = t ? sm.var[q] : sm.var[p];
          vsel[n] = t ? q : p;
          ++n;
        };
        auto max_lo = [&](int p, int q) {  // x = mx(x, mn(var[p], var[q]))
          is_min[n] = false;
          const bool t = sm.var[q] < sm.var[p];
          bound[n] = t ? sm.var[q] : sm.var[p];
          vsel[n] = t ? q : p;
          ++n;
        };
        if (jj == L) {
          min_hi(L, L - 1);
          max_lo(L, L - 1);
        }
        if (jj == 2) {
          min_hi(2, 1);
          max_lo(2, 1);
        }
        if (jj >= 3) {
          const int k = jj - 1;
          if (k + 2 > L || gm[k + 2] * gm[k] > 0) {
            min_hi(k, k + 1);
            max_lo(k, k + 1);
          } else if (gm[k + 2] > 0) {
            max_lo(k, k + 1);
          } else {
            min_hi(k, k + 1);
          }
        }
        bool sel[6];
        double x = lb[jj];
        for (int t = 0; t < n; ++t) {
          sel[t] = is_min[t] ? (bound[t] < x) : (x < bound[t]);
          if (sel[t]) x = bound[t];
        }
        double lam = sm.LL[jj];
        for (int t = n - 1; t >= 0 && lam != 0.; --t)
          if (sel[t]) {
            atomicAdd(&sm.Lsrc[vsel[t]], lam);
            lam = 0.;
          }
        sm.LL[jj] = lam;
      }
      __syncwarp();
      // back substitution (:317-318): LL(k-1) -= gam(k-1) LL(k), k = L+1..2,
      // a backward chain over i = L..1
      chain(
          L, sm.LL[L + 1], [&](int p) { return L - p; }, [&](int ii) { return Af{sm.LL[ii], -gm[ii]}; },
          [&](int ii, double y) { sm.LL[ii] = y; });
      for (int ii = lane + 1; ii <= L; ii += 32) sm.Lgam[ii] -= lb[ii] * sm.LL[ii + 1];
      __syncwarp();
      // the values before the forward substitution, lv(k) = lvb(k) + gam(k-1) lvb(k-1)
      auto lvs = [&](int k) { return k == 1 ? lb[1] : lb[k] + gm[k - 1] * lb[k - 1]; };
      // first interface value (:314-316); a2 is the alpha of the elimination's last pass
      if (lane == 0) {
        const double a2 = (sc[3] - sc[2]) / (sc[2] - sc[1]);
        const double b0 = 1. + a2 * (1.5 + a2);
        const double D1 = a2 * (.5 + a2) - b0 * gm[1];
        const double LN1 = sm.LL[1] / D1, LD1 = -lvs(1) / D1 * sm.LL[1];
        atomicAdd(&sm.Lsrc[1], 2. * a2 * (1. + a2) * LN1);
        atomicAdd(&sm.Lsrc[2], LN1);
        double Lb0 = -lvs(2) * LN1;
        sm.LL[2] -= b0 * LN1;
        double La2 = (2. + 4. * a2) * sm.var[1] * LN1 + (.5 + 2. * a2) * LD1;
        Lb0 -= gm[1] * LD1;
        sm.Lgam[1] -= b0 * LD1;
        La2 += (1.5 + 2. * a2) * Lb0;
        sm.La2 = La2;
      }
      __syncwarp();
      // elimination (:306-313), k = 2..L: the LL chain LL(k+1) -= LL(k) / beta(k),
      // then the gam chain gam_adj(k) += (gam(k-1) gam_adj(k-1) + lv(k) LL(k)) / beta(k)
      auto beta = [&](int k) {
        const double ak = (sc[k + 1] - sc[k]) / (sc[k] - sc[k - 1]);
        return 2. + 2. * ak - gm[k];
      };
      chain(
          L - 1, sm.LL[2], [&](int p) { return 3 + p; }, [&](int ii) { return Af{sm.LL[ii], -1. / beta(ii - 1)}; },
          [&](int ii, double y) { sm.LL[ii] = y; });
      chain(
          L - 1, sm.Lgam[1], [&](int p) { return 2 + p; },
          [&](int k) {
            const double be = beta(k);
            return Af{sm.Lgam[k] + lvs(k) / be * sm.LL[k], gm[k - 1] / be};
          },
          [&](int k, double y) { sm.Lgam[k] = y; });
      for (int k = lane + 2; k <= L; k += 32) {
        const double nn = sc[k + 1] - sc[k], dd = sc[k] - sc[k - 1];
        const double ak = nn / dd;
        const double bek = 2. + 2. * ak - gm[k];
        const double lg1 = sm.Lgam[k - 1];
        double La = (k == 2) ? sm.La2 : 0.;
        La += lg1 / bek;
        double Lbe = -gm[k - 1] / bek * lg1;
        const double LN = sm.LL[k] / bek;
        Lbe -= lvs(k) / bek * sm.LL[k];
        atomicAdd(&sm.Lsrc[k], 3. * LN);
        atomicAdd(&sm.Lsrc[k - 1], 3. * ak * LN);
        La += 3. * sm.var[k - 1] * LN;
        La += 2. * Lbe;
        const double Ld = -ak / dd * La;
        atomicAdd(&sm.Lsc[k + 1], La / dd);
        atomicAdd(&sm.Lsc[k], -La / dd + Ld);
        atomicAdd(&sm.Lsc[k - 1], -Ld);
      }
      __syncwarp();
      // top interface value and gam(nlay) (:301-305)
      if (lane == 0) {
        const double nn = sc[L] - sc[L - 1], dd = sc[L + 1] - sc[L];
        const double aL = nn / dd;
        const double bL = aL * (.5 + aL);
        const double LNL = sm.LL[L + 1] / bL;
        double LbL = -lvs(L + 1) / bL * sm.LL[L + 1];
        sm.Lsrc[L] += 2. * aL * (1. + aL) * LNL;
        sm.Lsrc[L - 1] += LNL;
        double LaL = (2. + 4. * aL) * sm.var[L] * LNL;
        const double LG = sm.Lgam[L] / bL;
        LbL -= gm[L] / bL * sm.Lgam[L];
        LaL += (1.5 + 2. * aL) * LG;
        LaL += (.5 + 2. * aL) * LbL;
        sm.Lsc[L] += LaL / dd;
        sm.Lsc[L - 1] -= LaL / dd;
        const double Ldd = -aL / dd * LaL;
        sm.Lsc[L + 1] += Ldd;
        sm.Lsc[L] -= Ldd;
      }
      __syncwarp();
      // outputs: the wind adjoint; the dp adjoints of the four columns through
      // sc(k) = 7/12 (pa + pb) - 1/12 (pc + pd), p(k) = ptop + sum of dp(m >= k),
      // and dc(k) = 7/12 (ta + tb) - 1/12 (tc + td), t = ak + bk (ps - ptop)
      double z = 0.;
      for (int k = lane + 1; k <= L; k += 32) {
        lf[oa + (long long)(k - 1) * S] += sm.Lsrc[k];
        z += ra.bk[k - 1] * sm.Ldc[k];
      }
      const double Z = warp_sum(z);
      chain(
          L, 0., [&](int p) { return 1 + p; }, [&](int m) { return Af{sm.Lsc[m], 1.}; },
          [&](int m, double P) {
            const double v = P + Z;
            if (v != 0.) {
              const long long kk = (long long)(m - 1) * S;
              atomicAdd(lam_dp + oa + kk, C7_12 * v);
              atomicAdd(lam_dp + ob + kk, C7_12 * v);
              atomicAdd(lam_dp + oc + kk, -C1_12 * v);
              atomicAdd(lam_dp + od + kk, -C1_12 * v);
            }
          });
    }
    __syncwarp();
  }
}

}  // namespace rwa
}  // namespace atm
