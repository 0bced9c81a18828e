// Column-marching sweep kernels of the B200 dynamical core.
//
// A warp owns a strip of one layer: 32 consecutive x columns (lane = column)
// of which the middle 26 are outputs (3 halo columns on each side feed the
// PPM stencils), and TYS output rows that it walks through in ascending y.
// Each lane keeps the y-direction stencil values of its column (the last
// few rows of every stage) in registers, so that every stage of the
// reference's layer loop is evaluated once per cell instead of once per
// cell of every overlapping tile halo; x-direction neighbours come from the
// neighbouring lanes by warp shuffles.  No shared memory and no block-wide
// barrier: the warps of a block are independent.
//
// Each iteration loads the inputs of the next row before working on the
// current one, so that the loads' latency overlaps a row of arithmetic.
//
// The stage formulas, index shifts and evaluation order are those of the
// tile kernels (atm_sweeps.cuh) and of the reference, so FP64 instances
// are bit-identical to them (the oracle's parity tests passed with the
// FP64 form built on these kernels).  The mixed form launches its four
// sweeps as marching kernels; in FP64 the tiles are faster (the marching
// FP64 sweeps execute about as many instructions per cell, at 140-174
// registers a thread and 17 % warps active), so the FP64 form keeps them.
// The persistent ensemble kernel runs the same strip functions with plain
// loads (RO = false), as it reads fields that it wrote earlier in the same
// launch.
#pragma once

#include <type_traits>

#include "atm_kernels.cuh"

namespace atm {

constexpr int MW = 32;              // lanes (columns) of a strip
constexpr int MXH = 3;              // halo columns on each side
constexpr int MOUT = MW - 2 * MXH;  // output columns of a strip
constexpr int MWARPS = 4;           // independent strips (warps) per block
// blocks per SM the register budget of the marching kernels is set for: 4
// (16 warps), which the FP32 sweeps reach without spilling (at most 128
// registers; the C-momentum sweep would take 131 and fall to 3 blocks)
#ifndef ATM_MARCH_MINB
#define ATM_MARCH_MINB 4
#endif

template <typename T>
__device__ __forceinline__ T shfl_at(T v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}
template <typename T>
__device__ __forceinline__ T shfl_dn(T v, int d) {
  return __shfl_down_sync(0xffffffffu, v, d);
}
template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) {
  return __shfl_up_sync(0xffffffffu, v, d);
}

// a * b + c.  The mixed form's translation unit is compiled without
// contraction (so that every kernel inlining these functions rounds them
// alike), and its FP32 arithmetic asks for its fused operations here; in
// FP64 the unfused expression, whose value equals the formula as written
// (an IEEE sum does not depend on the order of its two operands).
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmadd(double a, double b, double c) { return a * b + c; }

// Edge anomalies of a cell from its value and neighbours (qm, q0, qp) and
// their monotone slopes (mm, m0, mp): the operations of edges_pre.
template <typename T, int V>
__device__ __forceinline__ void edges_v(T qm, T q0, T qp, T mm, T m0, T mp, T& eL, T& eR) {
  eL = fmadd(qm - q0, T(0.5), div_const<3>(mm - m0));
  eR = fmadd(qp - q0, T(0.5), div_const<3>(m0 - mp));
  if (V == PPM_CON || V == PPM_NN) {
    const T d0 = (qp - qm) * T(0.25);
    const T lim = T(2) * fab(d0);
    eL = -cpsign(mn(lim, fab(eL)), d0);
    eR = +cpsign(mn(lim, fab(eR)), d0);
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

// Upwind flux with Courant number c from the values and monotone slopes
// around the upwind cell (cell i-1 for c > 0, cell i otherwise): the
// operations of flux_pre.
template <typename T, int V>
__device__ __forceinline__ T flux_v(T c, T qm, T q0, T qp, T mm, T m0, T mp) {
  const T sa = fab(c);
  const T k1 = fmadd(T(-2), sa, T(1)) * (T(1) - sa);
  const T k2 = sa * (sa - T(1));
  T eL, eR;
  edges_v<T, V>(qm, q0, qp, mm, m0, mp, eL, eR);
  return (c > T(0)) ? fmadd(k2, eL, fmadd(k1, eR, q0)) : fmadd(k2, eR, fmadd(k1, eL, q0));
}

// Flux with the edge values of the upwind candidates given (PPM_CONSTRAINED):
// the operations of flux_con_pre.  qm, q0 are the values of cells i-1 and
// i, (eLm, eRm) and (eL0, eR0) their edges.
template <typename T>
__device__ __forceinline__ T flux_con_v(T c, T qm, T q0, T eLm, T eRm, T eL0, T eR0) {
  if ((T(3) * fab(eL0 + eR0) > fab(eL0 - eR0)) && (T(3) * fab(eLm + eRm) > fab(eLm - eRm)))
    return (c > T(0)) ? qm : q0;
  const T sa = fab(c);
  const T k1 = fmadd(T(-2), sa, T(1)) * (T(1) - sa);
  const T k2 = sa * (sa - T(1));
  return (c > T(0)) ? fmadd(k2, eLm, fmadd(k1, eRm, qm)) : fmadd(k2, eR0, fmadd(k1, eL0, q0));
}

__device__ __forceinline__ double slope_v(double qm, double q0, double qp) {
  double d, m;
  slopes(qm, q0, qp, d, m);
  return m;
}
__device__ __forceinline__ float slope_v(float qm, float q0, float qp) {
  float d, m;
  slopes(qm, q0, qp, d, m);
  return m;
}

// Row accessor of one level of a stored field: value at (x, y) of the
// level, zero outside the stored (halo-padded) array.  RO: no thread writes
// the field during the launch, so it is read through the read-only data
// path; the persistent ensemble kernel, whose later stages read what earlier
// stages of the same launch wrote, uses plain (coherent) loads.
template <typename E, bool RO = true>
struct Lev {
  const E* p;  // element (0, 0) of the level
  int P, nx, ny;
  __device__ __forceinline__ E operator()(int x, int y) const {
    if (x < -H || x >= nx + H || y < -H || y >= ny + H) return E(0);
    const E* a = p + (long long)y * P + x;
    if constexpr (RO) return __ldg(a);
    else return *a;
  }
};
template <bool RO = true, typename E>
__device__ __forceinline__ Lev<E, RO> level(const E* f, const Geom& g, int k) {
  return Lev<E, RO>{f + g.at(0, 0, k), g.P, g.nx, g.ny};
}

// ---------------------------------------------------------------- mass ----
// The C-grid (CGRID) or D-grid mass and potential-temperature sweep of one
// layer (src/mod_sw_dyn.f90:96-268 and 439-598), as k_mass2: S the state
// type, C the C-grid fields' type, T the sweep arithmetic.  Output region
// [lo, nx-1+hi] x [lo, ny-1+hi]; strips of TYS rows.
template <typename T, bool CGRID, typename S, typename C>
struct MassM {
  using UB = std::conditional_t<CGRID, S, C>;  // u, v inputs
  using O = std::conditional_t<CGRID, C, S>;   // outputs
};

template <typename T, int TYS, bool CGRID, typename S, typename C, bool RO = true>
__device__ __forceinline__ void mass_strip(Geom g, Consts c, const S* dp,
                                                         const S* pt,
                                                         const typename MassM<T, CGRID, S, C>::UB* u,
                                                         const typename MassM<T, CGRID, S, C>::UB* v,
                                                         const double* heat,
                                                         typename MassM<T, CGRID, S, C>::O* dpo,
                                                         typename MassM<T, CGRID, S, C>::O* pto, int lo,
                                                         int hi, int* nonfinite, int sx, int sy, int k) {
  using UB = typename MassM<T, CGRID, S, C>::UB;
  using O = typename MassM<T, CGRID, S, C>::O;
  constexpr int V = CGRID ? PPM_UNC : PPM_NN;
  constexpr bool SAME = std::is_same_v<S, T>;
  const int lane = threadIdx.x & (MW - 1);
  const int ox = lo + sx * MOUT;
  const int oy = lo + sy * TYS;
  const int xhi = g.nx - 1 + hi, yhi = g.ny - 1 + hi;
  if (ox > xhi) return;  // the whole warp is past the region
  const int x = ox - MXH + lane;
  const bool out_lane = lane >= MXH && lane < MXH + MOUT && x <= xhi;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  const T dxv = dtdx * T(c.vdx), dyv = dtdy * T(c.vdy), vdx = T(c.vdx), vdy = T(c.vdy);
  const auto fdp = level<RO>(dp, g, k), fpt = level<RO>(pt, g, k);
  const auto fu = level<RO>(u, g, k), fv = level<RO>(v, g, k);

  // register windows of the column, named by their row offset from the
  // newest row j of the current iteration
  T d4 = 0, d3 = 0, d2 = 0, d1 = 0, d0 = 0;       // dp(j-4 .. j)
  T p4 = 0, p3 = 0, p2 = 0, p1 = 0, p0 = 0;       // pt(j-4 .. j)
  T tx4 = 0, tx3 = 0, tx2 = 0, tx1 = 0, tx0 = 0;  // inner x sweep of dp, rows j-4 .. j
  T tp4 = 0, tp3 = 0, tp2 = 0, tp1 = 0, tp0 = 0;  // ... of pt
  T my4 = 0, my3 = 0, my2 = 0, my1 = 0;           // its monotone y slopes, rows j-4 .. j-1
  T mp4 = 0, mp3 = 0, mp2 = 0, mp1 = 0;
  T fy1 = 0, fy0 = 0, fq1 = 0, fq0 = 0;           // y fluxes of dp and pt at rows j-3, j-2
  T ld2 = 0, ld1 = 0, ld0 = 0, lq2 = 0, lq1 = 0, lq0 = 0;  // Laplacians of dp, pt at rows j-4 .. j-2
  T uc3 = 0, uc2 = 0, uc1 = 0, uc0 = 0;           // C-grid u at rows j-3 .. j
  T vc1 = 0, vc0 = 0;                             // C-grid v at rows j-3, j-2
  T su_x = 0, su_xm = 0;                          // D-grid u at (x, j), (x-1, j) (C grid)
  T sv_x = 0, sv_xp = 0;                          // D-grid v at (x, j-3), (x+1, j-3) (C grid)
  if constexpr (CGRID) {
    su_x = T(fu(x, oy - 3));
    su_xm = T(fu(x - 1, oy - 3));
    sv_x = T(fv(x, oy - 6));
    sv_xp = T(fv(x + 1, oy - 6));
  }
  bool bad = false;
  const int jend = min(oy + TYS, yhi + 1) + 3;
  S dn_p = fdp(x, oy - 3), pn_p = fpt(x, oy - 3);
  UB ua_p = CGRID ? fu(x, oy - 2) : fu(x, oy - 3), ub_p = CGRID ? fu(x - 1, oy - 2) : UB(0);
  UB va_p = fv(x, oy - 5), vb_p = CGRID ? fv(x + 1, oy - 5) : UB(0);
  for (int j = oy - 3; j < jend; ++j) {
    // ---- row j: inputs, C-grid u, the inner x sweep (mod_sw_dyn.f90:109-117, 176-185; 503-511)
    const S d_upd = fdp(x, j - 3), p_upd = fpt(x, j - 3);  // the update's state values of row j-3
    const T dn = T(dn_p), pn = T(pn_p);
    const UB ua_c = ua_p, ub_c = ub_p, va_c = va_p, vb_c = vb_p;
    dn_p = fdp(x, j + 1);
    pn_p = fpt(x, j + 1);
    if constexpr (CGRID) {
      ua_p = fu(x, j + 2);
      ub_p = fu(x - 1, j + 2);
      vb_p = fv(x + 1, j - 1);
    } else {
      ua_p = fu(x, j + 1);
    }
    va_p = fv(x, j - 1);
    T ucn;
    if constexpr (CGRID) {
      const T a = T(ua_c), b = T(ub_c);
      const T ub = T(.5) * (su_x + su_xm);
      ucn = T(.5) * (ub + T(.5) * (a + b));
      su_x = a;
      su_xm = b;
    } else {
      ucn = T(ua_c);
    }
    const T ucR = shfl_dn(ucn, 1);
    const T dL = shfl_up(dn, 1), dR = shfl_dn(dn, 1);
    const T pL = shfl_up(pn, 1), pR = shfl_dn(pn, 1);
    T txn, tpn;
    {
      const T cx0 = dtdx * ucn, cx1 = dtdx * ucR;
      const T den = T(1) / fmadd(-dtdx, ucR - ucn, T(1));
      T f0 = (cx0 > T(0)) ? dL : dn;
      T f1 = (cx1 > T(0)) ? dn : dR;
      txn = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, dn), dn);
      f0 = (cx0 > T(0)) ? pL : pn;
      f1 = (cx1 > T(0)) ? pn : pR;
      tpn = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, pn), pn);
    }
    // shift the windows to the new row
    d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = dn;
    p4 = p3; p3 = p2; p2 = p1; p1 = p0; p0 = pn;
    tx4 = tx3; tx3 = tx2; tx2 = tx1; tx1 = tx0; tx0 = txn;
    tp4 = tp3; tp3 = tp2; tp2 = tp1; tp1 = tp0; tp0 = tpn;
    uc3 = uc2; uc2 = uc1; uc1 = uc0; uc0 = ucn;
    // monotone y slope of row j-1 (ppm, :870-875)
    my4 = my3; my3 = my2; my2 = my1; my1 = slope_v(tx2, tx1, tx0);
    mp4 = mp3; mp3 = mp2; mp2 = mp1; mp1 = slope_v(tp2, tp1, tp0);
    // C-grid v of row j-2 (:109-117)
    T vcn;
    if constexpr (CGRID) {
      const T a = T(va_c), b = T(vb_c);
      const T vb = T(.5) * (a + sv_x);
      vcn = T(.5) * (vb + T(.5) * (b + sv_xp));
      sv_x = a;
      sv_xp = b;
    } else {
      vcn = T(va_c);
    }
    vc1 = vc0;
    vc0 = vcn;
    {  // outer y sweep (PPM) at the interface below row j-2; the upwind
       // cell's values selected first: one flux evaluation per lane
      const T cy = dtdx * vc0;
      const bool up = cy > T(0);
      fy1 = fy0;
      fq1 = fq0;
      fy0 = flux_v<T, V>(cy, up ? tx4 : tx3, up ? tx3 : tx2, up ? tx2 : tx1, up ? my4 : my3, up ? my3 : my2,
                         up ? my2 : my1) * cy;
      fq0 = flux_v<T, V>(cy, up ? tp4 : tp3, up ? tp3 : tp2, up ? tp2 : tp1, up ? mp4 : mp3, up ? mp3 : mp2,
                         up ? mp2 : mp1);
    }
    // Laplacians of row j-2 (:158-173)
    {
      const T dl = shfl_up(d2, 1), dr = shfl_dn(d2, 1);
      const T pl = shfl_up(p2, 1), pr = shfl_dn(p2, 1);
      ld2 = ld1; ld1 = ld0;
      lq2 = lq1; lq1 = lq0;
      ld0 = fmadd(d1 + d3, rdy2, fmadd(dr + dl, rdx2, T(-2.) * d2 * rdxy));
      lq0 = fmadd(p1 + p3, rdy2, fmadd(pr + pl, rdx2, T(-2.) * p2 * rdxy));
    }
    const int y = j - 3;
    if (y < oy) continue;  // warm-up rows of the strip (warp-uniform)
    // ---- row y: inner y sweep, its x slopes, the outer x sweep, the update
    T tyd, typ;
    {
      const T cy0 = dtdx * vc1, cy1 = dtdx * vc0;
      const T den = T(1) / fmadd(-dtdy, vc0 - vc1, T(1));
      T f0 = (cy0 > T(0)) ? d4 : d3;
      T f1 = (cy1 > T(0)) ? d3 : d2;
      tyd = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, d3), d3);
      f0 = (cy0 > T(0)) ? p4 : p3;
      f1 = (cy1 > T(0)) ? p3 : p2;
      typ = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, p3), p3);
    }
    const T mxd = slope_v(shfl_up(tyd, 1), tyd, shfl_dn(tyd, 1));
    const T mxp = slope_v(shfl_up(typ, 1), typ, shfl_dn(typ, 1));
    T fxd, fxp;
    {
      const T cx = dtdx * uc3;
      const int s0 = lane + ((cx > T(0)) ? -1 : 0);  // the upwind cell's lane
      fxd = flux_v<T, V>(cx, shfl_at(tyd, s0 - 1), shfl_at(tyd, s0), shfl_at(tyd, s0 + 1), shfl_at(mxd, s0 - 1),
                         shfl_at(mxd, s0), shfl_at(mxd, s0 + 1)) * cx;
      fxp = flux_v<T, V>(cx, shfl_at(typ, s0 - 1), shfl_at(typ, s0), shfl_at(typ, s0 + 1), shfl_at(mxp, s0 - 1),
                         shfl_at(mxp, s0), shfl_at(mxp, s0 + 1));
    }
    const T fxd1 = shfl_dn(fxd, 1), fxp1 = shfl_dn(fxp, 1);
    const T lxm = shfl_up(ld1, 1), lxp = shfl_dn(ld1, 1);
    const T qxm = shfl_up(lq1, 1), qxp = shfl_dn(lq1, 1);
    if (!out_lane || y > yhi) continue;
    // updates, mod_sw_dyn.f90:163-172,193-202,230-237,258-267 (C); 490-499,519-528,555-562,582-591 (D)
    O vo, qo;
    const long long o = g.at(x, y, k);
    if constexpr (SAME) {  // the reference's operations, in order
      const T d = d3;
      T vv = d - (fxd1 - fxd + dxv * (lxp - T(2.) * ld1 + lxm));
      vv = vv - (fy0 - fy1 + dyv * (ld0 - T(2.) * ld1 + ld2));
      T q = d * p3 - (fxp1 * fxd1 - fxp * fxd + vdx * ((qxp - lq1) * fxd1 - (lq1 - qxm) * fxd));
      q = q - (fq0 * fy0 - fq1 * fy1 + vdy * ((lq0 - lq1) * fy0 - (lq1 - lq2) * fy1));
      if (heat) q = q + dt * d * T(heat[o]);
      q = q / vv;
      vo = O(vv);
      qo = O(q);
    } else {
      // the same update in flux form: interface fluxes (advective plus
      // vorticity-damping) in the sweep type, their differences applied to
      // the state's type, so that mass and dp*pt telescope in S
      const T Fx0 = fmadd(dxv, ld1 - lxm, fxd), Fx1 = fmadd(dxv, lxp - ld1, fxd1);
      const T Fy0 = fmadd(dyv, ld1 - ld2, fy1), Fy1 = fmadd(dyv, ld0 - ld1, fy0);
      const T Hx0 = fmadd(vdx, lq1 - qxm, fxp) * fxd, Hx1 = fmadd(vdx, qxp - lq1, fxp1) * fxd1;
      const T Hy0 = fmadd(vdy, lq1 - lq2, fq1) * fy1, Hy1 = fmadd(vdy, lq0 - lq1, fq0) * fy0;
      const S d = d_upd;
      const S vv = d - ((S(Fx1) - S(Fx0)) + (S(Fy1) - S(Fy0)));
      S q = d * p_upd - ((S(Hx1) - S(Hx0)) + (S(Hy1) - S(Hy0)));
      if (heat) q = q + S(c.dt) * d * S(heat[o]);
      q = q / vv;
      vo = O(vv);
      qo = O(q);
    }
    dpo[o] = vo;
    pto[o] = qo;
    const bool inside = x >= 0 && x < g.nx && y >= 0 && y < g.ny;
    bad = bad || (inside && !(finite_(vo) && finite_(qo)));
  }
  if (nonfinite) flag_nonfinite(nonfinite, bad);
}

// one warp per strip: blockIdx.x * MWARPS + warp across x, blockIdx.y
// across y, blockIdx.z the layer
template <typename T, int TYS, bool CGRID, typename S, typename C>
__global__ void __launch_bounds__(MW * MWARPS, ATM_MARCH_MINB) k_mass_m(Geom g, Consts c, const S* __restrict__ dp,
                                                         const S* __restrict__ pt,
                                                         const typename MassM<T, CGRID, S, C>::UB* __restrict__ u,
                                                         const typename MassM<T, CGRID, S, C>::UB* __restrict__ v,
                                                         const double* __restrict__ heat,
                                                         typename MassM<T, CGRID, S, C>::O* __restrict__ dpo,
                                                         typename MassM<T, CGRID, S, C>::O* __restrict__ pto, int lo,
                                                         int hi, int* nonfinite) {
  mass_strip<T, TYS, CGRID, S, C>(g, c, dp, pt, u, v, heat, dpo, pto, lo, hi, nonfinite, blockIdx.x * MWARPS + (threadIdx.x >> 5), blockIdx.y, blockIdx.z);
}

// ======================================================== C-grid momentum ==
// The C-grid momentum update of one layer (src/mod_sw_dyn.f90:294-414), as
// k_c_mom2: kinetic energy from PPM fluxes of the C-grid winds with the
// layer-nlay A-grid winds (:299-317), absolute vorticity (:319-323), the
// pressure-gradient force (:325-339) and the vorticity-flux updates of uc
// and vc (:344-412).  Outputs on the interior; strips of TYS rows.
template <typename T, int TYS, typename S, typename C, bool RO = true>
__device__ __forceinline__ void c_mom_strip(Geom g, Consts c, const S* ud,
                                                          const S* vd, const double* pkap,
                                                          const double* gz, C* uc,
                                                          C* vc, int sx, int sy, int k) {
  constexpr int UNC = PPM_UNC;
  const int lane = threadIdx.x & (MW - 1);
  const int ox = sx * MOUT;
  const int oy = sy * TYS;
  const int L = g.L;
  if (ox >= g.nx) return;  // the whole warp is past the region
  const int x = ox - MXH + lane;
  const bool out_lane = lane >= MXH && lane < MXH + MOUT && x < g.nx;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy), f = T(c.coriolis);
  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  const T vdx = T(c.vdx), vdy = T(c.vdy);
  const auto fud = level<RO>(ud, g, k), fvd = level<RO>(vd, g, k);
  const auto fuL = level<RO>(ud, g, L - 1), fvL = level<RO>(vd, g, L - 1);
  const auto fpk0 = level<RO>(pkap, g, k), fpk1 = level<RO>(pkap, g, k + 1);
  const auto fgz0 = level<RO>(gz, g, k), fgz1 = level<RO>(gz, g, k + 1);

  // register windows of the column, named by their row offset from the
  // newest row j of the iteration
  T u_x = T(fud(x, oy - 3)), u_xm = T(fud(x - 1, oy - 3));  // ud(x, j), ud(x-1, j)
  T v_x = T(fvd(x, oy - 4)), v_xp = T(fvd(x + 1, oy - 4));  // vd(x, j-1), vd(x+1, j-1)
  T uw3 = 0, uw2 = 0, uw1 = 0, uw0 = 0;           // ud(x, j-3 .. j)
  T vw4 = 0, vw3 = 0, vw2 = 0, vw1 = 0, vw0 = 0;  // vd(x, j-4 .. j)
  T a3 = 0, a2 = 0, a1 = 0, a0 = 0;               // C-grid u of this layer, rows j-3 .. j
  T b4 = 0, b3 = 0, b2 = 0, b1 = 0, b0 = 0;       // C-grid v, rows j-4 .. j
  T mv4 = 0, mv3 = 0, mv2 = 0, mv1 = 0;           // monotone y slopes of C-grid v, rows j-4 .. j-1
  T w4 = 0, w3 = 0, w2 = 0, w1 = 0, w0 = 0;       // absolute vorticity, rows j-4 .. j
  T t4 = 0, t3 = 0, t2 = 0, t1 = 0, t0 = 0;       // inner x sweep of the vorticity, rows j-4 .. j
  T mt4 = 0, mt3 = 0, mt2 = 0, mt1 = 0;           // its monotone y slopes, rows j-4 .. j-1
  T lp1 = 0, lp0 = 0;                             // Laplacian of the vorticity, rows j-3, j-2
  T ke1 = 0, ke0 = 0;                             // kinetic energy, rows j-4, j-3
  double pk0m = 0, pk1m = 0, gz0m = 0, gz1m = 0;  // pkap, gz at k and k+1, row j-4
  // layer-nlay ud at row y and vd at rows y-1, y of the first kinetic-energy row y = oy-1
  T uL1 = T(fuL(x, oy - 1)), vL2 = T(fvL(x, oy - 2)), vL1 = T(fvL(x, oy - 1));
  const int jend = min(oy + TYS, g.ny) + 3;
  S un_p = fud(x, oy - 2), unm_p = fud(x - 1, oy - 2), vn_p = fvd(x, oy - 3), vnp_p = fvd(x + 1, oy - 3);
  for (int j = oy - 3; j < jend; ++j) {
    // loads of row y = j-3 issued before this row's work
    const double pk0 = fpk0(x, j - 3), pk1 = fpk1(x, j - 3), gz0 = fgz0(x, j - 3), gz1 = fgz1(x, j - 3);
    const S uL0_r = fuL(x, j - 2), vL0_r = fvL(x, j - 2);
    // ---- row j: C-grid winds of the layer (:110-117), vorticity (:319-323),
    // inner x sweep of the vorticity (:353-367)
    const T un = T(un_p), unm = T(unm_p);
    const T vn = T(vn_p), vnp = T(vnp_p);
    un_p = fud(x, j + 2);
    unm_p = fud(x - 1, j + 2);
    vn_p = fvd(x, j + 1);
    vnp_p = fvd(x + 1, j + 1);
    const T ucn = T(.5) * (T(.5) * (u_x + u_xm) + T(.5) * (un + unm));
    const T vcn = T(.5) * (T(.5) * (vn + v_x) + T(.5) * (vnp + v_xp));
    const T vor = fmadd(vcn - shfl_up(vcn, 1), rdx, fmadd(-(ucn - a0), rdy, f));
    const T vl = shfl_up(vor, 1), vr = shfl_dn(vor, 1);
    T tun;
    {
      const T c0 = dtdx * u_xm, c1 = dtdx * u_x;
      const T den = T(1) / fmadd(-dtdx, u_x - u_xm, T(1));
      const T f0 = (c0 > T(0)) ? vl : vor;
      const T f1 = (c1 > T(0)) ? vor : vr;
      tun = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, vor), vor);
    }
    uw3 = uw2; uw2 = uw1; uw1 = uw0; uw0 = u_x;
    u_x = un;
    u_xm = unm;
    v_x = vn;
    v_xp = vnp;
    vw4 = vw3; vw3 = vw2; vw2 = vw1; vw1 = vw0; vw0 = vn;
    a3 = a2; a2 = a1; a1 = a0; a0 = ucn;
    b4 = b3; b3 = b2; b2 = b1; b1 = b0; b0 = vcn;
    w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = vor;
    t4 = t3; t3 = t2; t2 = t1; t1 = t0; t0 = tun;
    mv4 = mv3; mv3 = mv2; mv2 = mv1; mv1 = slope_v(b2, b1, b0);
    mt4 = mt3; mt3 = mt2; mt2 = mt1; mt1 = slope_v(t2, t1, t0);
    // Laplacian of the vorticity at row j-2
    lp1 = lp0;
    lp0 = fmadd(w1 + w3, rdy2, fmadd(shfl_dn(w2, 1) + shfl_up(w2, 1), rdx2, T(-2.) * w2 * rdxy));
    const int y = j - 3;
    if (y < oy - 1) continue;  // warm-up rows (warp-uniform)
    // ---- row y: kinetic energy (:299-317) with the layer-nlay A-grid winds
    // (:110-125 at k = nlay), recomputed where they are read
    const T uL0 = T(uL0_r), vL0 = T(vL0_r);
    T ken;
    {
      const T ub = T(.5) * (uL1 + shfl_up(uL1, 1));
      const T ucl = T(.5) * (ub + T(.5) * (uL0 + shfl_up(uL0, 1)));
      const T ua = T(.5) * (ucl + T(.25) * (shfl_dn(uL1, 1) + uL1 + shfl_dn(uL0, 1) + uL0));
      const T vb = T(.5) * (vL1 + vL2);
      const T vL1r = shfl_dn(vL1, 1);
      const T vcl = T(.5) * (vb + T(.5) * (vL1r + shfl_dn(vL2, 1)));
      const T va = T(.5) * (vcl + T(.25) * (vL0 + vL1 + shfl_dn(vL0, 1) + vL1r));
      const T cy = dtdy * va;
      const bool upy = cy > T(0);
      const T fy = flux_v<T, UNC>(cy, upy ? b4 : b3, upy ? b3 : b2, upy ? b2 : b1, upy ? mv4 : mv3,
                                  upy ? mv3 : mv2, upy ? mv2 : mv1);
      const T kv = va * fy;
      const T mux = slope_v(shfl_up(a3, 1), a3, shfl_dn(a3, 1));
      const T cx = dtdx * ua;
      const int s0 = lane + ((cx > T(0)) ? 0 : 1);  // the upwind cell's lane
      const T fx = flux_v<T, UNC>(cx, shfl_at(a3, s0 - 1), shfl_at(a3, s0), shfl_at(a3, s0 + 1),
                                  shfl_at(mux, s0 - 1), shfl_at(mux, s0), shfl_at(mux, s0 + 1));
      ken = T(.5) * fmadd(ua, fx, kv);
    }
    uL1 = uL0;
    vL2 = vL1;
    vL1 = vL0;
    ke1 = ke0;
    ke0 = ken;
    const double pk0l = shfl_up(pk0, 1), pk1l = shfl_up(pk1, 1), gz0l = shfl_up(gz0, 1), gz1l = shfl_up(gz1, 1);
    const double pk0d = pk0m, pk1d = pk1m, gz0d = gz0m, gz1d = gz1m;  // row y-1
    pk0m = pk0; pk1m = pk1; gz0m = gz0; gz1m = gz1;
    if (y < oy) continue;
    // ---- row y: inner y sweep of the vorticity (:388-397), its x slopes, the updates
    T tvn;
    {
      const T c0 = dtdx * vw4, c1 = dtdx * vw3;
      const T den = T(1) / fmadd(-dtdy, vw3 - vw4, T(1));
      const T f0 = (c0 > T(0)) ? w4 : w3;
      const T f1 = (c1 > T(0)) ? w3 : w2;
      tvn = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, w3), w3);
    }
    const T mtv = slope_v(shfl_up(tvn, 1), tvn, shfl_dn(tvn, 1));
    const T ke_l = shfl_up(ke0, 1);
    const T lp_r = shfl_dn(lp1, 1);
    const T udx = uw3, vdx_ = vw3;
    T fx;
    {
      const T cx = dtdx * udx;
      const int s0 = lane + ((cx > T(0)) ? 0 : 1);
      fx = flux_v<T, UNC>(cx, shfl_at(tvn, s0 - 1), shfl_at(tvn, s0), shfl_at(tvn, s0 + 1), shfl_at(mtv, s0 - 1),
                          shfl_at(mtv, s0), shfl_at(mtv, s0 + 1));
    }
    if (!out_lane || y >= g.ny) continue;
    const double pgx = ((pk0 - pk1l) * (gz0l - gz1) + (pk0l - pk1) * (gz1l - gz0)) / (pk0 - pk1l + pk0l - pk1);
    const double pgy = ((pk0 - pk1d) * (gz0d - gz1) + (pk0d - pk1) * (gz1d - gz0)) / (pk0 - pk1d + pk0d - pk1);
    T fy;
    {
      const T cy = dtdx * vdx_;
      const bool up = cy > T(0);
      fy = flux_v<T, UNC>(cy, up ? t4 : t3, up ? t3 : t2, up ? t2 : t1, up ? mt4 : mt3, up ? mt3 : mt2,
                          up ? mt2 : mt1);
    }
    const T u = fmadd(-dtdx, ke0 - ke_l - T(pgx), fmadd(dt, fmadd(vdy, lp0 - lp1, vdx_ * fy), a3));
    const T v = fmadd(-dtdy, ke0 - ke1 - T(pgy), fmadd(-dt, fmadd(vdx, lp_r - lp1, udx * fx), b3));
    const long long o = g.at(x, y, k);
    uc[o] = C(u);
    vc[o] = C(v);
  }
}

// one warp per strip: blockIdx.x * MWARPS + warp across x, blockIdx.y
// across y, blockIdx.z the layer
template <typename T, int TYS, typename S, typename C>
__global__ void __launch_bounds__(MW * MWARPS, ATM_MARCH_MINB) k_c_mom_m(Geom g, Consts c, const S* __restrict__ ud,
                                                          const S* __restrict__ vd, const double* __restrict__ pkap,
                                                          const double* __restrict__ gz, C* __restrict__ uc,
                                                          C* __restrict__ vc) {
  c_mom_strip<T, TYS, S, C>(g, c, ud, vd, pkap, gz, uc, vc, blockIdx.x * MWARPS + (threadIdx.x >> 5), blockIdx.y, blockIdx.z);
}

// ======================================================== D-grid momentum ==
// The D-grid momentum update of one layer (src/mod_sw_dyn.f90:634-771), as
// k_d_mom2: kinetic energy from constrained-PPM fluxes of ud, vd with the
// layer-nlay B-grid winds (:639-657, 441-444), vorticity (:659-663), the
// B-grid pressure-gradient force (:665-679), del^4 divergence damping
// (:682-702) and the vorticity-flux updates (:708-769).  Outputs on the
// interior; strips of TYS rows.
template <typename T, int TYS, typename S, typename C, bool RO = true>
__device__ __forceinline__ void d_mom_strip(Geom g, Consts c, const S* ud,
                                                          const S* vd, const C* uc,
                                                          const C* vc, const double* pkapb,
                                                          const double* gzb, S* udo,
                                                          S* vdo, int* nonfinite, int sx, int sy, int k) {
  constexpr int CON = PPM_CON;
  const int lane = threadIdx.x & (MW - 1);
  const int ox = sx * MOUT;
  const int oy = sy * TYS;
  const int L = g.L;
  if (ox >= g.nx) return;  // the whole warp is past the region
  const int x = ox - MXH + lane;
  const bool out_lane = lane >= MXH && lane < MXH + MOUT && x < g.nx;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy), f = T(c.coriolis);
  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  const T vdx = T(c.vdx), vdy = T(c.vdy), divdamp = T(c.divdamp);
  const auto fud = level<RO>(ud, g, k), fvd = level<RO>(vd, g, k);
  const auto fuL = level<RO>(uc, g, L - 1), fvL = level<RO>(vc, g, L - 1);
  const auto fuc = level<RO>(uc, g, k), fvc = level<RO>(vc, g, k);
  const auto fpb0 = level<RO>(pkapb, g, k), fpb1 = level<RO>(pkapb, g, k + 1);
  const auto fgb0 = level<RO>(gzb, g, k), fgb1 = level<RO>(gzb, g, k + 1);

  // register windows of the column, named by their row offset from the
  // newest row j of the iteration
  T s2 = 0, s1 = 0, s0 = T(fud(x, oy - 3));                     // ud(x, j-2 .. j)
  T v3 = 0, v2 = 0, v1 = 0, v0 = T(fvd(x, oy - 3));             // vd(x, j-3 .. j)
  T mv3 = 0, mv2 = 0, mv1 = 0;                                  // monotone y slopes of vd, rows j-3 .. j-1
  T lv3 = 0, rv3 = 0, lv2 = 0, rv2 = 0;                         // constrained edges of vd, rows j-3, j-2
  T q2 = 0, q1 = 0, q0 = 0;                                     // divergence, rows j-2 .. j
  T e3 = 0, e2 = 0, e1 = 0;                                     // its Laplacian, rows j-3 .. j-1
  T dd3 = 0, dd2 = 0;                                           // del^4 damping term, rows j-3, j-2
  T w4 = 0, w3 = 0, w2 = 0, w1 = 0;                             // vorticity, rows j-4 .. j-1
  T t4 = 0, t3 = 0, t2 = 0, t1 = 0;                             // inner x sweep of the vorticity, rows j-4 .. j-1
  T mt4 = 0, mt3 = 0, mt2 = 0;                                  // its monotone y slopes, rows j-4 .. j-2
  T lt4 = 0, rt4 = 0, lt3 = 0, rt3 = 0;                         // its constrained edges, rows j-4, j-3
  T ke3 = 0, ke2 = 0;                                           // kinetic energy, rows j-3, j-2
  T lp4 = 0, lp3 = 0, lp2 = 0;                                  // Laplacian of the vorticity, rows j-4 .. j-2
  T cu3 = 0, cu2 = T(fuL(x, oy - 5)), cu1 = T(fuL(x, oy - 4));  // layer-nlay uc, rows j-3 .. j-1
  T cv3 = 0, cv2 = T(fvL(x, oy - 5));                           // layer-nlay vc, rows j-3, j-2
  double pb0y = 0, pb1y = 0, gb0y = 0, gb1y = 0;                // pkapb, gzb at k, k+1, row j-3
  bool bad = false;
  const int jend = min(oy + TYS, g.ny) + 3;
  S sn_p = fud(x, oy - 2), vn_p = fvd(x, oy - 2);
  C cu_p = fuL(x, oy - 3), cv_p = fvL(x, oy - 4);
  for (int j = oy - 2; j < jend; ++j) {
    // loads of rows j-2 (pressure terms) and j-3 (the update) issued before this row's work
    const double pb0n = fpb0(x, j - 2), pb1n = fpb1(x, j - 2), gb0n = fgb0(x, j - 2), gb1n = fgb1(x, j - 2);
    const C svc_r = fvc(x, j - 3), suc_r = fuc(x, j - 3);
    const S uo_r = fud(x, j - 3), vo_r = fvd(x, j - 3);
    // ---- row j inputs; vorticity of row j-1 (:659-663), divergence of row j (:682-685)
    const T sn = T(sn_p), vn = T(vn_p);
    const C cu_c = cu_p, cv_c = cv_p;
    sn_p = fud(x, j + 1);
    vn_p = fvd(x, j + 1);
    cu_p = fuL(x, j);
    cv_p = fvL(x, j - 1);
    const T vorn = fmadd(shfl_dn(v0, 1) - v0, rdx, fmadd(-(sn - s0), rdy, f));
    const T dvn = fmadd(rdy, vn - v0, rdx * (sn - shfl_up(sn, 1)));
    s2 = s1; s1 = s0; s0 = sn;
    v3 = v2; v2 = v1; v1 = v0; v0 = vn;
    w4 = w3; w3 = w2; w2 = w1; w1 = vorn;
    q2 = q1; q1 = q0; q0 = dvn;
    cu3 = cu2; cu2 = cu1; cu1 = T(cu_c);
    cv3 = cv2; cv2 = T(cv_c);
    // monotone slope of vd at row j-1, its edges at row j-2 (:870-911)
    mv3 = mv2; mv2 = mv1; mv1 = slope_v(v2, v1, v0);
    lv3 = lv2; rv3 = rv2;
    edges_v<T, CON>(v3, v2, v1, mv3, mv2, mv1, lv2, rv2);
    // del^2 of the divergence at row j-1 (:688-692), del^4 at row j-2 (:695-702)
    e3 = e2; e2 = e1;
    e1 = fmadd(q0 + q2, rdy2, fmadd(shfl_dn(q1, 1) + shfl_up(q1, 1), rdx2, T(-2.) * q1 * rdxy));
    dd3 = dd2;
    dd2 = divdamp * (fmadd(e1 + e3, rdy2, fmadd(shfl_dn(e2, 1) + shfl_up(e2, 1), rdx2, T(-2.) * e2 * rdxy)));
    // inner x sweep of the vorticity at row j-1 with the layer-nlay Courant numbers (:708-722)
    {
      const T cR = shfl_dn(cu1, 1);
      const T c0 = dtdx * cu1, c1 = dtdx * cR;
      const T den = T(1) / fmadd(-dtdx, cR - cu1, T(1));
      const T wl = shfl_up(w1, 1), wr = shfl_dn(w1, 1);  // every lane takes part in the shuffles
      const T f0 = (c0 > T(0)) ? wl : w1;
      const T f1 = (c1 > T(0)) ? w1 : wr;
      t4 = t3; t3 = t2; t2 = t1;
      t1 = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, w1), w1);
    }
    mt4 = mt3; mt3 = mt2; mt2 = slope_v(t3, t2, t1);
    lt4 = lt3; rt4 = rt3;
    edges_v<T, CON>(t4, t3, t2, mt4, mt3, mt2, lt3, rt3);
    // Laplacian of the vorticity at row j-2
    lp4 = lp3; lp3 = lp2;
    lp2 = fmadd(w1 + w3, rdy2, fmadd(shfl_dn(w2, 1) + shfl_up(w2, 1), rdx2, T(-2.) * w2 * rdxy));
    // kinetic energy of row j-2 with PPM_CONSTRAINED (:639-657) and the
    // layer-nlay B-grid winds (:441-444)
    {
      const T ubL = T(.5) * (cu2 + cu3);
      const T vbL = T(.5) * (cv2 + shfl_up(cv2, 1));
      const T fy = flux_con_v(dtdy * vbL, v3, v2, lv3, rv3, lv2, rv2);
      const T kv = vbL * fy;
      const T sl = shfl_up(s2, 1), sr = shfl_dn(s2, 1);
      const T mux = slope_v(sl, s2, sr);
      T lux, rux;
      edges_v<T, CON>(sl, s2, sr, shfl_up(mux, 1), mux, shfl_dn(mux, 1), lux, rux);
      const T fx = flux_con_v(dtdx * ubL, sl, s2, shfl_up(lux, 1), shfl_up(rux, 1), lux, rux);
      ke3 = ke2;
      ke2 = T(.5) * fmadd(ubL, fx, kv);
    }
    const int y = j - 3;
    if (y >= oy) {
      // ---- row y: inner y sweep of the vorticity (:744-753), its x slopes and
      // edges, the updates of ud, vd (:724-738, 755-769) with the B-grid PGF
      T tv;
      {
        const T c0 = dtdx * cv3, c1 = dtdx * cv2;
        const T den = T(1) / fmadd(-dtdy, cv2 - cv3, T(1));
        const T f0 = (c0 > T(0)) ? w4 : w3;
        const T f1 = (c1 > T(0)) ? w3 : w2;
        tv = T(.5) * fmadd(den, fmadd(-rA, f1 - f0, w3), w3);
      }
      const T tl = shfl_up(tv, 1), tr = shfl_dn(tv, 1);
      const T mtv = slope_v(tl, tv, tr);
      T ltv, rtv;
      edges_v<T, CON>(tl, tv, tr, shfl_up(mtv, 1), mtv, shfl_dn(mtv, 1), ltv, rtv);
      const T fx = flux_con_v(dtdx * cu3, tl, tv, shfl_up(ltv, 1), shfl_up(rtv, 1), ltv, rtv);
      const T fy = flux_con_v(dtdx * cv3, t4, t3, lt4, rt4, lt3, rt3);
      const T ke_r = shfl_dn(ke3, 1), dd_r = shfl_dn(dd3, 1), lp_l = shfl_up(lp3, 1);
      const double pb0r = shfl_dn(pb0y, 1), pb1r = shfl_dn(pb1y, 1), gb0r = shfl_dn(gb0y, 1), gb1r = shfl_dn(gb1y, 1);
      if (out_lane && y < g.ny) {
        const double pgx = ((pb0r - pb1y) * (gb0y - gb1r) + (pb0y - pb1r) * (gb1y - gb0r)) / (pb0r - pb1y + pb0y - pb1r);
        const double pgy = ((pb0n - pb1y) * (gb0y - gb1n) + (pb0y - pb1n) * (gb1y - gb0n)) / (pb0n - pb1y + pb0y - pb1n);
        const long long o = g.at(x, y, k);
        const T svc = T(svc_r), suc = T(suc_r);
        S u, v;
        if constexpr (std::is_same_v<S, T>) {  // the reference's operations, in order
          u = uo_r + dt * (svc * fy + vdy * (lp3 - lp4)) - dtdx * (ke_r - ke3 - dd_r + dd3 - T(pgx));
          v = vo_r - dt * (suc * fx + vdx * (lp3 - lp_l)) - dtdy * (ke2 - ke3 - dd2 + dd3 - T(pgy));
        } else {  // the tendency in the sweep type added to the state's type
          const T du = fmadd(-dtdx, ke_r - ke3 - dd_r + dd3 - T(pgx), dt * fmadd(vdy, lp3 - lp4, svc * fy));
          const T dv = fmadd(-dtdy, ke2 - ke3 - dd2 + dd3 - T(pgy), -dt * fmadd(vdx, lp3 - lp_l, suc * fx));
          u = uo_r + S(du);
          v = vo_r + S(dv);
        }
        udo[o] = u;
        vdo[o] = v;
        bad = bad || !(finite_(u) && finite_(v));
      }
    }
    pb0y = pb0n; pb1y = pb1n; gb0y = gb0n; gb1y = gb1n;
  }
  flag_nonfinite(nonfinite, bad);
}

// one warp per strip: blockIdx.x * MWARPS + warp across x, blockIdx.y
// across y, blockIdx.z the layer
template <typename T, int TYS, typename S, typename C>
__global__ void __launch_bounds__(MW * MWARPS, ATM_MARCH_MINB) k_d_mom_m(Geom g, Consts c, const S* __restrict__ ud,
                                                          const S* __restrict__ vd, const C* __restrict__ uc,
                                                          const C* __restrict__ vc, const double* __restrict__ pkapb,
                                                          const double* __restrict__ gzb, S* __restrict__ udo,
                                                          S* __restrict__ vdo, int* nonfinite) {
  d_mom_strip<T, TYS, S, C>(g, c, ud, vd, uc, vc, pkapb, gzb, udo, vdo, nonfinite, blockIdx.x * MWARPS + (threadIdx.x >> 5), blockIdx.y, blockIdx.z);
}

}  // namespace atm
