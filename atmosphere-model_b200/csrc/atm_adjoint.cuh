// Adjoint kernels of the FP64 dynamical core.
//
// Each adjoint kernel takes the tile of its forward kernel (same TMA input
// boxes, same shared-memory intermediates recomputed with the same FP64
// operations, hence the same limiter and upwind branches), then walks the
// tile's stages in reverse: the adjoint of every intermediate lives in
// shared memory next to it, stages are separated by __syncthreads, and
// contributions that several points of one stage make to the same input
// are summed with shared-memory atomics.  The adjoints of the tile's input
// boxes are finally added to the global adjoint fields with atomics (tiles
// overlap in their halos).  The local derivatives of the PPM fluxes, edge
// limiters and monotone slopes are written out by hand, each following the
// branch the forward took: the derivative of the branch-frozen forward.
// Conventions at kinks (shared with the oracle's tangent-linear model):
// d|x|/dx = 0 at x = 0; d copysign(a, b)/da = sgn(a) * (sign of b);
// min/max pass the derivative of the argument they return.
//
// The reverse of each stage is cited by the forward lines it inverts; the
// forward is src/mod_sw_dyn.f90 (C grid :80-416, D grid :424-773).
#pragma once

#include "atm_sweeps.cuh"

namespace atm {

// threads per block of the adjoint tile kernels
constexpr int NTA = 256;
// The adjoint kernels also run the forward's merged region loops
// (regions() of atm_sweeps.cuh), which stride by NT: a block of any other
// size would visit some points twice and double their accumulations.
static_assert(NTA == NT, "adjoint blocks must have the forward kernels' NT threads");

// add to a shared-memory adjoint (p points into shared memory): a reduction
// in the shared state space, not a generic-address atomic
__device__ __forceinline__ void sadd(double* p, double v) {
  asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(smem_u32(p)), "d"(v) : "memory");
}

// zero the doubles of [a, b)
__device__ __forceinline__ void zero_smem(unsigned char* a, unsigned char* b) {
  double* p = reinterpret_cast<double*>(a);
  const int n = (int)((b - a) / 8);
  for (int i = threadIdx.x; i < n; i += NTA) p[i] = 0.;
}

// region loop of the adjoint kernels: body(x, y) over [x0, x0+W) x [y0, y0+Hh)
template <int W, int Hh, typename F>
__device__ __forceinline__ void aregion(int x0, int y0, F&& body) {
  for (int idx = threadIdx.x; idx < W * Hh; idx += NTA) {
    const int y = idx / W;
    const int x = idx - y * W;
    body(x0 + x, y0 + y);
  }
}

// ---- adjoint building blocks -------------------------------------------

// index (0, 1, 2) of the argument that mn3 / mx3 return
__device__ __forceinline__ int sel_mn3(double a, double b, double c) {
  int i = (b < a) ? 1 : 0;
  double t = (b < a) ? b : a;
  return (c < t) ? 2 : i;
}
__device__ __forceinline__ int sel_mx3(double a, double b, double c) {
  int i = (a < b) ? 1 : 0;
  double t = (a < b) ? b : a;
  return (t < c) ? 2 : i;
}

// mono = monotone slope of q(-s), q(0), q(+s) (src/mod_sw_dyn.f90:870-875):
// mono = copysign(mn3(|dqi|, dmin, dmax), dqi) with dqi = (q(+s) - q(-s))/4,
// dmin = q0 - mn3(q(+s), q0, q(-s)), dmax = mx3(q(+s), q0, q(-s)) - q0;
// the derivative follows the argument each mn3/mx3 returns
__device__ __forceinline__ void slope_adj(const double* q, int s, double lam, double* lq, int ls) {
  if (lam == 0.) return;
  const double qm = q[-s], q0 = q[0], qp = q[s];
  const double dqi = (qp - qm) * 0.25;
  const double A = fabs(dqi);
  const double B = q0 - mn3(qp, q0, qm);
  const double C = mx3(qp, q0, qm) - q0;
  const int sel = sel_mn3(A, B, C);
  const double m3 = sel == 0 ? A : (sel == 1 ? B : C);
  if (!(m3 > 0.)) return;
  const double l = (signbit(dqi) ? -lam : lam);
  double am = 0., a0 = 0., ap = 0.;
  if (sel == 0) {
    const double gq = (dqi > 0. ? .25 : -.25) * l;
    ap += gq;
    am -= gq;
  } else if (sel == 1) {
    a0 += l;
    const int j = sel_mn3(qp, q0, qm);
    if (j == 0) ap -= l; else if (j == 1) a0 -= l; else am -= l;
  } else {
    a0 -= l;
    const int j = sel_mx3(qp, q0, qm);
    if (j == 0) ap += l; else if (j == 1) a0 += l; else am += l;
  }
  if (am != 0.) sadd(lq - ls, am);
  if (a0 != 0.) sadd(lq, a0);
  if (ap != 0.) sadd(lq + ls, ap);
}

// F = flux_pre<PPM_UNC>(q, mono, c), by hand: with u the upwind cell,
// eL = (q(u-1) - q(u))/2 + (m(u-1) - m(u))/3, eR = (q(u+1) - q(u))/2 + (m(u) - m(u+1))/3,
// F = q(u) + k1 eR + k2 eL (c > 0) or q(u) + k1 eL + k2 eR, k1 = (1-2s)(1-s),
// k2 = s(s-1), s = |c|.  Adds lamF * dF/d(q, mono) to lq, lm (spacings
// slq, slm around cell i) and lamF * dF/dc to lamc; returns F.
__device__ __forceinline__ double flux_unc_adj(const double* q, int sq, const double* mono, int sm, double c,
                                               double lamF, double* lq, int slq, double* lm, int slm, double& lamc) {
  const int o = (c > 0.) ? -1 : 0;
  const double* qu = q + o * sq;
  const double* mu = mono + o * sm;
  const double qm = qu[-sq], q0 = qu[0], qp = qu[sq], mm = mu[-sm], m0 = mu[0], mp = mu[sm];
  const double eL = (qm - q0) * 0.5 + div_const<3>(mm - m0);
  const double eR = (qp - q0) * 0.5 + div_const<3>(m0 - mp);
  const double sa = fabs(c);
  const double k1 = (1. - 2. * sa) * (1. - sa);
  const double k2 = sa * (sa - 1.);
  const double F = (c > 0.) ? q0 + k1 * eR + k2 * eL : q0 + k1 * eL + k2 * eR;
  if (lamF != 0.) {
    const double aR = (c > 0.) ? k1 : k2, aL = (c > 0.) ? k2 : k1;
    const double lR = aR * lamF, lL = aL * lamF;
    double* lqu = lq + o * slq;
    double* lmu = lm + o * slm;
    sadd(lqu - slq, .5 * lL);
    sadd(lqu, lamF - .5 * (lL + lR));
    sadd(lqu + slq, .5 * lR);
    sadd(lmu - slm, lL / 3.);
    sadd(lmu, (lR - lL) / 3.);
    sadd(lmu + slm, -lR / 3.);
    const double sg = c > 0. ? 1. : (c < 0. ? -1. : 0.);
    const double dk1 = 4. * sa - 3., dk2 = 2. * sa - 1.;
    lamc += sg * ((c > 0.) ? dk1 * eR + dk2 * eL : dk1 * eL + dk2 * eR) * lamF;
  }
  return F;
}

// (eL, eR) = edges_pre<PPM_CONSTRAINED>(q, mono) of one cell, by hand
// (src/mod_sw_dyn.f90:877-893): the raw edges, limited by 2|dqi| with the
// sign of dqi: adds lamL * deL + lamR * deR with respect to q(-1..1) and
// mono(-1..1) to lq, lm.
__device__ __forceinline__ void edges_con_adj(const double* q, int sq, const double* mono, int sm, double lamL,
                                              double lamR, double* lq, int slq, double* lm, int slm) {
  if (lamL == 0. && lamR == 0.) return;
  const double qm = q[-sq], q0 = q[0], qp = q[sq], mm = mono[-sm], m0 = mono[0], mp = mono[sm];
  const double eLr = (qm - q0) * 0.5 + div_const<3>(mm - m0);
  const double eRr = (qp - q0) * 0.5 + div_const<3>(m0 - mp);
  const double d0 = (qp - qm) * 0.25;
  const double lim = 2. * fabs(d0);
  const double sb = signbit(d0) ? -1. : 1.;
  const double sd = d0 > 0. ? 1. : (d0 < 0. ? -1. : 0.);
  double lLr = 0., lRr = 0., ld0 = 0.;
  {  // eL = -copysign(mn(lim, |eLr|), d0)
    const double a = fabs(eLr);
    const bool raw = a < lim;
    const double av = raw ? a : lim;
    const double la = -(av > 0. ? sb : 0.) * lamL;
    if (raw) lLr = (eLr > 0. ? 1. : (eLr < 0. ? -1. : 0.)) * la;
    else ld0 += 2. * sd * la;
  }
  {  // eR = +copysign(mn(lim, |eRr|), d0)
    const double a = fabs(eRr);
    const bool raw = a < lim;
    const double av = raw ? a : lim;
    const double la = (av > 0. ? sb : 0.) * lamR;
    if (raw) lRr = (eRr > 0. ? 1. : (eRr < 0. ? -1. : 0.)) * la;
    else ld0 += 2. * sd * la;
  }
  const double a_m = .5 * lLr - .25 * ld0, a_0 = -.5 * (lLr + lRr), a_p = .5 * lRr + .25 * ld0;
  if (a_m != 0.) sadd(lq - slq, a_m);
  if (a_0 != 0.) sadd(lq, a_0);
  if (a_p != 0.) sadd(lq + slq, a_p);
  const double b_m = lLr / 3., b_0 = (lRr - lLr) / 3., b_p = -lRr / 3.;
  if (b_m != 0.) sadd(lm - slm, b_m);
  if (b_0 != 0.) sadd(lm, b_0);
  if (b_p != 0.) sadd(lm + slm, b_p);
}

// F = flux_pre<PPM_NONNEGATIVE>(q, mono, c), by hand: the upwind cell's
// edges go through the chain of src/mod_sw_dyn.f90:877-911 -- raw edges,
// the 2|dqi| clamp with the sign of dqi, the floor at -q0, and the
// curvature fix-up (both zero, or one edge twice the other's magnitude) --
// each step's derivative following the branch the forward took.  Same
// contract as flux_unc_adj.
__device__ __forceinline__ double flux_nn_adj(const double* q, int sq, const double* mono, int sm, double c,
                                              double lamF, double* lq, int slq, double* lm, int slm, double& lamc) {
  const int o = (c > 0.) ? -1 : 0;
  const double* qu = q + o * sq;
  const double* mu = mono + o * sm;
  const double qm = qu[-sq], q0 = qu[0], qp = qu[sq], mm = mu[-sm], m0 = mu[0], mp = mu[sm];
  // forward, with edges_pre's operations
  const double eLr = (qm - q0) * 0.5 + div_const<3>(mm - m0);
  const double eRr = (qp - q0) * 0.5 + div_const<3>(m0 - mp);
  const double d0 = (qp - qm) * 0.25;
  const double lim = 2. * fabs(d0);
  const bool rawL = fabs(eLr) < lim, rawR = fabs(eRr) < lim;
  const double eL1 = -copysign(mn(lim, fabs(eLr)), d0);
  const double eR1 = +copysign(mn(lim, fabs(eRr)), d0);
  const bool floorL = eL1 < -q0, floorR = eR1 < -q0;
  const double eL2 = mx(eL1, -q0), eR2 = mx(eR1, -q0);
  const double a = eR2 - eL2;
  const double b = -3. * (eR2 + eL2);
  int fix = 0;  // 0: none, 1: both zero, 2: eL = 2|eR|, 3: eR = 2|eL|
  if ((fabs(a) < -b) && (q0 + a * a / (4. * b) + div_const<12>(b) < 0.)) {
    if (eL2 * eR2 > 0.) fix = 1;
    else if (eL2 > eR2) fix = 2;
    else fix = 3;
  }
  const double eL3 = fix == 1 ? 0. : (fix == 2 ? 2. * fabs(eR2) : eL2);
  const double eR3 = fix == 1 ? 0. : (fix == 3 ? 2. * fabs(eL2) : eR2);
  const double sa = fabs(c);
  const double k1 = (1. - 2. * sa) * (1. - sa);
  const double k2 = sa * (sa - 1.);
  const double F = (c > 0.) ? q0 + k1 * eR3 + k2 * eL3 : q0 + k1 * eL3 + k2 * eR3;
  if (lamF == 0.) return F;
  // reverse
  const double lR3 = ((c > 0.) ? k1 : k2) * lamF, lL3 = ((c > 0.) ? k2 : k1) * lamF;
  const double sgL2 = eL2 > 0. ? 1. : (eL2 < 0. ? -1. : 0.), sgR2 = eR2 > 0. ? 1. : (eR2 < 0. ? -1. : 0.);
  double lL2, lR2;
  if (fix == 0) { lL2 = lL3; lR2 = lR3; }
  else if (fix == 1) { lL2 = 0.; lR2 = 0.; }
  else if (fix == 2) { lL2 = 0.; lR2 = lR3 + 2. * sgR2 * lL3; }
  else { lR2 = 0.; lL2 = lL3 + 2. * sgL2 * lR3; }
  double lq0 = lamF;  // F's own q(u)
  double lL1 = 0., lR1 = 0.;
  if (floorL) lq0 -= lL2; else lL1 = lL2;
  if (floorR) lq0 -= lR2; else lR1 = lR2;
  const double sb = signbit(d0) ? -1. : 1.;
  const double sd = d0 > 0. ? 1. : (d0 < 0. ? -1. : 0.);
  double lLr = 0., lRr = 0., ld0 = 0.;
  {  // eL1 = -copysign(mn(lim, |eLr|), d0)
    const double av = rawL ? fabs(eLr) : lim;
    const double la = -(av > 0. ? sb : 0.) * lL1;
    if (rawL) lLr = (eLr > 0. ? 1. : (eLr < 0. ? -1. : 0.)) * la;
    else ld0 += 2. * sd * la;
  }
  {  // eR1 = +copysign(mn(lim, |eRr|), d0)
    const double av = rawR ? fabs(eRr) : lim;
    const double la = (av > 0. ? sb : 0.) * lR1;
    if (rawR) lRr = (eRr > 0. ? 1. : (eRr < 0. ? -1. : 0.)) * la;
    else ld0 += 2. * sd * la;
  }
  double* lqu = lq + o * slq;
  double* lmu = lm + o * slm;
  const double a_m = .5 * lLr - .25 * ld0, a_0 = lq0 - .5 * (lLr + lRr), a_p = .5 * lRr + .25 * ld0;
  if (a_m != 0.) sadd(lqu - slq, a_m);
  if (a_0 != 0.) sadd(lqu, a_0);
  if (a_p != 0.) sadd(lqu + slq, a_p);
  const double b_m = lLr / 3., b_0 = (lRr - lLr) / 3., b_p = -lRr / 3.;
  if (b_m != 0.) sadd(lmu - slm, b_m);
  if (b_0 != 0.) sadd(lmu, b_0);
  if (b_p != 0.) sadd(lmu + slm, b_p);
  const double sg = c > 0. ? 1. : (c < 0. ? -1. : 0.);
  const double dk1 = 4. * sa - 3., dk2 = 2. * sa - 1.;
  lamc += sg * ((c > 0.) ? dk1 * eR3 + dk2 * eL3 : dk1 * eL3 + dk2 * eR3) * lamF;
  return F;
}

// flux adjoint of the variant V of the mass sweeps (PPM_UNCONSTRAINED on
// the C grid, PPM_NONNEGATIVE on the D grid)
template <int V>
__device__ __forceinline__ double flux_adj(const double* q, int sq, const double* mono, int sm, double c, double lamF,
                                           double* lq, int slq, double* lm, int slm, double& lamc) {
  static_assert(V == PPM_UNC || V == PPM_NN, "the mass sweeps use PPM_UNCONSTRAINED or PPM_NONNEGATIVE");
  if constexpr (V == PPM_UNC) return flux_unc_adj(q, sq, mono, sm, c, lamF, lq, slq, lm, slm, lamc);
  else return flux_nn_adj(q, sq, mono, sm, c, lamF, lq, slq, lm, slm, lamc);
}

// F = flux_con_pre(q, eL, eR, c) with precomputed PPM_CONSTRAINED edges
// (src/mod_sw_dyn.f90:802-825); returns F.
__device__ __forceinline__ double flux_con_adj(const double* q, int sq, const double* eL, const double* eR, int se,
                                               double c, double lamF, double* lq, int slq, double* leL, double* leR,
                                               int sle, double& lamc) {
  const double eLm = eL[-se], eRm = eR[-se], eL0 = eL[0], eR0 = eR[0];
  if ((3. * fabs(eL0 + eR0) > fabs(eL0 - eR0)) && (3. * fabs(eLm + eRm) > fabs(eLm - eRm))) {
    if (c > 0.) {
      if (lamF != 0.) sadd(lq - slq, lamF);
      return q[-sq];
    }
    if (lamF != 0.) sadd(lq, lamF);
    return q[0];
  }
  const double sa = fabs(c);
  const double k1 = (1. - 2. * sa) * (1. - sa);
  const double k2 = sa * (sa - 1.);
  const double dk1 = 4. * sa - 3., dk2 = 2. * sa - 1.;
  const double sg = c > 0. ? 1. : (c < 0. ? -1. : 0.);
  if (c > 0.) {
    if (lamF != 0.) {
      sadd(lq - slq, lamF);
      sadd(leR - sle, k1 * lamF);
      sadd(leL - sle, k2 * lamF);
      lamc += sg * (dk1 * eRm + dk2 * eLm) * lamF;
    }
    return q[-sq] + k1 * eRm + k2 * eLm;
  }
  if (lamF != 0.) {
    sadd(lq, lamF);
    sadd(leL, k1 * lamF);
    sadd(leR, k2 * lamF);
    lamc += sg * (dk1 * eL0 + dk2 * eR0) * lamF;
  }
  return q[0] + k1 * eL0 + k2 * eR0;
}

// t = .5 (q0 + den (q0 - rA (f1 - f0))) with f0, f1 the upwind values of
// the piecewise-constant inner sweep (Courant numbers c0, c1) and den the
// (fixed here) denominator: adds lamT * dt/dq to lq(-1..1) and
// lamT * dt/dden to lden.
__device__ __forceinline__ void inner_adj(const double* q, int s, double c0, double c1, double den, double rA,
                                          double lamT, double* lq, int sl, double& lden) {
  if (lamT == 0.) return;
  const double f0 = (c0 > 0.) ? q[-s] : q[0];
  const double f1 = (c1 > 0.) ? q[0] : q[s];
  const double lf = .5 * den * rA * lamT;  // d/df0 = +lf, d/df1 = -lf
  double am = 0., a0 = .5 * (1. + den) * lamT, ap = 0.;
  if (c0 > 0.) am += lf; else a0 += lf;
  if (c1 > 0.) a0 -= lf; else ap -= lf;
  if (am != 0.) sadd(lq - sl, am);
  sadd(lq, a0);
  if (ap != 0.) sadd(lq + sl, ap);
  lden += .5 * (q[0] - rA * (f1 - f0)) * lamT;
}

// Four-point pressure-gradient term (src/mod_sw_dyn.f90:325-339, 665-679):
// pg = (a b + c d) / (a + c) with a = p0 - p1, b = g0 - g1, c = p2 - p3,
// d = g2 - g3.  Adds lam * dpg/d(p0..p3, g0..g3) through the callbacks.
struct PgfAdj {
  double dp0, dp1, dp2, dp3, dg0, dg1, dg2, dg3;
};
__device__ __forceinline__ PgfAdj pgf_adj(double p0, double p1, double g0, double g1, double p2, double p3, double g2,
                                          double g3, double lam) {
  const double a = p0 - p1, b = g0 - g1, c = p2 - p3, d = g2 - g3;
  const double D = a + c;
  const double pg = (a * b + c * d) / D;
  const double la = (b - pg) / D * lam, lc = (d - pg) / D * lam, lb = a / D * lam, ld = c / D * lam;
  return PgfAdj{la, -la, lc, -lc, lb, -lb, ld, -ld};
}

// true in every thread when some output adjoint of the tile [ox, ox+TX) x
// [oy, oy+TY) (points with x <= xhi, y <= yhi) is nonzero: adjoint
// sensitivities are local (a loss over a sub-domain reaches only its
// domain of dependence), and a tile whose outputs carry no adjoint adds
// nothing to any input adjoint
template <int TX, int TY>
__device__ __forceinline__ bool tile_active(const double* a, const double* b, const Geom& g, int k, int ox, int oy,
                                            int xhi, int yhi, int* s_flag) {
  if (threadIdx.x == 0) *s_flag = 0;
  __syncthreads();
  for (int idx = threadIdx.x; idx < TX * TY; idx += NTA) {
    const int x = ox + idx % TX, y = oy + idx / TX;
    if (x <= xhi && y <= yhi) {
      const long long o = g.at(x, y, k);
      if (a[o] != 0. || b[o] != 0.) *s_flag = 1;
    }
  }
  __syncthreads();
  return *s_flag != 0;
}

// add a tile-local adjoint box to a global adjoint field (level k)
__device__ __forceinline__ void flush_box(const Sm<double>& a, int w, int h, double* dst, const Geom& g, int k) {
  if (!dst) return;
  for (int idx = threadIdx.x; idx < w * h; idx += NTA) {
    const int yy = idx / w, xx = idx - yy * w;
    const double v = a.p[idx];
    const int x = a.x0 + xx, y = a.y0 + yy;
    if (v != 0. && x >= -H && x < g.nx + H && y >= -H && y < g.ny + H) atomicAdd(dst + g.at(x, y, k), v);
  }
}

// ======================================================== mass adjoint ====
// Adjoint of k_mass2 (C grid: dpc, ptc from dp, pt, ud, vd; D grid: dp, pt
// from dp, pt, uc, vc), src/mod_sw_dyn.f90:94-270 and 439-600 (heating off).
// The update's adjoint needs only the new dp and pt (read from the step's
// outputs), so the reverse splits by sweep direction into two kernels that
// meet in global memory through the flush atomics: the x branch (inner
// y-sweep, its slopes, the outer x fluxes, the x terms of the damping, and
// the direct dependence of the new dp, pt on the old) and the y branch.
// Each holds about two thirds of the shared memory one kernel needed (3
// CTAs per SM on 32 x 8 tiles instead of 2); the D grid uses the split, the
// C grid the one-kernel form below.
template <int TX, int TY, bool CGRID>
struct MassAdjBL {
  using F = MassL<double, TX, TY, CGRID>;
  static constexpr int UW = CGRID ? TX + 2 : TX + 1, UH = CGRID ? TY + 7 : TY + 6;
  static constexpr int VW = CGRID ? TX + 7 : TX + 6, VH = CGRID ? TY + 2 : TY + 1;
  static constexpr size_t cwinds = CGRID ? box_bytes<double>(TX + 1, TY + 6) + box_bytes<double>(TX + 6, TY + 1) : 0;
  // the larger of the two branches (the y branch's arrays are the x
  // branch's transposed, up to the row padding)
  static constexpr size_t inner = box_bytes<double>(TX + 6, TY) > box_bytes<double>(TX, TY + 6)
                                      ? box_bytes<double>(TX + 6, TY) : box_bytes<double>(TX, TY + 6);
  static constexpr size_t slope = box_bytes<double>(TX + 4, TY) > box_bytes<double>(TX, TY + 4)
                                      ? box_bytes<double>(TX + 4, TY) : box_bytes<double>(TX, TY + 4);
  static constexpr size_t flux = box_bytes<double>(TX + 1, TY) > box_bytes<double>(TX, TY + 1)
                                     ? box_bytes<double>(TX + 1, TY) : box_bytes<double>(TX, TY + 1);
  static constexpr size_t fwd = cwinds + 2 * inner + box_bytes<double>(TX + 2, TY + 2) + 2 * slope + 2 * flux;
  static constexpr size_t lam = 2 * box_bytes<double>(TX, TY) + 2 * box_bytes<double>(TX + 2, TY + 2) + 2 * slope +
                                2 * inner + cwinds + 2 * box_bytes<double>(TX + 6, TY + 6) +
                                box_bytes<double>(UW, UH) + box_bytes<double>(VW, VH);
  static constexpr size_t bytes = F::boxes + fwd + lam + 128;
};

// XB: the x branch (and the direct terms); !XB: the y branch.  dpo, pto: the
// new dp and pt the forward wrote (outputs over [lo, n-1+hi]^2).
template <int TX, int TY, bool CGRID, bool XB>
__global__ void __launch_bounds__(NTA, 3) k_mass_adj(const __grid_constant__ CUtensorMap m_dp,
                                                 const __grid_constant__ CUtensorMap m_pt,
                                                 const __grid_constant__ CUtensorMap m_u,
                                                 const __grid_constant__ CUtensorMap m_v, Geom g, Consts c,
                                                 const double* __restrict__ dpo, const double* __restrict__ pto,
                                                 const double* __restrict__ lam_dpo, const double* __restrict__ lam_pto,
                                                 double* lam_dp, double* lam_pt, double* lam_u, double* lam_v, int lo,
                                                 int hi, int* timeout) {
  using T = double;
  using Lay = MassL<T, TX, TY, CGRID>;
  using ALay = MassAdjBL<TX, TY, CGRID>;
  constexpr int V = CGRID ? PPM_UNC : PPM_NN;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z;
  const int ox = lo + blockIdx.x * TX, oy = lo + blockIdx.y * TY;
  const T dtdx = c.dtdx, dtdy = c.dtdy, rA = c.rA;
  if (!tile_active<TX, TY>(lam_dpo, lam_pto, g, k, ox, oy, g.nx - 1 + hi, g.ny - 1 + hi, &s_ok)) return;

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  Sm<T> sdp = tbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<T> spt = tbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<T> su = CGRID ? tbox(ox - 1, oy - 3, Lay::WU, Lay::HU) : tbox(ox, oy - 3, Lay::WU, Lay::HU);
  Sm<T> sv = CGRID ? tbox(ox - 3, oy - 1, Lay::WV, Lay::HV) : tbox(ox - 3, oy, Lay::WV, Lay::HV);
  {
    const TmaBox boxes[4] = {{&m_dp, sdp.p, sdp.x0, sdp.y0, k},
                             {&m_pt, spt.p, spt.x0, spt.y0, k},
                             {&m_u, su.p, su.x0, su.y0, k},
                             {&m_v, sv.p, sv.x0, sv.y0, k}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  Sm<T> suc = su, svc = sv;
  if (CGRID) {
    suc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
    svc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  }
  // the branch's inner sweeps (x branch: the y-sweeps tyd, typ on
  // [ox-3, ox+TX+2] x [oy, oy+TY); y branch: the x-sweeps txd, txp), their
  // slopes along the outer direction, and its outer fluxes
  constexpr int IW = XB ? TX + 6 : TX, IH = XB ? TY : TY + 6;
  constexpr int MW = XB ? TX + 4 : TX, MH = XB ? TY : TY + 4;
  constexpr int FW = XB ? TX + 1 : TX, FH = XB ? TY : TY + 1;
  const int ix = XB ? ox - 3 : ox, iy = XB ? oy : oy - 3;
  const int mx = XB ? ox - 2 : ox, my = XB ? oy : oy - 2;
  constexpr int SO = XB ? 1 : IW;  // stride along the outer direction in the inner arrays
  constexpr int SM_ = XB ? 1 : MW;
  Sm<T> tid = carve<T>(p, ix, iy, IW, IH);
  Sm<T> tip = carve<T>(p, ix, iy, IW, IH);
  Sm<T> lpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> mid = carve<T>(p, mx, my, MW, MH);
  Sm<T> mip = carve<T>(p, mx, my, MW, MH);
  Sm<T> fod = carve<T>(p, ox, oy, FW, FH);
  Sm<T> fop = carve<T>(p, ox, oy, FW, FH);
  // adjoints
  unsigned char* lam0 = p;
  Sm<T> Lv = carve<T>(p, ox, oy, TX, TY);
  Sm<T> Lq = carve<T>(p, ox, oy, TX, TY);
  Sm<T> alpd = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> alpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> amid = carve<T>(p, mx, my, MW, MH);
  Sm<T> amip = carve<T>(p, mx, my, MW, MH);
  Sm<T> atid = carve<T>(p, ix, iy, IW, IH);
  Sm<T> atip = carve<T>(p, ix, iy, IW, IH);
  Sm<T> asuc{}, asvc{};
  if (CGRID) {
    asuc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
    asvc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  }
  Sm<T> asdp = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> aspt = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> asu = CGRID ? carve<T>(p, ox - 1, oy - 3, ALay::UW, ALay::UH) : carve<T>(p, ox, oy - 3, ALay::UW, ALay::UH);
  Sm<T> asv = CGRID ? carve<T>(p, ox - 3, oy - 1, ALay::VW, ALay::VH) : carve<T>(p, ox - 3, oy, ALay::VW, ALay::VH);
  if (!CGRID) {
    asuc = asu;
    asvc = asv;
  }
  zero_smem(lam0, p);

  // ---- forward recomputation (as k_mass2)
  if (CGRID) {  // mod_sw_dyn.f90:109-117
    regions(reg<TX + 1, TY + 6>(ox, oy - 3, [&](int x, int y) {
      T ub = T(.5) * (su(x, y) + su(x - 1, y));
      suc(x, y) = T(.5) * (ub + T(.5) * (su(x, y + 1) + su(x - 1, y + 1)));
    }),
            reg<TX + 6, TY + 1>(ox - 3, oy, [&](int x, int y) {
      T vb = T(.5) * (sv(x, y) + sv(x, y - 1));
      svc(x, y) = T(.5) * (vb + T(.5) * (sv(x + 1, y) + sv(x + 1, y - 1)));
    }));
    __syncthreads();
  }
  const T rdx2 = c.rdx2, rdy2 = c.rdy2, rdxy = c.rdx2rdy2;
  regions(reg<IW, IH>(ix, iy, [&](int x, int y) {
    if constexpr (XB) {
      T cy0 = dtdx * svc(x, y), cy1 = dtdx * svc(x, y + 1);
      T den = T(1) / (T(1) - dtdy * (svc(x, y + 1) - svc(x, y)));
      T f0 = (cy0 > T(0)) ? sdp(x, y - 1) : sdp(x, y);
      T f1 = (cy1 > T(0)) ? sdp(x, y) : sdp(x, y + 1);
      tid(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
      f0 = (cy0 > T(0)) ? spt(x, y - 1) : spt(x, y);
      f1 = (cy1 > T(0)) ? spt(x, y) : spt(x, y + 1);
      tip(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
    } else {
      T cx0 = dtdx * suc(x, y), cx1 = dtdx * suc(x + 1, y);
      T den = T(1) / (T(1) - dtdx * (suc(x + 1, y) - suc(x, y)));
      T f0 = (cx0 > T(0)) ? sdp(x - 1, y) : sdp(x, y);
      T f1 = (cx1 > T(0)) ? sdp(x, y) : sdp(x + 1, y);
      tid(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
      f0 = (cx0 > T(0)) ? spt(x - 1, y) : spt(x, y);
      f1 = (cx1 > T(0)) ? spt(x, y) : spt(x + 1, y);
      tip(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
    }
  }),
          reg<TX + 2, TY + 2>(ox - 1, oy - 1, [&](int x, int y) {
    lpp(x, y) = T(-2.) * spt(x, y) * rdxy + (spt(x + 1, y) + spt(x - 1, y)) * rdx2 +
                (spt(x, y + 1) + spt(x, y - 1)) * rdy2;
  }));
  __syncthreads();
  aregion<MW, MH>(mx, my, [&](int x, int y) {
    mid(x, y) = slope_at(tid.ptr(x, y), SO);
    mip(x, y) = slope_at(tip.ptr(x, y), SO);
  });
  __syncthreads();
  aregion<FW, FH>(ox, oy, [&](int x, int y) {
    T cw = dtdx * (XB ? suc(x, y) : svc(x, y));
    fod(x, y) = flux_pre<T, V>(tid.ptr(x, y), SO, mid.ptr(x, y), SM_, cw) * cw;
    fop(x, y) = flux_pre<T, V>(tip.ptr(x, y), SO, mip.ptr(x, y), SM_, cw);
  });
  __syncthreads();

  // ---- reverse
  const int xhi = g.nx - 1 + hi, yhi = g.ny - 1 + hi;
  const T dxv = dtdx * c.vdx, dyv = dtdy * c.vdy, vdx = c.vdx, vdy = c.vdy;
  // updates (:163-172,193-202,230-237,258-267 / :490-499,519-528,555-562,582-591):
  // Lv = adjoint of the new dp, Lq = adjoint of the numerator of the new pt
  aregion<TX, TY>(ox, oy, [&](int x, int y) {
    double lv = 0., lq = 0.;
    if (x <= xhi && y <= yhi) {
      const long long o = g.at(x, y, k);
      const double v = dpo[o], qv = pto[o];  // the new dp and pt = q / v
      const double lpo = lam_pto[o];
      lq = lpo / v;
      lv = lam_dpo[o] - qv / v * lpo;
      if (XB) {
        asdp(x, y) += lv + spt(x, y) * lq;
        aspt(x, y) += sdp(x, y) * lq;
      }
    }
    Lv(x, y) = lv;
    Lq(x, y) = lq;
  });
  __syncthreads();
  auto inT = [&](int x, int y) { return x >= ox && x < ox + TX && y >= oy && y < oy + TY; };
  auto LV = [&](int x, int y) { return inT(x, y) ? Lv(x, y) : 0.; };
  auto LQ = [&](int x, int y) { return inT(x, y) ? Lq(x, y) : 0.; };
  // the branch's terms of the Laplacians' adjoints (gather), and the outer
  // PPM sweep (:156-161,186-191 / :484-489,513-518)
  regions(reg<TX + 2, TY + 2>(ox - 1, oy - 1, [&](int x, int y) {
    double a = 0.;
    if constexpr (XB) {
      alpd(x, y) = dxv * (2. * LV(x, y) - LV(x - 1, y) - LV(x + 1, y));
      if (inT(x - 1, y)) a -= fod(x, y) * Lq(x - 1, y);
      if (inT(x, y)) a += (fod(x + 1, y) + fod(x, y)) * Lq(x, y);
      if (inT(x + 1, y)) a -= fod(x + 1, y) * Lq(x + 1, y);
      alpp(x, y) = vdx * a;
    } else {
      alpd(x, y) = dyv * (2. * LV(x, y) - LV(x, y - 1) - LV(x, y + 1));
      if (inT(x, y - 1)) a -= fod(x, y) * Lq(x, y - 1);
      if (inT(x, y)) a += (fod(x, y + 1) + fod(x, y)) * Lq(x, y);
      if (inT(x, y + 1)) a -= fod(x, y + 1) * Lq(x, y + 1);
      alpp(x, y) = vdy * a;
    }
  }),
          reg<FW, FH>(ox, oy, [&](int x, int y) {
    const int xm = XB ? x - 1 : x, ym = XB ? y : y - 1;  // the upstream cell of the face
    const double ql = LQ(xm, ym), qr = LQ(x, y);
    const double lfd = (LV(x, y) - LV(xm, ym)) + (fop(x, y) + (XB ? vdx : vdy) * (lpp(x, y) - lpp(xm, ym))) * (qr - ql);
    const double lfp = fod(x, y) * (qr - ql);
    if (lfd == 0. && lfp == 0.) return;
    const T cw = dtdx * (XB ? suc(x, y) : svc(x, y));
    double lc = 0.;
    double Fl = flux_adj<V>(tid.ptr(x, y), SO, mid.ptr(x, y), SM_, cw, lfd * cw, atid.ptr(x, y), SO, amid.ptr(x, y),
                            SM_, lc);
    lc += lfd * Fl;
    flux_adj<V>(tip.ptr(x, y), SO, mip.ptr(x, y), SM_, cw, lfp, atip.ptr(x, y), SO, amip.ptr(x, y), SM_, lc);
    if (XB) asuc(x, y) += dtdx * lc;
    else asvc(x, y) += dtdx * lc;
  }));
  __syncthreads();
  // slopes (:870-875) and the Laplacians (:148-153,178-183 / :476-481,505-510)
  auto inL = [&](int x, int y) { return x >= ox - 1 && x < ox + TX + 1 && y >= oy - 1 && y < oy + TY + 1; };
  regions(reg<MW, MH>(mx, my, [&](int x, int y) {
    slope_adj(tid.ptr(x, y), SO, amid(x, y), atid.ptr(x, y), SO);
    slope_adj(tip.ptr(x, y), SO, amip(x, y), atip.ptr(x, y), SO);
  }),
          reg<TX + 4, TY + 4>(ox - 2, oy - 2, [&](int x, int y) {
    double ad = 0., ap = 0.;
    if (inL(x, y)) { ad += -2. * rdxy * alpd(x, y); ap += -2. * rdxy * alpp(x, y); }
    if (inL(x - 1, y)) { ad += rdx2 * alpd(x - 1, y); ap += rdx2 * alpp(x - 1, y); }
    if (inL(x + 1, y)) { ad += rdx2 * alpd(x + 1, y); ap += rdx2 * alpp(x + 1, y); }
    if (inL(x, y - 1)) { ad += rdy2 * alpd(x, y - 1); ap += rdy2 * alpp(x, y - 1); }
    if (inL(x, y + 1)) { ad += rdy2 * alpd(x, y + 1); ap += rdy2 * alpp(x, y + 1); }
    asdp(x, y) += ad;
    aspt(x, y) += ap;
  }));
  __syncthreads();
  // inner sweeps (:142-147,176-177,210-216,238-243 / :470-475,503-504,531-536,563-568)
  aregion<IW, IH>(ix, iy, [&](int x, int y) {
    const double ld = atid(x, y), lp = atip(x, y);
    if (ld == 0. && lp == 0.) return;
    double lden = 0.;
    if constexpr (XB) {
      const T w0 = svc(x, y), w1 = svc(x, y + 1);
      const T cy0 = dtdx * w0, cy1 = dtdx * w1;
      const T den = T(1) / (T(1) - dtdy * (w1 - w0));
      inner_adj(sdp.ptr(x, y), sdp.w, cy0, cy1, den, rA, ld, asdp.ptr(x, y), TX + 6, lden);
      inner_adj(spt.ptr(x, y), spt.w, cy0, cy1, den, rA, lp, aspt.ptr(x, y), TX + 6, lden);
      const double lw = dtdy * den * den * lden;
      if (lw != 0.) {
        sadd(asvc.ptr(x, y + 1), lw);
        sadd(asvc.ptr(x, y), -lw);
      }
    } else {
      const T w0 = suc(x, y), w1 = suc(x + 1, y);
      const T cx0 = dtdx * w0, cx1 = dtdx * w1;
      const T den = T(1) / (T(1) - dtdx * (w1 - w0));
      inner_adj(sdp.ptr(x, y), 1, cx0, cx1, den, rA, ld, asdp.ptr(x, y), 1, lden);
      inner_adj(spt.ptr(x, y), 1, cx0, cx1, den, rA, lp, aspt.ptr(x, y), 1, lden);
      const double lw = dtdx * den * den * lden;
      if (lw != 0.) {
        sadd(asuc.ptr(x + 1, y), lw);
        sadd(asuc.ptr(x, y), -lw);
      }
    }
  });
  __syncthreads();
  if (CGRID) {  // C-grid winds from the D-grid winds (:109-117)
    regions(reg<TX + 1, TY + 6>(ox, oy - 3, [&](int x, int y) {
      const double l = .25 * asuc(x, y);
      if (l == 0.) return;
      sadd(asu.ptr(x, y), l);
      sadd(asu.ptr(x - 1, y), l);
      sadd(asu.ptr(x, y + 1), l);
      sadd(asu.ptr(x - 1, y + 1), l);
    }),
            reg<TX + 6, TY + 1>(ox - 3, oy, [&](int x, int y) {
      const double l = .25 * asvc(x, y);
      if (l == 0.) return;
      sadd(asv.ptr(x, y), l);
      sadd(asv.ptr(x, y - 1), l);
      sadd(asv.ptr(x + 1, y), l);
      sadd(asv.ptr(x + 1, y - 1), l);
    }));
    __syncthreads();
  }
  flush_box(asdp, TX + 6, TY + 6, lam_dp, g, k);
  flush_box(aspt, TX + 6, TY + 6, lam_pt, g, k);
  flush_box(asu, ALay::UW, ALay::UH, lam_u, g, k);
  flush_box(asv, ALay::VW, ALay::VH, lam_v, g, k);
}

// The mass adjoint in one kernel (both branches, the update recomputed from
// the fluxes), used on the C grid: there the halo-wide output range and the
// C-grid winds each branch would recompute make two kernels slower.
template <int TX, int TY, bool CGRID>
struct MassAdj1L {
  using F = MassL<double, TX, TY, CGRID>;
  static constexpr int UW = CGRID ? TX + 2 : TX + 1, UH = CGRID ? TY + 7 : TY + 6;
  static constexpr int VW = CGRID ? TX + 7 : TX + 6, VH = CGRID ? TY + 2 : TY + 1;
  static constexpr size_t lam =
      2 * box_bytes<double>(TX, TY) + 2 * box_bytes<double>(TX + 2, TY + 2) + 2 * box_bytes<double>(TX + 4, TY) +
      2 * box_bytes<double>(TX, TY + 4) + 2 * box_bytes<double>(TX + 6, TY) + 2 * box_bytes<double>(TX, TY + 6) +
      (CGRID ? box_bytes<double>(TX + 1, TY + 6) + box_bytes<double>(TX + 6, TY + 1) : 0) +
      2 * box_bytes<double>(TX + 6, TY + 6) + box_bytes<double>(UW, UH) + box_bytes<double>(VW, VH);
  static constexpr size_t bytes = F::bytes + lam;
};

template <int TX, int TY, bool CGRID>
__global__ void __launch_bounds__(NTA, 3) k_mass_adj1(const __grid_constant__ CUtensorMap m_dp,
                                                 const __grid_constant__ CUtensorMap m_pt,
                                                 const __grid_constant__ CUtensorMap m_u,
                                                 const __grid_constant__ CUtensorMap m_v, Geom g, Consts c,
                                                 const double* __restrict__ lam_dpo, const double* __restrict__ lam_pto,
                                                 double* lam_dp, double* lam_pt, double* lam_u, double* lam_v, int lo,
                                                 int hi, int* timeout) {
  using T = double;
  using Lay = MassL<T, TX, TY, CGRID>;
  using ALay = MassAdj1L<TX, TY, CGRID>;
  constexpr int V = CGRID ? PPM_UNC : PPM_NN;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z;
  const int ox = lo + blockIdx.x * TX, oy = lo + blockIdx.y * TY;
  const T dtdx = c.dtdx, dtdy = c.dtdy, rA = c.rA;
  if (!tile_active<TX, TY>(lam_dpo, lam_pto, g, k, ox, oy, g.nx - 1 + hi, g.ny - 1 + hi, &s_ok)) return;

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  Sm<T> sdp = tbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<T> spt = tbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<T> su = CGRID ? tbox(ox - 1, oy - 3, Lay::WU, Lay::HU) : tbox(ox, oy - 3, Lay::WU, Lay::HU);
  Sm<T> sv = CGRID ? tbox(ox - 3, oy - 1, Lay::WV, Lay::HV) : tbox(ox - 3, oy, Lay::WV, Lay::HV);
  {
    const TmaBox boxes[4] = {{&m_dp, sdp.p, sdp.x0, sdp.y0, k},
                             {&m_pt, spt.p, spt.x0, spt.y0, k},
                             {&m_u, su.p, su.x0, su.y0, k},
                             {&m_v, sv.p, sv.x0, sv.y0, k}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  Sm<T> suc = su, svc = sv;
  if (CGRID) {
    suc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
    svc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  }
  Sm<T> tyd = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> typ = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> txd = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> txp = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> lpd = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> lpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> mxd = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> mxp = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> myd = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> myp = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> fxd = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fxp = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fyd = carve<T>(p, ox, oy, TX, TY + 1);
  Sm<T> fyp = carve<T>(p, ox, oy, TX, TY + 1);
  // adjoints
  unsigned char* lam0 = p;
  Sm<T> Lv = carve<T>(p, ox, oy, TX, TY);
  Sm<T> Lq = carve<T>(p, ox, oy, TX, TY);
  Sm<T> alpd = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> alpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> amxd = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> amxp = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> amyd = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> amyp = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> atyd = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> atyp = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> atxd = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> atxp = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> asuc{}, asvc{};
  if (CGRID) {
    asuc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
    asvc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  }
  Sm<T> asdp = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> aspt = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> asu = CGRID ? carve<T>(p, ox - 1, oy - 3, ALay::UW, ALay::UH) : carve<T>(p, ox, oy - 3, ALay::UW, ALay::UH);
  Sm<T> asv = CGRID ? carve<T>(p, ox - 3, oy - 1, ALay::VW, ALay::VH) : carve<T>(p, ox - 3, oy, ALay::VW, ALay::VH);
  if (!CGRID) {
    asuc = asu;
    asvc = asv;
  }
  zero_smem(lam0, p);

  // ---- forward recomputation (as k_mass2)
  if (CGRID) {
    aregion<TX + 1, TY + 6>(ox, oy - 3, [&](int x, int y) {
      T ub = T(.5) * (su(x, y) + su(x - 1, y));
      suc(x, y) = T(.5) * (ub + T(.5) * (su(x, y + 1) + su(x - 1, y + 1)));
    });
    aregion<TX + 6, TY + 1>(ox - 3, oy, [&](int x, int y) {
      T vb = T(.5) * (sv(x, y) + sv(x, y - 1));
      svc(x, y) = T(.5) * (vb + T(.5) * (sv(x + 1, y) + sv(x + 1, y - 1)));
    });
    __syncthreads();
  }
  aregion<TX + 6, TY>(ox - 3, oy, [&](int x, int y) {
    T cy0 = dtdx * svc(x, y), cy1 = dtdx * svc(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (svc(x, y + 1) - svc(x, y)));
    T f0 = (cy0 > T(0)) ? sdp(x, y - 1) : sdp(x, y);
    T f1 = (cy1 > T(0)) ? sdp(x, y) : sdp(x, y + 1);
    tyd(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
    f0 = (cy0 > T(0)) ? spt(x, y - 1) : spt(x, y);
    f1 = (cy1 > T(0)) ? spt(x, y) : spt(x, y + 1);
    typ(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
  });
  aregion<TX, TY + 6>(ox, oy - 3, [&](int x, int y) {
    T cx0 = dtdx * suc(x, y), cx1 = dtdx * suc(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (suc(x + 1, y) - suc(x, y)));
    T f0 = (cx0 > T(0)) ? sdp(x - 1, y) : sdp(x, y);
    T f1 = (cx1 > T(0)) ? sdp(x, y) : sdp(x + 1, y);
    txd(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
    f0 = (cx0 > T(0)) ? spt(x - 1, y) : spt(x, y);
    f1 = (cx1 > T(0)) ? spt(x, y) : spt(x + 1, y);
    txp(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
  });
  const T rdx2 = c.rdx2, rdy2 = c.rdy2, rdxy = c.rdx2rdy2;
  aregion<TX + 2, TY + 2>(ox - 1, oy - 1, [&](int x, int y) {
    lpd(x, y) = T(-2.) * sdp(x, y) * rdxy + (sdp(x + 1, y) + sdp(x - 1, y)) * rdx2 +
                (sdp(x, y + 1) + sdp(x, y - 1)) * rdy2;
    lpp(x, y) = T(-2.) * spt(x, y) * rdxy + (spt(x + 1, y) + spt(x - 1, y)) * rdx2 +
                (spt(x, y + 1) + spt(x, y - 1)) * rdy2;
  });
  __syncthreads();
  aregion<TX + 4, TY>(ox - 2, oy, [&](int x, int y) {
    mxd(x, y) = slope_at(tyd.ptr(x, y), 1);
    mxp(x, y) = slope_at(typ.ptr(x, y), 1);
  });
  aregion<TX, TY + 4>(ox, oy - 2, [&](int x, int y) {
    myd(x, y) = slope_at(txd.ptr(x, y), TX);
    myp(x, y) = slope_at(txp.ptr(x, y), TX);
  });
  __syncthreads();
  aregion<TX + 1, TY>(ox, oy, [&](int x, int y) {
    T cx = dtdx * suc(x, y);
    fxd(x, y) = flux_pre<T, V>(tyd.ptr(x, y), 1, mxd.ptr(x, y), 1, cx) * cx;
    fxp(x, y) = flux_pre<T, V>(typ.ptr(x, y), 1, mxp.ptr(x, y), 1, cx);
  });
  aregion<TX, TY + 1>(ox, oy, [&](int x, int y) {
    T cy = dtdx * svc(x, y);
    fyd(x, y) = flux_pre<T, V>(txd.ptr(x, y), TX, myd.ptr(x, y), TX, cy) * cy;
    fyp(x, y) = flux_pre<T, V>(txp.ptr(x, y), TX, myp.ptr(x, y), TX, cy);
  });
  __syncthreads();

  // ---- reverse
  const int xhi = g.nx - 1 + hi, yhi = g.ny - 1 + hi;
  const T dxv = dtdx * c.vdx, dyv = dtdy * c.vdy, vdx = c.vdx, vdy = c.vdy;
  // updates (:163-172,193-202,230-237,258-267 / :490-499,519-528,555-562,582-591):
  // Lv = adjoint of the new dp, Lq = adjoint of the numerator of the new pt
  aregion<TX, TY>(ox, oy, [&](int x, int y) {
    double lv = 0., lq = 0.;
    if (x <= xhi && y <= yhi) {
      T d = sdp(x, y);
      T v = d - (fxd(x + 1, y) - fxd(x, y) + dxv * (lpd(x + 1, y) - T(2.) * lpd(x, y) + lpd(x - 1, y)));
      v = v - (fyd(x, y + 1) - fyd(x, y) + dyv * (lpd(x, y + 1) - T(2.) * lpd(x, y) + lpd(x, y - 1)));
      T q = d * spt(x, y) - (fxp(x + 1, y) * fxd(x + 1, y) - fxp(x, y) * fxd(x, y) +
                             vdx * ((lpp(x + 1, y) - lpp(x, y)) * fxd(x + 1, y) - (lpp(x, y) - lpp(x - 1, y)) * fxd(x, y)));
      q = q - (fyp(x, y + 1) * fyd(x, y + 1) - fyp(x, y) * fyd(x, y) +
               vdy * ((lpp(x, y + 1) - lpp(x, y)) * fyd(x, y + 1) - (lpp(x, y) - lpp(x, y - 1)) * fyd(x, y)));
      const long long o = g.at(x, y, k);
      const double lpo = lam_pto[o];
      lq = lpo / v;
      lv = lam_dpo[o] - (q / v) / v * lpo;
      asdp(x, y) += lv + spt(x, y) * lq;
      aspt(x, y) += d * lq;
    }
    Lv(x, y) = lv;
    Lq(x, y) = lq;
  });
  __syncthreads();
  auto inT = [&](int x, int y) { return x >= ox && x < ox + TX && y >= oy && y < oy + TY; };
  auto LV = [&](int x, int y) { return inT(x, y) ? Lv(x, y) : 0.; };
  auto LQ = [&](int x, int y) { return inT(x, y) ? Lq(x, y) : 0.; };
  // Laplacians' adjoints (gather)
  aregion<TX + 2, TY + 2>(ox - 1, oy - 1, [&](int x, int y) {
    alpd(x, y) = dxv * (2. * LV(x, y) - LV(x - 1, y) - LV(x + 1, y)) + dyv * (2. * LV(x, y) - LV(x, y - 1) - LV(x, y + 1));
    double a = 0., b = 0.;
    if (inT(x - 1, y)) a -= fxd(x, y) * Lq(x - 1, y);
    if (inT(x, y)) a += (fxd(x + 1, y) + fxd(x, y)) * Lq(x, y);
    if (inT(x + 1, y)) a -= fxd(x + 1, y) * Lq(x + 1, y);
    if (inT(x, y - 1)) b -= fyd(x, y) * Lq(x, y - 1);
    if (inT(x, y)) b += (fyd(x, y + 1) + fyd(x, y)) * Lq(x, y);
    if (inT(x, y + 1)) b -= fyd(x, y + 1) * Lq(x, y + 1);
    alpp(x, y) = vdx * a + vdy * b;
  });
  // outer PPM sweeps (:156-161,186-191 / :484-489,513-518)
  aregion<TX + 1, TY>(ox, oy, [&](int x, int y) {
    const double ql = LQ(x - 1, y), qr = LQ(x, y);
    const double lfd = (LV(x, y) - LV(x - 1, y)) + (fxp(x, y) + vdx * (lpp(x, y) - lpp(x - 1, y))) * (qr - ql);
    const double lfp = fxd(x, y) * (qr - ql);
    if (lfd == 0. && lfp == 0.) return;
    const T cx = dtdx * suc(x, y);
    double lc = 0.;
    double F = flux_adj<V>(tyd.ptr(x, y), 1, mxd.ptr(x, y), 1, cx, lfd * cx, atyd.ptr(x, y), 1, amxd.ptr(x, y), 1, lc);
    lc += lfd * F;
    flux_adj<V>(typ.ptr(x, y), 1, mxp.ptr(x, y), 1, cx, lfp, atyp.ptr(x, y), 1, amxp.ptr(x, y), 1, lc);
    asuc(x, y) += dtdx * lc;
  });
  aregion<TX, TY + 1>(ox, oy, [&](int x, int y) {
    const double ql = LQ(x, y - 1), qr = LQ(x, y);
    const double lfd = (LV(x, y) - LV(x, y - 1)) + (fyp(x, y) + vdy * (lpp(x, y) - lpp(x, y - 1))) * (qr - ql);
    const double lfp = fyd(x, y) * (qr - ql);
    if (lfd == 0. && lfp == 0.) return;
    const T cy = dtdx * svc(x, y);
    double lc = 0.;
    double F = flux_adj<V>(txd.ptr(x, y), TX, myd.ptr(x, y), TX, cy, lfd * cy, atxd.ptr(x, y), TX, amyd.ptr(x, y), TX, lc);
    lc += lfd * F;
    flux_adj<V>(txp.ptr(x, y), TX, myp.ptr(x, y), TX, cy, lfp, atxp.ptr(x, y), TX, amyp.ptr(x, y), TX, lc);
    asvc(x, y) += dtdx * lc;
  });
  __syncthreads();
  // slopes (:870-875) and the Laplacians (:148-153,178-183 / :476-481,505-510)
  aregion<TX + 4, TY>(ox - 2, oy, [&](int x, int y) {
    slope_adj(tyd.ptr(x, y), 1, amxd(x, y), atyd.ptr(x, y), 1);
    slope_adj(typ.ptr(x, y), 1, amxp(x, y), atyp.ptr(x, y), 1);
  });
  aregion<TX, TY + 4>(ox, oy - 2, [&](int x, int y) {
    slope_adj(txd.ptr(x, y), TX, amyd(x, y), atxd.ptr(x, y), TX);
    slope_adj(txp.ptr(x, y), TX, amyp(x, y), atxp.ptr(x, y), TX);
  });
  auto inL = [&](int x, int y) { return x >= ox - 1 && x < ox + TX + 1 && y >= oy - 1 && y < oy + TY + 1; };
  aregion<TX + 4, TY + 4>(ox - 2, oy - 2, [&](int x, int y) {
    double ad = 0., ap = 0.;
    if (inL(x, y)) { ad += -2. * rdxy * alpd(x, y); ap += -2. * rdxy * alpp(x, y); }
    if (inL(x - 1, y)) { ad += rdx2 * alpd(x - 1, y); ap += rdx2 * alpp(x - 1, y); }
    if (inL(x + 1, y)) { ad += rdx2 * alpd(x + 1, y); ap += rdx2 * alpp(x + 1, y); }
    if (inL(x, y - 1)) { ad += rdy2 * alpd(x, y - 1); ap += rdy2 * alpp(x, y - 1); }
    if (inL(x, y + 1)) { ad += rdy2 * alpd(x, y + 1); ap += rdy2 * alpp(x, y + 1); }
    asdp(x, y) += ad;
    aspt(x, y) += ap;
  });
  __syncthreads();
  // inner sweeps (:142-147,176-177,210-216,238-243 / :470-475,503-504,531-536,563-568)
  aregion<TX + 6, TY>(ox - 3, oy, [&](int x, int y) {
    const double ld = atyd(x, y), lp = atyp(x, y);
    if (ld == 0. && lp == 0.) return;
    const T w0 = svc(x, y), w1 = svc(x, y + 1);
    const T cy0 = dtdx * w0, cy1 = dtdx * w1;
    const T den = T(1) / (T(1) - dtdy * (w1 - w0));
    double lden = 0.;
    inner_adj(sdp.ptr(x, y), sdp.w, cy0, cy1, den, rA, ld, asdp.ptr(x, y), TX + 6, lden);
    inner_adj(spt.ptr(x, y), spt.w, cy0, cy1, den, rA, lp, aspt.ptr(x, y), TX + 6, lden);
    const double lw = dtdy * den * den * lden;
    if (lw != 0.) {
      sadd(asvc.ptr(x, y + 1), lw);
      sadd(asvc.ptr(x, y), -lw);
    }
  });
  aregion<TX, TY + 6>(ox, oy - 3, [&](int x, int y) {
    const double ld = atxd(x, y), lp = atxp(x, y);
    if (ld == 0. && lp == 0.) return;
    const T w0 = suc(x, y), w1 = suc(x + 1, y);
    const T cx0 = dtdx * w0, cx1 = dtdx * w1;
    const T den = T(1) / (T(1) - dtdx * (w1 - w0));
    double lden = 0.;
    inner_adj(sdp.ptr(x, y), 1, cx0, cx1, den, rA, ld, asdp.ptr(x, y), 1, lden);
    inner_adj(spt.ptr(x, y), 1, cx0, cx1, den, rA, lp, aspt.ptr(x, y), 1, lden);
    const double lw = dtdx * den * den * lden;
    if (lw != 0.) {
      sadd(asuc.ptr(x + 1, y), lw);
      sadd(asuc.ptr(x, y), -lw);
    }
  });
  __syncthreads();
  if (CGRID) {  // C-grid winds from the D-grid winds (:109-117)
    aregion<TX + 1, TY + 6>(ox, oy - 3, [&](int x, int y) {
      const double l = .25 * asuc(x, y);
      if (l == 0.) return;
      sadd(asu.ptr(x, y), l);
      sadd(asu.ptr(x - 1, y), l);
      sadd(asu.ptr(x, y + 1), l);
      sadd(asu.ptr(x - 1, y + 1), l);
    });
    aregion<TX + 6, TY + 1>(ox - 3, oy, [&](int x, int y) {
      const double l = .25 * asvc(x, y);
      if (l == 0.) return;
      sadd(asv.ptr(x, y), l);
      sadd(asv.ptr(x, y - 1), l);
      sadd(asv.ptr(x + 1, y), l);
      sadd(asv.ptr(x + 1, y - 1), l);
    });
    __syncthreads();
  }
  flush_box(asdp, TX + 6, TY + 6, lam_dp, g, k);
  flush_box(aspt, TX + 6, TY + 6, lam_pt, g, k);
  flush_box(asu, ALay::UW, ALay::UH, lam_u, g, k);
  flush_box(asv, ALay::VW, ALay::VH, lam_v, g, k);
}

// =================================================== C-momentum adjoint ====
// Adjoint of k_c_mom2: uc, vc of layer k from ud, vd of layers k and nlay
// and pkap, gz of levels k, k+1 (src/mod_sw_dyn.f90:294-414).
template <int TX, int TY>
struct CMomAdjL {
  using F = CMomL<double, TX, TY>;
  // the forward values the reverse reads (the layer-nlay A-grid winds are
  // recomputed where the reverse reads them; ke and lap are not needed)
  static constexpr size_t fwd = 2 * box_bytes<double>(TX + 6, TY + 6) +                       // uc1, vc1
                                box_bytes<double>(TX + 5, TY + 5) +                           // vor
                                box_bytes<double>(TX, TY + 5) + box_bytes<double>(TX + 5, TY) +  // tU, tV
                                box_bytes<double>(TX + 1, TY + 4) + box_bytes<double>(TX + 4, TY + 1) +  // mvy, mux
                                box_bytes<double>(TX, TY + 3) + box_bytes<double>(TX + 3, TY);  // mtU, mtV
  static constexpr size_t lam =
      2 * box_bytes<double>(TX + 6, TY + 6) + 2 * box_bytes<double>(TX + 1, TY + 1) +  // uc1, vc1, uaL, vaL
      box_bytes<double>(TX + 5, TY + 5) + box_bytes<double>(TX + 1, TY + 1) +          // vor, ke
      box_bytes<double>(TX, TY + 5) + box_bytes<double>(TX + 5, TY) +                  // tU, tV
      box_bytes<double>(TX + 1, TY + 1) +                                              // lap
      box_bytes<double>(TX + 1, TY + 4) + box_bytes<double>(TX + 4, TY + 1) +          // mvy, mux
      box_bytes<double>(TX, TY + 3) + box_bytes<double>(TX + 3, TY) +                  // mtU, mtV
      2 * box_bytes<double>(TX + 7, TY + 7) + 2 * box_bytes<double>(TX + 3, TY + 3) +  // ud, vd (k, nlay)
      4 * box_bytes<double>(TX + 1, TY + 1);                                           // pkap, gz (k, k+1)
  static constexpr size_t bytes = F::boxes + fwd + lam + 128;
};


// 3 CTAs per SM: shared memory (the layout above) and 85 registers a thread
template <int TX, int TY>
__global__ void __launch_bounds__(NTA, 3) k_c_mom_adj(const __grid_constant__ CUtensorMap m_ud,
                                                  const __grid_constant__ CUtensorMap m_vd,
                                                  const __grid_constant__ CUtensorMap m_udL,
                                                  const __grid_constant__ CUtensorMap m_vdL,
                                                  const __grid_constant__ CUtensorMap m_pk,
                                                  const __grid_constant__ CUtensorMap m_gz, Geom g, Consts c,
                                                  const double* __restrict__ lam_uc, const double* __restrict__ lam_vc,
                                                  double* lam_ud, double* lam_vd, double* lam_pk, double* lam_gz,
                                                  int* timeout) {
  using T = double;
  using Lay = CMomL<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = c.dt, dtdx = c.dtdx, dtdy = c.dtdy, rA = c.rA;
  const T rdx = c.rdx, rdy = c.rdy;
  if (!tile_active<TX, TY>(lam_uc, lam_vc, g, k, ox, oy, g.nx - 1, g.ny - 1, &s_ok)) return;

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  Sm<T> sud = tbox(ox - 4, oy - 3, Lay::WU, Lay::HU);
  Sm<T> svd = tbox(ox - 3, oy - 4, Lay::WV, Lay::HV);
  Sm<T> udL = tbox(ox - 2, oy - 2, Lay::WL, Lay::HL);
  Sm<T> vdL = tbox(ox - 2, oy - 2, Lay::WL, Lay::HL);
  Sm<T> pk0 = tbox(ox - 1, oy - 1, Lay::WP, Lay::HP);
  Sm<T> pk1 = tbox(ox - 1, oy - 1, Lay::WP, Lay::HP);
  Sm<T> gz0 = tbox(ox - 1, oy - 1, Lay::WP, Lay::HP);
  Sm<T> gz1 = tbox(ox - 1, oy - 1, Lay::WP, Lay::HP);
  {
    const TmaBox boxes[8] = {{&m_ud, sud.p, sud.x0, sud.y0, k},     {&m_vd, svd.p, svd.x0, svd.y0, k},
                             {&m_udL, udL.p, udL.x0, udL.y0, L - 1}, {&m_vdL, vdL.p, vdL.x0, vdL.y0, L - 1},
                             {&m_pk, pk0.p, pk0.x0, pk0.y0, k},      {&m_pk, pk1.p, pk1.x0, pk1.y0, k + 1},
                             {&m_gz, gz0.p, gz0.x0, gz0.y0, k},      {&m_gz, gz1.p, gz1.x0, gz1.y0, k + 1}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  Sm<T> uc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> vc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> vor = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> tU = carve<T>(p, ox, oy - 2, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 2, oy, TX + 5, TY);
  Sm<T> mvy = carve<T>(p, ox - 1, oy - 2, TX + 1, TY + 4);
  Sm<T> mux = carve<T>(p, ox - 2, oy - 1, TX + 4, TY + 1);
  Sm<T> mtU = carve<T>(p, ox, oy - 1, TX, TY + 3);
  Sm<T> mtV = carve<T>(p, ox - 1, oy, TX + 3, TY);
  unsigned char* lam0 = p;
  Sm<T> auc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> avc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> auaL = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> avaL = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> avor = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> ake = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> atU = carve<T>(p, ox, oy - 2, TX, TY + 5);
  Sm<T> atV = carve<T>(p, ox - 2, oy, TX + 5, TY);
  Sm<T> alap = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> amvy = carve<T>(p, ox - 1, oy - 2, TX + 1, TY + 4);
  Sm<T> amux = carve<T>(p, ox - 2, oy - 1, TX + 4, TY + 1);
  Sm<T> amtU = carve<T>(p, ox, oy - 1, TX, TY + 3);
  Sm<T> amtV = carve<T>(p, ox - 1, oy, TX + 3, TY);
  Sm<T> asud = carve<T>(p, ox - 4, oy - 3, TX + 7, TY + 7);
  Sm<T> asvd = carve<T>(p, ox - 3, oy - 4, TX + 7, TY + 7);
  Sm<T> audL = carve<T>(p, ox - 2, oy - 2, TX + 3, TY + 3);
  Sm<T> avdL = carve<T>(p, ox - 2, oy - 2, TX + 3, TY + 3);
  Sm<T> apk0 = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> apk1 = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> agz0 = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> agz1 = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  zero_smem(lam0, p);

  // ---- forward recomputation (as k_c_mom2)
  aregion<TX + 6, TY + 6>(ox - 3, oy - 3, [&](int x, int y) {
    T ub = T(.5) * (sud(x, y) + sud(x - 1, y));
    uc1(x, y) = T(.5) * (ub + T(.5) * (sud(x, y + 1) + sud(x - 1, y + 1)));
    T vb = T(.5) * (svd(x, y) + svd(x, y - 1));
    vc1(x, y) = T(.5) * (vb + T(.5) * (svd(x + 1, y) + svd(x + 1, y - 1)));
  });
  __syncthreads();
  const T f = c.coriolis;
  aregion<TX + 5, TY + 5>(ox - 2, oy - 2, [&](int x, int y) {
    vor(x, y) = f - (uc1(x, y) - uc1(x, y - 1)) * rdy + (vc1(x, y) - vc1(x - 1, y)) * rdx;
  });
  aregion<TX + 1, TY + 4>(ox - 1, oy - 2, [&](int x, int y) { mvy(x, y) = slope_at(vc1.ptr(x, y), TX + 6); });
  aregion<TX + 4, TY + 1>(ox - 2, oy - 1, [&](int x, int y) { mux(x, y) = slope_at(uc1.ptr(x, y), 1); });
  __syncthreads();
  aregion<TX, TY + 5>(ox, oy - 2, [&](int x, int y) {
    T c0 = dtdx * sud(x - 1, y), c1 = dtdx * sud(x, y);
    T den = T(1) / (T(1) - dtdx * (sud(x, y) - sud(x - 1, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  });
  aregion<TX + 5, TY>(ox - 2, oy, [&](int x, int y) {
    T c0 = dtdx * svd(x, y - 1), c1 = dtdx * svd(x, y);
    T den = T(1) / (T(1) - dtdy * (svd(x, y) - svd(x, y - 1)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  });
  const T rdx2 = c.rdx2, rdy2 = c.rdy2, rdxy = c.rdx2rdy2;
  __syncthreads();
  aregion<TX, TY + 3>(ox, oy - 1, [&](int x, int y) { mtU(x, y) = slope_at(tU.ptr(x, y), TX); });
  aregion<TX + 3, TY>(ox - 1, oy, [&](int x, int y) { mtV(x, y) = slope_at(tV.ptr(x, y), 1); });
  __syncthreads();

  // ---- reverse: uc, vc updates with the PGF (:325-339, 369-381, 399-411)
  const T vdx = c.vdx, vdy = c.vdy;
  aregion<TX, TY>(ox, oy, [&](int x, int y) {
    if (x >= g.nx || y >= g.ny) return;
    const long long o = g.at(x, y, k);
    const double lu = lam_uc[o], lv = lam_vc[o];
    if (lu != 0.) {
      sadd(auc1.ptr(x, y), lu);
      double lc = 0.;
      double F = flux_unc_adj(tU.ptr(x, y + 1), TX, mtU.ptr(x, y + 1), TX, dtdx * svd(x, y), dt * svd(x, y) * lu,
                                       atU.ptr(x, y + 1), TX, amtU.ptr(x, y + 1), TX, lc);
      sadd(asvd.ptr(x, y), dt * F * lu + dtdx * lc);
      sadd(alap.ptr(x, y + 1), dt * vdy * lu);
      sadd(alap.ptr(x, y), -dt * vdy * lu);
      sadd(ake.ptr(x, y), -dtdx * lu);
      sadd(ake.ptr(x - 1, y), dtdx * lu);
      PgfAdj a = pgf_adj(pk0(x, y), pk1(x - 1, y), gz0(x - 1, y), gz1(x, y), pk0(x - 1, y), pk1(x, y), gz1(x - 1, y),
                         gz0(x, y), dtdx * lu);
      sadd(apk0.ptr(x, y), a.dp0);
      sadd(apk1.ptr(x - 1, y), a.dp1);
      sadd(agz0.ptr(x - 1, y), a.dg0);
      sadd(agz1.ptr(x, y), a.dg1);
      sadd(apk0.ptr(x - 1, y), a.dp2);
      sadd(apk1.ptr(x, y), a.dp3);
      sadd(agz1.ptr(x - 1, y), a.dg2);
      sadd(agz0.ptr(x, y), a.dg3);
    }
    if (lv != 0.) {
      sadd(avc1.ptr(x, y), lv);
      double lc = 0.;
      double F = flux_unc_adj(tV.ptr(x + 1, y), 1, mtV.ptr(x + 1, y), 1, dtdx * sud(x, y), -dt * sud(x, y) * lv,
                                       atV.ptr(x + 1, y), 1, amtV.ptr(x + 1, y), 1, lc);
      sadd(asud.ptr(x, y), -dt * F * lv + dtdx * lc);
      sadd(alap.ptr(x + 1, y), -dt * vdx * lv);
      sadd(alap.ptr(x, y), dt * vdx * lv);
      sadd(ake.ptr(x, y), -dtdy * lv);
      sadd(ake.ptr(x, y - 1), dtdy * lv);
      PgfAdj a = pgf_adj(pk0(x, y), pk1(x, y - 1), gz0(x, y - 1), gz1(x, y), pk0(x, y - 1), pk1(x, y), gz1(x, y - 1),
                         gz0(x, y), dtdy * lv);
      sadd(apk0.ptr(x, y), a.dp0);
      sadd(apk1.ptr(x, y - 1), a.dp1);
      sadd(agz0.ptr(x, y - 1), a.dg0);
      sadd(agz1.ptr(x, y), a.dg1);
      sadd(apk0.ptr(x, y - 1), a.dp2);
      sadd(apk1.ptr(x, y), a.dp3);
      sadd(agz1.ptr(x, y - 1), a.dg2);
      sadd(agz0.ptr(x, y), a.dg3);
    }
  });
  __syncthreads();
  // slopes of the vorticity-flux sweeps; Laplacian (:388-397, gather);
  // kinetic energy (:299-317)
  aregion<TX, TY + 3>(ox, oy - 1, [&](int x, int y) { slope_adj(tU.ptr(x, y), TX, amtU(x, y), atU.ptr(x, y), TX); });
  aregion<TX + 3, TY>(ox - 1, oy, [&](int x, int y) { slope_adj(tV.ptr(x, y), 1, amtV(x, y), atV.ptr(x, y), 1); });
  auto inL = [&](int x, int y) { return x >= ox && x <= ox + TX && y >= oy && y <= oy + TY; };
  aregion<TX + 3, TY + 3>(ox - 1, oy - 1, [&](int x, int y) {
    double a = 0.;
    if (inL(x, y)) a += -2. * rdxy * alap(x, y);
    if (inL(x - 1, y)) a += rdx2 * alap(x - 1, y);
    if (inL(x + 1, y)) a += rdx2 * alap(x + 1, y);
    if (inL(x, y - 1)) a += rdy2 * alap(x, y - 1);
    if (inL(x, y + 1)) a += rdy2 * alap(x, y + 1);
    avor(x, y) += a;
  });
  aregion<TX + 1, TY + 1>(ox - 1, oy - 1, [&](int x, int y) {
    const double l = ake(x, y);
    if (l == 0.) return;
    T ua, va;
    al_winds<T>(udL, vdL, x, y, ua, va);
    double lcy = 0., lcx = 0.;
    double fy = flux_unc_adj(vc1.ptr(x, y + 1), TX + 6, mvy.ptr(x, y + 1), TX + 1, dtdy * va, .5 * va * l,
                                      avc1.ptr(x, y + 1), TX + 6, amvy.ptr(x, y + 1), TX + 1, lcy);
    double fx = flux_unc_adj(uc1.ptr(x + 1, y), 1, mux.ptr(x + 1, y), 1, dtdx * ua, .5 * ua * l,
                                      auc1.ptr(x + 1, y), 1, amux.ptr(x + 1, y), 1, lcx);
    avaL(x, y) += .5 * fy * l + dtdy * lcy;
    auaL(x, y) += .5 * fx * l + dtdx * lcx;
  });
  __syncthreads();
  // slopes of the KE sweeps; inner vorticity sweeps (:344-367, 383-397); layer-nlay A-grid winds
  aregion<TX + 1, TY + 4>(ox - 1, oy - 2, [&](int x, int y) { slope_adj(vc1.ptr(x, y), TX + 6, amvy(x, y), avc1.ptr(x, y), TX + 6); });
  aregion<TX + 4, TY + 1>(ox - 2, oy - 1, [&](int x, int y) { slope_adj(uc1.ptr(x, y), 1, amux(x, y), auc1.ptr(x, y), 1); });
  aregion<TX, TY + 5>(ox, oy - 2, [&](int x, int y) {
    const double l = atU(x, y);
    if (l == 0.) return;
    const T w0 = sud(x - 1, y), w1 = sud(x, y);
    const T den = T(1) / (T(1) - dtdx * (w1 - w0));
    double lden = 0.;
    inner_adj(vor.ptr(x, y), 1, dtdx * w0, dtdx * w1, den, rA, l, avor.ptr(x, y), 1, lden);
    const double lw = dtdx * den * den * lden;
    if (lw != 0.) {
      sadd(asud.ptr(x, y), lw);
      sadd(asud.ptr(x - 1, y), -lw);
    }
  });
  aregion<TX + 5, TY>(ox - 2, oy, [&](int x, int y) {
    const double l = atV(x, y);
    if (l == 0.) return;
    const T w0 = svd(x, y - 1), w1 = svd(x, y);
    const T den = T(1) / (T(1) - dtdy * (w1 - w0));
    double lden = 0.;
    inner_adj(vor.ptr(x, y), TX + 5, dtdx * w0, dtdx * w1, den, rA, l, avor.ptr(x, y), TX + 5, lden);
    const double lw = dtdy * den * den * lden;
    if (lw != 0.) {
      sadd(asvd.ptr(x, y), lw);
      sadd(asvd.ptr(x, y - 1), -lw);
    }
  });
  aregion<TX + 1, TY + 1>(ox - 1, oy - 1, [&](int x, int y) {
    const double lu = auaL(x, y), lv = avaL(x, y);
    if (lu != 0.) {
      sadd(audL.ptr(x, y), .25 * lu);
      sadd(audL.ptr(x - 1, y), .125 * lu);
      sadd(audL.ptr(x, y + 1), .25 * lu);
      sadd(audL.ptr(x - 1, y + 1), .125 * lu);
      sadd(audL.ptr(x + 1, y), .125 * lu);
      sadd(audL.ptr(x + 1, y + 1), .125 * lu);
    }
    if (lv != 0.) {
      sadd(avdL.ptr(x, y), .25 * lv);
      sadd(avdL.ptr(x, y - 1), .125 * lv);
      sadd(avdL.ptr(x + 1, y), .25 * lv);
      sadd(avdL.ptr(x + 1, y - 1), .125 * lv);
      sadd(avdL.ptr(x, y + 1), .125 * lv);
      sadd(avdL.ptr(x + 1, y + 1), .125 * lv);
    }
  });
  __syncthreads();
  // vorticity (:319-323)
  aregion<TX + 5, TY + 5>(ox - 2, oy - 2, [&](int x, int y) {
    const double l = avor(x, y);
    if (l == 0.) return;
    sadd(auc1.ptr(x, y), -rdy * l);
    sadd(auc1.ptr(x, y - 1), rdy * l);
    sadd(avc1.ptr(x, y), rdx * l);
    sadd(avc1.ptr(x - 1, y), -rdx * l);
  });
  __syncthreads();
  // C-grid winds of the layer (:110-117)
  aregion<TX + 6, TY + 6>(ox - 3, oy - 3, [&](int x, int y) {
    const double lu = .25 * auc1(x, y), lv = .25 * avc1(x, y);
    if (lu != 0.) {
      sadd(asud.ptr(x, y), lu);
      sadd(asud.ptr(x - 1, y), lu);
      sadd(asud.ptr(x, y + 1), lu);
      sadd(asud.ptr(x - 1, y + 1), lu);
    }
    if (lv != 0.) {
      sadd(asvd.ptr(x, y), lv);
      sadd(asvd.ptr(x, y - 1), lv);
      sadd(asvd.ptr(x + 1, y), lv);
      sadd(asvd.ptr(x + 1, y - 1), lv);
    }
  });
  __syncthreads();
  flush_box(asud, TX + 7, TY + 7, lam_ud, g, k);
  flush_box(asvd, TX + 7, TY + 7, lam_vd, g, k);
  flush_box(audL, TX + 3, TY + 3, lam_ud, g, L - 1);
  flush_box(avdL, TX + 3, TY + 3, lam_vd, g, L - 1);
  flush_box(apk0, TX + 1, TY + 1, lam_pk, g, k);
  flush_box(apk1, TX + 1, TY + 1, lam_pk, g, k + 1);
  flush_box(agz0, TX + 1, TY + 1, lam_gz, g, k);
  flush_box(agz1, TX + 1, TY + 1, lam_gz, g, k + 1);
}

// =================================================== D-momentum adjoint ====
// Adjoint of k_d_mom2: ud, vd of layer k from the old ud, vd, uc, vc of
// layers k and nlay and pkapb, gzb of levels k, k+1 (src/mod_sw_dyn.f90:634-771).
// The reverse splits into two chains that share only the adjoints of the
// inputs, which meet in global memory through the flush atomics: the
// kinetic-energy flux (:639-657: its PPM sweeps of ud, vd with the layer-nlay
// B-grid winds) and everything else (the vorticity-flux sweeps, the
// divergence and vorticity damping, the PGF and the direct terms).  One
// kernel each keeps the shared memory of a CTA small enough for 5 and 3
// CTAs per SM where one kernel held 2.

// the kinetic-energy chain: ud, vd and the layer-nlay C-grid winds
template <int TX, int TY>
struct DMomKeAdjL {
  using F = DMomL<double, TX, TY>;
  static constexpr size_t boxes = 2 * tma_box_bytes(F::WU, F::HU, 8) + tma_box_bytes(F::WUL, F::HUL, 8) +
                                  tma_box_bytes(F::WVL, F::HVL, 8);
  static constexpr uint32_t tx_bytes = (uint32_t)((2 * F::WU * F::HU + F::WUL * F::HUL + F::WVL * F::HVL) * 8);
  static constexpr size_t fwd = F::slopes_ke + F::edges_ke;
  static constexpr size_t lam = box_bytes<double>(TX + 1, TY + 1) + F::edges_ke + F::slopes_ke +
                                2 * box_bytes<double>(TX + 6, TY + 6) + box_bytes<double>(TX + 1, TY + 5) +
                                box_bytes<double>(TX + 5, TY + 1);
  static constexpr size_t bytes = boxes + fwd + lam + 128;
};

// the rest: all ten input boxes
template <int TX, int TY>
struct DMomVfAdjL {
  using F = DMomL<double, TX, TY>;
  static constexpr size_t fwd = box_bytes<double>(TX + 5, TY + 5) + box_bytes<double>(TX, TY + 5) +
                                box_bytes<double>(TX + 5, TY) + F::slopes_vf + F::edges_vf;
  static constexpr size_t lam = 2 * box_bytes<double>(TX + 5, TY + 5) + box_bytes<double>(TX + 3, TY + 3) +
                                2 * box_bytes<double>(TX + 1, TY + 1) + box_bytes<double>(TX, TY + 5) +
                                box_bytes<double>(TX + 5, TY) + F::slopes_vf + F::edges_vf +
                                2 * box_bytes<double>(TX + 6, TY + 6) + box_bytes<double>(TX + 1, TY + 5) +
                                box_bytes<double>(TX + 5, TY + 1) + 2 * box_bytes<double>(TX, TY) +
                                4 * box_bytes<double>(TX + 1, TY + 1);
  static constexpr size_t bytes = F::boxes + fwd + lam + 128;
};

template <int TX, int TY>
__global__ void __launch_bounds__(NTA, 4) k_d_mom_adj_ke(const __grid_constant__ CUtensorMap m_ud,
                                                     const __grid_constant__ CUtensorMap m_vd,
                                                     const __grid_constant__ CUtensorMap m_ucL,
                                                     const __grid_constant__ CUtensorMap m_vcL, Geom g, Consts c,
                                                     const double* __restrict__ lam_udo,
                                                     const double* __restrict__ lam_vdo, double* lam_ud,
                                                     double* lam_vd, double* lam_uc, double* lam_vc, int* timeout) {
  using T = double;
  using Lay = DMomL<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dtdx = c.dtdx, dtdy = c.dtdy;
  if (!tile_active<TX, TY>(lam_udo, lam_vdo, g, k, ox, oy, g.nx - 1, g.ny - 1, &s_ok)) return;

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  Sm<T> sud = tbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<T> svd = tbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<T> ucL = tbox(ox, oy - 3, Lay::WUL, Lay::HUL);
  Sm<T> vcL = tbox(ox - 3, oy, Lay::WVL, Lay::HVL);
  {
    const TmaBox boxes[4] = {{&m_ud, sud.p, sud.x0, sud.y0, k},
                             {&m_vd, svd.p, svd.x0, svd.y0, k},
                             {&m_ucL, ucL.p, ucL.x0, ucL.y0, L - 1},
                             {&m_vcL, vcL.p, vcL.x0, vcL.y0, L - 1}};
    if (!tma_fetch(boxes, DMomKeAdjL<TX, TY>::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  Sm<T> mvy = carve<T>(p, ox, oy - 2, TX + 1, TY + 4);
  Sm<T> mux = carve<T>(p, ox - 2, oy, TX + 4, TY + 1);
  Sm<T> lvy = carve<T>(p, ox, oy - 1, TX + 1, TY + 2), rvy = carve<T>(p, ox, oy - 1, TX + 1, TY + 2);
  Sm<T> lux = carve<T>(p, ox - 1, oy, TX + 2, TY + 1), rux = carve<T>(p, ox - 1, oy, TX + 2, TY + 1);
  unsigned char* lam0 = p;
  Sm<T> ake = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> alvy = carve<T>(p, ox, oy - 1, TX + 1, TY + 2), arvy = carve<T>(p, ox, oy - 1, TX + 1, TY + 2);
  Sm<T> alux = carve<T>(p, ox - 1, oy, TX + 2, TY + 1), arux = carve<T>(p, ox - 1, oy, TX + 2, TY + 1);
  Sm<T> amvy = carve<T>(p, ox, oy - 2, TX + 1, TY + 4);
  Sm<T> amux = carve<T>(p, ox - 2, oy, TX + 4, TY + 1);
  Sm<T> asud = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> asvd = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> aucL = carve<T>(p, ox, oy - 3, TX + 1, TY + 5);
  Sm<T> avcL = carve<T>(p, ox - 3, oy, TX + 5, TY + 1);
  zero_smem(lam0, p);

  // ---- forward recomputation (as k_d_mom2): slopes and edges of the KE sweeps
  regions(reg<TX + 1, TY + 4>(ox, oy - 2, [&](int x, int y) { mvy(x, y) = slope_at(svd.ptr(x, y), Lay::WU); }),
          reg<TX + 4, TY + 1>(ox - 2, oy, [&](int x, int y) { mux(x, y) = slope_at(sud.ptr(x, y), 1); }));
  __syncthreads();
  regions(reg<TX + 1, TY + 2>(ox, oy - 1, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(svd.ptr(x, y), Lay::WU, mvy.ptr(x, y), TX + 1, eL, eR);
    lvy(x, y) = eL;
    rvy(x, y) = eR;
  }),
          reg<TX + 2, TY + 1>(ox - 1, oy, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(sud.ptr(x, y), 1, mux.ptr(x, y), 1, eL, eR);
    lux(x, y) = eL;
    rux(x, y) = eR;
  }));
  __syncthreads();

  // ---- reverse: the kinetic-energy terms of the ud, vd updates (:665-679)
  aregion<TX, TY>(ox, oy, [&](int x, int y) {
    if (x >= g.nx || y >= g.ny) return;
    const long long o = g.at(x, y, k);
    const double lu = lam_udo[o], lv = lam_vdo[o];
    if (lu != 0.) {
      sadd(ake.ptr(x + 1, y), -dtdx * lu);
      sadd(ake.ptr(x, y), dtdx * lu);
    }
    if (lv != 0.) {
      sadd(ake.ptr(x, y + 1), -dtdy * lv);
      sadd(ake.ptr(x, y), dtdy * lv);
    }
  });
  __syncthreads();
  // kinetic energy (:639-657) with the layer-nlay B-grid winds (:441-444),
  // which the reverse recomputes where it reads them
  aregion<TX + 1, TY + 1>(ox, oy, [&](int x, int y) {
    const double l = ake(x, y);
    if (l == 0.) return;
    const T ub = T(.5) * (ucL(x, y) + ucL(x, y - 1));
    const T vb = T(.5) * (vcL(x, y) + vcL(x - 1, y));
    double lcy = 0., lcx = 0.;
    double fy = flux_con_adj(svd.ptr(x, y), Lay::WU, lvy.ptr(x, y), rvy.ptr(x, y), TX + 1, dtdy * vb, .5 * vb * l,
                             asvd.ptr(x, y), TX + 6, alvy.ptr(x, y), arvy.ptr(x, y), TX + 1, lcy);
    double fx = flux_con_adj(sud.ptr(x, y), 1, lux.ptr(x, y), rux.ptr(x, y), 1, dtdx * ub, .5 * ub * l, asud.ptr(x, y), 1,
                             alux.ptr(x, y), arux.ptr(x, y), 1, lcx);
    const double lu = .5 * (.5 * fx * l + dtdx * lcx), lv = .5 * (.5 * fy * l + dtdy * lcy);
    if (lu != 0.) {
      sadd(aucL.ptr(x, y), lu);
      sadd(aucL.ptr(x, y - 1), lu);
    }
    if (lv != 0.) {
      sadd(avcL.ptr(x, y), lv);
      sadd(avcL.ptr(x - 1, y), lv);
    }
  });
  __syncthreads();
  // edges of the KE sweeps
  regions(reg<TX + 1, TY + 2>(ox, oy - 1, [&](int x, int y) {
    edges_con_adj(svd.ptr(x, y), Lay::WU, mvy.ptr(x, y), TX + 1, alvy(x, y), arvy(x, y), asvd.ptr(x, y), TX + 6,
                  amvy.ptr(x, y), TX + 1);
  }),
          reg<TX + 2, TY + 1>(ox - 1, oy, [&](int x, int y) {
    edges_con_adj(sud.ptr(x, y), 1, mux.ptr(x, y), 1, alux(x, y), arux(x, y), asud.ptr(x, y), 1, amux.ptr(x, y), 1);
  }));
  __syncthreads();
  // slopes of the KE sweeps
  regions(reg<TX + 1, TY + 4>(ox, oy - 2, [&](int x, int y) {
    slope_adj(svd.ptr(x, y), Lay::WU, amvy(x, y), asvd.ptr(x, y), TX + 6);
  }),
          reg<TX + 4, TY + 1>(ox - 2, oy, [&](int x, int y) { slope_adj(sud.ptr(x, y), 1, amux(x, y), asud.ptr(x, y), 1); }));
  __syncthreads();
  flush_box(asud, TX + 6, TY + 6, lam_ud, g, k);
  flush_box(asvd, TX + 6, TY + 6, lam_vd, g, k);
  flush_box(aucL, TX + 1, TY + 5, lam_uc, g, L - 1);
  flush_box(avcL, TX + 5, TY + 1, lam_vc, g, L - 1);
}

template <int TX, int TY>
__global__ void __launch_bounds__(NTA, 3) k_d_mom_adj_vf(const __grid_constant__ CUtensorMap m_ud,
                                                     const __grid_constant__ CUtensorMap m_vd,
                                                     const __grid_constant__ CUtensorMap m_ucL,
                                                     const __grid_constant__ CUtensorMap m_vcL,
                                                     const __grid_constant__ CUtensorMap m_uc,
                                                     const __grid_constant__ CUtensorMap m_vc,
                                                     const __grid_constant__ CUtensorMap m_pkb,
                                                     const __grid_constant__ CUtensorMap m_gzb, Geom g, Consts c,
                                                     const double* __restrict__ lam_udo,
                                                     const double* __restrict__ lam_vdo, double* lam_ud,
                                                     double* lam_vd, double* lam_uc, double* lam_vc, double* lam_pkb,
                                                     double* lam_gzb, int* timeout) {
  using T = double;
  using Lay = DMomL<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = c.dt, dtdx = c.dtdx, dtdy = c.dtdy, rA = c.rA;
  const T rdx = c.rdx, rdy = c.rdy;
  if (!tile_active<TX, TY>(lam_udo, lam_vdo, g, k, ox, oy, g.nx - 1, g.ny - 1, &s_ok)) return;

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  Sm<T> sud = tbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<T> svd = tbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<T> ucL = tbox(ox, oy - 3, Lay::WUL, Lay::HUL);
  Sm<T> vcL = tbox(ox - 3, oy, Lay::WVL, Lay::HVL);
  Sm<T> suc = tbox(ox, oy, Lay::WC, Lay::HC);
  Sm<T> svc = tbox(ox, oy, Lay::WC, Lay::HC);
  Sm<T> pb0 = tbox(ox, oy, Lay::WP, Lay::HP);
  Sm<T> pb1 = tbox(ox, oy, Lay::WP, Lay::HP);
  Sm<T> gb0 = tbox(ox, oy, Lay::WP, Lay::HP);
  Sm<T> gb1 = tbox(ox, oy, Lay::WP, Lay::HP);
  {
    const TmaBox boxes[10] = {
        {&m_ud, sud.p, sud.x0, sud.y0, k},       {&m_vd, svd.p, svd.x0, svd.y0, k},
        {&m_ucL, ucL.p, ucL.x0, ucL.y0, L - 1},  {&m_vcL, vcL.p, vcL.x0, vcL.y0, L - 1},
        {&m_uc, suc.p, suc.x0, suc.y0, k},       {&m_vc, svc.p, svc.x0, svc.y0, k},
        {&m_pkb, pb0.p, pb0.x0, pb0.y0, k},      {&m_pkb, pb1.p, pb1.x0, pb1.y0, k + 1},
        {&m_gzb, gb0.p, gb0.x0, gb0.y0, k},      {&m_gzb, gb1.p, gb1.x0, gb1.y0, k + 1}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  Sm<T> vor = carve<T>(p, ox - 3, oy - 3, TX + 5, TY + 5);
  Sm<T> tU = carve<T>(p, ox, oy - 3, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 3, oy, TX + 5, TY);
  Sm<T> mtU = carve<T>(p, ox, oy - 2, TX, TY + 3);
  Sm<T> mtV = carve<T>(p, ox - 2, oy, TX + 3, TY);
  Sm<T> ltU = carve<T>(p, ox, oy - 1, TX, TY + 1), rtU = carve<T>(p, ox, oy - 1, TX, TY + 1);
  Sm<T> ltV = carve<T>(p, ox - 1, oy, TX + 1, TY), rtV = carve<T>(p, ox - 1, oy, TX + 1, TY);
  unsigned char* lam0 = p;
  Sm<T> avor = carve<T>(p, ox - 3, oy - 3, TX + 5, TY + 5);
  Sm<T> adv0 = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> adv2 = carve<T>(p, ox - 1, oy - 1, TX + 3, TY + 3);
  Sm<T> adv4 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> atU = carve<T>(p, ox, oy - 3, TX, TY + 5);
  Sm<T> atV = carve<T>(p, ox - 3, oy, TX + 5, TY);
  Sm<T> alap = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> amtU = carve<T>(p, ox, oy - 2, TX, TY + 3);
  Sm<T> amtV = carve<T>(p, ox - 2, oy, TX + 3, TY);
  Sm<T> altU = carve<T>(p, ox, oy - 1, TX, TY + 1), artU = carve<T>(p, ox, oy - 1, TX, TY + 1);
  Sm<T> altV = carve<T>(p, ox - 1, oy, TX + 1, TY), artV = carve<T>(p, ox - 1, oy, TX + 1, TY);
  Sm<T> asud = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> asvd = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> aucL = carve<T>(p, ox, oy - 3, TX + 1, TY + 5);
  Sm<T> avcL = carve<T>(p, ox - 3, oy, TX + 5, TY + 1);
  Sm<T> asuc = carve<T>(p, ox, oy, TX, TY);
  Sm<T> asvc = carve<T>(p, ox, oy, TX, TY);
  Sm<T> apb0 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> apb1 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> agb0 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> agb1 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  zero_smem(lam0, p);

  // ---- forward recomputation (as k_d_mom2): vorticity and its flux sweeps
  const T f = c.coriolis;
  aregion<TX + 5, TY + 5>(ox - 3, oy - 3, [&](int x, int y) {
    vor(x, y) = f - (sud(x, y + 1) - sud(x, y)) * rdy + (svd(x + 1, y) - svd(x, y)) * rdx;
  });
  __syncthreads();
  const T rdx2 = c.rdx2, rdy2 = c.rdy2, rdxy = c.rdx2rdy2;
  regions(reg<TX, TY + 5>(ox, oy - 3, [&](int x, int y) {
    T c0 = dtdx * ucL(x, y), c1 = dtdx * ucL(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (ucL(x + 1, y) - ucL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }),
          reg<TX + 5, TY>(ox - 3, oy, [&](int x, int y) {
    T c0 = dtdx * vcL(x, y), c1 = dtdx * vcL(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (vcL(x, y + 1) - vcL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }));
  __syncthreads();
  const T divdamp = c.divdamp;
  regions(reg<TX, TY + 3>(ox, oy - 2, [&](int x, int y) { mtU(x, y) = slope_at(tU.ptr(x, y), TX); }),
          reg<TX + 3, TY>(ox - 2, oy, [&](int x, int y) { mtV(x, y) = slope_at(tV.ptr(x, y), 1); }));
  __syncthreads();
  regions(reg<TX, TY + 1>(ox, oy - 1, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(tU.ptr(x, y), TX, mtU.ptr(x, y), TX, eL, eR);
    ltU(x, y) = eL;
    rtU(x, y) = eR;
  }),
          reg<TX + 1, TY>(ox - 1, oy, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(tV.ptr(x, y), 1, mtV.ptr(x, y), 1, eL, eR);
    ltV(x, y) = eL;
    rtV(x, y) = eR;
  }));
  __syncthreads();

  // ---- reverse: ud, vd updates without the KE terms, with the B-grid PGF
  // (:665-679, 724-738, 755-769)
  const T vdx = c.vdx, vdy = c.vdy;
  aregion<TX, TY>(ox, oy, [&](int x, int y) {
    if (x >= g.nx || y >= g.ny) return;
    const long long o = g.at(x, y, k);
    const double lu = lam_udo[o], lv = lam_vdo[o];
    if (lu != 0.) {
      sadd(asud.ptr(x, y), lu);
      double lc = 0.;
      double F = flux_con_adj(tU.ptr(x, y), TX, ltU.ptr(x, y), rtU.ptr(x, y), TX, dtdx * vcL(x, y), dt * svc(x, y) * lu,
                              atU.ptr(x, y), TX, altU.ptr(x, y), artU.ptr(x, y), TX, lc);
      sadd(avcL.ptr(x, y), dtdx * lc);
      sadd(asvc.ptr(x, y), dt * F * lu);
      sadd(alap.ptr(x, y), dt * vdy * lu);
      sadd(alap.ptr(x, y - 1), -dt * vdy * lu);
      sadd(adv4.ptr(x + 1, y), dtdx * lu);
      sadd(adv4.ptr(x, y), -dtdx * lu);
      PgfAdj a = pgf_adj(pb0(x + 1, y), pb1(x, y), gb0(x, y), gb1(x + 1, y), pb0(x, y), pb1(x + 1, y), gb1(x, y),
                         gb0(x + 1, y), dtdx * lu);
      sadd(apb0.ptr(x + 1, y), a.dp0);
      sadd(apb1.ptr(x, y), a.dp1);
      sadd(agb0.ptr(x, y), a.dg0);
      sadd(agb1.ptr(x + 1, y), a.dg1);
      sadd(apb0.ptr(x, y), a.dp2);
      sadd(apb1.ptr(x + 1, y), a.dp3);
      sadd(agb1.ptr(x, y), a.dg2);
      sadd(agb0.ptr(x + 1, y), a.dg3);
    }
    if (lv != 0.) {
      sadd(asvd.ptr(x, y), lv);
      double lc = 0.;
      double F = flux_con_adj(tV.ptr(x, y), 1, ltV.ptr(x, y), rtV.ptr(x, y), 1, dtdx * ucL(x, y), -dt * suc(x, y) * lv,
                              atV.ptr(x, y), 1, altV.ptr(x, y), artV.ptr(x, y), 1, lc);
      sadd(aucL.ptr(x, y), dtdx * lc);
      sadd(asuc.ptr(x, y), -dt * F * lv);
      sadd(alap.ptr(x, y), -dt * vdx * lv);
      sadd(alap.ptr(x - 1, y), dt * vdx * lv);
      sadd(adv4.ptr(x, y + 1), dtdy * lv);
      sadd(adv4.ptr(x, y), -dtdy * lv);
      PgfAdj a = pgf_adj(pb0(x, y + 1), pb1(x, y), gb0(x, y), gb1(x, y + 1), pb0(x, y), pb1(x, y + 1), gb1(x, y),
                         gb0(x, y + 1), dtdy * lv);
      sadd(apb0.ptr(x, y + 1), a.dp0);
      sadd(apb1.ptr(x, y), a.dp1);
      sadd(agb0.ptr(x, y), a.dg0);
      sadd(agb1.ptr(x, y + 1), a.dg1);
      sadd(apb0.ptr(x, y), a.dp2);
      sadd(apb1.ptr(x, y + 1), a.dp3);
      sadd(agb1.ptr(x, y), a.dg2);
      sadd(agb0.ptr(x, y + 1), a.dg3);
    }
  });
  __syncthreads();
  // edges of the vorticity-flux sweeps; del^4 (:695-702, gather); Laplacian
  // of the vorticity (:712-721, gather)
  auto in4 = [&](int x, int y) { return x >= ox && x <= ox + TX && y >= oy && y <= oy + TY; };
  auto inP = [&](int x, int y) { return x >= ox - 1 && x <= ox + TX - 1 && y >= oy - 1 && y <= oy + TY - 1; };
  regions(reg<TX, TY + 1>(ox, oy - 1, [&](int x, int y) {
    edges_con_adj(tU.ptr(x, y), TX, mtU.ptr(x, y), TX, altU(x, y), artU(x, y), atU.ptr(x, y), TX, amtU.ptr(x, y), TX);
  }),
          reg<TX + 1, TY>(ox - 1, oy, [&](int x, int y) {
    edges_con_adj(tV.ptr(x, y), 1, mtV.ptr(x, y), 1, altV(x, y), artV(x, y), atV.ptr(x, y), 1, amtV.ptr(x, y), 1);
  }),
          reg<TX + 3, TY + 3>(ox - 1, oy - 1, [&](int x, int y) {
    double a = 0.;
    if (in4(x, y)) a += -2. * rdxy * adv4(x, y);
    if (in4(x - 1, y)) a += rdx2 * adv4(x - 1, y);
    if (in4(x + 1, y)) a += rdx2 * adv4(x + 1, y);
    if (in4(x, y - 1)) a += rdy2 * adv4(x, y - 1);
    if (in4(x, y + 1)) a += rdy2 * adv4(x, y + 1);
    adv2(x, y) = divdamp * a;
  }),
          reg<TX + 3, TY + 3>(ox - 2, oy - 2, [&](int x, int y) {
    double a = 0.;
    if (inP(x, y)) a += -2. * rdxy * alap(x, y);
    if (inP(x - 1, y)) a += rdx2 * alap(x - 1, y);
    if (inP(x + 1, y)) a += rdx2 * alap(x + 1, y);
    if (inP(x, y - 1)) a += rdy2 * alap(x, y - 1);
    if (inP(x, y + 1)) a += rdy2 * alap(x, y + 1);
    avor(x, y) += a;
  }));
  __syncthreads();
  // slopes of the vorticity-flux sweeps; del^2 of the divergence (gather)
  auto in2 = [&](int x, int y) { return x >= ox - 1 && x <= ox + TX + 1 && y >= oy - 1 && y <= oy + TY + 1; };
  regions(reg<TX, TY + 3>(ox, oy - 2, [&](int x, int y) { slope_adj(tU.ptr(x, y), TX, amtU(x, y), atU.ptr(x, y), TX); }),
          reg<TX + 3, TY>(ox - 2, oy, [&](int x, int y) { slope_adj(tV.ptr(x, y), 1, amtV(x, y), atV.ptr(x, y), 1); }),
          reg<TX + 5, TY + 5>(ox - 2, oy - 2, [&](int x, int y) {
    double a = 0.;
    if (in2(x, y)) a += -2. * rdxy * adv2(x, y);
    if (in2(x - 1, y)) a += rdx2 * adv2(x - 1, y);
    if (in2(x + 1, y)) a += rdx2 * adv2(x + 1, y);
    if (in2(x, y - 1)) a += rdy2 * adv2(x, y - 1);
    if (in2(x, y + 1)) a += rdy2 * adv2(x, y + 1);
    adv0(x, y) = a;
  }));
  __syncthreads();
  // inner vorticity sweeps (:704-722, 740-753); divergence (:682-685)
  regions(reg<TX, TY + 5>(ox, oy - 3, [&](int x, int y) {
    const double l = atU(x, y);
    if (l == 0.) return;
    const T w0 = ucL(x, y), w1 = ucL(x + 1, y);
    const T den = T(1) / (T(1) - dtdx * (w1 - w0));
    double lden = 0.;
    inner_adj(vor.ptr(x, y), 1, dtdx * w0, dtdx * w1, den, rA, l, avor.ptr(x, y), 1, lden);
    const double lw = dtdx * den * den * lden;
    if (lw != 0.) {
      sadd(aucL.ptr(x + 1, y), lw);
      sadd(aucL.ptr(x, y), -lw);
    }
  }),
          reg<TX + 5, TY>(ox - 3, oy, [&](int x, int y) {
    const double l = atV(x, y);
    if (l == 0.) return;
    const T w0 = vcL(x, y), w1 = vcL(x, y + 1);
    const T den = T(1) / (T(1) - dtdy * (w1 - w0));
    double lden = 0.;
    inner_adj(vor.ptr(x, y), TX + 5, dtdx * w0, dtdx * w1, den, rA, l, avor.ptr(x, y), TX + 5, lden);
    const double lw = dtdy * den * den * lden;
    if (lw != 0.) {
      sadd(avcL.ptr(x, y + 1), lw);
      sadd(avcL.ptr(x, y), -lw);
    }
  }),
          reg<TX + 5, TY + 5>(ox - 2, oy - 2, [&](int x, int y) {
    const double l = adv0(x, y);
    if (l == 0.) return;
    sadd(asud.ptr(x, y), rdx * l);
    sadd(asud.ptr(x - 1, y), -rdx * l);
    sadd(asvd.ptr(x, y), rdy * l);
    sadd(asvd.ptr(x, y - 1), -rdy * l);
  }));
  __syncthreads();
  // vorticity (:659-663)
  aregion<TX + 5, TY + 5>(ox - 3, oy - 3, [&](int x, int y) {
    const double l = avor(x, y);
    if (l == 0.) return;
    sadd(asud.ptr(x, y + 1), -rdy * l);
    sadd(asud.ptr(x, y), rdy * l);
    sadd(asvd.ptr(x + 1, y), rdx * l);
    sadd(asvd.ptr(x, y), -rdx * l);
  });
  __syncthreads();
  flush_box(asud, TX + 6, TY + 6, lam_ud, g, k);
  flush_box(asvd, TX + 6, TY + 6, lam_vd, g, k);
  flush_box(aucL, TX + 1, TY + 5, lam_uc, g, L - 1);
  flush_box(avcL, TX + 5, TY + 1, lam_vc, g, L - 1);
  flush_box(asuc, TX, TY, lam_uc, g, k);
  flush_box(asvc, TX, TY, lam_vc, g, k);
  flush_box(apb0, TX + 1, TY + 1, lam_pkb, g, k);
  flush_box(apb1, TX + 1, TY + 1, lam_pkb, g, k + 1);
  flush_box(agb0, TX + 1, TY + 1, lam_gzb, g, k);
  flush_box(agb1, TX + 1, TY + 1, lam_gzb, g, k + 1);
}

// ===================================================== column adjoint ====
// Adjoint of k_column: plev = ptop + suffix sums of dp, pkap = plev**kappa,
// gz(k+1) = gz(k) + cp pt(k) (pkap(k) - pkap(k+1)) from the fixed surface
// gz (src/mod_sw_dyn.f90:276-292, 606-626).  pkap of level nlay+1 and gz of
// level 1 are constants.  One thread per column over [lo, n-1+hi]^2.
template <int LM>
__global__ void __launch_bounds__(128) k_column_adj(Geom g, Consts c, const double* __restrict__ dpl,
                                                    const double* __restrict__ ptl, const double* __restrict__ lam_pk,
                                                    const double* __restrict__ lam_gz, double* lam_dp, double* lam_pt,
                                                    int lo, int hi) {
  const int w = g.nx - lo + hi, hgt = g.ny - lo + hi;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w * hgt) return;
  const int x = lo + col % w, y = lo + col / w;
  const long long o = g.at(x, y), S = g.S;
  const int L = g.L;
  double lpl[LM];  // adjoint of plev(k), k = 0..L-1
  // top-down: recompute plev, pkap; reverse the gz recursion on the way
  double pl = c.ptop, pk_up = c.pk_top, pl_up = c.ptop;
  double lz = 0., lpk_up = 0.;  // adjoint of gz(k+1) so far, of pkap(k+1)
  for (int k = L - 1; k >= 0; --k) {
    const long long ok = o + (long long)k * S;
    pl = pl + dpl[ok];
    const double pk = atm_pow(pl, KAPPA);
    lz += lam_gz[ok + S];  // gz level k+1
    const double pt = ptl[ok];
    const double cpz = CP_DRY * pt * lz;
    lam_pt[ok] += CP_DRY * (pk - pk_up) * lz;
    double lpk = lam_pk[ok] + cpz;
    if (k + 1 < L) {
      lpk_up -= cpz;  // pkap(k+1) complete
      lpl[k + 1] = lpk_up * KAPPA * pk_up / pl_up;
    }
    lpk_up = lpk;
    pk_up = pk;
    pl_up = pl;
  }
  lpl[0] = lpk_up * KAPPA * pk_up / pl_up;
  double acc = 0.;
  for (int k = 0; k < L; ++k) {
    acc += lpl[k];
    lam_dp[o + (long long)k * S] += acc;
  }
}

// ==================================================== corners adjoint ====
// Adjoint of interpolate_to_corners (src/mod_sw_dyn.f90:921-956): the
// 4x4-point corner value has weights a(dx) b(dy) + b(dx) a(dy) with
// a = (-1/12, 7/12, 7/12, -1/12) and b = (-1/32, 9/32, 9/32, -1/32) over
// dx, dy = -2..1.  Gather over the corners [0, nx] x [0, ny] each point of
// [-2, nx+1]^2 feeds: pkapb(l) -> pkap(l) and gzb(l+1) -> gz(l+1), l < nlay.
__global__ void k_corners_adj(Geom g, const double* __restrict__ lam_pkb, const double* __restrict__ lam_gzb,
                              double* lam_pk, double* lam_gz) {
  // one thread per point and level (blockIdx.y): the 16-point gathers of a
  // block's row of points hit L1, and every level runs in parallel
  const int w = g.nx + 4, h = g.ny + 4;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= w * h) return;
  const int x = -2 + idx % w, y = -2 + idx / w;
  const int l = blockIdx.y;
  const double a[4] = {-C1_12, C7_12, C7_12, -C1_12};
  const double b[4] = {-C1_32, C9_32, C9_32, -C1_32};
  const double* pkb = lam_pkb + (long long)l * g.S;
  const double* gzb = lam_gzb + (long long)(l + 1) * g.S;
  double sp = 0., sg = 0.;
  for (int dy = -2; dy <= 1; ++dy) {
    const int cy = y - dy;
    if (cy < 0 || cy > g.ny) continue;
    const long long row = g.at(0, cy);
    for (int dx = -2; dx <= 1; ++dx) {
      const int cx = x - dx;
      if (cx < 0 || cx > g.nx) continue;
      const double wt = a[dx + 2] * b[dy + 2] + b[dx + 2] * a[dy + 2];
      sp += wt * pkb[row + cx];
      sg += wt * gzb[row + cx];
    }
  }
  lam_pk[g.at(x, y, l)] += sp;
  lam_gz[g.at(x, y, l + 1)] += sg;
}

// ======================================================= halo adjoints ====
// Adjoint of the periodic ring fill (k_ring, copy = false): every ring
// point's adjoint is added to its periodic image in the interior and
// cleared.
__global__ void k_ring_fold(Geom g, double* f0, double* f1, double* f2, double* f3, int K) {
  const int wide = g.nx + 2 * H;
  const int nband = 2 * H * wide;
  const int nring = nband + 2 * H * g.ny;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nring || (int)blockIdx.y >= K) return;
  int x, y;
  if (idx < nband) {
    int r = idx / wide;
    y = r < H ? r - H : g.ny + (r - H);
    x = idx % wide - H;
  } else {
    int q = idx - nband;
    y = q / (2 * H);
    int cc = q % (2 * H);
    x = cc < H ? cc - H : g.nx + (cc - H);
  }
  const int fld = blockIdx.z;
  double* f = fld == 0 ? f0 : fld == 1 ? f1 : fld == 2 ? f2 : f3;
  if (!f) return;
  const int k = blockIdx.y;
  const long long o = g.at(x, y, k);
  const double v = f[o];
  if (v == 0.) return;
  const int xs = x < 0 ? x + g.nx : (x >= g.nx ? x - g.nx : x);
  const int ys = y < 0 ? y + g.ny : (y >= g.ny ? y - g.ny : y);
  atomicAdd(f + g.at(xs, ys, k), v);
  f[o] = 0.;
}

// Adjoint of the ring copy old -> new time level (k_ring, copy = true)
// for the ring points that the following step did not overwrite: points
// of fields 0, 1 inside [-band01, n+band01)^2 and of fields 2, 3 inside
// [-band23, n+band23)^2 were recomputed and keep their adjoint.
__global__ void k_ring_copy_adj(Geom g, double* d0, double* d1, double* d2, double* d3, double* s0, double* s1,
                                double* s2, double* s3, int K, int band01, int band23) {
  const int wide = g.nx + 2 * H;
  const int nband = 2 * H * wide;
  const int nring = nband + 2 * H * g.ny;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nring || (int)blockIdx.y >= K) return;
  int x, y;
  if (idx < nband) {
    int r = idx / wide;
    y = r < H ? r - H : g.ny + (r - H);
    x = idx % wide - H;
  } else {
    int q = idx - nband;
    y = q / (2 * H);
    int cc = q % (2 * H);
    x = cc < H ? cc - H : g.nx + (cc - H);
  }
  const int fld = blockIdx.z;
  const int band = fld < 2 ? band01 : band23;
  if (x >= -band && x < g.nx + band && y >= -band && y < g.ny + band) return;
  double* d = fld == 0 ? d0 : fld == 1 ? d1 : fld == 2 ? d2 : d3;
  double* s = fld == 0 ? s0 : fld == 1 ? s1 : fld == 2 ? s2 : s3;
  const long long o = g.at(x, y, blockIdx.y);
  s[o] += d[o];
  d[o] = 0.;
}

// ======================================================= remap adjoint ====
// Reverse mode of remap_column (src/mod_remap.f90:165-356): the forward
// vertical_ppm is recomputed with its intermediates kept (solve, back
// substitution, limited interface values), the same layer pairs are
// visited, and the adjoints flow back to the source values and to both
// coordinates.
// The column arrays of the adjoint of vertical_ppm: the forward's lvs (after
// the elimination), lvb (after the back substitution), lvc (limited) and
// gam, and the adjoints.  The monotone path forms each layer's edges and
// curvature on the fly (PPMLayers); RemapAdjFull also stores them, for the
// all-pairs path of non-monotone coordinates.
template <int LM>
struct RemapAdjWork {
  double gam[LM + 2], lvs[LM + 2], lvb[LM + 2], lvc[LM + 2];
  double LL[LM + 2], Lgam[LM + 2], Ltop[LM + 2], Lbtm[LM + 2];
};
template <int LM>
struct RemapAdjFull : RemapAdjWork<LM> {
  double top[LM + 2], btm[LM + 2], curv[LM + 2];
};

// vertical_ppm (src/mod_remap.f90:287-356) keeping lvs, lvb, lvc, the
// edges and the curvature; the operations are those of vertical_ppm in
// atm_kernels.cuh.
template <int LM>
__device__ void vppm_record(RemapAdjFull<LM>& w, int L, const double* var, const double* coord) {
  double* gam = w.gam;
  double* lv = w.lvs;
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
  double* b = w.lvb;
  b[1] = lv[1];
  for (int k = 2; k <= L + 1; ++k) b[k] = lv[k] - gam[k - 1] * b[k - 1];
  double* c = w.lvc;
  for (int k = 1; k <= L + 1; ++k) c[k] = b[k];
  c[L] = mn(c[L], mx(var[L], var[L - 1]));
  c[L] = mx(c[L], mn(var[L], var[L - 1]));
  c[2] = mn(c[2], mx(var[2], var[1]));
  c[2] = mx(c[2], mn(var[2], var[1]));
  for (int k = 2; k <= L - 1; ++k) {
    double lo = mn(var[k], var[k + 1]), hi = mx(var[k], var[k + 1]);
    if (k + 2 > L || gam[k + 2] * gam[k] > 0) {
      c[k + 1] = mn(c[k + 1], hi);
      c[k + 1] = mx(c[k + 1], lo);
    } else if (gam[k + 2] > 0) {
      c[k + 1] = mx(c[k + 1], lo);
    } else {
      c[k + 1] = mn(c[k + 1], hi);
    }
  }
  for (int k = 1; k <= L; ++k) {
    w.top[k] = c[k + 1];
    w.btm[k] = c[k];
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

// adjoint of r = mn(mx(x0, mn3(a, b, c)), mx3(a, b, c)) for the edge limiter
// of src/mod_remap.f90:342-352 with a = var, b = var + s2 * gam(j2),
// c = b + s15 * gam(j15): returns the adjoint of x0.
__device__ __forceinline__ double edge_clamp_adj(double x0, double a, double b, double c, double lam, double& lvar,
                                                 double* Lgam, int j2, double s2, int j15, double s15) {
  const double lo = mn3(a, b, c), hi = mx3(a, b, c);
  const double inner = mx(x0, lo);
  int which;  // 0: x0, 1: lo, 2: hi
  if (hi < inner) which = 2;
  else if (x0 < lo) which = 1;
  else which = 0;
  if (which == 0) return lam;
  const int s = which == 1 ? sel_mn3(a, b, c) : sel_mx3(a, b, c);
  if (s == 0) {
    lvar += lam;
  } else {
    lvar += lam;
    Lgam[j2] += s2 * lam;
    if (s == 2) Lgam[j15] += s15 * lam;
  }
  return 0.;
}

// Adjoint of vertical_ppm given w.Ltop, w.Lbtm (curvature already folded
// into them and into Lvar): adds to Lvar (source values) and Lc (coordinate).
template <int LM>
__device__ void vppm_adj(RemapAdjWork<LM>& w, int L, const double* var, const double* coord, double* Lvar, double* Lc) {
  const double* gam = w.gam;
  double* LL = w.LL;
  double* Lgam = w.Lgam;
  for (int k = 0; k <= L + 1; ++k) {
    LL[k] = 0.;
    Lgam[k] = 0.;
  }
  // edge limiters of top/btm (:340-352), reverse order
  for (int k = L - 1; k >= 2; --k) {
    double lt = w.Ltop[k + 1];
    if (lt != 0.) {
      const double pmp1 = var[k + 1] - 2. * gam[k];
      const double lac1 = pmp1 + 1.5 * gam[k - 1];
      lt = edge_clamp_adj(w.lvc[k + 2], var[k + 1], pmp1, lac1, lt, Lvar[k + 1], Lgam, k, -2., k - 1, 1.5);
    }
    double lb = w.Lbtm[k + 1];
    if (lb != 0.) {
      const double pmp1 = var[k + 1] + 2. * gam[k + 1];
      const double lac1 = pmp1 - 1.5 * gam[k];
      lb = edge_clamp_adj(w.lvc[k + 1], var[k + 1], pmp1, lac1, lb, Lvar[k + 1], Lgam, k + 1, 2., k, -1.5);
    }
    w.Ltop[k + 1] = lt;
    w.Lbtm[k + 1] = lb;
  }
  for (int k = 1; k <= L; ++k) {
    LL[k + 1] += w.Ltop[k];
    LL[k] += w.Lbtm[k];
  }
  // interface-value limiters (:319-339): each entry's chain of clamps, reversed
  for (int j = 2; j <= L; ++j) {
    bool is_min[6];
    double bound[6];
    int vsel[6];
    int n = 0;
    auto min_hi = [&](int p, int q) {  // x = mn(x, mx(var[p], var[q]))
      is_min[n] = true;
      bool t = var[p] < var[q];
      bound[n] = t ? var[q] : var[p];
      vsel[n] = t ? q : p;
      ++n;
    };
    auto max_lo = [&](int p, int q) {  // x = mx(x, mn(var[p], var[q]))
      is_min[n] = false;
      bool t = var[q] < var[p];
      bound[n] = t ? var[q] : var[p];
      vsel[n] = t ? q : p;
      ++n;
    };
    if (j == L) { min_hi(L, L - 1); max_lo(L, L - 1); }
    if (j == 2) { min_hi(2, 1); max_lo(2, 1); }
    if (j >= 3) {
      const int k = j - 1;
      if (k + 2 > L || gam[k + 2] * gam[k] > 0) { min_hi(k, k + 1); max_lo(k, k + 1); }
      else if (gam[k + 2] > 0) max_lo(k, k + 1);
      else min_hi(k, k + 1);
    }
    bool sel[6];
    double x = w.lvb[j];
    for (int i = 0; i < n; ++i) {
      sel[i] = is_min[i] ? (bound[i] < x) : (x < bound[i]);
      if (sel[i]) x = bound[i];
    }
    double lam = LL[j];
    for (int i = n - 1; i >= 0 && lam != 0.; --i)
      if (sel[i]) {
        Lvar[vsel[i]] += lam;
        lam = 0.;
      }
    LL[j] = lam;
  }
  // back substitution (:317-318)
  for (int k = L + 1; k >= 2; --k) {
    LL[k - 1] -= gam[k - 1] * LL[k];
    Lgam[k - 1] -= w.lvb[k - 1] * LL[k];
  }
  // first interface value (:314-316); a2 is the alpha of the loop's last pass
  const double a2 = (coord[3] - coord[2]) / (coord[2] - coord[1]);
  double La2;
  {
    const double b0 = 1. + a2 * (1.5 + a2);
    const double D1 = a2 * (.5 + a2) - b0 * gam[1];
    const double LN1 = LL[1] / D1, LD1 = -w.lvs[1] / D1 * LL[1];
    Lvar[1] += 2. * a2 * (1. + a2) * LN1;
    Lvar[2] += LN1;
    double Lb0 = -w.lvs[2] * LN1;
    LL[2] -= b0 * LN1;
    La2 = (2. + 4. * a2) * var[1] * LN1 + (.5 + 2. * a2) * LD1;
    Lb0 -= gam[1] * LD1;
    Lgam[1] -= b0 * LD1;
    La2 += (1.5 + 2. * a2) * Lb0;
  }
  // elimination (:306-313), reverse order k = 2..L
  for (int k = 2; k <= L; ++k) {
    const double nn = coord[k + 1] - coord[k], dd = coord[k] - coord[k - 1];
    const double ak = nn / dd;
    const double bek = 2. + 2. * ak - gam[k];
    double La = (k == 2) ? La2 : 0.;
    La += Lgam[k - 1] / bek;
    double Lbe = -gam[k - 1] / bek * Lgam[k - 1];
    const double LN = LL[k] / bek;
    Lbe -= w.lvs[k] / bek * LL[k];
    Lvar[k] += 3. * LN;
    Lvar[k - 1] += 3. * ak * LN;
    La += 3. * var[k - 1] * LN;
    LL[k + 1] -= LN;
    La += 2. * Lbe;
    Lgam[k] -= Lbe;
    Lc[k + 1] += La / dd;
    Lc[k] -= La / dd;
    const double Ld = -ak / dd * La;
    Lc[k] += Ld;
    Lc[k - 1] -= Ld;
  }
  // top interface value and gam(nlay) (:301-305)
  {
    const double nn = coord[L] - coord[L - 1], dd = coord[L + 1] - coord[L];
    const double aL = nn / dd;
    const double bL = aL * (.5 + aL);
    const double LNL = LL[L + 1] / bL;
    double LbL = -w.lvs[L + 1] / bL * LL[L + 1];
    Lvar[L] += 2. * aL * (1. + aL) * LNL;
    Lvar[L - 1] += LNL;
    double LaL = (2. + 4. * aL) * var[L] * LNL;
    const double LG = Lgam[L] / bL;
    LbL -= gam[L] / bL * Lgam[L];
    LaL += (1.5 + 2. * aL) * LG;
    LaL += (.5 + 2. * aL) * LbL;
    Lc[L] += LaL / dd;
    Lc[L - 1] -= LaL / dd;
    const double Ldd = -aL / dd * LaL;
    Lc[L + 1] += Ldd;
    Lc[L] -= Ldd;
  }
}

// adjoint of one pair's contribution (remap_pair) given source layer k's
// edges, curvature and value: adds to Ltop/Lbtm (with the curvature folded
// in), Lsrc, Lsc, Ldc
template <int LM>
__device__ __forceinline__ void remap_pair_adj(RemapAdjWork<LM>& w, double btm, double top, double curv, double vk,
                                               double ldst, const double* sc, const double* dc, int k, int m,
                                               double* Lsrc, double* Lsc, double* Ldc) {
  const double dsrc = sc[k + 1] - sc[k];
  const double s1 = (dc[m] - sc[k]) / dsrc;
  const double s2 = (dc[m + 1] - sc[k]) / dsrc;
  const double ddst = dc[m + 1] - dc[m];
  const double IF = dsrc / ddst;
  const double tmp3 = 2. * s1 * s1;
  double Ls1 = 0., Ls2 = 0., LIF = 0., Lb = 0., Lt = 0., Lcv = 0.;
  if (dc[m + 1] <= sc[k + 1] && sc[k + 1] < dc[m] && dc[m] < sc[k]) {
    const double t1 = s1 - 1., t2 = s1 + 1.;
    const double A = 3. * (btm * t1 - top * t2) + curv * (tmp3 - t2);
    const double f = t1 / 6. * IF * ldst;
    Lb += f * 3. * t1;
    Lt -= f * 3. * t2;
    Lcv += f * (tmp3 - t2);
    LIF += t1 / 6. * A * ldst;
    Ls1 += (A / 6. * IF + t1 / 6. * IF * (3. * (btm - top) + curv * (4. * s1 - 1.))) * ldst;
  }
  if (sc[k + 1] < dc[m + 1] && dc[m + 1] < sc[k] && sc[k] <= dc[m]) {
    const double B = btm * (2. - s2) + s2 * (top + curv * (1. - C2_3 * s2));
    const double f = s2 / 2. * IF * ldst;
    Lb += f * (2. - s2);
    Lt += f * s2;
    Lcv += f * s2 * (1. - C2_3 * s2);
    LIF += s2 / 2. * B * ldst;
    Ls2 += (.5 * B * IF + s2 / 2. * IF * (-btm + top + curv * (1. - 2. * C2_3 * s2))) * ldst;
  }
  if (dc[m + 1] <= sc[k + 1] && sc[k] <= dc[m]) {
    Lsrc[k] += IF * ldst;
    LIF += vk * ldst;
  }
  if (sc[k + 1] < dc[m + 1] && dc[m] < sc[k]) {
    const double t1 = s1 + s2;
    const double C = 3. * (btm * (t1 - 2.) - top * t1) + curv * (tmp3 + t1 * (2. * s2 - 3.));
    const double f = (s1 - s2) / 6. * IF * ldst;
    Lb += f * 3. * (t1 - 2.);
    Lt -= f * 3. * t1;
    Lcv += f * (tmp3 + t1 * (2. * s2 - 3.));
    LIF += (s1 - s2) / 6. * C * ldst;
    const double dC1 = 3. * (btm - top) + curv * (4. * s1 + 2. * s2 - 3.);
    const double dC2 = 3. * (btm - top) + curv * (2. * s2 - 3. + 2. * t1);
    Ls1 += (C * IF / 6. + (s1 - s2) / 6. * IF * dC1) * ldst;
    Ls2 += (-C * IF / 6. + (s1 - s2) / 6. * IF * dC2) * ldst;
  }
  // curvature = 6 var - 3 (top + btm)
  Lsrc[k] += 6. * Lcv;
  w.Ltop[k] += Lt - 3. * Lcv;
  w.Lbtm[k] += Lb - 3. * Lcv;
  const double Ldsrc = -(Ls1 * s1 + Ls2 * s2) / dsrc + LIF / ddst;
  Ldc[m] += Ls1 / dsrc + LIF * IF / ddst;
  Ldc[m + 1] += Ls2 / dsrc - LIF * IF / ddst;
  Lsc[k] += -(Ls1 + Ls2) / dsrc - Ldsrc;
  Lsc[k + 1] += Ldsrc;
}

// All-pairs adjoint of remap_column for coordinates that are not monotone
// (every source layer against every target layer, as the reference loops),
// with its own column arrays.
template <int LM>
__device__ __noinline__ void remap_column_adj_full(int L, const double* src_var, const double* Ldst, const double* sc,
                                                   const double* dc, double* Lsrc, double* Lsc, double* Ldc) {
  RemapAdjFull<LM> w;
  vppm_record<LM>(w, L, src_var, sc);
  for (int k = 0; k <= L + 1; ++k) {
    w.Ltop[k] = 0.;
    w.Lbtm[k] = 0.;
  }
  for (int k = 1; k <= L; ++k)
    for (int m = 1; m <= L; ++m) {
      if (sc[k + 1] >= dc[m] || sc[k] <= dc[m + 1] || Ldst[m] == 0.) continue;
      remap_pair_adj<LM>(w, w.btm[k], w.top[k], w.curv[k], src_var[k], Ldst[m], sc, dc, k, m, Lsrc, Lsc, Ldc);
    }
  vppm_adj<LM>(w, L, src_var, sc, Lsrc, Lsc);
}

// Adjoint of remap_column: given the adjoint Ldst of the remapped values,
// adds to Lsrc (source values), Lsc (source coordinate), Ldc (target).
// Monotone coordinates (the usual case): the elimination of vertical_ppm
// as the forward's streaming remap does it (ppm_eliminate), then the pairs
// in the forward merge's order with each source layer's edges and curvature
// formed as the merge reaches it (PPMLayers, which also yields the back
// substituted and limited interface values the reverse of vertical_ppm
// reads); the same operations as vertical_ppm, so the same values.
template <int LM>
__device__ void remap_column_adj(RemapAdjWork<LM>& w, int L, const double* src_var, const double* Ldst, const double* sc,
                                 const double* dc, double* Lsrc, double* Lsc, double* Ldc) {
  bool mono = true;
  for (int k = 1; k <= L; ++k) mono = mono && (sc[k + 1] <= sc[k]) && (dc[k + 1] <= dc[k]);
  if (!mono) {
    remap_column_adj_full<LM>(L, src_var, Ldst, sc, dc, Lsrc, Lsc, Ldc);
    return;
  }
  const ColArr csc{const_cast<double*>(sc), 1}, clv{w.lvs, 1}, cgam{w.gam, 1};
  {
    int kc = L + 2, kv = L + 1;
    ppm_eliminate<false>(L, [&]() { return sc[--kc]; }, [&]() { return src_var[--kv]; }, csc, clv, cgam);
  }
  for (int k = 0; k <= L + 1; ++k) {
    w.Ltop[k] = 0.;
    w.Lbtm[k] = 0.;
  }
  auto var = [&](int k) { return src_var[k]; };
  PPMLayers<decltype(var)> ly(clv, cgam, L, var);
  w.lvb[1] = ly.lvf;
  w.lvc[1] = ly.lvc;
  auto advance = [&]() {  // to the next layer; its top interface values
    ly.next();
    w.lvb[ly.k + 1] = ly.lvf;
    w.lvc[ly.k + 1] = ly.lvc;
  };
  int k0 = 1;
  for (int m = 1; m <= L; ++m) {
    while (k0 <= L && sc[k0 + 1] >= dc[m]) ++k0;
    if (Ldst[m] == 0.) continue;
    for (int k = k0; k <= L && sc[k] > dc[m + 1]; ++k) {
      while (ly.k < k) advance();
      remap_pair_adj<LM>(w, ly.btm, ly.top, ly.curv, ly.vk, Ldst[m], sc, dc, k, m, Lsrc, Lsc, Ldc);
    }
  }
  while (ly.k < L) advance();
  vppm_adj<LM>(w, L, src_var, sc, Lsrc, Lsc);
}

// remap_column of the energy for coordinates that are not monotone, with
// its own column arrays
template <int LM>
__device__ __noinline__ void remap_energy_pairs(int L, const double* en, double* er, const double* plev,
                                                const double* tpl) {
  PPMWork<LM> wf;
  remap_column<LM>(wf, L, en, er, plev, tpl, nullptr, 1, nullptr);
}

// Adjoint of k_remap_energy (src/mod_remap.f90:42-78, 111-161) on the
// interior: adjoints of the remapped dp, pt, ud, vd in; adjoints of the
// pre-remap dp, pt (this column), ud, vd (its A-grid neighbours) and of the
// remapped face winds urem, vrem out.
// 16 blocks of 64 threads per SM (64 registers; more columns in flight to
// hide the local-memory latency of the column arrays): both remap adjoints
// 51.1 ms per remap at 1024x1024x64 against 73.9 at the compiler's own
// budget, 60.4 at 12 blocks, 58.0 at 24
template <int LM>
__global__ void __launch_bounds__(64, 16) k_remap_energy_adj(Geom g, RemapArgs ra, const double* __restrict__ dp,
                                                         const double* __restrict__ pt, const double* __restrict__ ud,
                                                         const double* __restrict__ vd, const double* __restrict__ urem,
                                                         const double* __restrict__ vrem, const double* __restrict__ gzs,
                                                         const double* __restrict__ lam_dpo,
                                                         const double* __restrict__ lam_pto,
                                                         const double* __restrict__ lam_udo,
                                                         const double* __restrict__ lam_vdo, double* lam_dp,
                                                         double* lam_pt, double* lam_ud, double* lam_vd, double* lam_ur,
                                                         double* lam_vr) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.nx * g.ny) return;
  const int i = col % g.nx, j = col / g.nx;
  const int L = g.L;
  const long long S = g.S;
  const long long o = g.at(i, j);
  const int P = g.P;
  double plev[LM + 2], pk[LM + 2], tpl[LM + 2], tpk[LM + 2];
  double en[LM + 2], ptr[LM + 2];
  double Lplev[LM + 2], Ltpl[LM + 2], Lpk[LM + 2], Ltpk[LM + 2], Ler[LM + 2];
  RemapAdjWork<LM> wk;
  // ud = urem and vd = vrem (:156-161); the column's energy and pressure
  // adjoints are zero unless its new dp or pt carry an adjoint
  bool any = false;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    if (lam_udo[ok] != 0.) atomicAdd(lam_ur + ok, lam_udo[ok]);
    if (lam_vdo[ok] != 0.) atomicAdd(lam_vr + ok, lam_vdo[ok]);
    any = any || lam_dpo[ok] != 0. || lam_pto[ok] != 0.;
  }
  if (!any) return;
  // forward recomputation, as k_remap_energy
  plev[L + 1] = ra.ptop;
  pk[L + 1] = ra.pk_top;
  double lyk[LM + 2], tlyk[LM + 2];
  for (int k = L; k >= 1; --k) {
    plev[k] = plev[k + 1] + dp[o + (long long)(k - 1) * S];
    pk[k] = atm_pow(plev[k], KAPPA);
    double plog = atm_log(pk[k + 1] / pk[k]);
    lyk[k] = (pk[k + 1] - pk[k]) / plog;
  }
  tpl[L + 1] = ra.ptop;
  tpk[L + 1] = ra.pk_top;
  for (int k = L; k >= 1; --k) {
    tpl[k] = ra.ak[k - 1] + ra.bk[k - 1] * (plev[1] - ra.ptop);
    tpk[k] = atm_pow(tpl[k], KAPPA);
    double plog = atm_log(tpk[k + 1] / tpk[k]);
    tlyk[k] = (tpk[k + 1] - tpk[k]) / plog;
  }
  {
    double gz0 = gzs[o];  // gz(k), streamed upward
    for (int k = 1; k <= L; ++k) {
      long long ok = o + (long long)(k - 1) * S;
      const double gz1 = gz0 + CP_DRY * pt[ok] * (pk[k] - pk[k + 1]);
      double ua = (.25 * (ud[ok] + ud[ok + P]) + .125 * (ud[ok - 1] + ud[ok - 1 + P] + ud[ok + 1] + ud[ok + 1 + P]));
      double va = (.25 * (vd[ok] + vd[ok + 1]) + .125 * (vd[ok - P] + vd[ok + 1 - P] + vd[ok + P] + vd[ok + 1 + P]));
      en[k] = CV_DRY * pt[ok] * lyk[k] + .5 * (gz1 + gz0 + ua * ua + va * va);
      gz0 = gz1;
    }
  }
  {
    // the remapped energy er(m), ascending, and the recovered pt (:127-150)
    double gzr = gzs[o];
    auto put = [&](int m, double erm) {
      long long ok = o + (long long)(m - 1) * S;
      double ua = (.25 * (urem[ok] + urem[ok + P]) + .125 * (urem[ok - 1] + urem[ok - 1 + P] + urem[ok + 1] + urem[ok + 1 + P]));
      double va = (.25 * (vrem[ok] + vrem[ok + 1]) + .125 * (vrem[ok - P] + vrem[ok + 1 - P] + vrem[ok + P] + vrem[ok + 1 + P]));
      ptr[m] = (erm - gzr - .5 * (ua * ua + va * va)) / (CV_DRY * tlyk[m] + .5 * CP_DRY * (tpk[m] - tpk[m + 1]));
      gzr = gzr + CP_DRY * ptr[m] * (tpk[m] - tpk[m + 1]);
    };
    bool mono = true;
    for (int k = 1; k <= L; ++k) mono = mono && (plev[k + 1] <= plev[k]) && (tpl[k + 1] <= tpl[k]);
    if (mono) {  // the forward's streaming remap (the energy kernel's path)
      const ColArr cpl{plev, 1}, clv{wk.lvs, 1}, cgam{wk.gam, 1};
      int kc = L + 2, kv = L + 1;
      ppm_eliminate<false>(L, [&]() { return plev[--kc]; }, [&]() { return en[--kv]; }, cpl, clv, cgam);
      remap_merge(L, cpl, clv, cgam, [&](int k) { return en[k]; }, [&](int k) { return tpl[k]; }, put, nullptr, 1);
    } else {  // all pairs, into Ler as scratch (it is cleared below)
      remap_energy_pairs<LM>(L, en, Ler, plev, tpl);
      for (int m = 1; m <= L; ++m) put(m, Ler[m]);
    }
  }
  for (int k = 0; k <= L + 1; ++k) {
    Lplev[k] = 0.; Ltpl[k] = 0.; Lpk[k] = 0.; Ltpk[k] = 0.; Ler[k] = 0.;
  }
  // outputs: dp = tpl(k) - tpl(k+1) (:156-161)
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    const double ld = lam_dpo[ok];
    Ltpl[k] += ld;
    Ltpl[k + 1] -= ld;
  }
  // pt recovery and the remapped geopotential (:130-150), reverse
  {
    double lgz = 0.;  // adjoint of gz_remap(k+1)
    for (int k = L; k >= 1; --k) {
      long long ok = o + (long long)(k - 1) * S;
      const double dtp = tpk[k] - tpk[k + 1];
      const double Dk = CV_DRY * tlyk[k] + .5 * CP_DRY * dtp;
      const double lp = lam_pto[ok] + CP_DRY * dtp * lgz;
      Ltpk[k] += CP_DRY * ptr[k] * lgz;
      Ltpk[k + 1] -= CP_DRY * ptr[k] * lgz;
      const double ln = lp / Dk;  // adjoint of the numerator
      Ler[k] += ln;
      lgz -= ln;
      const double LD = -ptr[k] / Dk * lp;
      // tlyk(k) = (tpk(k+1) - tpk(k)) / log(tpk(k+1) / tpk(k))
      const double lg = log(tpk[k + 1] / tpk[k]);
      const double Ly = CV_DRY * LD;
      Ltpk[k + 1] += Ly * (1. - tlyk[k] / tpk[k + 1]) / lg;
      Ltpk[k] += Ly * (-1. + tlyk[k] / tpk[k]) / lg;
      Ltpk[k] += .5 * CP_DRY * LD;
      Ltpk[k + 1] -= .5 * CP_DRY * LD;
      // ua, va of the remapped face winds
      const double ua = (.25 * (urem[ok] + urem[ok + P]) + .125 * (urem[ok - 1] + urem[ok - 1 + P] + urem[ok + 1] + urem[ok + 1 + P]));
      const double va = (.25 * (vrem[ok] + vrem[ok + 1]) + .125 * (vrem[ok - P] + vrem[ok + 1 - P] + vrem[ok + P] + vrem[ok + 1 + P]));
      const double lu = -ua * ln, lv = -va * ln;
      if (lu != 0.) {
        atomicAdd(lam_ur + ok, .25 * lu);
        atomicAdd(lam_ur + ok + P, .25 * lu);
        atomicAdd(lam_ur + ok - 1, .125 * lu);
        atomicAdd(lam_ur + ok - 1 + P, .125 * lu);
        atomicAdd(lam_ur + ok + 1, .125 * lu);
        atomicAdd(lam_ur + ok + 1 + P, .125 * lu);
      }
      if (lv != 0.) {
        atomicAdd(lam_vr + ok, .25 * lv);
        atomicAdd(lam_vr + ok + 1, .25 * lv);
        atomicAdd(lam_vr + ok - P, .125 * lv);
        atomicAdd(lam_vr + ok + 1 - P, .125 * lv);
        atomicAdd(lam_vr + ok + P, .125 * lv);
        atomicAdd(lam_vr + ok + 1 + P, .125 * lv);
      }
    }
  }
  // the energy remap (:107-110)
  double Lsrc[LM + 2];
  for (int k = 0; k <= L + 1; ++k) Lsrc[k] = 0.;
  remap_column_adj<LM>(wk, L, en, Ler, plev, tpl, Lsrc, Lplev, Ltpl);
  // target pressures (:57-71): tpk = tpl**kappa, tpl = ak + bk (ps - ptop)
  for (int k = 1; k <= L; ++k) {
    Ltpl[k] += Ltpk[k] * KAPPA * tpk[k] / tpl[k];
    Lplev[1] += ra.bk[k - 1] * Ltpl[k];
  }
  // energy (:72-78), hydrostatic gz (:53-56), playkap (:46-52)
  double Lpt[LM + 2];
  {
    for (int k = 1; k <= L; ++k) {
      long long ok = o + (long long)(k - 1) * S;
      const double le = Lsrc[k];
      Lpt[k] = CV_DRY * lyk[k] * le;
      // lyk(k) = (pk(k+1) - pk(k)) / log(pk(k+1) / pk(k))
      const double ly = CV_DRY * pt[ok] * le;
      const double lg = log(pk[k + 1] / pk[k]);
      Lpk[k + 1] += ly * (1. - lyk[k] / pk[k + 1]) / lg;
      Lpk[k] += ly * (-1. + lyk[k] / pk[k]) / lg;
      // the adjoint of en(k) (Lsrc(k)) also reaches .5 (gz(k+1) + gz(k)) and the kinetic energy
      const double ua = (.25 * (ud[ok] + ud[ok + P]) + .125 * (ud[ok - 1] + ud[ok - 1 + P] + ud[ok + 1] + ud[ok + 1 + P]));
      const double va = (.25 * (vd[ok] + vd[ok + 1]) + .125 * (vd[ok - P] + vd[ok + 1 - P] + vd[ok + P] + vd[ok + 1 + P]));
      const double lu = ua * le, lv = va * le;
      if (lu != 0.) {
        atomicAdd(lam_ud + ok, .25 * lu);
        atomicAdd(lam_ud + ok + P, .25 * lu);
        atomicAdd(lam_ud + ok - 1, .125 * lu);
        atomicAdd(lam_ud + ok - 1 + P, .125 * lu);
        atomicAdd(lam_ud + ok + 1, .125 * lu);
        atomicAdd(lam_ud + ok + 1 + P, .125 * lu);
      }
      if (lv != 0.) {
        atomicAdd(lam_vd + ok, .25 * lv);
        atomicAdd(lam_vd + ok + 1, .25 * lv);
        atomicAdd(lam_vd + ok - P, .125 * lv);
        atomicAdd(lam_vd + ok + 1 - P, .125 * lv);
        atomicAdd(lam_vd + ok + P, .125 * lv);
        atomicAdd(lam_vd + ok + 1 + P, .125 * lv);
      }
    }
    // gz(k+1) = gz(k) + cp pt(k) (pk(k) - pk(k+1)); d en(k) / d gz(k), gz(k+1) = .5
    double lz = 0.;
    for (int k = L; k >= 1; --k) {
      long long ok = o + (long long)(k - 1) * S;
      lz += .5 * Lsrc[k];  // gz(k+1)
      if (k + 1 <= L) lz += .5 * Lsrc[k + 1];  // gz(k+1) is also the lower level of layer k+1
      Lpt[k] += CP_DRY * (pk[k] - pk[k + 1]) * lz;
      Lpk[k] += CP_DRY * pt[ok] * lz;
      Lpk[k + 1] -= CP_DRY * pt[ok] * lz;
    }
  }
  // pk = plev**kappa; plev(k) = plev(k+1) + dp(k)
  for (int k = 1; k <= L; ++k) Lplev[k] += Lpk[k] * KAPPA * pk[k] / plev[k];
  double acc = 0.;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    acc += Lplev[k];
    lam_dp[ok] += acc;
    lam_pt[ok] += Lpt[k];
  }
}

// Adjoint of k_remap_winds (src/mod_remap.f90:80-105) on [-1, nx] x [-1, ny]:
// the adjoints of urem, vrem in; ud, vd of the column and dp of the seven
// columns that form its source and target interface pressures out.
template <int LM>
__global__ void __launch_bounds__(64, 16) k_remap_winds_adj(Geom g, RemapArgs ra, const double* __restrict__ dp,
                                                        const double* __restrict__ ud, const double* __restrict__ vd,
                                                        const double* __restrict__ lam_ur,
                                                        const double* __restrict__ lam_vr, double* lam_dp,
                                                        double* lam_ud, double* lam_vd) {
  const int w = g.nx + 2, h = g.ny + 2;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w * h) return;
  const int i = -1 + col % w, j = -1 + col / w;
  const int L = g.L;
  double sc[LM + 2], dc[LM + 2], var[LM + 2], Ld[LM + 2], Lv[LM + 2], Ls[LM + 2], Lt[LM + 2];
  RemapAdjWork<LM> wk;
  const int cx[7] = {i, i, i, i, i - 2, i - 1, i + 1};
  const int cy[7] = {j - 2, j - 1, j, j + 1, j, j, j};
  double ps[7];
  for (int q = 0; q < 7; ++q) {
    long long oq = g.at(cx[q], cy[q]);
    double pl = ra.ptop;
    for (int k = L - 1; k >= 0; --k) pl = pl + dp[oq + (long long)k * g.S];
    ps[q] = pl;
  }
  for (int dir = 0; dir < 2; ++dir) {
    const int qa = 2, qb = dir == 0 ? 1 : 5, qc = dir == 0 ? 3 : 6, qd = dir == 0 ? 0 : 4;
    long long oa = g.at(cx[qa], cy[qa]), ob = g.at(cx[qb], cy[qb]), oc = g.at(cx[qc], cy[qc]), od = g.at(cx[qd], cy[qd]);
    double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop;
    for (int k = L + 1; k >= 1; --k) {
      if (k <= L) {
        long long kk = (long long)(k - 1) * g.S;
        pa = pa + dp[oa + kk];
        pb = pb + dp[ob + kk];
        pc = pc + dp[oc + kk];
        pd = pd + dp[od + kk];
      }
      sc[k] = C7_12 * (pa + pb) - C1_12 * (pc + pd);
      double ta, tb, tc, td;
      if (k <= L) {
        double a = ra.ak[k - 1], b = ra.bk[k - 1];
        ta = a + b * (ps[qa] - ra.ptop);
        tb = a + b * (ps[qb] - ra.ptop);
        tc = a + b * (ps[qc] - ra.ptop);
        td = a + b * (ps[qd] - ra.ptop);
      } else {
        ta = tb = tc = td = ra.ptop;
      }
      dc[k] = C7_12 * (ta + tb) - C1_12 * (tc + td);
    }
    const double* f = dir == 0 ? ud : vd;
    const double* lr = dir == 0 ? lam_ur : lam_vr;
    long long o = g.at(i, j);
    bool any = false;
    for (int k = 1; k <= L; ++k) {
      var[k] = f[o + (long long)(k - 1) * g.S];
      Ld[k] = lr[o + (long long)(k - 1) * g.S];
      any = any || Ld[k] != 0.;
    }
    if (!any) continue;
    for (int k = 0; k <= L + 1; ++k) { Lv[k] = 0.; Ls[k] = 0.; Lt[k] = 0.; }
    remap_column_adj<LM>(wk, L, var, Ld, sc, dc, Lv, Ls, Lt);
    double* lf = dir == 0 ? lam_ud : lam_vd;
    for (int k = 1; k <= L; ++k) lf[o + (long long)(k - 1) * g.S] += Lv[k];
    // sc(k) = 7/12 (pa + pb) - 1/12 (pc + pd), p(k) = ptop + sum of dp(m >= k);
    // dc(k) = 7/12 (ta + tb) - 1/12 (tc + td), t = ak + bk (ps - ptop)
    double Z = 0.;
    for (int k = 1; k <= L; ++k) Z += ra.bk[k - 1] * Lt[k];
    double P = 0.;
    for (int m = 1; m <= L; ++m) {
      P += Ls[m];
      const double v = P + Z;
      if (v == 0.) continue;
      long long kk = (long long)(m - 1) * g.S;
      atomicAdd(lam_dp + oa + kk, C7_12 * v);
      atomicAdd(lam_dp + ob + kk, C7_12 * v);
      atomicAdd(lam_dp + oc + kk, -C1_12 * v);
      atomicAdd(lam_dp + od + kk, -C1_12 * v);
    }
  }
}

}  // namespace atm
