// Radiation of the reference (src/mod_radiation.f90, src/mod_gas_optics.f90,
// src/mod_solar.f90) on the device, FP64 in both forms:
//   calculate_radiative_heating (:41-156): layer pressures and temperatures
//   of each column, then for each of the 16 g-points a shortwave
//   (solve_shortwave_column, :158-268) and a longwave
//   (solve_longwave_column, :270-347) two-stream solution, both closed by
//   the adding method of calculate_fluxes (:349-381), summed into net_flux.
// Built with --fmad=false and the portable exp/log/pow of atm_math.h:
// every value is the reference's expression in its order, so the results
// are those of the FP64 restatement.  The table searches are binary
// searches for the index the reference's linear scans stop at (the first
// grid point not below the argument), which is the same index.
#include "atm_math.h"
#include "atm_ops.h"
#include "atm_radiation.h"

namespace atm {
namespace {

// mod_constants.f90:8 -- pi is a default-real literal
constexpr double PI_F = (double)3.1415926535897932384626433f;
// mod_solar.f90:33: 600*(1.+.2/(1.+(radius/100000e3)**2)); .2 and 100000e3
// are default-real literals
constexpr double SOLAR_BASE = 600.;
constexpr double SOLAR_PEAK = (double).2f;
constexpr double SOLAR_SCALE = (double)100000e3f;

// first k with xs[k] >= x for x in [xs[0], xs[n-1]]: where `k = 1; do while
// (x > xs(k)); k = k + 1` stops
__device__ __forceinline__ int first_not_below(const double* __restrict__ xs, int n, double x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xs[mid] >= x) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// lookup_1d (mod_gas_optics.f90:4556-4579) split in two: the bracket
// (where the reference's scan stops; outside the table the reference stops,
// :4562-4566, and the kernel flags it) and the interpolation at a known
// bracket.  The pressures, temperatures and level temperatures are the
// same for every g-point, so each column finds its brackets once.
__device__ __forceinline__ int bracket(double x, const double* __restrict__ xs, int n, bool& bad) {
  if (x < xs[0] || x > xs[n - 1] || x != x) {
    bad = true;
    return 1;
  }
  return first_not_below(xs, n, x);  // 0 only where x == xs[0], which interp_at returns exactly
}
__device__ __forceinline__ double interp_at(double x, const double* __restrict__ xs, const double* __restrict__ ys,
                                            int k) {
  if (x == xs[k]) return ys[k];
  return (ys[k] * (xs[k - 1] - x) + ys[k - 1] * (x - xs[k])) / (xs[k - 1] - xs[k]);
}

// lookup_pT_table (mod_gas_optics.f90:4581-4609): the brackets of one layer
// packed as kp | kt1 << 16 | kt2 << 24 (pressure; temperature in rows kp
// and kp - 1; kt2 unused when p is a grid pressure; atm_set_gas_optics
// keeps n_p below 2^16 and n_t below 2^8)
__device__ __forceinline__ unsigned bracket_pt(const RadTables& tb, double p, double t, bool& bad) {
  const int np = tb.np, nt = tb.nt;
  if (p < tb.pressures[0] || p > tb.pressures[np - 1] || p != p) {
    bad = true;
    return 1u | 1u << 16 | 1u << 24;
  }
  const int kp = first_not_below(tb.pressures, np, p);
  const int kt1 = bracket(t, tb.temps + kp * nt, nt, bad);
  const int kt2 = p == tb.pressures[kp] ? 1 : bracket(t, tb.temps + (kp - 1) * nt, nt, bad);
  return (unsigned)kp | (unsigned)kt1 << 16 | (unsigned)kt2 << 24;
}
__device__ __forceinline__ double lookup_pt_at(const RadTables& tb, double p, double t,
                                               const double* __restrict__ table, unsigned code) {
  const int nt = tb.nt, kp = code & 0xffff, kt1 = (code >> 16) & 0xff, kt2 = code >> 24;
  const double t1 = interp_at(t, tb.temps + kp * nt, table + kp * nt, kt1);
  if (p == tb.pressures[kp]) return t1;
  const double t2 = interp_at(t, tb.temps + (kp - 1) * nt, table + (kp - 1) * nt, kt2);
  return (t1 * (tb.pressures[kp - 1] - p) + t2 * (p - tb.pressures[kp])) / (tb.pressures[kp - 1] - tb.pressures[kp]);
}

// delta_eddington_rescaling (mod_radiation.f90:383-398)
__device__ __forceinline__ void delta_eddington(double& tau, double& ssa, double& asym) {
  const double forward_scatter = asym * asym;
  const double coefficient = 1. - ssa * forward_scatter;
  tau = tau * coefficient;
  ssa = ssa * (1. - forward_scatter) / coefficient;
  asym = asym / (1. + asym);
}

// Per-column working arrays of one g-point (1-based as in the reference).
template <int LM>
struct Column {
  double R[LM + 1], T[LM + 1], su[LM + 1], sd[LM + 1];  // reflectance, transmittance, sources
  double alb[LM + 2], em[LM + 2], beta[LM + 1];         // calculate_fluxes' albedo, emission_up, beta
  double beam[LM + 2];                                  // solar_beam
};

// calculate_fluxes (mod_radiation.f90:349-381) in two halves.  The upward
// sweep (:357-363) at layer k: beta(k), albedo(k+1), emission_up(k+1), the
// last two carried in registers; the longwave runs it inside its layer loop
// (both go upward), so its upward sources are never stored.
template <int LM>
__device__ __forceinline__ void adding_up(Column<LM>& c, int k, double R, double T, double su, double sd,
                                          double& alb, double& em) {
  const double beta = 1. / (1. - R * alb);
  const double alb1 = R + (T * T) * beta * alb;
  const double em1 = su + T * beta * (em + sd * alb);
  c.beta[k] = beta;
  c.alb[k + 1] = alb1;
  c.em[k + 1] = em1;
  alb = alb1;
  em = em1;
}

// the downward sweep (:365-380), each level's pair handed to
// emit(k, flux_up, flux_dn) from the top down
template <int LM, typename Emit>
__device__ __forceinline__ void adding_down(const Column<LM>& c, int L, double toa_dn, Emit emit) {
  double fdn = toa_dn;
  emit(L + 1, c.alb[L + 1] * toa_dn + c.em[L + 1], fdn);
  for (int k = L + 1; k >= 2; --k) {
    fdn = c.beta[k - 1] * (c.sd[k - 1] + c.T[k - 1] * fdn + c.R[k - 1] * c.em[k - 1]);
    emit(k - 1, c.alb[k - 1] * fdn + c.em[k - 1], fdn);
  }
}

// solve_shortwave_column (mod_radiation.f90:158-268) for g-point g: the
// layer coefficients top-down (the direct beam is attenuated layer by
// layer), then calculate_fluxes; the beam is added to the downward flux.
template <int LM>
__device__ void shortwave(const RadTables& tb, int g, int L, const double* play, const double* dm, const double* tlay,
                          const unsigned* code, double irradiance, double mu0, double sfc_albedo, Column<LM>& c,
                          double* up, double* dn) {
  const double* tab = tb.sw_abs + (long long)g * tb.np * tb.nt;
  c.beam[L + 1] = mu0 * irradiance;
  for (int k = L; k >= 1; --k) {
    const double k_abs = lookup_pt_at(tb, play[k], tlay[k], tab, code[k]);
    const double k_sca = tb.sw_sca[g];
    const double k_ext = k_abs + k_sca;
    double tau = k_ext * dm[k];
    double ssa = k_sca / k_ext;
    double asym = 0.;
    delta_eddington(tau, ssa, asym);
    // direct to diffuse: hybrid modified Eddington-delta (Meador & Weaver 1980)
    const double asy2 = asym * asym;
    double backscatter = (2. - 3. * asym * mu0) / 4.;
    double tmp1 = 4. * (1. - asy2 * (1. - mu0));
    double gamma3 = ssa * asy2;
    double gamma4 = 4. * backscatter + 3. * asym;
    double tmp2 = 3. * asym;
    double gamma1 = (7. - 3. * asy2 - ssa * (4. + tmp2) + gamma3 * gamma4) / tmp1;
    double gamma2 = (-1. + asy2 + ssa * (4. - tmp2) + gamma3 * (gamma4 - 4.)) / tmp1;
    gamma3 = backscatter;
    gamma4 = 1. - gamma3;
    const double alpha1 = gamma1 * gamma4 + gamma2 * gamma3;
    const double alpha2 = gamma2 * gamma3 + gamma2 * gamma4;
    double lambda = sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    const double lam_mu = lambda * mu0;
    const double e_minus = atm_exp(-(lambda * tau));
    double e_2minus = e_minus * e_minus;
    const double direct_t = atm_exp(-(tau / mu0));
    tmp1 = ssa / ((1. - lam_mu * lam_mu) * (lambda + gamma1 + (lambda - gamma1) * e_2minus));
    tmp2 = lambda * gamma3;
    const double diffuse_r = tmp1 * ((1. - lam_mu) * (alpha2 + tmp2) - (1. + lam_mu) * (alpha2 - tmp2) * e_2minus -
                                     2. * lambda * (gamma3 - alpha2 * mu0) * e_minus * direct_t);
    tmp2 = lambda * gamma4;
    const double diffuse_t = tmp1 * (2. * lambda * (gamma4 + alpha1 * mu0) * e_minus -
                                     direct_t * ((1. + lam_mu) * (alpha1 + tmp2) - (1. - lam_mu) * (alpha1 - tmp2) * e_2minus));
    c.beam[k] = direct_t * c.beam[k + 1];
    c.su[k] = diffuse_r * c.beam[k + 1];
    c.sd[k] = diffuse_t * c.beam[k + 1];
    // diffuse to diffuse: hemispheric constant (Meador & Weaver 1980) with
    // the backscatter of Ritter & Geleyn (1992); e_minus is the one above
    backscatter = (4. + asym) / (8. * (1. + asym));
    gamma1 = 2. * (1. - ssa * (1. - backscatter));
    gamma2 = 2. * ssa * backscatter;
    lambda = sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    e_2minus = e_minus * e_minus;
    tmp1 = 1. / (lambda + gamma1 + (lambda - gamma1) * e_2minus);
    c.R[k] = tmp1 * gamma2 * (1. - e_2minus);
    c.T[k] = 2. * tmp1 * lambda * e_minus;
  }
  double alb = sfc_albedo, em = 0.;
  c.alb[1] = alb;
  c.em[1] = em;
  for (int k = 1; k <= L; ++k) adding_up(c, k, c.R[k], c.T[k], c.su[k], c.sd[k], alb, em);
  adding_down(c, L, c.beam[L + 1], [&](int k, double fu, double fd) {
    up[k] = up[k] + fu;
    dn[k] = dn[k] + (fd + c.beam[k]);
  });
}

// solve_longwave_column (mod_radiation.f90:270-347) for g-point g: no
// scattering, a Planck source linear in optical depth
template <int LM>
__device__ void longwave(const RadTables& tb, int g, int L, const double* play, const double* dm, const double* tlay,
                         const double* tlev, const unsigned* code, const int* kb, double ts, int kbs,
                         double emissivity, Column<LM>& c, double* up, double* dn) {
  const double* tab = tb.lw_abs + (long long)g * tb.np * tb.nt;
  const double* plk = tb.plk + (long long)g * tb.npl;
  const double surface_planckian = interp_at(ts, tb.plk_t, plk, kbs);
  double lp_k = interp_at(tlev[1], tb.plk_t, plk, kb[1]);
  double alb = 1. - emissivity, em = emissivity * PI_F * surface_planckian;  // calculate_fluxes' arguments (:345)
  c.alb[1] = alb;
  c.em[1] = em;
  for (int k = 1; k <= L; ++k) {
    const double k_abs = lookup_pt_at(tb, play[k], tlay[k], tab, code[k]);
    const double k_sca = 0.;
    const double k_ext = k_abs + k_sca;
    double tau = k_ext * dm[k];
    double ssa = k_sca / k_ext;
    double asym = 0.;
    delta_eddington(tau, ssa, asym);
    const double backscatter = (4. - 3. * asym) / 8.;
    const double gamma1 = 2. * (1. - ssa * (1. - backscatter));
    const double gamma2 = 2. * ssa * backscatter;
    const double lambda = sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    const double e_minus = atm_exp(-(lambda * tau));
    const double e_2minus = e_minus * e_minus;
    double tmp1 = 1. / (lambda + gamma1 + (lambda - gamma1) * e_2minus);
    const double R = tmp1 * gamma2 * (1. - e_2minus);
    const double T = 2. * tmp1 * lambda * e_minus;
    const double lp_k1 = interp_at(tlev[k + 1], tb.plk_t, plk, kb[k + 1]);
    const double pdiff = (1. + R - T) * (lp_k - lp_k1) / (tau * (gamma1 + gamma2));
    tmp1 = 1. - R;
    const double su = PI_F * (tmp1 * lp_k1 - T * lp_k + pdiff);
    const double sd = PI_F * (tmp1 * lp_k - T * lp_k1 - pdiff);
    c.R[k] = R;
    c.T[k] = T;
    c.sd[k] = sd;
    lp_k = lp_k1;
    adding_up(c, k, R, T, su, sd, alb, em);
  }
  adding_down(c, L, 0., [&](int k, double fu, double fd) {
    up[k] = up[k] + fu;
    dn[k] = dn[k] + fd;
  });
}

// One thread per interior column: the layer pressures and temperatures
// (mod_radiation.f90:54-103), then for g = 1..16 in order the shortwave
// and longwave fluxes added into the four sums the reference keeps
// (:113-147), and net_flux = (down sw + down lw) - (up sw + up lw) (:149-152).
// The reference also overwrites plev, pkap, play and playkap of the shared
// fields here; every later reader recomputes them first, so they stay
// local.  Its domain is the interior plus 3 halo cells, whose values the
// halo exchange that follows replaces: the interior is computed here and
// atm_radiation_halo fills the halo.
template <int LM>
__global__ void __launch_bounds__(128, 8) k_radiation(Geom g, RadTables tb, RadArgs a) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.nx * g.ny) return;
  const int i = col % g.nx, j = col / g.nx;
  const int L = g.L;
  const long long S = g.S, o = g.at(i, j);
  double play[LM + 1], tlay[LM + 1], tlev[LM + 2], dm[LM + 1];
  double usw[LM + 2], dsw[LM + 2], ulw[LM + 2], dlw[LM + 2];
  // layer properties, from the model top down (:54-84)
  double plev_up = a.ptop, pk_up = a.pk_top;  // plev(k + 1), pkap(k + 1)
  for (int k = L; k >= 1; --k) {
    const double dpk = a.dp[o + (long long)(k - 1) * S];
    const double plev_k = plev_up + dpk;
    const double pk_k = atm_pow(plev_k, KAPPA);
    double plog = atm_log(plev_k / plev_up);
    play[k] = dpk / plog;
    const double playkap = (pk_up - pk_k) / (-(plog * KAPPA));
    tlay[k] = a.pt[o + (long long)(k - 1) * S] * playkap;
    if (k < L) {  // linear interpolation of T in log p
      const double p1 = atm_log(play[k]), p2 = atm_log(play[k + 1]);
      plog = atm_log(plev_up);
      tlev[k + 1] = (tlay[k] * (p2 - plog) + tlay[k + 1] * (plog - p1)) / (p2 - p1);
    }
    plev_up = plev_k;
    pk_up = pk_k;
  }
  {  // linear extrapolation in log p to the model top (:86-93) and bottom (:95-102)
    double p1 = atm_log(play[L - 1]), p2 = atm_log(play[L]), plog = atm_log(a.ptop);
    tlev[L + 1] = (tlay[L - 1] * (p2 - plog) + tlay[L] * (plog - p1)) / (p2 - p1);
    p1 = atm_log(play[1]);
    p2 = atm_log(play[2]);
    plog = atm_log(plev_up);
    tlev[1] = (tlay[1] * (p2 - plog) + tlay[2] * (plog - p1)) / (p2 - p1);
  }
  for (int k = 1; k <= L; ++k) dm[k] = a.dp[o + (long long)(k - 1) * S] / a.gravity;  // :118
  for (int k = 1; k <= L + 1; ++k) usw[k] = dsw[k] = ulw[k] = dlw[k] = 0.;          // :112-116
  // solar_irradiance (mod_solar.f90:26-35)
  const double r = a.radius[col] / SOLAR_SCALE;
  const double irradiance = SOLAR_BASE * (1. + SOLAR_PEAK / (1. + r * r));
  const double ts = a.ts[o];
  // the table brackets of every layer and level, shared by the g-points
  bool bad = false;
  unsigned code[LM + 1];
  int kb[LM + 2];
  for (int k = 1; k <= L; ++k) code[k] = bracket_pt(tb, play[k], tlay[k], bad);
  for (int k = 1; k <= L + 1; ++k) kb[k] = bracket(tlev[k], tb.plk_t, tb.npl, bad);
  const int kbs = bracket(ts, tb.plk_t, tb.npl, bad);
  Column<LM> c;
  if (!bad)
    for (int gp = 0; gp < tb.ng; ++gp) {
      shortwave<LM>(tb, gp, L, play, dm, tlay, code, tb.frac[gp] * irradiance, a.mu0, a.albedo, c, usw, dsw);
      longwave<LM>(tb, gp, L, play, dm, tlay, tlev, code, kb, ts, kbs, a.emissivity, c, ulw, dlw);
    }
  for (int k = 1; k <= L + 1; ++k) a.nf[o + (long long)(k - 1) * S] = (dsw[k] + dlw[k]) - (usw[k] + ulw[k]);
  if (bad) atomicOr(a.range_error, 1);
}

template <int LM>
cudaError_t launch(const Geom& g, const RadTables& t, const RadArgs& a, cudaStream_t s) {
  const int n = g.nx * g.ny;
  k_radiation<LM><<<(n + 127) / 128, 128, 0, s>>>(g, t, a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t radiative_heating(const Geom& g, const RadTables& t, const RadArgs& a, cudaStream_t s) {
  if (g.L <= 32) return launch<32>(g, t, a, s);
  if (g.L <= 64) return launch<64>(g, t, a, s);
  return launch<MAX_LAYERS>(g, t, a, s);
}

}  // namespace atm
