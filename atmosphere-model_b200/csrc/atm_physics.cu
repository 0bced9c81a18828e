// Column physics of the reference (src/mod_physics.f90) on the device, FP64
// in both forms (the prognostic state is FP64 in both):
//   calculate_physics_tendencies (:27-79) with dry_convective_adjustment
//   (:81-176) and surface_heating (:178-185)  -> k_physics_tend
//   apply_physics_tendencies (:187-211)       -> k_physics_apply
// Built with --fmad=false: every value is the reference's expression,
// evaluated in its order, so the results are those of the FP64 restatement.
#include "atm_ops.h"
#include "atm_physics.h"

namespace atm {
namespace {

// mod_physics.f90:86-88 (min_v2 is a default-real literal) and :179
constexpr double MIN_V2 = (double)1e-4f;
constexpr double CRITICAL_RI = .25;
constexpr double MIXING_TIMESCALE = 600.;
constexpr double SURFACE_HEAT_CAPACITY = 41680. * 5.;

// One thread per column over [isd-2, ied+2]^2.  The reference computes the
// A-grid winds, plev, pkap, gz and playkap as whole-domain arrays and then
// adjusts each column; a column reads only its own levels and the D-grid
// winds of its neighbours, so each thread forms its column here: a
// downward pass stores plev and pkap (the suffix sum from the model top),
// then one upward pass forms gz, playkap and the energy of layer k + 1,
// mixes across interface k, and finishes layer k (its wind tendencies and
// the potential temperature recovered from its energy), which no later
// interface touches.  Every quantity is the reference's expression.
template <int LM>
__global__ void __launch_bounds__(128) k_physics_tend(Geom g, double ptop, double pk_top,
                                                      const double* __restrict__ dp, const double* __restrict__ pt,
                                                      const double* __restrict__ ud, const double* __restrict__ vd,
                                                      const double* __restrict__ gzs, const double* __restrict__ nf,
                                                      double* __restrict__ pt_tend, double* __restrict__ u_tend,
                                                      double* __restrict__ v_tend, double* __restrict__ ts_tend) {
  const int w = g.nx + 4;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w * (g.ny + 4)) return;
  const int i = -2 + col % w, j = -2 + col / w;
  const int L = g.L;
  const long long S = g.S;
  const int P = g.P;
  const long long o = g.at(i, j);
  double plev[LM + 2], pk[LM + 2];
  // plev, pkap downward (:49-57); plev(nlay+1), pkap(nlay+1): mod_input.f90:229-231
  plev[L + 1] = ptop;
  pk[L + 1] = pk_top;
  for (int k = L; k >= 1; --k) {
    plev[k] = plev[k + 1] + dp[o + (long long)(k - 1) * S];
    pk[k] = atm_pow(plev[k], KAPPA);
  }
  // layer k's A-grid winds (:39-47)
  auto ua = [&](long long ok) {
    return (.25 * (ud[ok] + ud[ok + P]) + .125 * (ud[ok - 1] + ud[ok - 1 + P] + ud[ok + 1] + ud[ok + 1 + P]));
  };
  auto va = [&](long long ok) {
    return (.25 * (vd[ok] + vd[ok + 1]) + .125 * (vd[ok - P] + vd[ok + 1 - P] + vd[ok + P] + vd[ok + 1 + P]));
  };
  // playkap (:66-69)
  auto playkap = [&](int k) { return (pk[k + 1] - pk[k]) / atm_log(plev[k + 1] / plev[k]) / KAPPA; };

  // layer 1: gz(1) is the surface geopotential, gz(2) from :60-64
  long long ok = o;
  double pt_c = pt[ok], dp_c = dp[ok], ua_c = ua(ok), va_c = va(ok);
  double gz_c = gzs[o];
  double gz_c1 = gz_c + CP_DRY * pt_c * (pk[1] - pk[2]);
  double ply_c = playkap(1);
  double e_c = CV_DRY * pt_c * ply_c + .5 * (gz_c1 + gz_c + ua_c * ua_c + va_c * va_c);  // :95-97
  double u_c = ua_c, v_c = va_c;
  double gza = gz_c;  // gz_adj(1) = gz(1) (:157)
  for (int k = 1; k <= L; ++k) {
    double pt_n = 0., dp_n = 0., ua_n = 0., va_n = 0., gz_n1 = 0., e_n = 0., u_n = 0., v_n = 0., ply_n = 0.;
    if (k < L) {
      const long long on = ok + S;
      pt_n = pt[on];
      dp_n = dp[on];
      ua_n = ua(on);
      va_n = va(on);
      gz_n1 = gz_c1 + CP_DRY * pt_n * (pk[k + 1] - pk[k + 2]);
      ply_n = playkap(k + 1);
      e_n = CV_DRY * pt_n * ply_n + .5 * (gz_n1 + gz_c1 + ua_n * ua_n + va_n * va_n);
      u_n = ua_n;
      v_n = va_n;
      // Richardson number on interface k (:103-109) and the mixing (:111-133)
      const double du = ua_n - ua_c, dv = va_n - va_c;
      const double ri = (pt_n - pt_c) * (dp_c * (gz_c1 - gz_c) + dp_n * (gz_n1 - gz_c1)) /
                        ((dp_c * pt_c + dp_n * pt_n) * (du * du + dv * dv + MIN_V2));
      if (ri < CRITICAL_RI) {
        const double q = ri / CRITICAL_RI;
        const double t = 1. - (q > 0. ? q : 0.);  // 1 - max(0.0, q)
        const double mixing_fraction = t * t * dp_c * dp_n / (dp_c + dp_n);
        double exchange = mixing_fraction * (u_c - u_n);
        u_c = u_c - exchange / dp_c;
        u_n = u_n + exchange / dp_n;
        exchange = mixing_fraction * (v_c - v_n);
        v_c = v_c - exchange / dp_c;
        v_n = v_n + exchange / dp_n;
        exchange = mixing_fraction * (e_c - e_n);
        e_c = e_c - exchange / dp_c;
        e_n = e_n + exchange / dp_n;
      }
    }
    // layer k is final: wind tendencies (:139-142, the tendencies start at
    // zero, :31-34) and the recovered potential temperature (:146-166)
    u_tend[ok] = 0. + (u_c - ua_c) / MIXING_TIMESCALE;
    v_tend[ok] = 0. + (v_c - va_c) / MIXING_TIMESCALE;
    const double pta = (e_c - gza - .5 * (u_c * u_c + v_c * v_c)) / (CV_DRY * ply_c + .5 * CP_DRY * (pk[k] - pk[k + 1]));
    gza = gza + CP_DRY * pta * (pk[k] - pk[k + 1]);
    pt_tend[ok] = 0. + (pta - pt_c) / MIXING_TIMESCALE;
    pt_c = pt_n;
    dp_c = dp_n;
    ua_c = ua_n;
    va_c = va_n;
    gz_c = gz_c1;
    gz_c1 = gz_n1;
    e_c = e_n;
    u_c = u_n;
    v_c = v_n;
    ply_c = ply_n;
    ok += S;
  }
  // surface_heating on the interior (:178-185)
  if (i >= 0 && i < g.nx && j >= 0 && j < g.ny) ts_tend[o] = (nf ? nf[o] : 0.) / SURFACE_HEAT_CAPACITY;
}

// apply_physics_tendencies on the interior (:187-211); dp_tend is zero
// (:31), kept as dp + dt * 0 so that dp is what the reference makes of it.
__global__ void k_physics_apply(Geom g, double dt, double* __restrict__ dp, double* __restrict__ pt,
                                double* __restrict__ ud, double* __restrict__ vd, double* __restrict__ ts,
                                const double* __restrict__ pt_tend, const double* __restrict__ u_tend,
                                const double* __restrict__ v_tend, const double* __restrict__ ts_tend) {
  const long long n = (long long)g.nx * g.ny;
  const long long total = n * g.L;
  const int P = g.P;
  const double dp_tend = 0.;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q / n);
    const long long r = q - (long long)k * n;
    const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
    const long long o = g.at(i, j, k);
    dp[o] = dp[o] + dt * dp_tend;
    pt[o] = pt[o] + dt * pt_tend[o];
    if (k == 0) {
      const long long o2 = g.at(i, j);
      ts[o2] = ts[o2] + dt * ts_tend[o2];
    }
    ud[o] = ud[o] + dt * (C7_12 * (u_tend[o] + u_tend[o - P]) - C1_12 * (u_tend[o + P] + u_tend[o - 2 * P]));
    vd[o] = vd[o] + dt * (C7_12 * (v_tend[o] + v_tend[o - 1]) - C1_12 * (v_tend[o + 1] + v_tend[o - 2]));
  }
}

template <int LM>
cudaError_t physics_tend_lm(const Geom& g, const PhysicsArgs& a, cudaStream_t s) {
  const int n = (g.nx + 4) * (g.ny + 4);
  k_physics_tend<LM><<<(n + 127) / 128, 128, 0, s>>>(g, a.ptop, a.pk_top, a.dp, a.pt, a.ud, a.vd, a.gzs, a.nf,
                                                     a.pt_tend, a.u_tend, a.v_tend, a.ts_tend);
  return cudaGetLastError();
}

}  // namespace

cudaError_t physics_tend(const Geom& g, const PhysicsArgs& a, cudaStream_t s) {
  if (g.L <= 32) return physics_tend_lm<32>(g, a, s);
  if (g.L <= 64) return physics_tend_lm<64>(g, a, s);
  return physics_tend_lm<MAX_LAYERS>(g, a, s);
}

cudaError_t physics_apply(const Geom& g, double dt, const PhysicsArgs& a, double* dp, double* pt, double* ud,
                          double* vd, double* ts, cudaStream_t s) {
  k_physics_apply<<<1184, 256, 0, s>>>(g, dt, dp, pt, ud, vd, ts, a.pt_tend, a.u_tend, a.v_tend, a.ts_tend);
  return cudaGetLastError();
}

}  // namespace atm
