// CPU oracle (test infrastructure only) for the radiation of
// felix-goddard/atmosphere-model: a line-faithful FP64 restatement of
//   src/mod_radiation.f90:41-156   calculate_radiative_heating
//   src/mod_radiation.f90:158-268  solve_shortwave_column
//   src/mod_radiation.f90:270-347  solve_longwave_column
//   src/mod_radiation.f90:349-381  calculate_fluxes
//   src/mod_radiation.f90:383-398  delta_eddington_rescaling
//   src/mod_gas_optics.f90:4556-4609  lookup_1d, lookup_pT_table (linear
//                                     scans, as written)
//   src/mod_solar.f90:26-35        solar_irradiance
//   src/mod_input.f90:233-243      radius from the xc, yc axes
// Loops, evaluation order and the default-real literals (.3, .99, .2,
// 100000e3, pi) follow the Fortran.  Build with -ffp-contract=off.
// The reference stops on a lookup outside its table; here the call returns 1.
#include "atm_oracle.h"

#include <cmath>
#include <thread>
#include <vector>

#ifdef ORC_LIBM
static inline double rad_pow(double x, double y) { return std::pow(x, y); }
static inline double rad_log(double x) { return std::log(x); }
static inline double rad_exp(double x) { return std::exp(x); }
#else
#include "../atmosphere-model_b200/csrc/atm_math.h"
static inline double rad_pow(double x, double y) { return atm_pow(x, y); }
static inline double rad_log(double x) { return atm_log(x); }
static inline double rad_exp(double x) { return atm_exp(x); }
#endif

namespace {

const double R_DRY = (double)287.052874f;  // mod_constants.f90:11-14
const double CP_DRY = 1005.0;
const double KAPPA = R_DRY / CP_DRY;
const double PI = (double)3.1415926535897932384626433f;  // mod_constants.f90:8

struct Abort {};  // logger%fatal + abort_now

// lookup_1d (mod_gas_optics.f90:4556-4579); xs, ys 1-based through the lambda
double lookup_1d(double x, const double* xs, const double* ys, int n) {
  auto X = [&](int k) { return xs[k - 1]; };
  auto Y = [&](int k) { return ys[k - 1]; };
  if (x < X(1) || x > X(n)) throw Abort();
  if (x != x) throw Abort();  // the reference would read xs(0) here
  int k = 1;
  while (x > X(k)) k = k + 1;
  if (x == X(k)) return Y(k);
  return (Y(k) * (X(k - 1) - x) + Y(k - 1) * (x - X(k))) / (X(k - 1) - X(k));
}

// lookup_pT_table (mod_gas_optics.f90:4581-4609); table(t, p) of one g-point
double lookup_pt(const orc_gas_optics& go, double pressure, double temperature, const double* table) {
  const int np = go.n_p, nt = go.n_t;
  auto P = [&](int k) { return go.pressures[k - 1]; };
  if (pressure < P(1) || pressure > P(np)) throw Abort();
  if (pressure != pressure) throw Abort();
  int k = 1;
  while (pressure > P(k)) k = k + 1;
  const double* tk = go.temperatures + (size_t)(k - 1) * nt;
  const double* yk = table + (size_t)(k - 1) * nt;
  if (pressure == P(k)) return lookup_1d(temperature, tk, yk, nt);
  const double t1 = lookup_1d(temperature, tk, yk, nt);
  const double t2 = lookup_1d(temperature, tk - nt, yk - nt, nt);
  return (t1 * (P(k - 1) - pressure) + t2 * (pressure - P(k))) / (P(k - 1) - P(k));
}

void delta_eddington_rescaling(double& optical_thickness, double& single_scattering_albedo, double& asymmetry) {
  double forward_scatter = asymmetry * asymmetry;
  double coefficient = 1. - single_scattering_albedo * forward_scatter;
  optical_thickness = optical_thickness * coefficient;
  single_scattering_albedo = single_scattering_albedo * (1. - forward_scatter) / coefficient;
  asymmetry = asymmetry / (1. + asymmetry);
}

// the module arrays of one column solve (mod_radiation.f90:34-38), 1-based
struct Work {
  int nlay;
  std::vector<double> flux_up, flux_dn, transmittance, reflectance, albedo, emission_up, beta, source_up, source_dn,
      solar_beam;
  explicit Work(int n)
      : nlay(n), flux_up(n + 2), flux_dn(n + 2), transmittance(n + 1), reflectance(n + 1), albedo(n + 2),
        emission_up(n + 2), beta(n + 1), source_up(n + 2), source_dn(n + 2), solar_beam(n + 2) {}
};

}  // namespace

namespace {

// calculate_fluxes (mod_radiation.f90:349-381)
void calculate_fluxes(Work& w, double toa_downward_flux, double sfc_upward_flux, double sfc_albedo) {
  const int nlay = w.nlay;
  auto& R = w.reflectance;
  auto& T = w.transmittance;
  w.albedo[1] = sfc_albedo;
  w.emission_up[1] = sfc_upward_flux;
  for (int k = 1; k <= nlay; ++k) {
    w.beta[k] = 1. / (1. - R[k] * w.albedo[k]);
    w.albedo[k + 1] = R[k] + (T[k] * T[k]) * w.beta[k] * w.albedo[k];
    w.emission_up[k + 1] = w.source_up[k] + T[k] * w.beta[k] * (w.emission_up[k] + w.source_dn[k] * w.albedo[k]);
  }
  w.flux_dn[nlay + 1] = toa_downward_flux;
  w.flux_up[nlay + 1] = w.albedo[nlay + 1] * toa_downward_flux + w.emission_up[nlay + 1];
  for (int k = nlay + 1; k >= 2; --k) {
    w.flux_dn[k - 1] =
        w.beta[k - 1] * (w.source_dn[k - 1] + T[k - 1] * w.flux_dn[k] + R[k - 1] * w.emission_up[k - 1]);
    w.flux_up[k - 1] = w.albedo[k - 1] * w.flux_dn[k - 1] + w.emission_up[k - 1];
  }
}

// solve_shortwave_column (mod_radiation.f90:158-268); pressure, layer_mass,
// temperature 1-based
void solve_shortwave_column(Work& w, const orc_gas_optics& go, int g_point, const double* pressure,
                            const double* layer_mass, const double* temperature, double irradiance, double sza,
                            double surface_albedo) {
  const int nlay = w.nlay;
  const double* lut = go.sw_absorption + (size_t)(g_point - 1) * go.n_p * go.n_t;
  double mu0 = std::cos(sza);
  w.solar_beam[nlay + 1] = mu0 * irradiance;
  for (int k = nlay; k >= 1; --k) {
    double k_abs = lookup_pt(go, pressure[k], temperature[k], lut);
    double k_sca = go.sw_scattering[g_point - 1];
    double k_ext = k_abs + k_sca;
    double optical_thickness = k_ext * layer_mass[k];
    double single_scattering_albedo = k_sca / k_ext;
    double asymmetry = 0.;
    delta_eddington_rescaling(optical_thickness, single_scattering_albedo, asymmetry);
    double asy2 = asymmetry * asymmetry;
    double backscatter = (2. - 3. * asymmetry * mu0) / 4.;
    double tmp1 = 4. * (1. - asy2 * (1. - mu0));
    double gamma3 = single_scattering_albedo * asy2;
    double gamma4 = 4. * backscatter + 3. * asymmetry;
    double tmp2 = 3. * asymmetry;
    double gamma1 = (7. - 3. * asy2 - single_scattering_albedo * (4. + tmp2) + gamma3 * gamma4) / tmp1;
    double gamma2 = (-1. + asy2 + single_scattering_albedo * (4. - tmp2) + gamma3 * (gamma4 - 4.)) / tmp1;
    gamma3 = backscatter;
    gamma4 = 1. - gamma3;
    double alpha1 = gamma1 * gamma4 + gamma2 * gamma3;
    double alpha2 = gamma2 * gamma3 + gamma2 * gamma4;
    double lambda = std::sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    double lam_mu = lambda * mu0;
    double e_minus = rad_exp(-lambda * optical_thickness);
    double e_2minus = e_minus * e_minus;
    double direct_transmittance = rad_exp(-optical_thickness / mu0);
    tmp1 = single_scattering_albedo / ((1. - lam_mu * lam_mu) * (lambda + gamma1 + (lambda - gamma1) * e_2minus));
    tmp2 = lambda * gamma3;
    double diffuse_reflectance =
        tmp1 * ((1. - lam_mu) * (alpha2 + tmp2) - (1. + lam_mu) * (alpha2 - tmp2) * e_2minus -
                2. * lambda * (gamma3 - alpha2 * mu0) * e_minus * direct_transmittance);
    tmp2 = lambda * gamma4;
    double diffuse_transmittance =
        tmp1 * (2. * lambda * (gamma4 + alpha1 * mu0) * e_minus -
                direct_transmittance * ((1. + lam_mu) * (alpha1 + tmp2) - (1. - lam_mu) * (alpha1 - tmp2) * e_2minus));
    w.solar_beam[k] = direct_transmittance * w.solar_beam[k + 1];
    w.source_up[k] = diffuse_reflectance * w.solar_beam[k + 1];
    w.source_dn[k] = diffuse_transmittance * w.solar_beam[k + 1];
    backscatter = (4. + asymmetry) / (8. * (1. + asymmetry));
    gamma1 = 2. * (1. - single_scattering_albedo * (1. - backscatter));
    gamma2 = 2. * single_scattering_albedo * backscatter;
    lambda = std::sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    e_2minus = e_minus * e_minus;
    tmp1 = 1. / (lambda + gamma1 + (lambda - gamma1) * e_2minus);
    w.reflectance[k] = tmp1 * gamma2 * (1. - e_2minus);
    w.transmittance[k] = 2. * tmp1 * lambda * e_minus;
  }
  calculate_fluxes(w, w.solar_beam[nlay + 1], 0., surface_albedo);
  for (int k = 1; k <= nlay + 1; ++k) w.flux_dn[k] = w.flux_dn[k] + w.solar_beam[k];
}

// planck_function (mod_gas_optics.f90:3575-4554)
double planck_function(const orc_gas_optics& go, int g_point, double temperature) {
  return lookup_1d(temperature, go.planck_temperatures, go.planck + (size_t)(g_point - 1) * go.n_planck,
                   go.n_planck);
}

// solve_longwave_column (mod_radiation.f90:270-347)
void solve_longwave_column(Work& w, const orc_gas_optics& go, int g_point, const double* pressure,
                           const double* layer_mass, const double* temperature, const double* level_temperature,
                           double surface_temperature, double surface_emissivity) {
  const int nlay = w.nlay;
  const double* lut = go.lw_absorption + (size_t)(g_point - 1) * go.n_p * go.n_t;
  std::vector<double> level_planckian(nlay + 2);
  double surface_planckian = planck_function(go, g_point, surface_temperature);
  level_planckian[1] = planck_function(go, g_point, level_temperature[1]);
  for (int k = 1; k <= nlay; ++k) {
    double k_abs = lookup_pt(go, pressure[k], temperature[k], lut);
    double k_sca = 0.;
    double k_ext = k_abs + k_sca;
    double optical_thickness = k_ext * layer_mass[k];
    double single_scattering_albedo = k_sca / k_ext;
    double asymmetry = 0.;
    delta_eddington_rescaling(optical_thickness, single_scattering_albedo, asymmetry);
    double backscatter = (4. - 3. * asymmetry) / 8.;
    double gamma1 = 2. * (1. - single_scattering_albedo * (1. - backscatter));
    double gamma2 = 2. * single_scattering_albedo * backscatter;
    double lambda = std::sqrt(gamma1 * gamma1 - gamma2 * gamma2);
    double e_minus = rad_exp(-lambda * optical_thickness);
    double e_2minus = e_minus * e_minus;
    double tmp1 = 1. / (lambda + gamma1 + (lambda - gamma1) * e_2minus);
    w.reflectance[k] = tmp1 * gamma2 * (1. - e_2minus);
    w.transmittance[k] = 2. * tmp1 * lambda * e_minus;
    level_planckian[k + 1] = planck_function(go, g_point, level_temperature[k + 1]);
    double planckian_difference = (1. + w.reflectance[k] - w.transmittance[k]) *
                                  (level_planckian[k] - level_planckian[k + 1]) /
                                  (optical_thickness * (gamma1 + gamma2));
    tmp1 = 1. - w.reflectance[k];
    w.source_up[k] =
        PI * (tmp1 * level_planckian[k + 1] - w.transmittance[k] * level_planckian[k] + planckian_difference);
    w.source_dn[k] =
        PI * (tmp1 * level_planckian[k] - w.transmittance[k] * level_planckian[k + 1] - planckian_difference);
  }
  calculate_fluxes(w, 0., surface_emissivity * PI * surface_planckian, 1. - surface_emissivity);
}

}  // namespace

namespace {

// calculate_radiative_heating (mod_radiation.f90:41-156) for the columns
// c0 <= c < c1 (c = j nx + i); returns 1 on a lookup outside the tables
int heating_columns(int nx, int ny, int nlay, const double* dp, const double* pt, const double* ts,
                    const double* radius, double ptop, double gravity, const orc_gas_optics& go, double sza,
                    double surface_albedo, double surface_emissivity, double* net_flux, long long c0, long long c1) {
  (void)ny;
  const long long n2 = (long long)nx * ny;
  Work w(nlay);
  std::vector<double> plev(nlay + 2), pkap(nlay + 2), play(nlay + 1), playkap(nlay + 1), layer_temperature(nlay + 1),
      level_temperature(nlay + 2), dm(nlay + 1), usw(nlay + 2), dsw(nlay + 2), ulw(nlay + 2), dlw(nlay + 2);
  try {
    for (long long c = c0; c < c1; ++c) {
      auto DP = [&](int k) { return dp[(long long)(k - 1) * n2 + c]; };
      auto PT = [&](int k) { return pt[(long long)(k - 1) * n2 + c]; };
      // layer properties (:54-103); plev(nlay+1), pkap(nlay+1): mod_input.f90:229-231
      plev[nlay + 1] = ptop;
      pkap[nlay + 1] = rad_pow(ptop, KAPPA);
      double plog, p1, p2;
      for (int k = nlay; k >= 1; --k) {
        plev[k] = plev[k + 1] + DP(k);
        pkap[k] = rad_pow(plev[k], KAPPA);
        plog = rad_log(plev[k] / plev[k + 1]);
        play[k] = DP(k) / plog;
        playkap[k] = (pkap[k + 1] - pkap[k]) / (-plog * KAPPA);
        layer_temperature[k] = PT(k) * playkap[k];
        if (k < nlay) {
          p1 = rad_log(play[k]);
          p2 = rad_log(play[k + 1]);
          plog = rad_log(plev[k + 1]);
          level_temperature[k + 1] =
              (layer_temperature[k] * (p2 - plog) + layer_temperature[k + 1] * (plog - p1)) / (p2 - p1);
        }
      }
      p1 = rad_log(play[nlay - 1]);
      p2 = rad_log(play[nlay]);
      plog = rad_log(plev[nlay + 1]);
      level_temperature[nlay + 1] =
          (layer_temperature[nlay - 1] * (p2 - plog) + layer_temperature[nlay] * (plog - p1)) / (p2 - p1);
      p1 = rad_log(play[1]);
      p2 = rad_log(play[2]);
      plog = rad_log(plev[1]);
      level_temperature[1] = (layer_temperature[1] * (p2 - plog) + layer_temperature[2] * (plog - p1)) / (p2 - p1);
      // the column's two-stream solutions (:105-153)
      for (int k = 1; k <= nlay + 1; ++k) usw[k] = dsw[k] = ulw[k] = dlw[k] = 0.;
      for (int k = 1; k <= nlay; ++k) dm[k] = DP(k) / gravity;
      // solar_irradiance (mod_solar.f90:26-35)
      double irradiance = 600 * (1. + (double).2f / (1. + (radius[c] / (double)100000e3f) * (radius[c] / (double)100000e3f)));
      for (int g = 1; g <= go.n_g; ++g) {
        solve_shortwave_column(w, go, g, play.data(), dm.data(), layer_temperature.data(),
                               go.irradiance_fraction[g - 1] * irradiance, sza, surface_albedo);
        for (int k = 1; k <= nlay + 1; ++k) {
          usw[k] = usw[k] + w.flux_up[k];
          dsw[k] = dsw[k] + w.flux_dn[k];
        }
        solve_longwave_column(w, go, g, play.data(), dm.data(), layer_temperature.data(), level_temperature.data(),
                              ts[c], surface_emissivity);
        for (int k = 1; k <= nlay + 1; ++k) {
          ulw[k] = ulw[k] + w.flux_up[k];
          dlw[k] = dlw[k] + w.flux_dn[k];
        }
      }
      for (int k = 1; k <= nlay + 1; ++k)
        net_flux[(long long)(k - 1) * n2 + c] = (dsw[k] + dlw[k]) - (usw[k] + ulw[k]);
    }
  } catch (const Abort&) {
    return 1;
  }
  return 0;
}

}  // namespace

extern "C" int orc_radiative_heating(int nx, int ny, int nlay, const double* dp, const double* pt, const double* ts,
                                     const double* xc, const double* yc, double ptop, double gravity,
                                     const orc_gas_optics* go, double sza, double surface_albedo,
                                     double surface_emissivity, double* net_flux, int nthreads) {
  if (nx < 1 || ny < 1 || nlay < 2 || !go) return 2;
  // radius (mod_input.f90:233-243)
  std::vector<double> radius((size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double r = xc[i] * xc[i];
      r = r + yc[j] * yc[j];
      radius[(size_t)j * nx + i] = std::sqrt(r);
    }
  const long long n2 = (long long)nx * ny;
  const int nt = nthreads < 1 ? 1 : nthreads;
  std::vector<int> bad(nt, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    long long c0 = n2 * t / nt, c1 = n2 * (t + 1) / nt;
    th.emplace_back([&, t, c0, c1] {
      bad[t] = heating_columns(nx, ny, nlay, dp, pt, ts, radius.data(), ptop, gravity, *go, sza, surface_albedo,
                               surface_emissivity, net_flux, c0, c1);
    });
  }
  for (auto& x : th) x.join();
  for (int b : bad)
    if (b) return 1;
  return 0;
}
