// Device radiation (src/mod_radiation.f90, src/mod_gas_optics.f90,
// src/mod_solar.f90), FP64 in both forms.
#pragma once

#include <cuda_runtime.h>
#include "atm_common.cuh"

namespace atm {

// The gas-optics tables on the device, in the reference's index order
// (flattened from the last Fortran index): temps[p][t] is temperatures(t, p),
// sw_abs[g][p][t] is shortwave_absorption_lut(t, p, g), planck[g][t] is
// planckian_lut(t, g).
struct RadTables {
  int ng, np, nt, npl;
  const double* pressures;  // [np]
  const double* temps;      // [np][nt]
  const double* sw_abs;     // [ng][np][nt]
  const double* sw_sca;     // [ng]
  const double* lw_abs;     // [ng][np][nt]
  const double* plk_t;      // [npl]
  const double* plk;        // [ng][npl]
  const double* frac;       // [ng], irradiance_fraction
};

struct RadArgs {
  double ptop, pk_top;           // plev(nlay+1) and pkap(nlay+1) (mod_input.f90:229-231)
  double gravity;
  double mu0;                    // cos(solar_zenith_angle) (mod_radiation.f90:174)
  double albedo, emissivity;     // surface_albedo, surface_emissivity (:108-109)
  const double *dp, *pt, *ts;    // state fields (pitched, with halo)
  const double* radius;          // [ny][nx], distance of each cell centre from the origin
  double* nf;                    // net_flux (pitched, nlay + 1 levels)
  int* range_error;              // set when a lookup leaves its table (the reference stops there)
};

// calculate_radiative_heating (src/mod_radiation.f90:41-156) on the interior
cudaError_t radiative_heating(const Geom& g, const RadTables& t, const RadArgs& a, cudaStream_t s);

}  // namespace atm
