// Device column physics (src/mod_physics.f90), FP64 in both forms.
#pragma once

#include <cuda_runtime.h>
#include "atm_common.cuh"

namespace atm {

struct PhysicsArgs {
  double ptop, pk_top;           // plev(nlay+1) and pkap(nlay+1) (mod_input.f90:229-231)
  const double *dp, *pt, *ud, *vd;
  const double* gzs;             // a field whose level 1 is the surface geopotential
  const double* nf;              // net_flux (level 1 feeds surface_heating) or nullptr (zero)
  double *pt_tend, *u_tend, *v_tend, *ts_tend;
};

// calculate_physics_tendencies (src/mod_physics.f90:27-79): tendencies on
// [isd-2, ied+2]^2, ts_tend on the interior
cudaError_t physics_tend(const Geom& g, const PhysicsArgs& a, cudaStream_t s);
// apply_physics_tendencies (src/mod_physics.f90:187-211) on the interior
cudaError_t physics_apply(const Geom& g, double dt, const PhysicsArgs& a, double* dp, double* pt, double* ud,
                          double* vd, double* ts, cudaStream_t s);

}  // namespace atm
