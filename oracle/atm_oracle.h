/*
 * CPU oracle for the dynamical-core step of felix-goddard/atmosphere-model.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-faithful FP64 restatement of the
 * reference's Fortran (src/mod_sw_dyn.f90, src/mod_remap.f90, the single-image
 * path of src/mod_sync.f90 / src/mod_tiles.f90, src/mod_fields.f90:69-106,
 * src/mod_physics.f90 and the constants of src/mod_constants.f90).  It is the
 * checker for the CUDA library and the timed CPU baseline; no product code
 * path may link or call it.
 *
 * PARITY UNPINNED: the reference is Fortran 2008 with coarrays and needs
 * gfortran + OpenCoarrays + netCDF-Fortran, none of which exist on this
 * machine, and the reference ships no tests, golden vectors or FP64 output
 * (its netCDF files are written as FP32, src/mod_netcdf.f90:197,243,412).
 * The restatement is therefore pinned only by analytic known-answer tests
 * (resting-atmosphere steadiness, remap identity, mass conservation, halo
 * wrap) and by agreement between its serial and layer-parallel modes.
 *
 * Arrays use the reference's layout: Fortran column-major, i fastest, with
 * bounds (is:ie, js:je, 1:K), is = isd - 7 (src/mod_tiles.f90:12,222-241).
 */
#ifndef ATM_ORACLE_H
#define ATM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

/* field identifiers, shared with include/atmdyn.h */
enum {
  ORC_DP = 0, ORC_PT = 1, ORC_UD = 2, ORC_VD = 3,
  ORC_GZ = 4, ORC_PLEV = 5, ORC_PKAP = 6, ORC_NET_FLUX = 7,
  /* the C-grid half step's module arrays (private in mod_sw_dyn.f90:23-27) */
  ORC_DPC = 8, ORC_PTC = 9, ORC_UC = 10, ORC_VC = 11,
  /* surface temperature (mod_fields.f90:51), one level */
  ORC_TS = 12
};

orc_state* orc_create(int nx, int ny, int nlay, double dx, double dy,
                      const double* ak, const double* bk, double gravity,
                      double coriolis, double divdamp, double vortdamp);
void orc_destroy(orc_state* s);

/* with_halo = 1: a is the full (is:ie, js:je, K) array; 0: interior (nx, ny, K) */
int orc_set_field(orc_state* s, int field, const double* a, int with_halo);
int orc_get_field(orc_state* s, int field, double* a, int with_halo);
/* extent of a field in levels (nlay or nlay+1), or -1 */
int orc_field_levels(orc_state* s, int field);

/* mod_input.f90:229-231 (plev/pkap top) + initial_halo_exchange (:247) +
   init_sw_dyn (mod_sw_dyn.f90:958) + allocate_remapping_arrays (mod_remap.f90:358) */
void orc_init(orc_state* s);

void orc_cgrid_step(orc_state* s, double dt);   /* dt is the half step */
void orc_cgrid_halo(orc_state* s);
void orc_dgrid_step(orc_state* s, double dt);
void orc_remap(orc_state* s);
void orc_dgrid_halo(orc_state* s);
/* src/mod_physics.f90: calculate_physics_tendencies (:27-79, with
   dry_convective_adjustment and surface_heating), apply_physics_tendencies
   (:187-211), physics_halo_exchange (:213-217) */
void orc_physics_tendencies(orc_state* s);
void orc_apply_physics(orc_state* s, double dt);
void orc_physics_halo(orc_state* s);
int  orc_check_stability(orc_state* s);          /* 1 = all finite */
double orc_mass(orc_state* s);                   /* sum of interior dp */

/* 0 or 1 thread: the faithful serial loops; n > 1: OpenMP over layers with
   thread-private scratch (bit-identical results) */
void orc_set_threads(orc_state* s, int nthreads);
/* re-fill every 2-D scratch array with NaN before each layer (debug) */
void orc_set_poison(orc_state* s, int on);

/* Remap pair trace.  buf holds int32[3][ny+2][nx+2][nlay][5]; for every
   remapped variable (0 = u, 1 = v, 2 = energy), every column over
   [isd-1, ied+1]^2 and every destination layer m it records
   {first k, last k, case of first, case of last, number of pairs}
   of the source layers that contribute (src/mod_remap.f90:176-283).
   Columns that a variable does not remap hold -1. NULL disables. */
void orc_set_remap_trace(orc_state* s, int32_t* buf);

/* Tangent-linear model: the same restatement on dual numbers (dual.h).  A
   field carries values and tangents; the value part is bit-identical to the
   FP64 run, so the tangents are the derivative of the branch-frozen step. */
typedef struct orc_tlm orc_tlm;
orc_tlm* tlm_create(int nx, int ny, int nlay, double dx, double dy, const double* ak, const double* bk,
                    double gravity, double coriolis, double divdamp, double vortdamp);
void tlm_destroy(orc_tlm* s);
/* tan may be NULL (zero tangents on set; not returned on get) */
int tlm_set_field(orc_tlm* s, int field, const double* val, const double* tan, int with_halo);
int tlm_get_field(orc_tlm* s, int field, double* val, double* tan, int with_halo);
void tlm_init(orc_tlm* s);
void tlm_cgrid_step(orc_tlm* s, double dt);
void tlm_cgrid_halo(orc_tlm* s);
void tlm_dgrid_step(orc_tlm* s, double dt);
void tlm_remap(orc_tlm* s);
void tlm_dgrid_halo(orc_tlm* s);
void tlm_set_threads(orc_tlm* s, int nthreads);

/* the x**y and log(x) the oracle uses, element-wise (accuracy tests) */
void orc_pow_array(const double* x, double y, double* out, int n);
void orc_log_array(const double* x, double* out, int n);

/* radiation (src/mod_radiation.f90:41-398, src/mod_gas_optics.f90,
   src/mod_solar.f90), atm_oracle_radiation.cpp.  Tables in the layout of
   include/atmdyn.h's atm_gas_optics; fields interior-only, i fastest:
   dp, pt (nlay, ny, nx), ts (ny, nx), net_flux out (nlay + 1, ny, nx).
   Returns 0, 1 when a lookup leaves a table (where the reference stops),
   2 on bad sizes. */
typedef struct {
  int n_g, n_p, n_t, n_planck;
  const double *pressures, *temperatures, *sw_absorption, *sw_scattering, *lw_absorption, *planck_temperatures,
      *planck, *irradiance_fraction;
} orc_gas_optics;
int orc_radiative_heating(int nx, int ny, int nlay, const double* dp, const double* pt, const double* ts,
                          const double* xc, const double* yc, double ptop, double gravity,
                          const orc_gas_optics* go, double sza, double surface_albedo,
                          double surface_emissivity, double* net_flux, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
