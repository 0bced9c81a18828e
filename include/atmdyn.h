/*
 * libatmdyn -- B200 (sm_100a) dynamical-core step of
 * felix-goddard/atmosphere-model behind a plain C ABI.
 *
 * The reference has no plugin API: its dycore is the Fortran module
 * interface of mod_sw_dyn / mod_remap / mod_sync, whose routines take only
 * dt and work on module-global arrays (src/mod_fields.f90:16-37).  Each
 * entry point below replaces one of those routines; the Fortran host binds
 * them through ISO_C_BINDING with the same call order as run_model
 * (src/mod_model.f90:146-177).
 *
 * Conventions
 *  - Every function returns an int status: ATM_OK (0) or an ATM_ERR_* code;
 *    atm_last_error(ctx) returns a message for the last failure.  The
 *    reference logs a fatal message and stops (src/mod_util.f90:13-19); the
 *    Fortran wrapper does the same on a non-zero status.
 *  - Host field arrays are the reference's allocatable arrays passed with
 *    c_loc: FP64, Fortran order (i fastest), bounds (is:ie, js:je, 1:K) with
 *    is = 1 - 7, ie = nx + 7, js = 1 - 7, je = ny + 7 (the single-image
 *    tiling of src/mod_tiles.f90:222-241), K = nlay or nlay + 1 (see the
 *    field table).  The library copies and keeps no host pointer.
 *  - Device memory and one CUDA stream belong to the context; calls are
 *    asynchronous on that stream until a download, atm_sync,
 *    atm_check_stability or atm_mass.  A context is not thread-safe.
 */
#ifndef ATMDYN_H
#define ATMDYN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct atm_ctx atm_ctx;

/* fields (host arrays are (is:ie, js:je, 1:K)) */
enum {
  ATM_DP = 0,        /* pressure thickness dp, K = nlay          (mod_fields.f90:17) */
  ATM_PT = 1,        /* potential temperature pt, K = nlay       (:18) */
  ATM_UD = 2,        /* D-grid u, K = nlay                        (:19) */
  ATM_VD = 3,        /* D-grid v, K = nlay                        (:20) */
  ATM_GZ = 4,        /* geopotential on interfaces, K = nlay + 1; level 1 is the
                        surface geopotential gzs, the only level read on upload (:29) */
  ATM_PLEV = 5,      /* interface pressure, K = nlay + 1 (download only; see below) */
  ATM_PKAP = 6,      /* plev**kappa, K = nlay + 1 (download only) */
  ATM_NET_FLUX = 7,  /* radiative net flux, K = nlay + 1 (upload via atm_set_net_flux) */
  /* download only: the C-grid half step's arrays dpc, ptc, uc, vc, private
     module variables of the reference (src/mod_sw_dyn.f90:23-27), K = nlay;
     valid on the ranges cgrid_dynamics_step writes and, after
     atm_cgrid_halo, everywhere */
  ATM_DPC = 8, ATM_PTC = 9, ATM_UC = 10, ATM_VC = 11,
  ATM_TS = 12        /* surface temperature ts, K = 1 (mod_fields.f90:51); upload,
                        download; the physics updates it (src/mod_physics.f90:172) */
};

/* forms */
enum {
  ATM_FP64 = 0,      /* the reference's FP64 arithmetic, bit-identical to the FP64 restatement */
  ATM_MIXED = 1      /* FP32 horizontal sweeps, FP64 column sums / pkap / gz / remap / mass */
};

/* status codes */
enum {
  ATM_OK = 0,
  ATM_ERR_ARG = 1,       /* invalid argument (sizes, field id, null pointer) */
  ATM_ERR_CUDA = 2,      /* a CUDA call failed; the message names it */
  ATM_ERR_STATE = 3,     /* call out of order (e.g. a step before atm_init) */
  ATM_ERR_NOMEM = 4,     /* device allocation failed */
  ATM_ERR_UNSUPPORTED = 5,
  ATM_ERR_TOO_LARGE = 6, /* atm_remap_noalloc: the domain needs more than its fixed scratch */
  ATM_ERR_RANGE = 7      /* atm_radiative_heating: a lookup outside the gas-optics tables */
};

/* flags for atm_create */
#define ATM_FLAG_NONE 0

/* init_sw_dyn + allocate_remapping_arrays + allocate_sync_buffers
   (src/mod_sw_dyn.f90:958-1023, src/mod_remap.f90:358-388,
   src/mod_sync.f90:219-230): allocates the device state for an
   nx x ny x nlay single-image domain.  ak, bk: the hybrid coordinate,
   nlay+1 entries (Ak(1) is the model-top pressure, src/mod_remap.f90:362).
   g, f, divdamp, vortdamp: the physics_parameters namelist
   (src/mod_config.f90:47-51, src/mod_constants.f90:20-27).
   Requires nx, ny >= 7 and 3 <= nlay <= 128. */
int atm_create(atm_ctx** out, int nx, int ny, int nlay, double dx, double dy, const double* ak,
               const double* bk, double g, double f, double divdamp, double vortdamp,
               int precision, int flags);

/* copy a field from / to a host (is:ie, js:je, 1:K) FP64 array.  Upload
   accepts ATM_DP, ATM_PT, ATM_UD, ATM_VD, ATM_GZ (level 1 only) and ATM_TS.
   Download of ATM_PLEV / ATM_PKAP / ATM_GZ returns the column diagnostics
   recomputed from the current dp and pt (plev = Ak(1) + suffix sum of dp,
   pkap = plev**kappa, hydrostatic gz), on the whole array. */
int atm_upload(atm_ctx* ctx, int field, const double* host);
int atm_download(atm_ctx* ctx, int field, double* host);

/* initial_halo_exchange (src/mod_input.f90:247-252) of dp, pt, gz, ud, vd
   and ts, and the set-up that needs gz (src/mod_sw_dyn.f90:990-996).  Call
   after the uploads and before the first step. */
int atm_init(atm_ctx* ctx);

/* cgrid_dynamics_step(dt) (src/mod_sw_dyn.f90:80-416); dt_half is the
   argument the reference receives (run_model passes dt/2.). */
int atm_cgrid_step(atm_ctx* ctx, double dt_half);
/* cgrid_halo_exchange (src/mod_sw_dyn.f90:418-422): periodic halo fill */
int atm_cgrid_halo(atm_ctx* ctx);
/* dgrid_dynamics_step(dt) (src/mod_sw_dyn.f90:424-773) */
int atm_dgrid_step(atm_ctx* ctx, double dt);
/* perform_vertical_remapping (src/mod_remap.f90:27-163); call it where
   run_model does, after the D-grid step and before the D-grid halo */
int atm_remap(atm_ctx* ctx);
/* dgrid_halo_exchange (src/mod_sw_dyn.f90:775-779): periodic halo fill */
int atm_dgrid_halo(atm_ctx* ctx);

/* check_stability (src/mod_fields.f90:69-106) with the co_reduce of
   src/mod_model.f90:176: *stable = 1 when dp, pt, ud, vd are finite on the
   interior.  Synchronises the stream. */
int atm_check_stability(atm_ctx* ctx, int* stable);
/* total mass: FP64 sum of the interior dp, in a fixed order (no reference
   counterpart; conservation diagnostic).  Synchronises the stream. */
int atm_mass(atm_ctx* ctx, double* total);
/* net_flux, the radiative input of the heating term
   (src/mod_sw_dyn.f90:103-106,461-464); a host (is:ie, js:je, 1:nlay+1)
   array.  NULL restores the default of zero flux (no heating). */
int atm_set_net_flux(atm_ctx* ctx, const double* host);

/* one full model step as run_model orders it (src/mod_model.f90:146-177):
   C-grid half step, halo, D-grid step, remap when do_remap != 0, halo; then
   *stable as atm_check_stability when stable != NULL (no reference
   counterpart as a single call; it is the sequence above). */
int atm_step(atm_ctx* ctx, double dt, int do_remap, int* stable);

int atm_sync(atm_ctx* ctx);
int atm_destroy(atm_ctx* ctx);
const char* atm_last_error(atm_ctx* ctx);

/* ---- device-resident access (the PyTorch binding; no reference counterpart) ----
   Copy a field between the context and a caller-owned device buffer holding
   the interior only: FP64 (for ATM_FP64) or the form's sweep type, shape
   (K, ny, nx) contiguous, i fastest.  Stream-ordered on the context's stream. */
int atm_upload_device(atm_ctx* ctx, int field, const void* dev, int dtype_bytes);
int atm_download_device(atm_ctx* ctx, int field, void* dev, int dtype_bytes);
/* use an external CUDA stream (cudaStream_t passed as void*; NULL = own) */
int atm_set_stream(atm_ctx* ctx, void* stream);

/* ---- validation (no reference counterpart) ----
   When buf != NULL, the next atm_remap also writes the set of contributing
   source layers of every remap_column call into buf, a host int32 array
   [3][ny+2][nx+2][nlay][5]: for variable 0 = u, 1 = v, 2 = energy, each
   column of [isd-1, ied+1]^2 and each destination layer m, {first k, last k,
   case of the first pair, case of the last pair, number of pairs}
   (src/mod_remap.f90:176-283); columns a variable does not remap hold -1.
   *fallback_columns (may be NULL) receives how many columns used the
   reference's all-pairs search because a coordinate was not monotone. */
int atm_remap_trace(atm_ctx* ctx, int32_t* buf, int* fallback_columns);

/* ---- measurement (no reference counterpart) ----
   atm_profile(ctx, 1) starts bracketing every kernel the step entry points
   launch with CUDA events on the context's stream (and clears earlier
   records); atm_profile_read synchronises and returns, per stage, the total
   milliseconds and the number of launches since then.  Stage i is named by
   atm_profile_stage(i) (NULL past the last).  atm_launch_count returns how
   many kernels the context's step entry points have launched. */
int atm_profile(atm_ctx* ctx, int enable);
int atm_profile_read(atm_ctx* ctx, double* ms, int* count, int nstage);
const char* atm_profile_stage(int i);
int atm_launch_count(atm_ctx* ctx, long long* n);

/* the portable x**y and log(x) the FP64 form evaluates on the device, on n
   host values (accuracy and bit-identity tests) */
int atm_device_pow_log(const double* x, double y, double* pow_out, double* log_out, int n);
/* p**kappa (kappa = R_dry / cp_dry) as the mixed form's column and remap
   kernels evaluate it on the device (a table method, within a few ulp), on n
   host values (accuracy tests) */
int atm_device_kappa_pow(const double* x, double* out, int n);

/* ---- vertical remap without allocation (no counterpart in the reference) ----
   perform_vertical_remapping (src/mod_remap.f90:27-163) for callers that
   cannot let the library allocate device memory: a host loop that fixes
   its device-memory budget at start-up, or one that must not meet the
   device-wide synchronisation cudaMalloc/cudaFree can cause mid-step.  It
   needs no context and calls no cudaMalloc, cudaFree or other allocating
   routine: its scratch (the remapped face winds of every column) is one
   file-scope device array of 2^20 doubles (8 MiB) that every GPU loading
   the library holds until the process exits.  Sizes with
   2 (nx+14)(ny+14) nlay + 2 (nlay+1) + 64 > 2^20 (e.g. above 64x64x64 or
   128x128x24) return ATM_ERR_TOO_LARGE.
   Inputs dp, pt, ud, vd and outputs dp_out .. vd_out are caller-owned FP64
   device arrays in the reference's layout (is:ie, js:je, 1:nlay) without
   row padding; gzs is the (is:ie, js:je) surface geopotential on the
   device; ak, bk are host arrays of nlay+1 hybrid coefficients.  Like the
   reference, ud and vd are read one point outside the interior, where they
   still hold the halo of the previous step.  Only the interior of the
   outputs is written; outputs must not alias inputs.  The call is
   asynchronous on stream (a cudaStream_t, NULL = the default stream); its
   result is bit-identical to atm_remap of the FP64 form.  Every call shares
   the one scratch array, so calls that overlap on the GPU (other streams,
   other threads) race and must be serialised by the caller.  The first
   call on a device looks up the array's device address
   (cudaGetSymbolAddress) with that device current; make that first call
   before any stream capture.  The address is kept for the life of the
   process: a cudaDeviceReset unloads the array, and the entry point must
   not be called on that device afterwards.
   stable and fallback_columns (either may be NULL) report what
   atm_check_stability and atm_remap_trace report for atm_remap: when
   either is non-NULL the call waits for the remap to finish on stream,
   stores 1 in *stable when every remapped value is finite (0 otherwise) and
   the number of columns whose coordinates were not monotone (the
   all-pairs search) in *fallback_columns.  When both are NULL the call
   stays asynchronous and reports no non-finite result: the caller checks
   the outputs itself. */
int atm_remap_noalloc(int nx, int ny, int nlay, const double* ak, const double* bk, const double* dp,
                      const double* pt, const double* ud, const double* vd, const double* gzs,
                      double* dp_out, double* pt_out, double* ud_out, double* vd_out, void* stream,
                      int* stable, int* fallback_columns);

/* ---- persistent ensemble (config 5; no counterpart in the reference) ----
   Many independent domains of the mixed form (members of uneven sizes, each
   a context made by atm_create/atm_init) advanced together by ONE
   cooperative launch of a persistent kernel: every stage of a step is a
   work queue of warp-sized items over all members, and the stages are
   separated by grid-wide barriers whose waits are bounded (about two
   seconds; a wait that runs out raises the status word read by
   atm_ensemble_status and ends the launch).  Members hold at most 64
   layers, use no net flux, live on the current device; dts gives each
   member's time step.  A member's results are bit-identical to stepping it
   alone with atm_step.
   atm_ensemble_prepare copies the members' descriptors (their current time
   levels and strip heights) to the device; call it after changing a
   member outside the ensemble and before stream capture.
   atm_ensemble_run enqueues one launch of nsteps steps on the ensemble's
   stream (the first member's unless set), the remap after every
   remap_every-th step counted from the launch (0: none); successive launches
   after one prepare must each swap the time levels an even number of times
   (nsteps + nsteps / remap_every even), so that a captured launch can be
   replayed.  atm_ensemble_set_strips sets a member's strip height of the
   marching sweeps (16, 32 or 64 rows; default 32).
   atm_ensemble_barrier_check launches the barrier schedule with no members and a
   barrier that waits for one block more than the grid holds: *timed_out
   reports that the bounded wait ran out and the launch ended. */
typedef struct atm_ens atm_ens;
int atm_ensemble_create(atm_ens** out, atm_ctx* const* members, const double* dts, int n);
int atm_ensemble_set_strips(atm_ens* e, int member, int rows);
int atm_ensemble_set_stream(atm_ens* e, void* stream);
int atm_ensemble_prepare(atm_ens* e);
int atm_ensemble_run(atm_ens* e, int nsteps, int remap_every);
int atm_ensemble_status(atm_ens* e, int* barrier_timed_out);
int atm_ensemble_blocks(atm_ens* e, int* blocks);
/* atm_ensemble_profile(e, 1) zeroes and enables per-stage timing of the
   following launches (block 0 reads the global timer at every barrier exit;
   0 disables it); atm_ensemble_stage_ms writes, for each of the 13 stages in
   step order (C mass, C column, C momentum, C halo, D ring copy, D mass,
   D column, corners, D momentum, remap ring copy, wind remap, energy remap,
   D halo), the milliseconds between the exit of the barrier before it and
   its own, summed over the timed launches (n >= 13). */
int atm_ensemble_profile(atm_ens* e, int enable);
/* The schedule of the following launches: 0 (default) every stage of every
   member, then a grid barrier; 1 dataflow -- no grid barrier: each member
   advances through its stages on its own, a warp claiming the next item of
   any member whose current stage has items left (an atomic ticket per
   member), so the stages of different members overlap; an idle wait longer
   than the limit raises the status word.  Profiled launches
   (atm_ensemble_profile) use the barriers. */
int atm_ensemble_set_schedule(atm_ens* e, int dataflow);
int atm_ensemble_stage_ms(atm_ens* e, double* ms, int n);
int atm_ensemble_destroy(atm_ens* e);
int atm_ensemble_barrier_check(long long timeout_ns, int* timed_out);

/* the number of the n pseudo-random FP64 arguments (all exponents, plus
   integers) for which the FP64 form's FMA-corrected division by the
   constants 3 and 12 differs from IEEE division (expected: 0) */
int atm_device_div_check(long long n, long long seed, long long* mismatches);
/* failure-detection check of the tile kernels' bounded wait: a kernel arms
   an mbarrier for transactions that never arrive (no copy is issued) and
   waits with the poll limit the TMA loads use, here max_polls polls of at
   most ~1 us (1..100000); *timed_out = 1 when the wait gave up and the
   kernel returned, as a tile kernel then does (it records
   Status.tma_timeout, which atm_check_stability reports as an error). */
int atm_device_wait_check(int max_polls, int* timed_out);

/* ---- adjoint of the FP64 step (the gradient work; no reference counterpart) ----
   Hand-written reverse mode of cgrid_dynamics_step, dgrid_dynamics_step
   (src/mod_sw_dyn.f90:80-773), perform_vertical_remapping
   (src/mod_remap.f90:27-356) and the halo exchanges (src/mod_sync.f90:67-217)
   with every limiter, upwind and remap-overlap branch frozen at the forward
   trajectory (the forward is recomputed bit for bit inside the adjoint).
   Adjoints are FP64 fields shaped like the state, in two slots:
   ATM_ADJ_OUT holds the adjoint of the state after a step and
   ATM_ADJ_IN receives the adjoint of the state before it.  FP64 contexts
   only, with the heating term off (net_flux unset). */
enum { ATM_ADJ_IN = 0, ATM_ADJ_OUT = 1 };
/* allocate (or clear) the adjoint fields */
int atm_adj_enable(atm_ctx* ctx);
int atm_adj_zero(atm_ctx* ctx);
/* adjoint field of a slot (ATM_DP..ATM_VD) or a C-grid adjoint
   (ATM_DPC..ATM_VC, slot ignored) from / to a host (is:ie, js:je, 1:nlay)
   array, halo included */
int atm_adj_set(atm_ctx* ctx, int slot, int field, const double* host);
int atm_adj_get(atm_ctx* ctx, int slot, int field, double* host);
/* the same for device (nlay, ny, nx) interiors; set clears the halo */
int atm_adj_set_device(atm_ctx* ctx, int slot, int field, const double* dev);
int atm_adj_get_device(atm_ctx* ctx, int slot, int field, double* dev);
/* one step reversed: on entry slot OUT is the adjoint of the state after
   atm_step(ctx, dt, do_remap) taken from the context's current state; on
   return slot OUT is the adjoint of the current state (its halo still
   holds the ring's share: atm_adj_halo folds it).  The state is not
   advanced; the other time level and the C-grid fields are overwritten. */
int atm_adj_step(atm_ctx* ctx, double dt, int do_remap);
/* the same with the step's forward products recorded by atm_step_tape
   instead of recomputed: atm_step_tape advances the state like atm_step
   and writes the state before the step, the C-grid fields (after their
   halo), the pre-remap state and the D step's corner pkap and gz into a
   device buffer of atm_tape_bytes bytes; atm_adj_step_tape reverses that
   step from the tape alone (the context's state is neither read nor
   changed) */
int atm_tape_bytes(atm_ctx* ctx, long long* bytes);
int atm_step_tape(atm_ctx* ctx, double dt, int do_remap, void* tape);
int atm_adj_step_tape(atm_ctx* ctx, double dt, int do_remap, const void* tape);
/* adjoint of a periodic halo fill: each ring adjoint added to its interior
   image and cleared (slot ATM_ADJ_IN or ATM_ADJ_OUT; C-grid adjoints) */
int atm_adj_halo(atm_ctx* ctx, int slot);
int atm_adj_cgrid_halo(atm_ctx* ctx);
/* single stages at the current state: slot IN += C^T (C-grid adjoints);
   slot IN, C-grid += D^T slot OUT (after the call's own C step and halo;
   slot OUT is consumed); slot IN += R^T slot OUT */
int atm_adj_cgrid_step(atm_ctx* ctx, double dt_half);
int atm_adj_dgrid_step(atm_ctx* ctx, double dt);
int atm_adj_remap(atm_ctx* ctx);
/* checkpoints: the whole prognostic state (both halos) to / from a device
   buffer of atm_state_bytes bytes */
int atm_state_bytes(atm_ctx* ctx, long long* bytes);
int atm_state_save(atm_ctx* ctx, void* dev);
int atm_state_load(atm_ctx* ctx, const void* dev);

/* ---- column physics (src/mod_physics.f90), FP64 in both forms ----
   atm_physics_tendencies: calculate_physics_tendencies (:27-79): A-grid
   winds, plev / pkap / gz / playkap of the current state, the dry
   convective adjustment (:81-176) on [isd-2, ied+2]^2 and the surface
   heating from level 1 of the net flux set by atm_set_net_flux (zero when
   none is set, :178-185).  The tendencies stay on the device until the next
   call.  Called where run_model calls it: at the start of a step when the
   physics is due (src/mod_model.f90:138-143).
   atm_apply_physics(dt): apply_physics_tendencies (:187-211) to the
   interior of dp, pt, ts, ud, vd, after the D-grid step of every step
   (src/mod_model.f90:153-155); ATM_ERR_STATE before the first tendencies.
   atm_physics_halo: physics_halo_exchange (:213-217), the periodic halo
   of ts, after atm_dgrid_halo (src/mod_model.f90:165-166). */
int atm_physics_tendencies(atm_ctx* ctx);
int atm_apply_physics(atm_ctx* ctx, double dt);
int atm_physics_halo(atm_ctx* ctx);

/* ---- radiation (src/mod_radiation.f90, src/mod_gas_optics.f90,
   src/mod_solar.f90), FP64 in both forms ----
   The correlated-k tables, which the reference compiles in as parameter
   arrays, are an input: arrays in the reference's index order flattened
   from the last Fortran index (temperatures[p][t] is temperatures(t, p) of
   mod_gas_optics.f90:50-132, sw_absorption[g][p][t] is
   shortwave_absorption_lut(t, p, g) of :143-1841, lw_absorption likewise of
   :1870-3568, planck[g][t] is planckian_lut(t, g) of :3623-4549;
   sw_scattering is rayleigh_scattering_lut (:1852-1857), irradiance_fraction
   that of mod_solar.f90:16-23).  atm_set_gas_optics copies them to the
   device (strictly ascending axes required). */
typedef struct {
  int n_g, n_p, n_t, n_planck;        /* 16, 53, 6, 231 in the reference; n_t <= 255 */
  const double* pressures;            /* [n_p], Pa */
  const double* temperatures;         /* [n_p][n_t], K */
  const double* sw_absorption;        /* [n_g][n_p][n_t], m2/kg */
  const double* sw_scattering;        /* [n_g], m2/kg */
  const double* lw_absorption;        /* [n_g][n_p][n_t], m2/kg */
  const double* planck_temperatures;  /* [n_planck], K */
  const double* planck;               /* [n_g][n_planck] */
  const double* irradiance_fraction;  /* [n_g] */
} atm_gas_optics;

/* the reference's fixed radiation parameters (mod_radiation.f90:107-109;
   .3 and .99 are default-real literals) */
#define ATM_SOLAR_ZENITH_ANGLE 0.0
#define ATM_SURFACE_ALBEDO ((double)0.3f)
#define ATM_SURFACE_EMISSIVITY ((double)0.99f)

int atm_set_gas_optics(atm_ctx* ctx, const atm_gas_optics* tables);
/* the cell-centre axes xc[nx], yc[ny] of the initial file; the solar
   irradiance of a column depends on radius = sqrt(xc^2 + yc^2)
   (src/mod_input.f90:233-243, src/mod_solar.f90:26-35) */
int atm_set_cell_coordinates(atm_ctx* ctx, const double* xc, const double* yc);
/* calculate_radiative_heating(time) (src/mod_radiation.f90:41-156): net_flux
   on the interior from the current dp, pt and ts: layer pressures and
   temperatures, then per g-point a shortwave and a longwave two-stream
   solution closed by the adding method.  The heating term and the surface
   heating use it from then on (as after atm_set_net_flux).  Called where
   run_model calls it: at the start of a step when radiation is due
   (src/mod_model.f90:117-127).  Synchronises the stream; ATM_ERR_RANGE when
   a layer pressure or temperature lies outside the tables (where the
   reference stops).
   atm_radiation_halo: radiation_halo_exchange (:400-404), the periodic halo
   of net_flux. */
int atm_radiative_heating(atm_ctx* ctx, double time, double solar_zenith_angle, double surface_albedo,
                          double surface_emissivity);
int atm_radiation_halo(atm_ctx* ctx);

/* ---- output accumulation on the device (accumulate_output / write_output,
   src/mod_output.f90:94-176) ----
   atm_accumulate_output(ctx, dt) adds dt * (dp, pt, u, v, net_flux, ts) of
   the current state to device sums, with u, v the cell-centre averages of
   the D-grid winds, exactly as the reference (whose compensated sum keeps
   no compensation: plain FP64 adds); atm_output_read returns one mean (sum /
   accumulated time) as a host (nlay, nlay+1 or 1, ny, nx) array, field
   ATM_OUT_DP..ATM_OUT_TS; atm_output_reset starts a new interval. */
enum { ATM_OUT_DP = 0, ATM_OUT_PT = 1, ATM_OUT_U = 2, ATM_OUT_V = 3, ATM_OUT_NFLX = 4, ATM_OUT_TS = 5 };
int atm_output_enable(atm_ctx* ctx);
int atm_output_reset(atm_ctx* ctx);
int atm_accumulate_output(atm_ctx* ctx, double dt);
int atm_output_read(atm_ctx* ctx, int which, double* host);
int atm_output_time(atm_ctx* ctx, double* t);

/* library version string */
const char* atm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ATMDYN_H */
