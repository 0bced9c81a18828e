// Precision-independent table of the device operations of one form of the
// dynamical core.  atm_fp64.cu fills it for the FP64 form (compiled without
// fused multiply-add so that it matches the FP64 restatement bit for bit),
// atm_mixed.cu for the FP32-sweep form.  Buffers are passed as void* and
// hold the form's sweep type; pressure, pkap and geopotential are double.
#pragma once

#include <cuda_runtime.h>
#include "atm_common.cuh"

namespace atm {

struct Ops {
  int elem;     // bytes of an element of the prognostic state (dp, pt, ud, vd)
  int cg_elem;  // bytes of an element of the C-grid fields (dpc, ptc, uc, vc)
  cudaError_t (*setup)();
  // C- or D-grid mass/potential-temperature sweep of every layer
  cudaError_t (*mass)(const Geom&, const Consts&, const void* dp, const void* pt, const void* u, const void* v,
                      const double* heat, void* dpo, void* pto, int lo, int hi, int* nonfinite, int* timeout,
                      bool cgrid, cudaStream_t);
  // plev/pkap/gz columns over [lo, n-1+hi]^2 from dp, pt of element size es
  cudaError_t (*column)(const Geom&, const Consts&, const void* dpl, const void* ptl, int es, double* pkap,
                        double* gz, int lo, int hi, double* plev, cudaStream_t);
  cudaError_t (*heating)(const Geom&, const Consts&, const void* dpl, int es, const double* net_flux, double* heat,
                         cudaStream_t);
  cudaError_t (*c_mom)(const Geom&, const Consts&, const void* ud, const void* vd, const double* pkap,
                       const double* gz, void* uc, void* vc, int* timeout, cudaStream_t);
  cudaError_t (*d_mom)(const Geom&, const Consts&, const void* ud, const void* vd, const void* uc, const void* vc,
                       const double* pkapb, const double* gzb, void* udo, void* vdo, int* nonfinite, int* timeout,
                       cudaStream_t);
  // periodic halo fill (copy = false) or ring copy src -> f (copy = true) of
  // nf state fields (ring) or C-grid fields (ring_cg)
  cudaError_t (*ring)(const Geom&, void* const* f, const void* const* src, int nf, int K, bool copy, cudaStream_t);
  cudaError_t (*ring_cg)(const Geom&, void* const* f, const void* const* src, int nf, int K, bool copy,
                         cudaStream_t);
  cudaError_t (*remap_winds)(const Geom&, const RemapArgs&, const void* dp, const void* ud, const void* vd,
                             void* urem, void* vrem, int* trace, Status*, cudaStream_t);
  cudaError_t (*remap_energy)(const Geom&, const RemapArgs&, const void* dp, const void* pt, const void* ud,
                              const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo,
                              void* pto, void* udo, void* vdo, int* trace, Status*, cudaStream_t);
  cudaError_t (*check_finite)(const Geom&, const void* const* f, int* flag, cudaStream_t);
  cudaError_t (*mass_sum)(const Geom&, const void* dp, double* partial, int nblocks, double* out, cudaStream_t);
  // C-grid-type <-> double conversion of whole padded fields
  cudaError_t (*to_double)(const void* src, double* dst, long long n, cudaStream_t);
  cudaError_t (*from_double)(const double* src, void* dst, long long n, cudaStream_t);
};

extern const Ops ops_fp64;
extern const Ops ops_mixed;

// interpolate_to_corners of pkap/gz (double in both forms)
cudaError_t corners(const Geom&, const double* pkap, const double* gz, double* pkapb, double* gzb, int with_pkap,
                    int lev0, int nlev, cudaStream_t);

// x**y and log(x) of the portable math on the device (tests)
cudaError_t device_pow_log(const double* x, double y, double* p, double* l, int n, cudaStream_t);
// p**kappa as the mixed form evaluates it (atm_mixed.cu)
cudaError_t device_kappa_pow(const double* x, double* out, int n, cudaStream_t);

// count of arguments where div_const<3>/<12> differs from IEEE division (tests)
cudaError_t device_div_check(unsigned long long n, unsigned long long seed, unsigned long long* bad, cudaStream_t);
// the TMA loads' bounded mbarrier wait on a barrier nothing completes: *flag = 1 when it gave up
cudaError_t device_wait_timeout(int max_polls, int* flag, cudaStream_t);

// ---- FP64 adjoint (atm_adjoint.cu); lam_* are adjoint fields laid out like
// the fields they belong to, accumulated with +=
cudaError_t adj_setup();
// dpo, pto: the new dp and pt the forward sweep wrote; parts (D grid): 1
// the x branch, 2 the y branch, 3 both (the C grid is one kernel)
cudaError_t adj_mass(const Geom&, const Consts&, const double* dp, const double* pt, const double* u, const double* v,
                     const double* dpo, const double* pto, const double* lam_dpo, const double* lam_pto, double* lam_dp,
                     double* lam_pt, double* lam_u, double* lam_v, int lo, int hi, int* timeout, bool cgrid,
                     cudaStream_t, int parts = 3);
cudaError_t adj_c_mom(const Geom&, const Consts&, const double* ud, const double* vd, const double* pkap,
                      const double* gz, const double* lam_uc, const double* lam_vc, double* lam_ud, double* lam_vd,
                      double* lam_pk, double* lam_gz, int* timeout, cudaStream_t);
// parts: 1 the kinetic-energy chain, 2 the rest, 3 both
cudaError_t adj_d_mom(const Geom&, const Consts&, const double* ud, const double* vd, const double* uc,
                      const double* vc, const double* pkapb, const double* gzb, const double* lam_udo,
                      const double* lam_vdo, double* lam_ud, double* lam_vd, double* lam_uc, double* lam_vc,
                      double* lam_pkb, double* lam_gzb, int* timeout, cudaStream_t, int parts = 3);
cudaError_t adj_column(const Geom&, const Consts&, const double* dp, const double* pt, const double* lam_pk,
                       const double* lam_gz, double* lam_dp, double* lam_pt, int lo, int hi, cudaStream_t);
cudaError_t adj_corners(const Geom&, const double* lam_pkb, const double* lam_gzb, double* lam_pk, double* lam_gz,
                        cudaStream_t);
cudaError_t adj_ring_fold(const Geom&, double* const* f, int nf, int K, cudaStream_t);
cudaError_t adj_ring_copy(const Geom&, double* const* dst, double* const* src, int K, int band01, int band23,
                          cudaStream_t);
cudaError_t adj_remap_energy(const Geom&, const RemapArgs&, const double* dp, const double* pt, const double* ud,
                             const double* vd, const double* urem, const double* vrem, const double* gzs,
                             const double* lam_dpo, const double* lam_pto, const double* lam_udo,
                             const double* lam_vdo, double* lam_dp, double* lam_pt, double* lam_ud, double* lam_vd,
                             double* lam_ur, double* lam_vr, cudaStream_t);
cudaError_t adj_remap_winds(const Geom&, const RemapArgs&, const double* dp, const double* ud, const double* vd,
                            const double* lam_ur, const double* lam_vr, double* lam_dp, double* lam_ud, double* lam_vd,
                            cudaStream_t);

// the persistent ensemble kernel of the mixed form (atm_ensemble.cuh): its
// largest cooperative grid on the current device, and one launch of a plan
struct EnsPlan;
int ensemble_max_blocks();
cudaError_t ensemble_launch(const EnsPlan& plan, int blocks, cudaStream_t);

// largest number of layers the vertical remap supports
constexpr int MAX_LAYERS = 128;

}  // namespace atm
