// Launch wrappers of one form of the dynamical core (T = sweep type).
// Included once by atm_fp64.cu (T = double) and once by atm_mixed.cu
// (T = float), which each define ATM_FORM_T and ATM_OPS_NAME.
#pragma once

#include "atm_kernels.cuh"
#include "atm_march.cuh"
#include "atm_ops.h"
#include "atm_remap_warp.cuh"

namespace atm {
namespace {

using T = ATM_FORM_T;  // sweep arithmetic
using S = double;      // prognostic state (dp, pt, ud, vd), both forms
using C = T;           // C-grid fields (dpc, ptc, uc, vc)
constexpr bool FP64_FORM = std::is_same_v<T, double>;
// Strip height (output rows a warp walks through) of each column-marching
// sweep: 6 warm-up rows per strip are recomputed halo, more strips per
// layer fill the GPU.
constexpr int TYS_MASS = 64;
constexpr int TYS_CMOM = 64;
constexpr int TYS_DMOM = 64;

inline dim3 strips(int lo, int hi, const Geom& g, int tys) {
  int w = g.nx - lo + hi, h = g.ny - lo + hi;
  return dim3((w + MOUT * MWARPS - 1) / (MOUT * MWARPS), (h + tys - 1) / tys, g.L);
}

// the column-marching sweeps need no shared memory: nothing to set up
cudaError_t setup() { return cudaSuccess; }

cudaError_t mass(const Geom& g, const Consts& c, const void* dp, const void* pt, const void* u, const void* v,
                 const double* heat, void* dpo, void* pto, int lo, int hi, int* nonfinite, int* timeout, bool cgrid,
                 cudaStream_t s) {
  (void)timeout;
  const dim3 grid = strips(lo, hi, g, TYS_MASS);
  if (cgrid)  // state in, C-grid fields out
    k_mass_m<T, TYS_MASS, true, S, C><<<grid, MW * MWARPS, 0, s>>>(g, c, (const S*)dp, (const S*)pt, (const S*)u,
                                                                    (const S*)v, heat, (C*)dpo, (C*)pto, lo, hi,
                                                                    nonfinite);
  else  // state and C-grid winds in, state out
    k_mass_m<T, TYS_MASS, false, S, C><<<grid, MW * MWARPS, 0, s>>>(g, c, (const S*)dp, (const S*)pt, (const C*)u,
                                                                     (const C*)v, heat, (S*)dpo, (S*)pto, lo, hi,
                                                                     nonfinite);
  return cudaGetLastError();
}

cudaError_t column(const Geom& g, const Consts& c, const void* dpl, const void* ptl, int es, double* pkap, double* gz,
                   int lo, int hi, double* plev, cudaStream_t s) {
  int n = (g.nx - lo + hi) * (g.ny - lo + hi);
  if (es == 8)
    k_column<double><<<(n + 127) / 128, 128, 0, s>>>(g, c, (const double*)dpl, (const double*)ptl, pkap, gz, lo, hi,
                                                     plev);
  else
    k_column<float><<<(n + 127) / 128, 128, 0, s>>>(g, c, (const float*)dpl, (const float*)ptl, pkap, gz, lo, hi,
                                                    plev);
  return cudaGetLastError();
}

cudaError_t heating(const Geom& g, const Consts& c, const void* dpl, int es, const double* nf, double* heat,
                    cudaStream_t s) {
  int n = (g.nx + 2 * H) * g.NYP;
  if (es == 8) k_heating<double><<<(n + 63) / 64, 64, 0, s>>>(g, c, (const double*)dpl, nf, heat);
  else k_heating<float><<<(n + 63) / 64, 64, 0, s>>>(g, c, (const float*)dpl, nf, heat);
  return cudaGetLastError();
}

cudaError_t c_mom(const Geom& g, const Consts& c, const void* ud, const void* vd, const double* pkap, const double* gz,
                  void* uc, void* vc, int* timeout, cudaStream_t s) {
  (void)timeout;
  k_c_mom_m<T, TYS_CMOM, S, C><<<strips(0, 0, g, TYS_CMOM), MW * MWARPS, 0, s>>>(g, c, (const S*)ud, (const S*)vd,
                                                                                pkap, gz, (C*)uc, (C*)vc);
  return cudaGetLastError();
}

cudaError_t d_mom(const Geom& g, const Consts& c, const void* ud, const void* vd, const void* uc, const void* vc,
                  const double* pkapb, const double* gzb, void* udo, void* vdo, int* nonfinite, int* timeout,
                  cudaStream_t s) {
  (void)timeout;
  k_d_mom_m<T, TYS_DMOM, S, C><<<strips(0, 0, g, TYS_DMOM), MW * MWARPS, 0, s>>>(
      g, c, (const S*)ud, (const S*)vd, (const C*)uc, (const C*)vc, pkapb, gzb, (S*)udo, (S*)vdo, nonfinite);
  return cudaGetLastError();
}

template <typename E>
cudaError_t ring_t(const Geom& g, void* const* f, const void* const* src, int nf, int K, bool copy, cudaStream_t s) {
  int nring = 2 * H * (g.nx + 2 * H) + 2 * H * g.ny;
  dim3 grid((nring + 255) / 256, K, nf);
  E* d[4] = {nullptr, nullptr, nullptr, nullptr};
  const E* q[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int i = 0; i < nf; ++i) {
    d[i] = (E*)f[i];
    if (src) q[i] = (const E*)src[i];
  }
  if (copy)
    k_ring<E, true><<<grid, 256, 0, s>>>(g, d[0], d[1], d[2], d[3], q[0], q[1], q[2], q[3], K);
  else
    k_ring<E, false><<<grid, 256, 0, s>>>(g, d[0], d[1], d[2], d[3], q[0], q[1], q[2], q[3], K);
  return cudaGetLastError();
}

// halo passes of the state fields and of the C-grid fields
cudaError_t ring(const Geom& g, void* const* f, const void* const* src, int nf, int K, bool copy, cudaStream_t s) {
  return ring_t<S>(g, f, src, nf, K, copy, s);
}
cudaError_t ring_cg(const Geom& g, void* const* f, const void* const* src, int nf, int K, bool copy, cudaStream_t s) {
  return ring_t<C>(g, f, src, nf, K, copy, s);
}

template <int LM>
cudaError_t remap_winds_lm(const Geom& g, const RemapArgs& ra, const void* dp, const void* ud, const void* vd,
                           void* urem, void* vrem, int* trace, Status* st, cudaStream_t s) {
  int n = (g.nx + 2) * (g.ny + 2);
  k_remap_winds<S, LM><<<dim3((n + 63) / 64, 2), 64, 0, s>>>(g, ra, (const S*)dp, (const S*)ud, (const S*)vd, (S*)urem,
                                                    (S*)vrem, trace, st);
  return cudaGetLastError();
}
template <int LM>
cudaError_t remap_energy_lm(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                            const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo,
                            void* pto, void* udo, void* vdo, int* trace, Status* st, cudaStream_t s) {
  int n = g.nx * g.ny;
  k_remap_energy<S, LM><<<(n + 63) / 64, 64, 0, s>>>(g, ra, (const S*)dp, (const S*)pt, (const S*)ud, (const S*)vd,
                                                     (const S*)urem, (const S*)vrem, gzs, (S*)dpo, (S*)pto, (S*)udo,
                                                     (S*)vdo, trace, st);
  return cudaGetLastError();
}

// The mixed form remaps with the warp-cooperative kernels (its sums in a
// different association); the FP64 form, and any remap whose pair trace is
// requested, with the sequential ones.
template <int LPL>
cudaError_t remap_winds_wl(const Geom& g, const RemapArgs& ra, const void* dp, const void* ud, const void* vd,
                           void* urem, void* vrem, Status* st, cudaStream_t s) {
  const long long warps = 2LL * (g.nx + 2) * (g.ny + 2);
  k_remap_winds_w<LPL><<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(g, ra, (const double*)dp, (const double*)ud,
                                                                    (const double*)vd, (double*)urem, (double*)vrem, st);
  return cudaGetLastError();
}
template <int LPL>
cudaError_t remap_energy_wl(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                            const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo,
                            void* pto, void* udo, void* vdo, Status* st, cudaStream_t s) {
  const long long warps = (long long)g.nx * g.ny;
  k_remap_energy_w<LPL><<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(
      g, ra, (const double*)dp, (const double*)pt, (const double*)ud, (const double*)vd, (const double*)urem,
      (const double*)vrem, gzs, (double*)dpo, (double*)pto, (double*)udo, (double*)vdo, st);
  return cudaGetLastError();
}

cudaError_t remap_winds(const Geom& g, const RemapArgs& ra, const void* dp, const void* ud, const void* vd, void* urem,
                        void* vrem, int* trace, Status* st, cudaStream_t s) {
  if (!FP64_FORM && !trace) {
    if (g.L <= 32) return remap_winds_wl<1>(g, ra, dp, ud, vd, urem, vrem, st, s);
    if (g.L <= 64) return remap_winds_wl<2>(g, ra, dp, ud, vd, urem, vrem, st, s);
    return remap_winds_wl<4>(g, ra, dp, ud, vd, urem, vrem, st, s);
  }
  if (g.L <= 32) return remap_winds_lm<32>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
  if (g.L <= 64) return remap_winds_lm<64>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
  return remap_winds_lm<MAX_LAYERS>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
}

cudaError_t remap_energy(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                         const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo, void* pto,
                         void* udo, void* vdo, int* trace, Status* st, cudaStream_t s) {
  if (!FP64_FORM && !trace) {
    if (g.L <= 32) return remap_energy_wl<1>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, st, s);
    if (g.L <= 64) return remap_energy_wl<2>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, st, s);
    return remap_energy_wl<4>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, st, s);
  }
  if (g.L <= 32) return remap_energy_lm<32>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
  if (g.L <= 64) return remap_energy_lm<64>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
  return remap_energy_lm<MAX_LAYERS>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
}

cudaError_t check_finite(const Geom& g, const void* const* f, int* flag, cudaStream_t s) {
  k_check_finite<S><<<296, 256, 0, s>>>(g, (const S*)f[0], (const S*)f[1], (const S*)f[2], (const S*)f[3], flag);
  return cudaGetLastError();
}

cudaError_t mass_sum(const Geom& g, const void* dp, double* partial, int nblocks, double* out, cudaStream_t s) {
  k_mass_partial<S><<<nblocks, 256, 0, s>>>(g, (const S*)dp, partial);
  k_mass_final<<<1, 32, 0, s>>>(partial, nblocks, out);
  return cudaGetLastError();
}

cudaError_t to_double(const void* src, double* dst, long long n, cudaStream_t s) {
  k_convert<T, double><<<1184, 256, 0, s>>>((const T*)src, dst, n);
  return cudaGetLastError();
}
cudaError_t from_double(const double* src, void* dst, long long n, cudaStream_t s) {
  k_convert<double, T><<<1184, 256, 0, s>>>(src, (T*)dst, n);
  return cudaGetLastError();
}

}  // namespace

const Ops ATM_OPS_NAME = {(int)sizeof(S), (int)sizeof(C), setup,        mass,       column,
                          heating,        c_mom,          d_mom,        ring,       ring_cg,
                          remap_winds,    remap_energy,   check_finite, mass_sum,   to_double,
                          from_double};

}  // namespace atm
