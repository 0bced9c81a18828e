// Launch wrappers of one form of the dynamical core (T = sweep type).
// Included once by atm_fp64.cu (T = double) and once by atm_mixed.cu
// (T = float), which each define ATM_FORM_T and ATM_OPS_NAME.
#pragma once

#include "atm_kernels.cuh"
#include "atm_ops.h"

namespace atm {
namespace {

using T = ATM_FORM_T;
constexpr int TX = 32, TY = 8;

inline dim3 tiles(int lo, int hi, const Geom& g, int layers) {
  int w = g.nx - lo + hi, h = g.ny - lo + hi;
  return dim3((w + TX - 1) / TX, (h + TY - 1) / TY, layers);
}

cudaError_t setup() {
  cudaError_t e;
  e = cudaFuncSetAttribute(k_mass<T, TX, TY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MassSmem<T, TX, TY>::bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_mass<T, TX, TY, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MassSmem<T, TX, TY>::bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_c_mom<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CMomSmem<T, TX, TY>::bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_d_mom<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DMomSmem<T, TX, TY>::bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_column<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (MAX_LAYERS + 1) * 64 * 8);
}

cudaError_t mass(const Geom& g, const Consts& c, const void* dp, const void* pt, const void* u, const void* v,
                 const double* heat, void* dpo, void* pto, int lo, int hi, int* nonfinite, bool cgrid, cudaStream_t s) {
  dim3 grid = tiles(lo, hi, g, g.L);
  if (cgrid)
    k_mass<T, TX, TY, true><<<grid, NT, MassSmem<T, TX, TY>::bytes, s>>>(
        g, c, (const T*)dp, (const T*)pt, (const T*)u, (const T*)v, heat, (T*)dpo, (T*)pto, lo, hi, nonfinite);
  else
    k_mass<T, TX, TY, false><<<grid, NT, MassSmem<T, TX, TY>::bytes, s>>>(
        g, c, (const T*)dp, (const T*)pt, (const T*)u, (const T*)v, heat, (T*)dpo, (T*)pto, lo, hi, nonfinite);
  return cudaGetLastError();
}

cudaError_t column(const Geom& g, const Consts& c, const void* dpl, const void* ptl, double* pkap, double* gz, int lo,
                   int hi, double* plev, cudaStream_t s) {
  int n = (g.nx - lo + hi) * (g.ny - lo + hi);
  k_column<T><<<(n + 63) / 64, 64, (size_t)(g.L + 1) * 64 * 8, s>>>(g, c, (const T*)dpl, (const T*)ptl, pkap, gz, lo, hi,
                                                                     plev);
  return cudaGetLastError();
}

cudaError_t heating(const Geom& g, const Consts& c, const void* dpl, const double* nf, double* heat, cudaStream_t s) {
  int n = (g.nx + 2 * H) * g.NYP;
  k_heating<T><<<(n + 63) / 64, 64, 0, s>>>(g, c, (const T*)dpl, nf, heat);
  return cudaGetLastError();
}

cudaError_t c_mom(const Geom& g, const Consts& c, const void* ud, const void* vd, const double* pkap, const double* gz,
                  void* uc, void* vc, cudaStream_t s) {
  k_c_mom<T, TX, TY><<<tiles(0, 0, g, g.L), NT, CMomSmem<T, TX, TY>::bytes, s>>>(g, c, (const T*)ud, (const T*)vd, pkap,
                                                                                gz, (T*)uc, (T*)vc);
  return cudaGetLastError();
}

cudaError_t d_mom(const Geom& g, const Consts& c, const void* ud, const void* vd, const void* uc, const void* vc,
                  const double* pkapb, const double* gzb, void* udo, void* vdo, int* nonfinite, cudaStream_t s) {
  k_d_mom<T, TX, TY><<<tiles(0, 0, g, g.L), NT, DMomSmem<T, TX, TY>::bytes, s>>>(
      g, c, (const T*)ud, (const T*)vd, (const T*)uc, (const T*)vc, pkapb, gzb, (T*)udo, (T*)vdo, nonfinite);
  return cudaGetLastError();
}

cudaError_t ring(const Geom& g, void* const* f, const void* const* src, int nf, int K, bool copy, cudaStream_t s) {
  int nring = 2 * H * (g.nx + 2 * H) + 2 * H * g.ny;
  dim3 grid((nring + 255) / 256, K, nf);
  T* d[4] = {nullptr, nullptr, nullptr, nullptr};
  const T* q[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int i = 0; i < nf; ++i) {
    d[i] = (T*)f[i];
    if (src) q[i] = (const T*)src[i];
  }
  if (copy)
    k_ring<T, true><<<grid, 256, 0, s>>>(g, d[0], d[1], d[2], d[3], q[0], q[1], q[2], q[3], K);
  else
    k_ring<T, false><<<grid, 256, 0, s>>>(g, d[0], d[1], d[2], d[3], q[0], q[1], q[2], q[3], K);
  return cudaGetLastError();
}

template <int LM>
cudaError_t remap_winds_lm(const Geom& g, const RemapArgs& ra, const void* dp, const void* ud, const void* vd,
                           void* urem, void* vrem, int* trace, Status* st, cudaStream_t s) {
  int n = (g.nx + 2) * (g.ny + 2);
  k_remap_winds<T, LM><<<(n + 63) / 64, 64, 0, s>>>(g, ra, (const T*)dp, (const T*)ud, (const T*)vd, (T*)urem,
                                                    (T*)vrem, trace, st);
  return cudaGetLastError();
}
template <int LM>
cudaError_t remap_energy_lm(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                            const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo,
                            void* pto, void* udo, void* vdo, int* trace, Status* st, cudaStream_t s) {
  int n = g.nx * g.ny;
  k_remap_energy<T, LM><<<(n + 63) / 64, 64, 0, s>>>(g, ra, (const T*)dp, (const T*)pt, (const T*)ud, (const T*)vd,
                                                     (const T*)urem, (const T*)vrem, gzs, (T*)dpo, (T*)pto, (T*)udo,
                                                     (T*)vdo, trace, st);
  return cudaGetLastError();
}

cudaError_t remap_winds(const Geom& g, const RemapArgs& ra, const void* dp, const void* ud, const void* vd, void* urem,
                        void* vrem, int* trace, Status* st, cudaStream_t s) {
  if (g.L <= 32) return remap_winds_lm<32>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
  if (g.L <= 64) return remap_winds_lm<64>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
  return remap_winds_lm<MAX_LAYERS>(g, ra, dp, ud, vd, urem, vrem, trace, st, s);
}

cudaError_t remap_energy(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                         const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo, void* pto,
                         void* udo, void* vdo, int* trace, Status* st, cudaStream_t s) {
  if (g.L <= 32) return remap_energy_lm<32>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
  if (g.L <= 64) return remap_energy_lm<64>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
  return remap_energy_lm<MAX_LAYERS>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto, udo, vdo, trace, st, s);
}

cudaError_t check_finite(const Geom& g, const void* const* f, int* flag, cudaStream_t s) {
  k_check_finite<T><<<296, 256, 0, s>>>(g, (const T*)f[0], (const T*)f[1], (const T*)f[2], (const T*)f[3], flag);
  return cudaGetLastError();
}

cudaError_t mass_sum(const Geom& g, const void* dp, double* partial, int nblocks, double* out, cudaStream_t s) {
  k_mass_partial<T><<<nblocks, 256, 0, s>>>(g, (const T*)dp, partial);
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

const Ops ATM_OPS_NAME = {(int)sizeof(T), setup,        mass,         column,       heating,
                          c_mom,          d_mom,        ring,         remap_winds,  remap_energy,
                          check_finite,   mass_sum,     to_double,    from_double};

}  // namespace atm
