// Launch wrappers of one form of the dynamical core (T = sweep type).
// Included once by atm_fp64.cu (T = double) and once by atm_mixed.cu
// (T = float), which each define ATM_FORM_T and ATM_OPS_NAME.
#pragma once

#include "atm_kernels.cuh"
#include "atm_march.cuh"
#include "atm_ops.h"
#include "atm_sweeps.cuh"
#include "atm_tmap.h"

namespace atm {
namespace {

using T = ATM_FORM_T;  // sweep arithmetic
using S = double;      // prognostic state (dp, pt, ud, vd), both forms
using C = T;           // C-grid fields (dpc, ptc, uc, vc)
// Tile of each sweep kernel (TX x TY_*), measured per kernel and form on
// B200 at 1024x1024x64 (heights 3 to 16 and 64x8 tried, with the CTAs per
// SM each layout's register budget is set for): smaller tiles hold more
// CTAs per SM, taller ones recompute less halo.
constexpr bool FP64_FORM = std::is_same_v<T, double>;
constexpr int TX = 32;
constexpr int TY_CMASS = FP64_FORM ? 4 : 16;
constexpr int TY_DMASS = FP64_FORM ? 6 : 16;
constexpr int TY_CMOM = 8;
constexpr int TY_DMOM = 4;
// The mixed form (ATM_MARCH_SWEEPS) runs its four sweeps as column-marching
// kernels (atm_march.cuh): measured on B200 at 1024x1024x64, C mass 1.79 /
// C momentum 2.21 / D mass 1.84 / D momentum 2.43 ms against its tiles'
// 2.70 / 3.01 / 2.66 / 4.05 (and the persistent ensemble kernel, which has
// only the marching sweeps, is bit-identical to it).  The FP64 form keeps
// the tiles: its marching sweeps took 29.1 ms a step against 17.4 (at
// 136-174 registers a thread they hold too few warps to hide the FP64
// latency, and they execute about as many instructions per cell).
#ifdef ATM_MARCH_SWEEPS
constexpr bool MARCH = true;
#else
constexpr bool MARCH = false;
#endif
// strip height (output rows a warp walks through) of the marching sweeps,
// chosen per launch: 128 rows where that grid still fills eight waves of
// resident blocks, else 32.  Measured on B200 (ms a step, mixed form, rows
// 32 / 64 / 96 / 128 / 256): 11.46 / 11.10 / 11.03 / 10.96 / 11.25 at
// 1024x1024x64 and 3.14 / 3.13 / 3.20 / 3.30 / 3.80 at 512x512x64, where 128
// rows leave 2.2 waves and the tail dominates.
constexpr int TYS_TALL = 128, TYS_SHORT = 32;

inline dim3 strips(int lo, int hi, const Geom& g, int tys) {
  int w = g.nx - lo + hi, h = g.ny - lo + hi;
  return dim3((w + MOUT * MWARPS - 1) / (MOUT * MWARPS), (h + tys - 1) / tys, g.L);
}

inline bool tall_strips(int lo, int hi, const Geom& g) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms = 148;
  dim3 b = strips(lo, hi, g, TYS_TALL);
  return (long long)b.x * b.y * b.z >= 8LL * sms * ATM_MARCH_MINB;
}

// calls f(std::integral_constant<int, rows>) with the strip height picked above
template <typename F>
cudaError_t with_rows(int lo, int hi, const Geom& g, F&& f) {
  if (tall_strips(lo, hi, g)) f(std::integral_constant<int, TYS_TALL>{});
  else f(std::integral_constant<int, TYS_SHORT>{});
  return cudaGetLastError();
}

inline dim3 tiles(int lo, int hi, const Geom& g, int layers, int ty) {
  int w = g.nx - lo + hi, h = g.ny - lo + hi;
  return dim3((w + TX - 1) / TX, (h + ty - 1) / ty, layers);
}

template <typename K>
cudaError_t smem_attr(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t setup() {
  cudaError_t e;
  if ((e = smem_attr(k_mass2<T, TX, TY_CMASS, true, S, C>, MassL<T, TX, TY_CMASS, true, S, C>::bytes)) != cudaSuccess)
    return e;
  if ((e = smem_attr(k_mass2<T, TX, TY_DMASS, false, S, C>, MassL<T, TX, TY_DMASS, false, S, C>::bytes)) !=
      cudaSuccess)
    return e;
  if constexpr (!MARCH) {
    if ((e = smem_attr(k_c_mom2<T, TX, TY_CMOM, S, C>, CMomL<T, TX, TY_CMOM, S>::bytes)) != cudaSuccess) return e;
    if ((e = smem_attr(k_d_mom2<T, TX, TY_DMOM, S, C>, DMomL<T, TX, TY_DMOM, S, C>::bytes)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t mass(const Geom& g, const Consts& c, const void* dp, const void* pt, const void* u, const void* v,
                 const double* heat, void* dpo, void* pto, int lo, int hi, int* nonfinite, int* timeout, bool cgrid,
                 cudaStream_t s) {
#ifdef ATM_MARCH_SWEEPS
  if constexpr (MARCH) {
    return with_rows(lo, hi, g, [&](auto rows) {
      constexpr int R = decltype(rows)::value;
      if (cgrid)  // state in, C-grid fields out
        k_mass_m<T, R, true, S, C><<<strips(lo, hi, g, R), MW * MWARPS, 0, s>>>(
            g, c, (const S*)dp, (const S*)pt, (const S*)u, (const S*)v, heat, (C*)dpo, (C*)pto, lo, hi, nonfinite);
      else  // state and C-grid winds in, state out
        k_mass_m<T, R, false, S, C><<<strips(lo, hi, g, R), MW * MWARPS, 0, s>>>(
            g, c, (const S*)dp, (const S*)pt, (const C*)u, (const C*)v, heat, (S*)dpo, (S*)pto, lo, hi, nonfinite);
    });
  }
#endif
  CUtensorMap md, mp, mu, mv;
  cudaError_t e;
  if (cgrid) {  // state in, C-grid fields out
    using Lay = MassL<T, TX, TY_CMASS, true, S, C>;
    dim3 grid = tiles(lo, hi, g, g.L, TY_CMASS);
    constexpr int eu = sizeof(typename Lay::UB);
    if ((e = tmap(dp, sizeof(S), g, g.L, Lay::WD, Lay::HD, &md)) ||
        (e = tmap(pt, sizeof(S), g, g.L, Lay::WD, Lay::HD, &mp)) || (e = tmap(u, eu, g, g.L, Lay::WU, Lay::HU, &mu)) ||
        (e = tmap(v, eu, g, g.L, Lay::WV, Lay::HV, &mv)))
      return e;
    k_mass2<T, TX, TY_CMASS, true, S, C><<<grid, NT, Lay::bytes, s>>>(md, mp, mu, mv, g, c, heat, (C*)dpo,
                                                                       (C*)pto, lo, hi, nonfinite, timeout);
  } else {
    using Lay = MassL<T, TX, TY_DMASS, false, S, C>;
    dim3 grid = tiles(lo, hi, g, g.L, TY_DMASS);
    constexpr int eu = sizeof(typename Lay::UB);
    if ((e = tmap(dp, sizeof(S), g, g.L, Lay::WD, Lay::HD, &md)) ||
        (e = tmap(pt, sizeof(S), g, g.L, Lay::WD, Lay::HD, &mp)) || (e = tmap(u, eu, g, g.L, Lay::WU, Lay::HU, &mu)) ||
        (e = tmap(v, eu, g, g.L, Lay::WV, Lay::HV, &mv)))
      return e;
    k_mass2<T, TX, TY_DMASS, false, S, C><<<grid, NT, Lay::bytes, s>>>(md, mp, mu, mv, g, c, heat, (S*)dpo,
                                                                        (S*)pto, lo, hi, nonfinite, timeout);
  }
  return cudaGetLastError();
}

cudaError_t column(const Geom& g, const Consts& c, const void* dpl, const void* ptl, int es, double* pkap, double* gz,
                   int lo, int hi, double* plev, cudaStream_t s) {
  int n = (g.nx - lo + hi) * (g.ny - lo + hi);
  if (es == 8)
    k_column<double, FormPow<T>><<<(n + 127) / 128, 128, 0, s>>>(g, c, (const double*)dpl, (const double*)ptl, pkap, gz, lo, hi,
                                                     plev);
  else
    k_column<float, FormPow<T>><<<(n + 127) / 128, 128, 0, s>>>(g, c, (const float*)dpl, (const float*)ptl, pkap, gz, lo, hi,
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
#ifdef ATM_MARCH_SWEEPS
  if constexpr (MARCH) {
    return with_rows(0, 0, g, [&](auto rows) {
      constexpr int R = decltype(rows)::value;
      k_c_mom_m<T, R, S, C><<<strips(0, 0, g, R), MW * MWARPS, 0, s>>>(g, c, (const S*)ud, (const S*)vd, pkap, gz,
                                                                        (C*)uc, (C*)vc);
    });
  }
#endif
  using Lay = CMomL<T, TX, TY_CMOM, S>;
  constexpr int es = sizeof(S);
  CUtensorMap mu, mv, muL, mvL, mpk, mgz;
  cudaError_t e;
  if ((e = tmap(ud, es, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(vd, es, g, g.L, Lay::WV, Lay::HV, &mv)) ||
      (e = tmap(ud, es, g, g.L, Lay::WL, Lay::HL, &muL)) || (e = tmap(vd, es, g, g.L, Lay::WL, Lay::HL, &mvL)) ||
      (e = tmap(pkap, 8, g, g.L + 1, Lay::WP, Lay::HP, &mpk)) || (e = tmap(gz, 8, g, g.L + 1, Lay::WP, Lay::HP, &mgz)))
    return e;
  k_c_mom2<T, TX, TY_CMOM, S, C><<<tiles(0, 0, g, g.L, TY_CMOM), NT, Lay::bytes, s>>>(
      mu, mv, muL, mvL, mpk, mgz, g, c, (const S*)ud, (const S*)vd, (C*)uc, (C*)vc, timeout);
  return cudaGetLastError();
}

cudaError_t d_mom(const Geom& g, const Consts& c, const void* ud, const void* vd, const void* uc, const void* vc,
                  const double* pkapb, const double* gzb, void* udo, void* vdo, int* nonfinite, int* timeout,
                  cudaStream_t s) {
#ifdef ATM_MARCH_SWEEPS
  if constexpr (MARCH) {
    return with_rows(0, 0, g, [&](auto rows) {
      constexpr int R = decltype(rows)::value;
      k_d_mom_m<T, R, S, C><<<strips(0, 0, g, R), MW * MWARPS, 0, s>>>(
          g, c, (const S*)ud, (const S*)vd, (const C*)uc, (const C*)vc, pkapb, gzb, (S*)udo, (S*)vdo, nonfinite);
    });
  }
#endif
  using Lay = DMomL<T, TX, TY_DMOM, S, C>;
  constexpr int es = sizeof(S), ec = sizeof(C);
  CUtensorMap mu, mv, muL, mvL, muc, mvc, mpb, mgb;
  cudaError_t e;
  if ((e = tmap(ud, es, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(vd, es, g, g.L, Lay::WU, Lay::HU, &mv)) ||
      (e = tmap(uc, ec, g, g.L, Lay::WUL, Lay::HUL, &muL)) || (e = tmap(vc, ec, g, g.L, Lay::WVL, Lay::HVL, &mvL)) ||
      (e = tmap(uc, ec, g, g.L, Lay::WC, Lay::HC, &muc)) || (e = tmap(vc, ec, g, g.L, Lay::WC, Lay::HC, &mvc)) ||
      (e = tmap(pkapb, 8, g, g.L + 1, Lay::WP, Lay::HP, &mpb)) || (e = tmap(gzb, 8, g, g.L + 1, Lay::WP, Lay::HP, &mgb)))
    return e;
  k_d_mom2<T, TX, TY_DMOM, S, C><<<tiles(0, 0, g, g.L, TY_DMOM), NT, Lay::bytes, s>>>(
      mu, mv, muL, mvL, muc, mvc, mpb, mgb, g, c, (const S*)ud, (const S*)vd, (S*)udo, (S*)vdo, nonfinite, timeout);
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
  k_remap_winds<S, LM, T><<<dim3((n + 63) / 64, 2), 64, 0, s>>>(g, ra, (const S*)dp, (const S*)ud, (const S*)vd, (S*)urem,
                                                    (S*)vrem, trace, st);
  return cudaGetLastError();
}
template <int LM>
cudaError_t remap_energy_lm(const Geom& g, const RemapArgs& ra, const void* dp, const void* pt, const void* ud,
                            const void* vd, const void* urem, const void* vrem, const double* gzs, void* dpo,
                            void* pto, void* udo, void* vdo, int* trace, Status* st, cudaStream_t s) {
  int n = g.nx * g.ny;
  k_remap_energy<S, LM, FormPow<T>><<<(n + 63) / 64, 64, 0, s>>>(g, ra, (const S*)dp, (const S*)pt, (const S*)ud, (const S*)vd,
                                                     (const S*)urem, (const S*)vrem, gzs, (S*)dpo, (S*)pto, (S*)udo,
                                                     (S*)vdo, trace, st);
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
