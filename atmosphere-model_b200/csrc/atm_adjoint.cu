// Launchers of the FP64 adjoint kernels (atm_adjoint.cuh).  Compiled with
// --fmad=false like the FP64 form: the adjoint kernels recompute the
// forward's intermediates with the forward's exact operations, so every
// limiter and upwind branch is taken as in the forward step.
#include "atm_adjoint.cuh"
#include "atm_ops.h"
#include "atm_tmap.h"

namespace atm {
namespace {

// tiles of the adjoints, measured: C-grid mass TXA x TYC (3 CTAs per SM),
// D-grid mass TXA x TYA (2 CTAs per SM; 32 x 4 is no faster there), the
// momentum adjoints TXA x TYM
constexpr int TXA = 32, TYC = 4, TYA = 8, TYM = 4;

inline dim3 tiles_a(int lo, int hi, const Geom& g, int ty) {
  int w = g.nx - lo + hi, h = g.ny - lo + hi;
  return dim3((w + TXA - 1) / TXA, (h + ty - 1) / ty, g.L);
}

template <typename K>
cudaError_t smem_attr(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

cudaError_t adj_setup() {
  cudaError_t e;
  if ((e = smem_attr(k_mass_adj1<TXA, TYC, true>, MassAdj1L<TXA, TYC, true>::bytes))) return e;
  if ((e = smem_attr(k_mass_adj<TXA, TYA, false, true>, MassAdjBL<TXA, TYA, false>::bytes))) return e;
  if ((e = smem_attr(k_mass_adj<TXA, TYA, false, false>, MassAdjBL<TXA, TYA, false>::bytes))) return e;
  if ((e = smem_attr(k_c_mom_adj<TXA, TYM>, CMomAdjL<TXA, TYM>::bytes))) return e;
  if ((e = smem_attr(k_d_mom_adj_ke<TXA, TYM>, DMomKeAdjL<TXA, TYM>::bytes))) return e;
  if ((e = smem_attr(k_d_mom_adj_vf<TXA, TYM>, DMomVfAdjL<TXA, TYM>::bytes))) return e;
  return cudaSuccess;
}

cudaError_t adj_mass(const Geom& g, const Consts& c, const double* dp, const double* pt, const double* u,
                     const double* v, const double* dpo, const double* pto, const double* lam_dpo,
                     const double* lam_pto, double* lam_dp, double* lam_pt, double* lam_u, double* lam_v, int lo,
                     int hi, int* timeout, bool cgrid, cudaStream_t s, int parts) {
  CUtensorMap md, mp, mu, mv;
  cudaError_t e;
  if (cgrid) {  // one kernel (the update recomputed from the fluxes)
    using Lay = MassL<double, TXA, TYC, true>;
    if ((e = tmap(dp, 8, g, g.L, Lay::WD, Lay::HD, &md)) || (e = tmap(pt, 8, g, g.L, Lay::WD, Lay::HD, &mp)) ||
        (e = tmap(u, 8, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(v, 8, g, g.L, Lay::WV, Lay::HV, &mv)))
      return e;
    (void)dpo;
    (void)pto;
    k_mass_adj1<TXA, TYC, true><<<tiles_a(lo, hi, g, TYC), NTA, MassAdj1L<TXA, TYC, true>::bytes, s>>>(
        md, mp, mu, mv, g, c, lam_dpo, lam_pto, lam_dp, lam_pt, lam_u, lam_v, lo, hi, timeout);
  } else {  // the x branch (with the direct terms) and the y branch, both adding into the same global adjoints
    using Lay = MassL<double, TXA, TYA, false>;
    constexpr size_t bytes = MassAdjBL<TXA, TYA, false>::bytes;
    if ((e = tmap(dp, 8, g, g.L, Lay::WD, Lay::HD, &md)) || (e = tmap(pt, 8, g, g.L, Lay::WD, Lay::HD, &mp)) ||
        (e = tmap(u, 8, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(v, 8, g, g.L, Lay::WV, Lay::HV, &mv)))
      return e;
    const dim3 grid = tiles_a(lo, hi, g, TYA);
    if (parts & 1)
      k_mass_adj<TXA, TYA, false, true><<<grid, NTA, bytes, s>>>(md, mp, mu, mv, g, c, dpo, pto, lam_dpo, lam_pto,
                                                                  lam_dp, lam_pt, lam_u, lam_v, lo, hi, timeout);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (parts & 2)
      k_mass_adj<TXA, TYA, false, false><<<grid, NTA, bytes, s>>>(md, mp, mu, mv, g, c, dpo, pto, lam_dpo, lam_pto,
                                                                   lam_dp, lam_pt, lam_u, lam_v, lo, hi, timeout);
  }
  return cudaGetLastError();
}

cudaError_t adj_c_mom(const Geom& g, const Consts& c, const double* ud, const double* vd, const double* pkap,
                      const double* gz, const double* lam_uc, const double* lam_vc, double* lam_ud, double* lam_vd,
                      double* lam_pk, double* lam_gz, int* timeout, cudaStream_t s) {
  using Lay = CMomL<double, TXA, TYM>;
  CUtensorMap mu, mv, muL, mvL, mpk, mgz;
  cudaError_t e;
  if ((e = tmap(ud, 8, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(vd, 8, g, g.L, Lay::WV, Lay::HV, &mv)) ||
      (e = tmap(ud, 8, g, g.L, Lay::WL, Lay::HL, &muL)) || (e = tmap(vd, 8, g, g.L, Lay::WL, Lay::HL, &mvL)) ||
      (e = tmap(pkap, 8, g, g.L + 1, Lay::WP, Lay::HP, &mpk)) || (e = tmap(gz, 8, g, g.L + 1, Lay::WP, Lay::HP, &mgz)))
    return e;
  k_c_mom_adj<TXA, TYM><<<tiles_a(0, 0, g, TYM), NTA, CMomAdjL<TXA, TYM>::bytes, s>>>(
      mu, mv, muL, mvL, mpk, mgz, g, c, lam_uc, lam_vc, lam_ud, lam_vd, lam_pk, lam_gz, timeout);
  return cudaGetLastError();
}

cudaError_t adj_d_mom(const Geom& g, const Consts& c, const double* ud, const double* vd, const double* uc,
                      const double* vc, const double* pkapb, const double* gzb, const double* lam_udo,
                      const double* lam_vdo, double* lam_ud, double* lam_vd, double* lam_uc, double* lam_vc,
                      double* lam_pkb, double* lam_gzb, int* timeout, cudaStream_t s, int parts) {
  using Lay = DMomL<double, TXA, TYM>;
  CUtensorMap mu, mv, muL, mvL, muc, mvc, mpb, mgb;
  cudaError_t e;
  if ((e = tmap(ud, 8, g, g.L, Lay::WU, Lay::HU, &mu)) || (e = tmap(vd, 8, g, g.L, Lay::WU, Lay::HU, &mv)) ||
      (e = tmap(uc, 8, g, g.L, Lay::WUL, Lay::HUL, &muL)) || (e = tmap(vc, 8, g, g.L, Lay::WVL, Lay::HVL, &mvL)) ||
      (e = tmap(uc, 8, g, g.L, Lay::WC, Lay::HC, &muc)) || (e = tmap(vc, 8, g, g.L, Lay::WC, Lay::HC, &mvc)) ||
      (e = tmap(pkapb, 8, g, g.L + 1, Lay::WP, Lay::HP, &mpb)) || (e = tmap(gzb, 8, g, g.L + 1, Lay::WP, Lay::HP, &mgb)))
    return e;
  // the kinetic-energy chain and the rest, both adding into the same
  // global adjoints
  if (parts & 1)
    k_d_mom_adj_ke<TXA, TYM><<<tiles_a(0, 0, g, TYM), NTA, DMomKeAdjL<TXA, TYM>::bytes, s>>>(
        mu, mv, muL, mvL, g, c, lam_udo, lam_vdo, lam_ud, lam_vd, lam_uc, lam_vc, timeout);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (parts & 2)
    k_d_mom_adj_vf<TXA, TYM><<<tiles_a(0, 0, g, TYM), NTA, DMomVfAdjL<TXA, TYM>::bytes, s>>>(
        mu, mv, muL, mvL, muc, mvc, mpb, mgb, g, c, lam_udo, lam_vdo, lam_ud, lam_vd, lam_uc, lam_vc, lam_pkb,
        lam_gzb, timeout);
  return cudaGetLastError();
}

cudaError_t adj_column(const Geom& g, const Consts& c, const double* dp, const double* pt, const double* lam_pk,
                       const double* lam_gz, double* lam_dp, double* lam_pt, int lo, int hi, cudaStream_t s) {
  const int n = (g.nx - lo + hi) * (g.ny - lo + hi);
  const int nb = (n + 127) / 128;
  if (g.L <= 32) k_column_adj<32><<<nb, 128, 0, s>>>(g, c, dp, pt, lam_pk, lam_gz, lam_dp, lam_pt, lo, hi);
  else if (g.L <= 64) k_column_adj<64><<<nb, 128, 0, s>>>(g, c, dp, pt, lam_pk, lam_gz, lam_dp, lam_pt, lo, hi);
  else k_column_adj<MAX_LAYERS><<<nb, 128, 0, s>>>(g, c, dp, pt, lam_pk, lam_gz, lam_dp, lam_pt, lo, hi);
  return cudaGetLastError();
}

cudaError_t adj_corners(const Geom& g, const double* lam_pkb, const double* lam_gzb, double* lam_pk, double* lam_gz,
                        cudaStream_t s) {
  const int n = (g.nx + 4) * (g.ny + 4);
  k_corners_adj<<<dim3((n + 255) / 256, g.L), 256, 0, s>>>(g, lam_pkb, lam_gzb, lam_pk, lam_gz);
  return cudaGetLastError();
}

cudaError_t adj_ring_fold(const Geom& g, double* const* f, int nf, int K, cudaStream_t s) {
  const int nring = 2 * H * (g.nx + 2 * H) + 2 * H * g.ny;
  double* d[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int i = 0; i < nf; ++i) d[i] = f[i];
  k_ring_fold<<<dim3((nring + 255) / 256, K, nf), 256, 0, s>>>(g, d[0], d[1], d[2], d[3], K);
  return cudaGetLastError();
}

cudaError_t adj_ring_copy(const Geom& g, double* const* dst, double* const* src, int K, int band01, int band23,
                          cudaStream_t s) {
  const int nring = 2 * H * (g.nx + 2 * H) + 2 * H * g.ny;
  k_ring_copy_adj<<<dim3((nring + 255) / 256, K, 4), 256, 0, s>>>(g, dst[0], dst[1], dst[2], dst[3], src[0], src[1],
                                                                   src[2], src[3], K, band01, band23);
  return cudaGetLastError();
}

template <int LM>
static cudaError_t remap_energy_adj_lm(const Geom& g, const RemapArgs& ra, const double* dp, const double* pt,
                                       const double* ud, const double* vd, const double* urem, const double* vrem,
                                       const double* gzs, const double* lam_dpo, const double* lam_pto,
                                       const double* lam_udo, const double* lam_vdo, double* lam_dp, double* lam_pt,
                                       double* lam_ud, double* lam_vd, double* lam_ur, double* lam_vr, cudaStream_t s) {
  const int n = g.nx * g.ny;
  k_remap_energy_adj<LM><<<(n + 63) / 64, 64, 0, s>>>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, lam_dpo, lam_pto,
                                                      lam_udo, lam_vdo, lam_dp, lam_pt, lam_ud, lam_vd, lam_ur, lam_vr);
  return cudaGetLastError();
}

cudaError_t adj_remap_energy(const Geom& g, const RemapArgs& ra, const double* dp, const double* pt, const double* ud,
                             const double* vd, const double* urem, const double* vrem, const double* gzs,
                             const double* lam_dpo, const double* lam_pto, const double* lam_udo,
                             const double* lam_vdo, double* lam_dp, double* lam_pt, double* lam_ud, double* lam_vd,
                             double* lam_ur, double* lam_vr, cudaStream_t s) {
  if (g.L <= 32)
    return remap_energy_adj_lm<32>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, lam_dpo, lam_pto, lam_udo, lam_vdo, lam_dp,
                                   lam_pt, lam_ud, lam_vd, lam_ur, lam_vr, s);
  if (g.L <= 64)
    return remap_energy_adj_lm<64>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, lam_dpo, lam_pto, lam_udo, lam_vdo, lam_dp,
                                   lam_pt, lam_ud, lam_vd, lam_ur, lam_vr, s);
  return remap_energy_adj_lm<MAX_LAYERS>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, lam_dpo, lam_pto, lam_udo, lam_vdo,
                                         lam_dp, lam_pt, lam_ud, lam_vd, lam_ur, lam_vr, s);
}

cudaError_t adj_remap_winds(const Geom& g, const RemapArgs& ra, const double* dp, const double* ud, const double* vd,
                            const double* lam_ur, const double* lam_vr, double* lam_dp, double* lam_ud, double* lam_vd,
                            cudaStream_t s) {
  const int n = (g.nx + 2) * (g.ny + 2);
  const int nb = (n + 63) / 64;
  if (g.L <= 32) k_remap_winds_adj<32><<<nb, 64, 0, s>>>(g, ra, dp, ud, vd, lam_ur, lam_vr, lam_dp, lam_ud, lam_vd);
  else if (g.L <= 64) k_remap_winds_adj<64><<<nb, 64, 0, s>>>(g, ra, dp, ud, vd, lam_ur, lam_vr, lam_dp, lam_ud, lam_vd);
  else k_remap_winds_adj<MAX_LAYERS><<<nb, 64, 0, s>>>(g, ra, dp, ud, vd, lam_ur, lam_vr, lam_dp, lam_ud, lam_vd);
  return cudaGetLastError();
}

}  // namespace atm
