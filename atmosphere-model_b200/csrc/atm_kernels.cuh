// Kernels of the B200 dynamical core, templated on the sweep type T
// (double for the FP64 form, float for the mixed form).  Column sums,
// pkap, gz and the vertical remap always run in double.
//
// Every per-layer kernel processes one TX x TY tile of one layer: it stages
// the tile plus the stencil halo of its inputs in shared memory, runs the
// stages of the reference's layer loop on that tile, and writes its outputs.
// Index ranges, staggering shifts and evaluation order follow the
// reference line by line (cited per stage).
#pragma once

#include "atm_common.cuh"

namespace atm {

constexpr int NT = 256;  // threads per block of the per-layer kernels

// ---------------------------------------------------------------- loads ----
// s[(y - y0) * w + (x - x0)] = field(x, y, k) for the box [x0, x0+w) x
// [y0, y0+h); points outside the stored (halo-padded) array read as zero and
// only ever feed outputs outside the kernel's output region.
template <typename T>
__device__ __forceinline__ void load_box(T* s, const T* __restrict__ f, const Geom& g, int k, int x0, int y0, int w,
                                         int h) {
  const T* base = f + (long long)k * g.S;
  for (int idx = threadIdx.x; idx < w * h; idx += blockDim.x) {
    int y = idx / w, x = idx - y * w;
    int gx = x0 + x, gy = y0 + y;
    T v = T(0);
    if (gx >= -H && gx < g.nx + H && gy >= -H && gy < g.ny + H) v = base[g.at(gx, gy)];
    s[idx] = v;
  }
}

template <typename T>
__device__ __forceinline__ Sm<T> carve(unsigned char*& p, int x0, int y0, int w, int h) {
  Sm<T> s{reinterpret_cast<T*>(p), x0, y0, w};
  p += ((size_t)w * h * sizeof(T) + 15) & ~(size_t)15;
  return s;
}
template <typename T>
__host__ __device__ constexpr size_t box_bytes(int w, int h) {
  return ((size_t)w * h * sizeof(T) + 15) & ~(size_t)15;
}

// Raise a context's non-finite flag (bad values are rare: one atomic each).
__device__ __forceinline__ void flag_nonfinite(int* flag, bool bad) {
  if (bad) atomicOr(flag, 1);
}
__device__ __forceinline__ bool finite_(double v) { return isfinite(v); }
__device__ __forceinline__ bool finite_(float v) { return isfinite(v); }

// ====================================================== column pressure ====
// plev = ptop + suffix sum of dp from the model top, pkap = plev**kappa,
// hydrostatic gz from the bottom (src/mod_sw_dyn.f90:276-292 and 606-626).
// One thread per column over [lo, n-1+hi]^2.  The downward pass writes
// pkap; the upward pass reads it back (from L2: a block's columns were just
// written), so no shared memory limits the occupancy.  The next layer's dp
// is loaded one iteration ahead so that its latency overlaps atm_pow.
template <typename T>
__global__ void __launch_bounds__(128) k_column(Geom g, Consts c, const T* __restrict__ dpl, const T* __restrict__ ptl,
                                                double* __restrict__ pkap, double* __restrict__ gz, int lo, int hi,
                                                double* __restrict__ plev_out) {
  const int w = g.nx - lo + hi;
  const int hgt = g.ny - lo + hi;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w * hgt) return;
  const int x = lo + col % w, y = lo + col / w;
  const long long o = g.at(x, y);
  const long long S = g.S;
  const int L = g.L;
  double plev = c.ptop;
  if (plev_out) plev_out[o + (long long)L * S] = plev;
  double dnext = (double)dpl[o + (long long)(L - 1) * S];
  for (int k = L - 1; k >= 0; --k) {
    const double d = dnext;
    if (k > 0) dnext = (double)dpl[o + (long long)(k - 1) * S];
    plev = plev + d;
    if (plev_out) plev_out[o + (long long)k * S] = plev;
    pkap[o + (long long)k * S] = atm_pow(plev, KAPPA);
  }
  double z = gz[o];
  double pk0 = pkap[o];
  double ptn = (double)ptl[o];
  for (int k = 0; k < L; ++k) {
    const double pk1 = k + 1 < L ? pkap[o + (long long)(k + 1) * S] : c.pk_top;
    const double pt = ptn;
    if (k + 1 < L) ptn = (double)ptl[o + (long long)(k + 1) * S];
    z = z + CP_DRY * pt * (pk0 - pk1);
    gz[o + (long long)(k + 1) * S] = z;
    pk0 = pk1;
  }
}

// Heating rate of the layer from the radiative net flux,
// src/mod_sw_dyn.f90:89-106 (C) and 433-464 (D): pkap from dp (C step) or
// dpc (D step) over the whole padded domain, playkap, then
// heat = (nf(k+1) - nf(k)) / (cp dp / g) / playkap.
template <typename T>
__global__ void __launch_bounds__(64) k_heating(Geom g, Consts c, const T* __restrict__ dpl,
                                                const double* __restrict__ nf, double* __restrict__ heat) {
  const int w = g.nx + 2 * H;
  const int col = blockIdx.x * 64 + threadIdx.x;
  if (col >= w * g.NYP) return;
  const int x = -H + col % w, y = -H + col / w;
  const long long o = g.at(x, y);
  const int L = g.L;
  double plev = c.ptop, pk_up = c.pk_top;
  for (int k = L - 1; k >= 0; --k) {
    long long ok = o + (long long)k * g.S;
    double d = (double)dpl[ok];
    plev = plev + d;
    double pk = atm_pow(plev, KAPPA);
    double playkap = (pk_up - pk) / atm_log(pk_up / pk);
    heat[ok] = (nf[ok + g.S] - nf[ok]) / (CP_DRY * d / c.gravity) / playkap;
    pk_up = pk;
  }
}

// ============================================================= corners ====
// interpolate_to_corners (src/mod_sw_dyn.f90:921-956) of pkap (levels
// 1..L -> pkapb) and gz (levels 2..L+1 -> gzb) on [0, nx] x [0, ny]; the
// first level of gzb is done once at set-up (level0 = 0, nlev = 1).
__device__ __forceinline__ double tx_(const double* q, long long o, int P) {
  return C7_12 * (q[o] + q[o - 1]) - C1_12 * (q[o + 1] + q[o - 2]);
}
__device__ __forceinline__ double ty_(const double* q, long long o, int P) {
  return C7_12 * (q[o] + q[o - P]) - C1_12 * (q[o + P] + q[o - 2 * P]);
}
__device__ __forceinline__ double corner(const double* q, long long o, int P) {
  double out = C9_32 * (tx_(q, o, P) + tx_(q, o - P, P)) - C1_32 * (tx_(q, o + P, P) + tx_(q, o - 2 * P, P));
  out = out + C9_32 * (ty_(q, o, P) + ty_(q, o - 1, P)) - C1_32 * (ty_(q, o + 1, P) + ty_(q, o - 2, P));
  return out;
}

static __global__ void k_corners(Geom g, const double* __restrict__ pkap, const double* __restrict__ gz,
                          double* __restrict__ pkapb, double* __restrict__ gzb, int with_pkap, int lev0, int nlev) {
  const int w = g.nx + 1, h = g.ny + 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= w * h) return;
  const int x = idx % w, y = idx / w;
  for (int l = lev0; l < lev0 + nlev; ++l) {
    long long o = g.at(x, y, l);
    if (with_pkap) pkapb[o] = corner(pkap, o, g.P);
    long long o1 = g.at(x, y, l + (with_pkap ? 1 : 0));
    gzb[o1] = corner(gz, o1, g.P);
  }
}

// =============================================================== halos ====
// Periodic fill of the 7-wide ring (the single-image halo_exchange,
// src/mod_sync.f90:67-217): every ring point takes the value of its
// periodic image in the interior.  With copy = true the ring of src is
// copied to dst instead (the ring of a new time level keeps the old ring).
template <typename T, bool COPY>
__global__ void k_ring(Geom g, T* f0, T* f1, T* f2, T* f3, const T* s0, const T* s1, const T* s2, const T* s3, int K) {
  const int wide = g.nx + 2 * H;
  const int nband = 2 * H * wide;
  const int nring = nband + 2 * H * g.ny;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nring) return;
  int x, y;
  if (idx < nband) {
    int r = idx / wide;
    y = r < H ? r - H : g.ny + (r - H);
    x = idx % wide - H;
  } else {
    int q = idx - nband;
    y = q / (2 * H);
    int cc = q % (2 * H);
    x = cc < H ? cc - H : g.nx + (cc - H);
  }
  const int k = blockIdx.y;
  if (k >= K) return;
  const int fld = blockIdx.z;
  T* f = fld == 0 ? f0 : fld == 1 ? f1 : fld == 2 ? f2 : f3;
  const T* s = fld == 0 ? s0 : fld == 1 ? s1 : fld == 2 ? s2 : s3;
  long long o = g.at(x, y, k);
  if (COPY) {
    f[o] = s[o];
  } else {
    int xs = x < 0 ? x + g.nx : (x >= g.nx ? x - g.nx : x);
    int ys = y < 0 ? y + g.ny : (y >= g.ny ? y - g.ny : y);
    f[o] = f[g.at(xs, ys, k)];
  }
}

// ========================================================= vertical remap ==
template <int LM>
struct PPMWork {
  double gam[LM + 2], lv[LM + 2], top[LM + 2], btm[LM + 2], curv[LM + 2];
};

// vertical_ppm, src/mod_remap.f90:287-356; arrays are 1-based.  The test of
// the last interface reads gam(nlay+1), past the end of gam in the
// reference; level_var(nlay) is already clamped to the same bounds at
// :319-320, so both clamps are applied there (any branch leaves it as is).
template <int LM>
__device__ void vertical_ppm(PPMWork<LM>& w, int L, const double* var, const double* coord) {
  double* gam = w.gam;
  double* lv = w.lv;
  double alpha, beta;
  alpha = (coord[L] - coord[L - 1]) / (coord[L + 1] - coord[L]);
  beta = alpha * (.5 + alpha);
  lv[L + 1] = (2. * alpha * (1. + alpha) * var[L] + var[L - 1]) / beta;
  gam[L] = (1. + alpha * (1.5 + alpha)) / beta;
  for (int k = L; k >= 2; --k) {
    alpha = (coord[k + 1] - coord[k]) / (coord[k] - coord[k - 1]);
    beta = 2. + 2. * alpha - gam[k];
    lv[k] = (3. * (var[k] + alpha * var[k - 1]) - lv[k + 1]) / beta;
    gam[k - 1] = alpha / beta;
  }
  beta = 1. + alpha * (1.5 + alpha);
  lv[1] = (2. * alpha * (1. + alpha) * var[1] + var[2] - beta * lv[2]) / (alpha * (.5 + alpha) - beta * gam[1]);
  for (int k = 2; k <= L + 1; ++k) lv[k] = lv[k] - gam[k - 1] * lv[k - 1];
  lv[L] = mn(lv[L], mx(var[L], var[L - 1]));
  lv[L] = mx(lv[L], mn(var[L], var[L - 1]));
  lv[2] = mn(lv[2], mx(var[2], var[1]));
  lv[2] = mx(lv[2], mn(var[2], var[1]));
  for (int k = 2; k <= L - 1; ++k) {
    double lo = mn(var[k], var[k + 1]), hi = mx(var[k], var[k + 1]);
    if (k + 2 > L || gam[k + 2] * gam[k] > 0) {
      lv[k + 1] = mn(lv[k + 1], hi);
      lv[k + 1] = mx(lv[k + 1], lo);
    } else if (gam[k + 2] > 0) {
      lv[k + 1] = mx(lv[k + 1], lo);
    } else {
      lv[k + 1] = mn(lv[k + 1], hi);
    }
  }
  for (int k = 1; k <= L; ++k) {
    w.top[k] = lv[k + 1];
    w.btm[k] = lv[k];
  }
  for (int k = 2; k <= L - 1; ++k) {
    double pmp1 = var[k + 1] - 2. * gam[k];
    double lac1 = pmp1 + 1.5 * gam[k - 1];
    w.top[k + 1] = mn(mx(w.top[k + 1], mn3(var[k + 1], pmp1, lac1)), mx3(var[k + 1], pmp1, lac1));
    pmp1 = var[k + 1] + 2. * gam[k + 1];
    lac1 = pmp1 - 1.5 * gam[k];
    w.btm[k + 1] = mn(mx(w.btm[k + 1], mn3(var[k + 1], pmp1, lac1)), mx3(var[k + 1], pmp1, lac1));
  }
  for (int k = 1; k <= L; ++k) w.curv[k] = 6. * var[k] - 3. * (w.top[k] + w.btm[k]);
}

// Contribution of source layer k to destination layer m, the body of the
// pair loop of src/mod_remap.f90:188-280.  Returns the case tag(s).
template <int LM>
__device__ __forceinline__ int remap_pair(const PPMWork<LM>& w, const double* src_var, double* dst_var,
                                          const double* sc, const double* dc, int k, int m) {
  double dsrc = sc[k + 1] - sc[k];
  double s1 = (dc[m] - sc[k]) / dsrc;
  double s2 = (dc[m + 1] - sc[k]) / dsrc;
  double integral_factor = dsrc / (dc[m + 1] - dc[m]);
  int which = 0;
  double tmp3 = 2. * s1 * s1;
  if (dc[m + 1] <= sc[k + 1] && sc[k + 1] < dc[m] && dc[m] < sc[k]) {
    double tmp1 = s1 - 1., tmp2 = s1 + 1.;
    dst_var[m] = dst_var[m] + tmp1 / 6. * (3. * (w.btm[k] * tmp1 - w.top[k] * tmp2) + w.curv[k] * (tmp3 - tmp2)) *
                                  integral_factor;
    which = 3;
  }
  if (sc[k + 1] < dc[m + 1] && dc[m + 1] < sc[k] && sc[k] <= dc[m]) {
    dst_var[m] = dst_var[m] + (s2 / 2.) * (w.btm[k] * (2. - s2) + s2 * (w.top[k] + w.curv[k] * (1. - C2_3 * s2))) *
                                  integral_factor;
    which = which * 10 + 4;
  }
  if (dc[m + 1] <= sc[k + 1] && sc[k] <= dc[m]) {
    dst_var[m] = dst_var[m] + src_var[k] * integral_factor;
    which = which * 10 + 5;
  }
  if (sc[k + 1] < dc[m + 1] && dc[m] < sc[k]) {
    double tmp1 = s1 + s2;
    dst_var[m] = dst_var[m] + (s1 - s2) / 6. *
                                  (3. * (w.btm[k] * (tmp1 - 2.) - w.top[k] * tmp1) + w.curv[k] * (tmp3 + tmp1 * (2. * s2 - 3.))) *
                                  integral_factor;
    which = which * 10 + 6;
  }
  return which;
}

// remap_column, src/mod_remap.f90:165-285.  When both coordinates are
// non-increasing the pairs that pass the reference's overlap test are, for
// each destination layer m, a contiguous run of source layers whose ends
// move monotonically with m; they are visited in that order (ascending k
// for each m, the order in which the reference accumulates dst_var(m)).
// Otherwise the reference's all-pairs loop runs.  trace, when non-null,
// receives {first k, last k, case of first, case of last, count} per m.
template <int LM>
__device__ void remap_column(PPMWork<LM>& w, int L, const double* src_var, double* dst_var, const double* sc,
                             const double* dc, int* trace, long long tstride, int* fallback) {
  for (int m = 1; m <= L; ++m) dst_var[m] = 0.;
  vertical_ppm<LM>(w, L, src_var, sc);
  bool mono = true;
  for (int k = 1; k <= L; ++k) mono = mono && (sc[k + 1] <= sc[k]) && (dc[k + 1] <= dc[k]);
  if (trace)
    for (int m = 1; m <= L; ++m) {
      int* t = trace + (long long)(m - 1) * 5 * tstride;
      t[0] = -1; t[tstride] = -1; t[2 * tstride] = -1; t[3 * tstride] = -1; t[4 * tstride] = 0;
    }
  if (mono) {
    int k0 = 1;
    for (int m = 1; m <= L; ++m) {
      while (k0 <= L && sc[k0 + 1] >= dc[m]) ++k0;
      for (int k = k0; k <= L && sc[k] > dc[m + 1]; ++k) {
        int which = remap_pair<LM>(w, src_var, dst_var, sc, dc, k, m);
        if (trace) {
          int* t = trace + (long long)(m - 1) * 5 * tstride;
          if (t[0] < 0) { t[0] = k; t[2 * tstride] = which; }
          t[tstride] = k;
          t[3 * tstride] = which;
          t[4 * tstride] += 1;
        }
      }
    }
  } else {
    if (fallback) atomicAdd(fallback, 1);
    for (int k = 1; k <= L; ++k)
      for (int m = 1; m <= L; ++m) {
        if (sc[k + 1] >= dc[m] || sc[k] <= dc[m + 1]) continue;
        int which = remap_pair<LM>(w, src_var, dst_var, sc, dc, k, m);
        if (trace) {
          int* t = trace + (long long)(m - 1) * 5 * tstride;
          if (t[0] < 0) { t[0] = k; t[2 * tstride] = which; }
          else if (t[tstride] != k - 1) t[4 * tstride] = -1000000;
          t[tstride] = k;
          t[3 * tstride] = which;
          if (t[4 * tstride] >= 0) t[4 * tstride] += 1;
        }
      }
  }
}

// Winds on the cell faces over [isd-1, ied+1]^2, src/mod_remap.f90:80-105.
// The D-grid winds here still carry last step's halo (the remap runs before
// the D-grid halo exchange), exactly as in the reference.
template <typename T, int LM>
__global__ void __launch_bounds__(64) k_remap_winds(Geom g, RemapArgs ra, const T* __restrict__ dp,
                                                    const T* __restrict__ ud, const T* __restrict__ vd,
                                                    T* __restrict__ urem, T* __restrict__ vrem, int* trace,
                                                    Status* st) {
  const int w = g.nx + 2, h = g.ny + 2;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w * h) return;
  const int i = -1 + col % w, j = -1 + col / w;
  const int L = g.L;
  double sc[LM + 2], dc[LM + 2], var[LM + 2], out[LM + 2];
  PPMWork<LM> wk;
  // surface pressures of the seven columns involved
  const int cx[7] = {i, i, i, i, i - 2, i - 1, i + 1};
  const int cy[7] = {j - 2, j - 1, j, j + 1, j, j, j};
  double ps[7];
  for (int q = 0; q < 7; ++q) {
    long long o = g.at(cx[q], cy[q]);
    double pl = ra.ptop;
    for (int k = L - 1; k >= 0; --k) pl = pl + (double)dp[o + (long long)k * g.S];
    ps[q] = pl;
  }
  for (int dir = 0; dir < 2; ++dir) {
    // u: columns (i, j-2..j+1) -> q = 0..3 ; v: (i-2..i+1, j) -> q = 4, 5, 2, 6
    const int qa = dir == 0 ? 2 : 2, qb = dir == 0 ? 1 : 5, qc = dir == 0 ? 3 : 6, qd = dir == 0 ? 0 : 4;
    long long oa = g.at(cx[qa], cy[qa]), ob = g.at(cx[qb], cy[qb]), oc = g.at(cx[qc], cy[qc]), od = g.at(cx[qd], cy[qd]);
    double pa = ra.ptop, pb = ra.ptop, pc = ra.ptop, pd = ra.ptop;
    for (int k = L + 1; k >= 1; --k) {
      if (k <= L) {
        long long kk = (long long)(k - 1) * g.S;
        pa = pa + (double)dp[oa + kk];
        pb = pb + (double)dp[ob + kk];
        pc = pc + (double)dp[oc + kk];
        pd = pd + (double)dp[od + kk];
      }
      sc[k] = C7_12 * (pa + pb) - C1_12 * (pc + pd);
      double ta, tb, tc, td;
      if (k <= L) {
        double a = ra.ak[k - 1], b = ra.bk[k - 1];
        ta = a + b * (ps[qa] - ra.ptop);
        tb = a + b * (ps[qb] - ra.ptop);
        tc = a + b * (ps[qc] - ra.ptop);
        td = a + b * (ps[qd] - ra.ptop);
      } else {
        ta = tb = tc = td = ra.ptop;
      }
      dc[k] = C7_12 * (ta + tb) - C1_12 * (tc + td);
    }
    const T* f = dir == 0 ? ud : vd;
    long long o = g.at(i, j);
    for (int k = 1; k <= L; ++k) var[k] = (double)f[o + (long long)(k - 1) * g.S];
    int* tr = nullptr;
    long long ts = 1;
    if (trace) {
      // layout [3][ny+2][nx+2][L][5]
      tr = trace + ((long long)dir * h * w + (long long)(j + 1) * w + (i + 1)) * L * 5;
    }
    remap_column<LM>(wk, L, var, out, sc, dc, tr, ts, &st->fallback_pairs);
    T* r = dir == 0 ? urem : vrem;
    for (int k = 1; k <= L; ++k) r[o + (long long)(k - 1) * g.S] = T(out[k]);
  }
}

// Energy remap and potential-temperature recovery on the interior,
// src/mod_remap.f90:42-78 (columns) and 111-161.
template <typename T, int LM>
__global__ void __launch_bounds__(64) k_remap_energy(Geom g, RemapArgs ra, const T* __restrict__ dp,
                                                     const T* __restrict__ pt, const T* __restrict__ ud,
                                                     const T* __restrict__ vd, const T* __restrict__ urem,
                                                     const T* __restrict__ vrem, const double* __restrict__ gzs,
                                                     T* __restrict__ dpo, T* __restrict__ pto, T* __restrict__ udo,
                                                     T* __restrict__ vdo, int* trace, Status* st) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= g.nx * g.ny) return;
  const int i = col % g.nx, j = col / g.nx;
  const int L = g.L;
  const long long S = g.S;
  const long long o = g.at(i, j);
  double plev[LM + 2], pk[LM + 2], tpl[LM + 2], tpk[LM + 2], lyk[LM + 2], tlyk[LM + 2], gzv[LM + 2];
  double en[LM + 2], er[LM + 2];
  PPMWork<LM> wk;
  plev[L + 1] = ra.ptop;
  pk[L + 1] = ra.pk_top;
  for (int k = L; k >= 1; --k) {
    plev[k] = plev[k + 1] + (double)dp[o + (long long)(k - 1) * S];
    pk[k] = atm_pow(plev[k], KAPPA);
    double plog = atm_log(pk[k + 1] / pk[k]);
    lyk[k] = (pk[k + 1] - pk[k]) / plog;
  }
  tpl[L + 1] = ra.ptop;
  tpk[L + 1] = ra.pk_top;
  for (int k = L; k >= 1; --k) {
    tpl[k] = ra.ak[k - 1] + ra.bk[k - 1] * (plev[1] - ra.ptop);
    tpk[k] = atm_pow(tpl[k], KAPPA);
    double plog = atm_log(tpk[k + 1] / tpk[k]);
    tlyk[k] = (tpk[k + 1] - tpk[k]) / plog;
  }
  gzv[1] = gzs[o];
  for (int k = 1; k <= L; ++k) gzv[k + 1] = gzv[k] + CP_DRY * (double)pt[o + (long long)(k - 1) * S] * (pk[k] - pk[k + 1]);
  const int P = g.P;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    double ua = (.25 * ((double)ud[ok] + (double)ud[ok + P]) +
                 .125 * ((double)ud[ok - 1] + (double)ud[ok - 1 + P] + (double)ud[ok + 1] + (double)ud[ok + 1 + P]));
    double va = (.25 * ((double)vd[ok] + (double)vd[ok + 1]) +
                 .125 * ((double)vd[ok - P] + (double)vd[ok + 1 - P] + (double)vd[ok + P] + (double)vd[ok + 1 + P]));
    en[k] = CV_DRY * (double)pt[ok] * lyk[k] + .5 * (gzv[k + 1] + gzv[k] + ua * ua + va * va);
  }
  int* tr = nullptr;
  if (trace) {
    const int w = g.nx + 2, h = g.ny + 2;
    tr = trace + ((long long)2 * h * w + (long long)(j + 1) * w + (i + 1)) * L * 5;
  }
  remap_column<LM>(wk, L, en, er, plev, tpl, tr, 1, &st->fallback_pairs);
  double gzr = gzv[1];
  bool bad = false;
  for (int k = 1; k <= L; ++k) {
    long long ok = o + (long long)(k - 1) * S;
    double ua = (.25 * ((double)urem[ok] + (double)urem[ok + P]) +
                 .125 * ((double)urem[ok - 1] + (double)urem[ok - 1 + P] + (double)urem[ok + 1] + (double)urem[ok + 1 + P]));
    double va = (.25 * ((double)vrem[ok] + (double)vrem[ok + 1]) +
                 .125 * ((double)vrem[ok - P] + (double)vrem[ok + 1 - P] + (double)vrem[ok + P] + (double)vrem[ok + 1 + P]));
    double ptr = (er[k] - gzr - .5 * (ua * ua + va * va)) / (CV_DRY * tlyk[k] + .5 * CP_DRY * (tpk[k] - tpk[k + 1]));
    gzr = gzr + CP_DRY * ptr * (tpk[k] - tpk[k + 1]);
    T dpn = T(tpl[k] - tpl[k + 1]);
    T un = urem[ok], vn = vrem[ok], tn = T(ptr);
    dpo[ok] = dpn;
    pto[ok] = tn;
    udo[ok] = un;
    vdo[ok] = vn;
    bad = bad || !(finite_(dpn) && finite_(tn) && finite_(un) && finite_(vn));
  }
  flag_nonfinite(&st->nonfinite_remap, bad);
}

// ============================================================ reductions ===
// Finite check of the interior of four fields (src/mod_fields.f90:69-106).
template <typename T>
__global__ void k_check_finite(Geom g, const T* f0, const T* f1, const T* f2, const T* f3, int* flag) {
  const int n = g.nx * g.ny;
  bool bad = false;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * g.L; idx += gridDim.x * blockDim.x) {
    int k = idx / n, r = idx - k * n;
    long long o = g.at(r % g.nx, r / g.nx, k);
    bad = bad || !(finite_(f0[o]) && finite_(f1[o]) && finite_(f2[o]) && finite_(f3[o]));
  }
  flag_nonfinite(flag, bad);
}

// Sum of the interior pressure thickness in FP64, in a fixed order: each
// block reduces a fixed slice of the (level, row) pairs with a fixed tree,
// the host-visible result sums the block partials in index order.
template <typename T>
__global__ void k_mass_partial(Geom g, const T* dp, double* partial) {
  __shared__ double red[256];
  const int rows = g.ny * g.L;
  double acc = 0.;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    int k = r / g.ny, j = r - k * g.ny;
    const T* row = dp + g.at(0, j, k);
    for (int i = threadIdx.x; i < g.nx; i += blockDim.x) acc += (double)row[i];
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}
static __global__ void k_mass_final(const double* partial, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.;
    for (int i = 0; i < n; ++i) s += partial[i];
    *out = s;
  }
}

// Precision conversion of whole padded fields (mixed-precision uploads and
// downloads go through an FP64 staging field).
template <typename A, typename B>
__global__ void k_convert(const A* __restrict__ src, B* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = B(src[i]);
}

}  // namespace atm
