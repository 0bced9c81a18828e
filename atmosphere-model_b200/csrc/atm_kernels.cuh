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

// ============================================================ mass sweeps ==
// One kernel serves both the C-grid half step (CGRID: C-grid winds built
// from the D-grid winds, PPM_UNCONSTRAINED, src/mod_sw_dyn.f90:109-268) and
// the D-grid step (C-grid winds read directly, PPM_NONNEGATIVE,
// src/mod_sw_dyn.f90:441-598).  Outputs: the new pressure thickness and
// potential temperature on [lo, n-1+hi]^2 (C: is+5:ie-5, D: is+4:ie-4).
template <typename T, int TX, int TY>
struct MassSmem {
  static constexpr size_t bytes =
      2 * box_bytes<T>(TX + 6, TY + 6) +              // dp, pt
      box_bytes<T>(TX + 2, TY + 7) + box_bytes<T>(TX + 7, TY + 2) +  // ud, vd boxes (C grid only)
      box_bytes<T>(TX + 1, TY + 6) + box_bytes<T>(TX + 6, TY + 1) +  // uc, vc
      2 * box_bytes<T>(TX + 6, TY) + 2 * box_bytes<T>(TX, TY + 6) +  // tmp (y-inner), tmp (x-inner)
      2 * box_bytes<T>(TX + 2, TY + 2) +                            // laplacians
      2 * box_bytes<T>(TX + 1, TY) + 2 * box_bytes<T>(TX, TY + 1);  // x and y fluxes
};

template <typename T, int TX, int TY, bool CGRID>
__global__ void __launch_bounds__(NT) k_mass(Geom g, Consts c, const T* __restrict__ dp, const T* __restrict__ pt,
                                             const T* __restrict__ uin, const T* __restrict__ vin,
                                             const double* __restrict__ heat, T* __restrict__ dpo,
                                             T* __restrict__ pto, int lo, int hi, int* nonfinite) {
  constexpr int V = CGRID ? PPM_UNC : PPM_NN;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* p = smem;
  const int k = blockIdx.z;
  const int ox = lo + blockIdx.x * TX, oy = lo + blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);

  Sm<T> sdp = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> spt = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> sud = carve<T>(p, ox - 1, oy - 3, TX + 2, TY + 7);
  Sm<T> svd = carve<T>(p, ox - 3, oy - 1, TX + 7, TY + 2);
  Sm<T> suc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
  Sm<T> svc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  Sm<T> tyd = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> typ = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> txd = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> txp = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> lpd = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> lpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> fxd = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fxp = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fyd = carve<T>(p, ox, oy, TX, TY + 1);
  Sm<T> fyp = carve<T>(p, ox, oy, TX, TY + 1);

  load_box(sdp.p, dp, g, k, ox - 3, oy - 3, TX + 6, TY + 6);
  load_box(spt.p, pt, g, k, ox - 3, oy - 3, TX + 6, TY + 6);
  if (CGRID) {
    load_box(sud.p, uin, g, k, ox - 1, oy - 3, TX + 2, TY + 7);
    load_box(svd.p, vin, g, k, ox - 3, oy - 1, TX + 7, TY + 2);
  } else {
    load_box(suc.p, uin, g, k, ox, oy - 3, TX + 1, TY + 6);
    load_box(svc.p, vin, g, k, ox - 3, oy, TX + 6, TY + 1);
  }
  __syncthreads();

  if (CGRID) {  // C-grid winds from the D-grid winds, mod_sw_dyn.f90:109-117
    for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 6); idx += NT) {
      int x = ox + idx % (TX + 1), y = oy - 3 + idx / (TX + 1);
      T ub = T(.5) * (sud(x, y) + sud(x - 1, y));
      suc(x, y) = T(.5) * (ub + T(.5) * (sud(x, y + 1) + sud(x - 1, y + 1)));
    }
    for (int idx = threadIdx.x; idx < (TX + 6) * (TY + 1); idx += NT) {
      int x = ox - 3 + idx % (TX + 6), y = oy + idx / (TX + 6);
      T vb = T(.5) * (svd(x, y) + svd(x, y - 1));
      svc(x, y) = T(.5) * (vb + T(.5) * (svd(x + 1, y) + svd(x + 1, y - 1)));
    }
    __syncthreads();
  }

  // inner sweeps (piecewise constant) and Laplacians
  // y-inner for the x-outer sweep: mod_sw_dyn.f90:142-155 (C), 470-482 (D)
  for (int idx = threadIdx.x; idx < (TX + 6) * TY; idx += NT) {
    int x = ox - 3 + idx % (TX + 6), y = oy + idx / (TX + 6);
    T cy0 = dtdx * svc(x, y), cy1 = dtdx * svc(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (svc(x, y + 1) - svc(x, y)));
    T f0 = (cy0 > T(0)) ? sdp(x, y - 1) : sdp(x, y);
    T f1 = (cy1 > T(0)) ? sdp(x, y) : sdp(x, y + 1);
    tyd(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
    f0 = (cy0 > T(0)) ? spt(x, y - 1) : spt(x, y);
    f1 = (cy1 > T(0)) ? spt(x, y) : spt(x, y + 1);
    typ(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
  }
  // x-inner for the y-outer sweep: mod_sw_dyn.f90:176-185 (C), 503-511 (D)
  for (int idx = threadIdx.x; idx < TX * (TY + 6); idx += NT) {
    int x = ox + idx % TX, y = oy - 3 + idx / TX;
    T cx0 = dtdx * suc(x, y), cx1 = dtdx * suc(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (suc(x + 1, y) - suc(x, y)));
    T f0 = (cx0 > T(0)) ? sdp(x - 1, y) : sdp(x, y);
    T f1 = (cx1 > T(0)) ? sdp(x, y) : sdp(x + 1, y);
    txd(x, y) = T(.5) * (sdp(x, y) + den * (sdp(x, y) - rA * (f1 - f0)));
    f0 = (cx0 > T(0)) ? spt(x - 1, y) : spt(x, y);
    f1 = (cx1 > T(0)) ? spt(x, y) : spt(x + 1, y);
    txp(x, y) = T(.5) * (spt(x, y) + den * (spt(x, y) - rA * (f1 - f0)));
  }
  {
    const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
    for (int idx = threadIdx.x; idx < (TX + 2) * (TY + 2); idx += NT) {
      int x = ox - 1 + idx % (TX + 2), y = oy - 1 + idx / (TX + 2);
      lpd(x, y) = T(-2.) * sdp(x, y) * rdxy + (sdp(x + 1, y) + sdp(x - 1, y)) * rdx2 +
                  (sdp(x, y + 1) + sdp(x, y - 1)) * rdy2;
      lpp(x, y) = T(-2.) * spt(x, y) * rdxy + (spt(x + 1, y) + spt(x - 1, y)) * rdx2 +
                  (spt(x, y + 1) + spt(x, y - 1)) * rdy2;
    }
  }
  __syncthreads();

  // outer sweeps (PPM): x fluxes on the tile's rows, y fluxes on its columns
  for (int idx = threadIdx.x; idx < (TX + 1) * TY; idx += NT) {
    int x = ox + idx % (TX + 1), y = oy + idx / (TX + 1);
    T cx = dtdx * suc(x, y);
    fxd(x, y) = flux<T, V>(tyd.ptr(x, y), 1, cx) * cx;
    fxp(x, y) = flux<T, V>(typ.ptr(x, y), 1, cx);
  }
  for (int idx = threadIdx.x; idx < TX * (TY + 1); idx += NT) {
    int x = ox + idx % TX, y = oy + idx / TX;
    T cy = dtdx * svc(x, y);
    fyd(x, y) = flux<T, V>(txd.ptr(x, y), TX, cy) * cy;
    fyp(x, y) = flux<T, V>(txp.ptr(x, y), TX, cy);
  }
  __syncthreads();

  // updates, mod_sw_dyn.f90:163-172,193-202,230-237,258-267 (C);
  // 490-499,519-528,555-562,582-591 (D)
  const int xhi = g.nx - 1 + hi, yhi = g.ny - 1 + hi;
  const T dxv = dtdx * T(c.vdx), dyv = dtdy * T(c.vdy), vdx = T(c.vdx), vdy = T(c.vdy);
  for (int idx = threadIdx.x; idx < TX * TY; idx += NT) {
    int x = ox + idx % TX, y = oy + idx / TX;
    if (x > xhi || y > yhi) continue;
    T d = sdp(x, y);
    T v = d - (fxd(x + 1, y) - fxd(x, y) + dxv * (lpd(x + 1, y) - T(2.) * lpd(x, y) + lpd(x - 1, y)));
    v = v - (fyd(x, y + 1) - fyd(x, y) + dyv * (lpd(x, y + 1) - T(2.) * lpd(x, y) + lpd(x, y - 1)));
    T q = d * spt(x, y) - (fxp(x + 1, y) * fxd(x + 1, y) - fxp(x, y) * fxd(x, y) +
                           vdx * ((lpp(x + 1, y) - lpp(x, y)) * fxd(x + 1, y) - (lpp(x, y) - lpp(x - 1, y)) * fxd(x, y)));
    q = q - (fyp(x, y + 1) * fyd(x, y + 1) - fyp(x, y) * fyd(x, y) +
             vdy * ((lpp(x, y + 1) - lpp(x, y)) * fyd(x, y + 1) - (lpp(x, y) - lpp(x, y - 1)) * fyd(x, y)));
    if (heat) q = q + dt * d * T(heat[g.at(x, y, k)]);
    q = q / v;
    long long o = g.at(x, y, k);
    dpo[o] = v;
    pto[o] = q;
    if (nonfinite) {
      bool inside = x >= 0 && x < g.nx && y >= 0 && y < g.ny;
      flag_nonfinite(nonfinite, inside && !(finite_(v) && finite_(q)));
    }
  }
}

// ====================================================== column pressure ====
// plev = ptop + suffix sum of dp from the model top, pkap = plev**kappa,
// hydrostatic gz from the bottom (src/mod_sw_dyn.f90:276-292 and 606-626).
// One thread per column over [lo, n-1+hi]^2; pkap of the column is kept in
// shared memory between the downward and the upward pass.
template <typename T>
__global__ void __launch_bounds__(64) k_column(Geom g, Consts c, const T* __restrict__ dpl, const T* __restrict__ ptl,
                                               double* __restrict__ pkap, double* __restrict__ gz, int lo, int hi,
                                               double* __restrict__ plev_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* spk = reinterpret_cast<double*>(smem);  // [L+1][64]
  const int w = g.nx - lo + hi;
  const int hgt = g.ny - lo + hi;
  const int col = blockIdx.x * 64 + threadIdx.x;
  if (col >= w * hgt) return;
  const int x = lo + col % w, y = lo + col / w;
  const long long o = g.at(x, y);
  const int L = g.L;
  double plev = c.ptop;
  spk[L * 64 + threadIdx.x] = c.pk_top;
  if (plev_out) plev_out[o + (long long)L * g.S] = plev;
  for (int k = L - 1; k >= 0; --k) {
    plev = plev + (double)dpl[o + (long long)k * g.S];
    if (plev_out) plev_out[o + (long long)k * g.S] = plev;
    double pk = atm_pow(plev, KAPPA);
    spk[k * 64 + threadIdx.x] = pk;
    pkap[o + (long long)k * g.S] = pk;
  }
  double z = gz[o];
  for (int k = 0; k < L; ++k) {
    z = z + CP_DRY * (double)ptl[o + (long long)k * g.S] * (spk[k * 64 + threadIdx.x] - spk[(k + 1) * 64 + threadIdx.x]);
    gz[o + (long long)(k + 1) * g.S] = z;
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

// ======================================================== C-grid momentum ==
// Second layer loop of the C-grid half step, src/mod_sw_dyn.f90:294-412:
// kinetic energy (PPM, with the A-grid winds of layer nlay that the first
// loop leaves in ua/va), vorticity, pressure-gradient force, and the
// vorticity-flux update of uc and vc on the interior.
template <typename T, int TX, int TY>
struct CMomSmem {
  static constexpr size_t bytes =
      2 * box_bytes<T>(TX + 7, TY + 7) + 2 * box_bytes<T>(TX + 3, TY + 3) + 4 * box_bytes<double>(TX + 1, TY + 1) +
      2 * box_bytes<T>(TX + 6, TY + 6) + 2 * box_bytes<T>(TX + 1, TY + 1) + box_bytes<T>(TX + 5, TY + 5) +
      box_bytes<T>(TX + 1, TY + 1) + box_bytes<T>(TX, TY + 5) + box_bytes<T>(TX + 5, TY) + box_bytes<T>(TX + 1, TY + 1);
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(NT) k_c_mom(Geom g, Consts c, const T* __restrict__ ud, const T* __restrict__ vd,
                                              const double* __restrict__ pkap, const double* __restrict__ gz,
                                              T* __restrict__ uc, T* __restrict__ vc) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* p = smem;
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy);

  Sm<T> sud = carve<T>(p, ox - 4, oy - 3, TX + 7, TY + 7);
  Sm<T> svd = carve<T>(p, ox - 3, oy - 4, TX + 7, TY + 7);
  Sm<T> udL = carve<T>(p, ox - 2, oy - 2, TX + 3, TY + 3);
  Sm<T> vdL = carve<T>(p, ox - 2, oy - 2, TX + 3, TY + 3);
  Sm<double> pk0 = carve<double>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<double> pk1 = carve<double>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<double> gz0 = carve<double>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<double> gz1 = carve<double>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> uc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> vc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> uaL = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> vaL = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> vor = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> ke = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> tU = carve<T>(p, ox, oy - 2, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 2, oy, TX + 5, TY);
  Sm<T> lap = carve<T>(p, ox, oy, TX + 1, TY + 1);

  load_box(sud.p, ud, g, k, ox - 4, oy - 3, TX + 7, TY + 7);
  load_box(svd.p, vd, g, k, ox - 3, oy - 4, TX + 7, TY + 7);
  load_box(udL.p, ud, g, L - 1, ox - 2, oy - 2, TX + 3, TY + 3);
  load_box(vdL.p, vd, g, L - 1, ox - 2, oy - 2, TX + 3, TY + 3);
  load_box(pk0.p, pkap, g, k, ox - 1, oy - 1, TX + 1, TY + 1);
  load_box(pk1.p, pkap, g, k + 1, ox - 1, oy - 1, TX + 1, TY + 1);
  load_box(gz0.p, gz, g, k, ox - 1, oy - 1, TX + 1, TY + 1);
  load_box(gz1.p, gz, g, k + 1, ox - 1, oy - 1, TX + 1, TY + 1);
  __syncthreads();

  // C-grid winds of this layer (first-loop values, mod_sw_dyn.f90:110-117)
  for (int idx = threadIdx.x; idx < (TX + 6) * (TY + 6); idx += NT) {
    int x = ox - 3 + idx % (TX + 6), y = oy - 3 + idx / (TX + 6);
    T ub = T(.5) * (sud(x, y) + sud(x - 1, y));
    uc1(x, y) = T(.5) * (ub + T(.5) * (sud(x, y + 1) + sud(x - 1, y + 1)));
    T vb = T(.5) * (svd(x, y) + svd(x, y - 1));
    vc1(x, y) = T(.5) * (vb + T(.5) * (svd(x + 1, y) + svd(x + 1, y - 1)));
  }
  // A-grid winds of layer nlay (mod_sw_dyn.f90:110-125 at k = nlay)
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox - 1 + idx % (TX + 1), y = oy - 1 + idx / (TX + 1);
    T ub = T(.5) * (udL(x, y) + udL(x - 1, y));
    T ucl = T(.5) * (ub + T(.5) * (udL(x, y + 1) + udL(x - 1, y + 1)));
    uaL(x, y) = T(.5) * (ucl + T(.25) * (udL(x + 1, y) + udL(x, y) + udL(x + 1, y + 1) + udL(x, y + 1)));
    T vb = T(.5) * (vdL(x, y) + vdL(x, y - 1));
    T vcl = T(.5) * (vb + T(.5) * (vdL(x + 1, y) + vdL(x + 1, y - 1)));
    vaL(x, y) = T(.5) * (vcl + T(.25) * (vdL(x, y + 1) + vdL(x, y) + vdL(x + 1, y + 1) + vdL(x + 1, y)));
  }
  __syncthreads();

  // vorticity (mod_sw_dyn.f90:319-323) and kinetic energy (:299-317)
  const T f = T(c.coriolis);
  for (int idx = threadIdx.x; idx < (TX + 5) * (TY + 5); idx += NT) {
    int x = ox - 2 + idx % (TX + 5), y = oy - 2 + idx / (TX + 5);
    vor(x, y) = f - (uc1(x, y) - uc1(x, y - 1)) * rdy + (vc1(x, y) - vc1(x - 1, y)) * rdx;
  }
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox - 1 + idx % (TX + 1), y = oy - 1 + idx / (TX + 1);
    // q(j) = vc(i, j+1) and q(i) = uc(i+1, j): the shifted sections of :300,310
    T fy = flux<T, PPM_UNC>(vc1.ptr(x, y + 1), TX + 6, dtdy * vaL(x, y));
    T kv = vaL(x, y) * fy;
    T fx = flux<T, PPM_UNC>(uc1.ptr(x + 1, y), 1, dtdx * uaL(x, y));
    ke(x, y) = T(.5) * (kv + uaL(x, y) * fx);
  }
  __syncthreads();

  // vorticity advection: inner sweeps and Laplacian (mod_sw_dyn.f90:344-367, 388-397)
  for (int idx = threadIdx.x; idx < TX * (TY + 5); idx += NT) {
    int x = ox + idx % TX, y = oy - 2 + idx / TX;
    // c(i) = cx(i-1, j): the shifted section cx(is+1:ie-3, j) of :355
    T c0 = dtdx * sud(x - 1, y), c1 = dtdx * sud(x, y);
    T den = T(1) / (T(1) - dtdx * (sud(x, y) - sud(x - 1, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }
  for (int idx = threadIdx.x; idx < (TX + 5) * TY; idx += NT) {
    int x = ox - 2 + idx % (TX + 5), y = oy + idx / (TX + 5);
    // c(j) = cy(i, j-1): the shifted section cy(i, js+1:je-3) of :390
    T c0 = dtdx * svd(x, y - 1), c1 = dtdx * svd(x, y);
    T den = T(1) / (T(1) - dtdy * (svd(x, y) - svd(x, y - 1)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }
  {
    const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
    for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
      int x = ox + idx % (TX + 1), y = oy + idx / (TX + 1);
      lap(x, y) = T(-2.) * vor(x, y) * rdxy + (vor(x + 1, y) + vor(x - 1, y)) * rdx2 +
                  (vor(x, y + 1) + vor(x, y - 1)) * rdy2;
    }
  }
  __syncthreads();

  // uc, vc updates (mod_sw_dyn.f90:369-381, 399-411) with the PGF (:325-339)
  const T vdx = T(c.vdx), vdy = T(c.vdy);
  for (int idx = threadIdx.x; idx < TX * TY; idx += NT) {
    int x = ox + idx % TX, y = oy + idx / TX;
    if (x >= g.nx || y >= g.ny) continue;
    double pgx = ((pk0(x, y) - pk1(x - 1, y)) * (gz0(x - 1, y) - gz1(x, y)) +
                  (pk0(x - 1, y) - pk1(x, y)) * (gz1(x - 1, y) - gz0(x, y))) /
                 (pk0(x, y) - pk1(x - 1, y) + pk0(x - 1, y) - pk1(x, y));
    double pgy = ((pk0(x, y) - pk1(x, y - 1)) * (gz0(x, y - 1) - gz1(x, y)) +
                  (pk0(x, y - 1) - pk1(x, y)) * (gz1(x, y - 1) - gz0(x, y))) /
                 (pk0(x, y) - pk1(x, y - 1) + pk0(x, y - 1) - pk1(x, y));
    // q(j) = tmp(i, j+1) (the section tmp(i, js+5:je-3) of :370)
    T fy = flux<T, PPM_UNC>(tU.ptr(x, y + 1), TX, dtdx * svd(x, y));
    T u = uc1(x, y) + dt * (svd(x, y) * fy + vdy * (lap(x, y + 1) - lap(x, y))) -
          dtdx * (ke(x, y) - ke(x - 1, y) - T(pgx));
    // q(i) = tmp(i+1, j) (the section tmp(is+5:ie-3, j) of :400)
    T fx = flux<T, PPM_UNC>(tV.ptr(x + 1, y), 1, dtdx * sud(x, y));
    T v = vc1(x, y) - dt * (sud(x, y) * fx + vdx * (lap(x + 1, y) - lap(x, y))) -
          dtdy * (ke(x, y) - ke(x, y - 1) - T(pgy));
    long long o = g.at(x, y, k);
    uc[o] = u;
    vc[o] = v;
  }
}

// ======================================================== D-grid momentum ==
// Third layer loop of the D-grid step, src/mod_sw_dyn.f90:634-771.  The
// B-grid winds ub/vb, the Courant numbers cx/cy and denom_x/denom_y are the
// ones the first loop leaves behind for layer nlay (:441-454), so they are
// built from uc/vc of layer nlay.
template <typename T, int TX, int TY>
struct DMomSmem {
  static constexpr size_t bytes =
      2 * box_bytes<T>(TX + 6, TY + 6) + box_bytes<T>(TX + 1, TY + 5) + box_bytes<T>(TX + 5, TY + 1) +
      4 * box_bytes<double>(TX + 1, TY + 1) + box_bytes<T>(TX + 5, TY + 5) + box_bytes<T>(TX + 5, TY + 5) +
      box_bytes<T>(TX + 3, TY + 3) + box_bytes<T>(TX + 1, TY + 1) * 4 + box_bytes<T>(TX, TY + 5) +
      box_bytes<T>(TX + 5, TY) + box_bytes<T>(TX + 1, TY + 1);
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(NT) k_d_mom(Geom g, Consts c, const T* __restrict__ ud, const T* __restrict__ vd,
                                              const T* __restrict__ uc, const T* __restrict__ vc,
                                              const double* __restrict__ pkapb, const double* __restrict__ gzb,
                                              T* __restrict__ udo, T* __restrict__ vdo, int* nonfinite) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* p = smem;
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy);

  Sm<T> sud = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> svd = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> ucL = carve<T>(p, ox, oy - 3, TX + 1, TY + 5);
  Sm<T> vcL = carve<T>(p, ox - 3, oy, TX + 5, TY + 1);
  Sm<double> pb0 = carve<double>(p, ox, oy, TX + 1, TY + 1);
  Sm<double> pb1 = carve<double>(p, ox, oy, TX + 1, TY + 1);
  Sm<double> gb0 = carve<double>(p, ox, oy, TX + 1, TY + 1);
  Sm<double> gb1 = carve<double>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> vor = carve<T>(p, ox - 3, oy - 3, TX + 5, TY + 5);
  Sm<T> dv0 = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> dv2 = carve<T>(p, ox - 1, oy - 1, TX + 3, TY + 3);
  Sm<T> dv4 = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> ubL = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> vbL = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> ke = carve<T>(p, ox, oy, TX + 1, TY + 1);
  Sm<T> tU = carve<T>(p, ox, oy - 3, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 3, oy, TX + 5, TY);
  Sm<T> lap = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);

  load_box(sud.p, ud, g, k, ox - 3, oy - 3, TX + 6, TY + 6);
  load_box(svd.p, vd, g, k, ox - 3, oy - 3, TX + 6, TY + 6);
  load_box(ucL.p, uc, g, L - 1, ox, oy - 3, TX + 1, TY + 5);
  load_box(vcL.p, vc, g, L - 1, ox - 3, oy, TX + 5, TY + 1);
  load_box(pb0.p, pkapb, g, k, ox, oy, TX + 1, TY + 1);
  load_box(pb1.p, pkapb, g, k + 1, ox, oy, TX + 1, TY + 1);
  load_box(gb0.p, gzb, g, k, ox, oy, TX + 1, TY + 1);
  load_box(gb1.p, gzb, g, k + 1, ox, oy, TX + 1, TY + 1);
  __syncthreads();

  const T f = T(c.coriolis);
  // vorticity (mod_sw_dyn.f90:659-663), divergence (:682-685), B-grid winds of layer nlay (:441-444)
  for (int idx = threadIdx.x; idx < (TX + 5) * (TY + 5); idx += NT) {
    int x = ox - 3 + idx % (TX + 5), y = oy - 3 + idx / (TX + 5);
    vor(x, y) = f - (sud(x, y + 1) - sud(x, y)) * rdy + (svd(x + 1, y) - svd(x, y)) * rdx;
    int xd = x + 1, yd = y + 1;
    dv0(xd, yd) = rdx * (sud(xd, yd) - sud(xd - 1, yd)) + rdy * (svd(xd, yd) - svd(xd, yd - 1));
  }
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox + idx % (TX + 1), y = oy + idx / (TX + 1);
    ubL(x, y) = T(.5) * (ucL(x, y) + ucL(x, y - 1));
    vbL(x, y) = T(.5) * (vcL(x, y) + vcL(x - 1, y));
  }
  __syncthreads();

  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  // kinetic energy with PPM_CONSTRAINED (:639-657)
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox + idx % (TX + 1), y = oy + idx / (TX + 1);
    T fy = flux<T, PPM_CON>(svd.ptr(x, y), TX + 6, dtdy * vbL(x, y));
    T kv = vbL(x, y) * fy;
    T fx = flux<T, PPM_CON>(sud.ptr(x, y), 1, dtdx * ubL(x, y));
    ke(x, y) = T(.5) * (kv + ubL(x, y) * fx);
  }
  // del^2 of the divergence (:688-692)
  for (int idx = threadIdx.x; idx < (TX + 3) * (TY + 3); idx += NT) {
    int x = ox - 1 + idx % (TX + 3), y = oy - 1 + idx / (TX + 3);
    dv2(x, y) = T(-2.) * dv0(x, y) * rdxy + (dv0(x + 1, y) + dv0(x - 1, y)) * rdx2 + (dv0(x, y + 1) + dv0(x, y - 1)) * rdy2;
  }
  // inner sweeps of the vorticity with the layer-nlay Courant numbers (:708-722, 744-753)
  for (int idx = threadIdx.x; idx < TX * (TY + 5); idx += NT) {
    int x = ox + idx % TX, y = oy - 3 + idx / TX;
    T c0 = dtdx * ucL(x, y), c1 = dtdx * ucL(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (ucL(x + 1, y) - ucL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }
  for (int idx = threadIdx.x; idx < (TX + 5) * TY; idx += NT) {
    int x = ox - 3 + idx % (TX + 5), y = oy + idx / (TX + 5);
    T c0 = dtdx * vcL(x, y), c1 = dtdx * vcL(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (vcL(x, y + 1) - vcL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox - 1 + idx % (TX + 1), y = oy - 1 + idx / (TX + 1);
    lap(x, y) = T(-2.) * vor(x, y) * rdxy + (vor(x + 1, y) + vor(x - 1, y)) * rdx2 + (vor(x, y + 1) + vor(x, y - 1)) * rdy2;
  }
  __syncthreads();
  // del^4 damping (:695-702)
  const T divdamp = T(c.divdamp);
  for (int idx = threadIdx.x; idx < (TX + 1) * (TY + 1); idx += NT) {
    int x = ox + idx % (TX + 1), y = oy + idx / (TX + 1);
    T d4 = T(-2.) * dv2(x, y) * rdxy + (dv2(x + 1, y) + dv2(x - 1, y)) * rdx2 + (dv2(x, y + 1) + dv2(x, y - 1)) * rdy2;
    dv4(x, y) = divdamp * d4;
  }
  __syncthreads();

  // ud, vd updates (:724-738, 755-769) with the B-grid PGF (:665-679)
  const T vdx = T(c.vdx), vdy = T(c.vdy);
  for (int idx = threadIdx.x; idx < TX * TY; idx += NT) {
    int x = ox + idx % TX, y = oy + idx / TX;
    if (x >= g.nx || y >= g.ny) continue;
    double pgx = ((pb0(x + 1, y) - pb1(x, y)) * (gb0(x, y) - gb1(x + 1, y)) +
                  (pb0(x, y) - pb1(x + 1, y)) * (gb1(x, y) - gb0(x + 1, y))) /
                 (pb0(x + 1, y) - pb1(x, y) + pb0(x, y) - pb1(x + 1, y));
    double pgy = ((pb0(x, y + 1) - pb1(x, y)) * (gb0(x, y) - gb1(x, y + 1)) +
                  (pb0(x, y) - pb1(x, y + 1)) * (gb1(x, y) - gb0(x, y + 1))) /
                 (pb0(x, y + 1) - pb1(x, y) + pb0(x, y) - pb1(x, y + 1));
    long long o = g.at(x, y, k);
    T fy = flux<T, PPM_CON>(tU.ptr(x, y), TX, dtdx * vcL(x, y));
    T u = sud(x, y) + dt * (vc[o] * fy + vdy * (lap(x, y) - lap(x, y - 1))) -
          dtdx * (ke(x + 1, y) - ke(x, y) - dv4(x + 1, y) + dv4(x, y) - T(pgx));
    T fx = flux<T, PPM_CON>(tV.ptr(x, y), 1, dtdx * ucL(x, y));
    T v = svd(x, y) - dt * (uc[o] * fx + vdx * (lap(x, y) - lap(x - 1, y))) -
          dtdy * (ke(x, y + 1) - ke(x, y) - dv4(x, y + 1) + dv4(x, y) - T(pgy));
    udo[o] = u;
    vdo[o] = v;
    flag_nonfinite(nonfinite, !(finite_(u) && finite_(v)));
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
