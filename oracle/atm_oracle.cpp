// CPU oracle (test infrastructure only) for the dynamical-core step of
// felix-goddard/atmosphere-model.  PARITY UNPINNED: see atm_oracle.h.
//
// Line-faithful FP64 restatement of
//   src/mod_sw_dyn.f90:80-1023   (C-grid half step, D-grid step, flux, ppm,
//                                 interpolate_to_corners, init_sw_dyn)
//   src/mod_remap.f90:27-388     (perform_vertical_remapping, remap_column,
//                                 vertical_ppm, allocate_remapping_arrays)
//   src/mod_sync.f90:67-217      (4/5-argument halo exchange, one image)
//   src/mod_fields.f90:69-106    (check_stability)
//   src/mod_constants.f90:8-14   (constants, default-real literals kept)
// Index ranges, array-section shifts, evaluation order and the single
// precision literals (7./12., 1./12., 2./3., R_dry) follow the Fortran.
// Build with -ffp-contract=off so that no multiply-add is fused.
#include "atm_oracle.h"
#include "dual.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>

#ifdef ORC_LIBM
// the C library's pow/log (the reference calls them through gfortran's **
// and log intrinsics); used to measure how sensitive results are to them
static inline double orc_pow_impl(double x, double y) { return std::pow(x, y); }
static inline double orc_log_impl(double x) { return std::log(x); }
#else
// the portable table-driven pow/log that the CUDA library evaluates
// bit-identically on the device
#include "../atmosphere-model_b200/csrc/atm_math.h"
static inline double orc_pow_impl(double x, double y) { return atm_pow(x, y); }
static inline double orc_log_impl(double x) { return atm_log(x); }
#endif
// x**y and log(x) of a dual number: d(x**y) = y x**y / x dx, d log x = dx / x
static inline Dual orc_pow_impl(const Dual& x, double y) {
  double p = orc_pow_impl(x.v, y);
  return Dual(p, y * p / x.v * x.d);
}
static inline Dual orc_log_impl(const Dual& x) { return Dual(orc_log_impl(x.v), x.d / x.v); }

namespace {

// src/mod_constants.f90:11 -- R_dry is a default-real literal
const double R_DRY = (double)287.052874f;
const double CP_DRY = 1005.0;
const double CV_DRY = CP_DRY - R_DRY;
const double KAPPA = R_DRY / CP_DRY;
// default-real constant expressions used in mod_sw_dyn.f90:933-953 and
// mod_remap.f90:86-100,243
const double C7_12 = (double)(7.0f / 12.0f);
const double C1_12 = (double)(1.0f / 12.0f);
const double C9_32 = (double)(9.0f / 32.0f);
const double C1_32 = (double)(1.0f / 32.0f);
const double C2_3 = (double)(2.0f / 3.0f);
const int HALO = 7;  // mod_tiles.f90:12

enum { PIECEWISE_CONSTANT = 0, PPM_UNCONSTRAINED = 1, PPM_CONSTRAINED = 2,
       PPM_NONNEGATIVE = 3 };  // mod_sw_dyn.f90:73-76

[[noreturn]] [[maybe_unused]] void die(const char* what, int a, int b, int c) {
  std::fprintf(stderr, "oracle: index out of bounds in %s (%d,%d,%d)\n", what, a, b, c);
  std::abort();
}

#ifdef ORC_BOUNDS
#define CHK(cond, what, a, b, c) do { if (!(cond)) die(what, a, b, c); } while (0)
#else
#define CHK(cond, what, a, b, c) do { } while (0)
#endif

template <class R>
struct A1 {
  std::vector<R> v;
  int lb = 0, ub = -1;
  void alloc(int l, int u) { lb = l; ub = u; v.assign((size_t)(u - l + 1), R(NAN)); }
  R& operator()(int i) {
    CHK(i >= lb && i <= ub, "A1", i, lb, ub);
    return v[(size_t)(i - lb)];
  }
};

template <class R>
struct A2 {
  std::vector<R> v;
  int i0 = 0, i1 = -1, j0 = 0, j1 = -1, ni = 0;
  void alloc(int a, int b, int c, int d) {
    i0 = a; i1 = b; j0 = c; j1 = d; ni = b - a + 1;
    v.assign((size_t)ni * (size_t)(d - c + 1), R(NAN));
  }
  void poison() { std::fill(v.begin(), v.end(), R(NAN)); }
  R& operator()(int i, int j) {
    CHK(i >= i0 && i <= i1 && j >= j0 && j <= j1, "A2", i, j, 0);
    return v[(size_t)(i - i0) + (size_t)(j - j0) * (size_t)ni];
  }
};

template <class R>
struct A3 {
  std::vector<R> v;
  int i0 = 0, i1 = -1, j0 = 0, j1 = -1, k0 = 1, k1 = 0, ni = 0, nj = 0;
  void alloc(int a, int b, int c, int d, int e, int f, R init = R(NAN)) {
    i0 = a; i1 = b; j0 = c; j1 = d; k0 = e; k1 = f;
    ni = b - a + 1; nj = d - c + 1;
    v.assign((size_t)ni * nj * (size_t)(f - e + 1), init);
  }
  R& operator()(int i, int j, int k) {
    CHK(i >= i0 && i <= i1 && j >= j0 && j <= j1 && k >= k0 && k <= k1, "A3", i, j, k);
    return v[(size_t)(i - i0) + (size_t)ni * ((size_t)(j - j0) + (size_t)nj * (size_t)(k - k0))];
  }
  ptrdiff_t sj() const { return ni; }
};

// A 1-D window onto an array section, indexed with the callee's bounds
// (Fortran passes e.g. vc(i, js+3:je-1, k) to a dummy q(js+2:je-2)).
template <class R>
struct V {
  R* p;
  ptrdiff_t s;
  int lb;
  R& operator()(int i) const { return p[(ptrdiff_t)(i - lb) * s]; }
};

template <class R> inline V<R> row(A2<R>& a, int ifirst, int j, int lb) { return V<R>{&a(ifirst, j), 1, lb}; }
template <class R> inline V<R> col(A2<R>& a, int i, int jfirst, int lb) { return V<R>{&a(i, jfirst), (ptrdiff_t)a.ni, lb}; }
template <class R> inline V<R> row3(A3<R>& a, int ifirst, int j, int k, int lb) { return V<R>{&a(ifirst, j, k), 1, lb}; }
template <class R> inline V<R> col3(A3<R>& a, int i, int jfirst, int k, int lb) { return V<R>{&a(i, jfirst, k), a.sj(), lb}; }

template <class R> inline R fmax3(const R& a, const R& b, const R& c) { return std::max(std::max(a, b), c); }
template <class R> inline R fmin3(const R& a, const R& b, const R& c) { return std::min(std::min(a, b), c); }

// The module-level scratch of mod_sw_dyn (mod_sw_dyn.f90:29-71).  In the
// serial mode there is one instance shared by every layer, exactly like the
// Fortran module variables; the layer-parallel mode gives each thread one.
template <class R>
struct Scratch {
  A2<R> vorticity, kinetic_energy, divergence, laplacian, pgfx, pgfy;
  A2<R> ua, va, ub, vb, tmp, cx, cy, dpfx, dpfy, denom_x, denom_y;
  A1<R> fx, fy, edge_L, edge_R, dqi, dqi_mono, ctmp;
  void alloc(int is, int ie, int js, int je) {
    A2<R>* a2[] = {&vorticity, &kinetic_energy, &divergence, &laplacian, &pgfx, &pgfy,
                &ua, &va, &ub, &vb, &tmp, &cx, &cy, &dpfx, &dpfy, &denom_x, &denom_y};
    for (A2<R>* a : a2) a->alloc(is, ie, js, je);
    int lo = std::min(is, js), hi = std::max(ie, je);
    A1<R>* a1[] = {&fx, &fy, &edge_L, &edge_R, &dqi, &dqi_mono, &ctmp};
    for (A1<R>* a : a1) a->alloc(lo, hi);
  }
  void poison() {
    A2<R>* a2[] = {&vorticity, &kinetic_energy, &divergence, &laplacian, &pgfx, &pgfy,
                &tmp, &dpfx, &dpfy};
    for (A2<R>* a : a2) a->poison();
  }
  void poison_courant() {
    A2<R>* a2[] = {&cx, &cy, &denom_x, &denom_y};
    for (A2<R>* a : a2) a->poison();
  }
  void poison_winds() {
    A2<R>* a2[] = {&ua, &va, &ub, &vb};
    for (A2<R>* a : a2) a->poison();
    poison_courant();
  }
};

// mod_sw_dyn.f90:848-919
template <class R>
void ppm(Scratch<R>& sc, const V<R>& q, int isl, int iel, int variant) {
  A1<R>& dqi = sc.dqi;
  A1<R>& dqi_mono = sc.dqi_mono;
  A1<R>& edge_L = sc.edge_L;
  A1<R>& edge_R = sc.edge_R;
  for (int i = isl + 1; i <= iel - 1; ++i) {
    dqi(i) = (q(i + 1) - q(i - 1)) / 4.;
    R dqi_max = fmax3(q(i + 1), q(i), q(i - 1)) - q(i);
    R dqi_min = q(i) - fmin3(q(i + 1), q(i), q(i - 1));
    dqi_mono(i) = copysign_(fmin3(fabs_(dqi(i)), dqi_min, dqi_max), dqi(i));
  }
  for (int i = isl + 2; i <= iel - 2; ++i) {
    edge_L(i) = (q(i - 1) - q(i)) / 2. + (dqi_mono(i - 1) - dqi_mono(i)) / 3.;
    edge_R(i) = (q(i + 1) - q(i)) / 2. + (dqi_mono(i) - dqi_mono(i + 1)) / 3.;
    if (variant == PPM_CONSTRAINED || variant == PPM_NONNEGATIVE) {
      edge_L(i) = -copysign_(std::min(R(2. * fabs_(dqi(i))), fabs_(edge_L(i))), dqi(i));
      edge_R(i) = +copysign_(std::min(R(2. * fabs_(dqi(i))), fabs_(edge_R(i))), dqi(i));
      if (variant == PPM_NONNEGATIVE) {
        edge_L(i) = std::max(edge_L(i), R(-q(i)));
        edge_R(i) = std::max(edge_R(i), R(-q(i)));
        R a = edge_R(i) - edge_L(i);
        R b = -3. * (edge_R(i) + edge_L(i));
        if ((fabs_(a) < -b) && (q(i) + a * a / (4. * b) + b / 12. < 0.)) {
          if (edge_L(i) * edge_R(i) > 0.) {
            edge_L(i) = 0.;
            edge_R(i) = 0.;
          } else if (edge_L(i) > edge_R(i)) {
            edge_L(i) = 2. * fabs_(edge_R(i));
          } else {
            edge_R(i) = 2. * fabs_(edge_L(i));
          }
        }
      }
    }
  }
}

// mod_sw_dyn.f90:781-846
template <class R>
void flux(Scratch<R>& sc, const V<R>& f, const V<R>& q, const V<R>& c, int isl, int iel, int variant) {
  if (variant == PPM_UNCONSTRAINED || variant == PPM_CONSTRAINED || variant == PPM_NONNEGATIVE) {
    ppm(sc, q, isl, iel, variant);
    A1<R>& edge_L = sc.edge_L;
    A1<R>& edge_R = sc.edge_R;
    for (int i = isl + 3; i <= iel - 2; ++i) {
      R s = fabs_(c(i));
      R k1 = (1. - 2. * s) * (1. - s);
      R k2 = s * (s - 1.);
      if (variant == PPM_CONSTRAINED &&
          (3. * fabs_(edge_L(i) + edge_R(i)) > fabs_(edge_L(i) - edge_R(i))) &&
          (3. * fabs_(edge_L(i - 1) + edge_R(i - 1)) > fabs_(edge_L(i - 1) - edge_R(i - 1)))) {
        if (c(i) > 0.) f(i) = q(i - 1);
        else f(i) = q(i);
      } else {
        if (c(i) > 0.) f(i) = q(i - 1) + k1 * edge_R(i - 1) + k2 * edge_L(i - 1);
        else f(i) = q(i) + k1 * edge_L(i) + k2 * edge_R(i);
      }
    }
  } else {
    for (int i = isl + 1; i <= iel; ++i) {
      if (c(i) > 0.) f(i) = q(i - 1);
      else f(i) = q(i);
    }
  }
}

// Fortran passes the expression dtdy*va(i, js+2:je-2) as a temporary array.
template <class R>
V<R> scaled_temp(Scratch<R>& sc, double a, const V<R>& src, int lo, int hi) {
  for (int i = lo; i <= hi; ++i) sc.ctmp(i) = a * src(i);
  return V<R>{&sc.ctmp(lo), 1, lo};
}

// mod_sw_dyn.f90:921-956; out/q are windows with bounds (isl:iel, jsl:jel)
template <class R>
struct W2 {
  R* p;
  ptrdiff_t sj;
  int i0, j0;
  R& operator()(int i, int j) const { return p[(ptrdiff_t)(i - i0) + (ptrdiff_t)(j - j0) * sj]; }
};
template <class R>
void interpolate_to_corners(const W2<R>& out, const W2<R>& q, int isl, int iel, int jsl, int jel) {
  int ni = iel - isl + 1;
  std::vector<R> t((size_t)ni * (size_t)(jel - jsl + 1), R(NAN));
  W2<R> tmpl{t.data(), ni, isl, jsl};
  for (int j = jsl; j <= jel; ++j)
    for (int i = isl + 2; i <= iel - 1; ++i)
      tmpl(i, j) = C7_12 * (q(i, j) + q(i - 1, j)) - C1_12 * (q(i + 1, j) + q(i - 2, j));
  for (int j = jsl + 2; j <= jel - 1; ++j)
    for (int i = isl + 2; i <= iel - 1; ++i)
      out(i, j) = C9_32 * (tmpl(i, j) + tmpl(i, j - 1)) - C1_32 * (tmpl(i, j + 1) + tmpl(i, j - 2));
  for (int j = jsl + 2; j <= jel - 1; ++j)
    for (int i = isl; i <= iel; ++i)
      tmpl(i, j) = C7_12 * (q(i, j) + q(i, j - 1)) - C1_12 * (q(i, j + 1) + q(i, j - 2));
  for (int j = jsl + 2; j <= jel - 1; ++j)
    for (int i = isl + 2; i <= iel - 1; ++i)
      out(i, j) = out(i, j) + C9_32 * (tmpl(i, j) + tmpl(i - 1, j)) - C1_32 * (tmpl(i + 1, j) + tmpl(i - 2, j));
}

template <class R>
W2<R> w3(A3<R>& a, int i0, int j0, int k) { return W2<R>{&a(i0, j0, k), a.sj(), i0, j0}; }

}  // namespace

template <class R>
struct StateT {
  int nx, ny, nlay;
  double dx, dy;
  int is, ie, js, je, isd, ied, jsd, jed;
  double gravity, coriolis, divergence_damping, vorticity_damping;
  double rdx, rdx2, rdy, rdy2, rdx2rdy2, rA;
  double divdamp_coeff, vortdamp_xcoeff, vortdamp_ycoeff;
  A1<double> coord_Ak, coord_Bk;
  // mod_fields
  A3<R> dp, pt, ud, vd, plev, pkap, playkap, gz, net_flux;
  // mod_sw_dyn module arrays
  A3<R> dpc, ptc, uc, vc, heating_rate, pkapb, gzb;
  Scratch<R> sc;
  // mod_physics module arrays (tendencies on isd-2:ied+2, A-grid winds on
  // is:ie) and the surface temperature ts (mod_fields.f90:51), 2-D arrays
  // held as one-level 3-D arrays
  A3<R> ts, ts_tend, dp_tend, pt_tend, u_tend, v_tend, ua, va;
  // mod_remap module arrays
  double top_pressure;
  A3<R> u_remap, v_remap, pt_remap, target_plev, target_pkap, target_playkap;
  // mod_sync buffers (single image: every neighbour is this image)
  std::vector<R> edge_buffer, corner_buffer;
  int nthreads = 1;
  bool poison = false;
  int32_t* trace = nullptr;
};

struct orc_state : StateT<double> {};
struct orc_tlm : StateT<Dual> {};

namespace {

// ---------------------------------------------------------------- halo ----
// mod_sync.f90:109-135 and 164-190 with neighbours(:) == this_image()
template <class R>
struct Halo {
  StateT<R>* s;
  size_t nb;  // max(nx, ny)
  R& eb(int a, int w, int k, int n, int idx) {
    size_t L1 = (size_t)s->nlay + 1;
    return s->edge_buffer[(size_t)(a - 1) + nb * ((size_t)(w - 1) + HALO * ((size_t)(k - 1) + L1 * ((size_t)(n - 1) + 4 * (size_t)(idx - 1))))];
  }
  R& cb(int a, int w, int k, int n, int idx) {
    size_t L1 = (size_t)s->nlay + 1;
    return s->corner_buffer[(size_t)(a - 1) + HALO * ((size_t)(w - 1) + HALO * ((size_t)(k - 1) + L1 * ((size_t)(n - 1) + 4 * (size_t)(idx - 1))))];
  }
  void to_buffer(A3<R>& q, int idx, int kmax) {
    int isd = s->isd, ied = s->ied, jsd = s->jsd, jed = s->jed;
    for (int i = 0; i <= HALO - 1; ++i)
      for (int k = 1; k <= kmax; ++k) {
        for (int j = jsd; j <= jed; ++j) {
          eb(j, i + 1, k, 1, idx) = q(isd + i, j, k);
          eb(j, i + 1, k, 2, idx) = q(ied - i, j, k);
        }
        for (int ii = isd; ii <= ied; ++ii) {
          eb(ii, i + 1, k, 3, idx) = q(ii, jsd + i, k);
          eb(ii, i + 1, k, 4, idx) = q(ii, jed - i, k);
        }
        for (int m = 1; m <= HALO; ++m) {
          cb(i + 1, m, k, 1, idx) = q(isd + i, jed - HALO + m, k);
          cb(i + 1, m, k, 2, idx) = q(ied - i, jed - HALO + m, k);
          cb(i + 1, m, k, 3, idx) = q(isd + i, jsd + m - 1, k);
          cb(i + 1, m, k, 4, idx) = q(ied - i, jsd + m - 1, k);
        }
      }
  }
  void from_buffer(A3<R>& q, int idx, int kmax) {
    int isd = s->isd, ied = s->ied, jsd = s->jsd, jed = s->jed, js = s->js;
    for (int i = 1; i <= HALO; ++i)
      for (int k = 1; k <= kmax; ++k) {
        for (int j = jsd; j <= jed; ++j) {
          q(isd - i, j, k) = eb(j, i, k, 2, idx);
          q(ied + i, j, k) = eb(j, i, k, 1, idx);
        }
        for (int ii = isd; ii <= ied; ++ii) {
          q(ii, jsd - i, k) = eb(ii, i, k, 4, idx);
          q(ii, jed + i, k) = eb(ii, i, k, 3, idx);
        }
        for (int m = 1; m <= HALO; ++m) {
          q(isd - i, jed + m, k) = cb(i, m, k, 4, idx);
          q(ied + i, jed + m, k) = cb(i, m, k, 3, idx);
          q(isd - i, js + m - 1, k) = cb(i, m, k, 2, idx);
          q(ied + i, js + m - 1, k) = cb(i, m, k, 1, idx);
        }
      }
  }
};

template <class R>
void halo_exchange(StateT<R>* s, A3<R>* const* f, int n, int kmax) {
  Halo<R> h{s, (size_t)std::max(s->nx, s->ny)};
  for (int a = 0; a < n; ++a) h.to_buffer(*f[a], a + 1, kmax);
  for (int a = 0; a < n; ++a) h.from_buffer(*f[a], a + 1, kmax);
}

// ------------------------------------------------------------ C grid ----
// first layer loop body, mod_sw_dyn.f90:99-268
template <class R>
void c_winds(StateT<R>* s, Scratch<R>& sc, int k) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  for (int j = js + 1; j <= je - 1; ++j)
    for (int i = is + 1; i <= ie - 1; ++i) {
      sc.ub(i, j) = .5 * (s->ud(i, j, k) + s->ud(i - 1, j, k));
      sc.vb(i, j) = .5 * (s->vd(i, j, k) + s->vd(i, j - 1, k));
      s->uc(i, j, k) = .5 * (sc.ub(i, j) + .5 * (s->ud(i, j + 1, k) + s->ud(i - 1, j + 1, k)));
      s->vc(i, j, k) = .5 * (sc.vb(i, j) + .5 * (s->vd(i + 1, j, k) + s->vd(i + 1, j - 1, k)));
      sc.ua(i, j) = .5 * (s->uc(i, j, k) + .25 * (s->ud(i + 1, j, k) + s->ud(i, j, k) +
                                                   s->ud(i + 1, j + 1, k) + s->ud(i, j + 1, k)));
      sc.va(i, j) = .5 * (s->vc(i, j, k) + .25 * (s->vd(i, j + 1, k) + s->vd(i, j, k) +
                                                   s->vd(i + 1, j + 1, k) + s->vd(i + 1, j, k)));
    }
}

template <class R>
void c_layer1(StateT<R>* s, Scratch<R>& sc, int k, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  double dtdx = dt * s->rdx, dtdy = dt * s->rdy, rA = s->rA;
  A3<R> &dp = s->dp, &pt = s->pt, &uc = s->uc, &vc = s->vc, &dpc = s->dpc, &ptc = s->ptc;
  A3<R> &pkap = s->pkap;
  if (s->poison) { sc.poison(); sc.poison_winds(); }

  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      s->playkap(i, j, k) = (pkap(i, j, k + 1) - pkap(i, j, k)) / orc_log_impl(pkap(i, j, k + 1) / pkap(i, j, k));
      s->heating_rate(i, j, k) = (s->net_flux(i, j, k + 1) - s->net_flux(i, j, k)) /
                                 (CP_DRY * dp(i, j, k) / s->gravity) / s->playkap(i, j, k);
    }

  c_winds(s, sc, k);

  for (int j = js + 1; j <= je - 1; ++j)
    for (int i = is + 1; i <= ie - 1; ++i) {
      sc.cx(i, j) = dtdx * uc(i, j, k);
      sc.cy(i, j) = dtdx * vc(i, j, k);
    }
  for (int j = js + 2; j <= je - 2; ++j)
    for (int i = is + 2; i <= ie - 2; ++i) {
      sc.denom_x(i, j) = 1. / (1. - dtdx * (uc(i + 1, j, k) - uc(i, j, k)));
      sc.denom_y(i, j) = 1. / (1. - dtdy * (vc(i, j + 1, k) - vc(i, j, k)));
    }

  A1<R> &fx = sc.fx, &fy = sc.fy;
  A2<R> &tmp = sc.tmp, &lap = sc.laplacian, &dpfx = sc.dpfx, &dpfy = sc.dpfy;
  V<R> fxv{&fx.v[0], 1, fx.lb}, fyv{&fy.v[0], 1, fy.lb};

  // ---- dpc
  for (int i = is + 2; i <= ie - 2; ++i) {
    flux(sc, fyv, col3(dp, i, js + 1, k, js + 1), col(sc.cy, i, js + 1, js + 1), js + 1, je - 1, PIECEWISE_CONSTANT);
    for (int j = js + 2; j <= je - 2; ++j) {
      tmp(i, j) = .5 * (dp(i, j, k) + sc.denom_y(i, j) * (dp(i, j, k) - rA * (fy(j + 1) - fy(j))));
      lap(i, j) = -2. * dp(i, j, k) * s->rdx2rdy2 + (dp(i + 1, j, k) + dp(i - 1, j, k)) * s->rdx2 +
                  (dp(i, j + 1, k) + dp(i, j - 1, k)) * s->rdy2;
    }
  }
  for (int j = js + 5; j <= je - 5; ++j) {
    flux(sc, fxv, row(tmp, is + 2, j, is + 2), row(sc.cx, is + 2, j, is + 2), is + 2, ie - 2, PPM_UNCONSTRAINED);
    dpfx(is + 5, j) = fx(is + 5) * sc.cx(is + 5, j);
    for (int i = is + 5; i <= ie - 5; ++i) {
      dpfx(i + 1, j) = fx(i + 1) * sc.cx(i + 1, j);
      dpc(i, j, k) = dp(i, j, k) - (dpfx(i + 1, j) - dpfx(i, j) +
                                    dtdx * s->vortdamp_xcoeff * (lap(i + 1, j) - 2. * lap(i, j) + lap(i - 1, j)));
    }
  }
  for (int j = js + 2; j <= je - 2; ++j) {
    flux(sc, fxv, row3(dp, is + 1, j, k, is + 1), row(sc.cx, is + 1, j, is + 1), is + 1, ie - 1, PIECEWISE_CONSTANT);
    for (int i = is + 2; i <= ie - 2; ++i)
      tmp(i, j) = .5 * (dp(i, j, k) + sc.denom_x(i, j) * (dp(i, j, k) - rA * (fx(i + 1) - fx(i))));
  }
  for (int i = is + 5; i <= ie - 5; ++i) {
    flux(sc, fyv, col(tmp, i, js + 2, js + 2), col(sc.cy, i, js + 2, js + 2), js + 2, je - 2, PPM_UNCONSTRAINED);
    dpfy(i, js + 5) = fy(js + 5) * sc.cy(i, js + 5);
    for (int j = js + 5; j <= je - 5; ++j) {
      dpfy(i, j + 1) = fy(j + 1) * sc.cy(i, j + 1);
      dpc(i, j, k) = dpc(i, j, k) - (dpfy(i, j + 1) - dpfy(i, j) +
                                     dtdy * s->vortdamp_ycoeff * (lap(i, j + 1) - 2. * lap(i, j) + lap(i, j - 1)));
    }
  }

  // ---- ptc
  for (int i = is + 2; i <= ie - 2; ++i) {
    flux(sc, fyv, col3(pt, i, js + 1, k, js + 1), col(sc.cy, i, js + 1, js + 1), js + 1, je - 1, PIECEWISE_CONSTANT);
    for (int j = js + 2; j <= je - 2; ++j) {
      tmp(i, j) = .5 * (pt(i, j, k) + sc.denom_y(i, j) * (pt(i, j, k) - rA * (fy(j + 1) - fy(j))));
      lap(i, j) = -2. * pt(i, j, k) * s->rdx2rdy2 + (pt(i + 1, j, k) + pt(i - 1, j, k)) * s->rdx2 +
                  (pt(i, j + 1, k) + pt(i, j - 1, k)) * s->rdy2;
    }
  }
  for (int j = js + 5; j <= je - 5; ++j) {
    flux(sc, fxv, row(tmp, is + 2, j, is + 2), row(sc.cx, is + 2, j, is + 2), is + 2, ie - 2, PPM_UNCONSTRAINED);
    for (int i = is + 5; i <= ie - 5; ++i)
      ptc(i, j, k) = dp(i, j, k) * pt(i, j, k) -
                     (fx(i + 1) * dpfx(i + 1, j) - fx(i) * dpfx(i, j) +
                      s->vortdamp_xcoeff * ((lap(i + 1, j) - lap(i, j)) * dpfx(i + 1, j) -
                                            (lap(i, j) - lap(i - 1, j)) * dpfx(i, j)));
  }
  for (int j = js + 2; j <= je - 2; ++j) {
    flux(sc, fxv, row3(pt, is + 1, j, k, is + 1), row(sc.cx, is + 1, j, is + 1), is + 1, ie - 1, PIECEWISE_CONSTANT);
    for (int i = is + 2; i <= ie - 2; ++i)
      tmp(i, j) = .5 * (pt(i, j, k) + sc.denom_x(i, j) * (pt(i, j, k) - rA * (fx(i + 1) - fx(i))));
  }
  for (int i = is + 5; i <= ie - 5; ++i) {
    flux(sc, fyv, col(tmp, i, js + 2, js + 2), col(sc.cy, i, js + 2, js + 2), js + 2, je - 2, PPM_UNCONSTRAINED);
    for (int j = js + 5; j <= je - 5; ++j)
      ptc(i, j, k) = (ptc(i, j, k) -
                      (fy(j + 1) * dpfy(i, j + 1) - fy(j) * dpfy(i, j) +
                       s->vortdamp_ycoeff * ((lap(i, j + 1) - lap(i, j)) * dpfy(i, j + 1) -
                                             (lap(i, j) - lap(i, j - 1)) * dpfy(i, j))) +
                      dt * dp(i, j, k) * s->heating_rate(i, j, k)) /
                     dpc(i, j, k);
  }
}

// second layer loop body, mod_sw_dyn.f90:296-412.  ua/va are the module
// arrays left by the LAST iteration of the first loop (layer nlay).
template <class R>
void c_layer2(StateT<R>* s, Scratch<R>& sc, int k, double dt, A2<R>& ua, A2<R>& va) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  double dtdx = dt * s->rdx, dtdy = dt * s->rdy, rA = s->rA;
  A3<R> &ud = s->ud, &vd = s->vd, &uc = s->uc, &vc = s->vc, &pkap = s->pkap, &gz = s->gz;
  A1<R> &fx = sc.fx, &fy = sc.fy;
  A2<R> &tmp = sc.tmp, &lap = sc.laplacian, &ke = sc.kinetic_energy, &vort = sc.vorticity;
  V<R> fxv{&fx.v[0], 1, fx.lb}, fyv{&fy.v[0], 1, fy.lb};
  if (s->poison) { sc.poison(); sc.poison_courant(); }

  for (int i = is + 5; i <= ie - 5; ++i) {
    V<R> cv = scaled_temp(sc, dtdy, col(va, i, js + 2, js + 2), js + 2, je - 2);
    flux(sc, fyv, col3(vc, i, js + 3, k, js + 2), cv, js + 2, je - 2, PPM_UNCONSTRAINED);
    for (int j = js + 5; j <= je - 5; ++j) ke(i, j) = va(i, j) * fy(j);
  }
  for (int j = js + 5; j <= je - 5; ++j) {
    V<R> cv = scaled_temp(sc, dtdx, row(ua, is + 2, j, is + 2), is + 2, ie - 2);
    flux(sc, fxv, row3(uc, is + 3, j, k, is + 2), cv, is + 2, ie - 2, PPM_UNCONSTRAINED);
    for (int i = is + 5; i <= ie - 5; ++i) ke(i, j) = .5 * (ke(i, j) + ua(i, j) * fx(i));
  }
  for (int j = js + 2; j <= je - 2; ++j)
    for (int i = is + 2; i <= ie - 2; ++i)
      vort(i, j) = s->coriolis - (uc(i, j, k) - uc(i, j - 1, k)) * s->rdy + (vc(i, j, k) - vc(i - 1, j, k)) * s->rdx;
  for (int j = js + 7; j <= je - 7; ++j)
    for (int i = is + 7; i <= ie - 7; ++i) {
      sc.pgfx(i, j) = ((pkap(i, j, k) - pkap(i - 1, j, k + 1)) * (gz(i - 1, j, k) - gz(i, j, k + 1)) +
                       (pkap(i - 1, j, k) - pkap(i, j, k + 1)) * (gz(i - 1, j, k + 1) - gz(i, j, k))) /
                      (pkap(i, j, k) - pkap(i - 1, j, k + 1) + pkap(i - 1, j, k) - pkap(i, j, k + 1));
      sc.pgfy(i, j) = ((pkap(i, j, k) - pkap(i, j - 1, k + 1)) * (gz(i, j - 1, k) - gz(i, j, k + 1)) +
                       (pkap(i, j - 1, k) - pkap(i, j, k + 1)) * (gz(i, j - 1, k + 1) - gz(i, j, k))) /
                      (pkap(i, j, k) - pkap(i, j - 1, k + 1) + pkap(i, j - 1, k) - pkap(i, j, k + 1));
    }
  for (int j = js + 1; j <= je - 1; ++j)
    for (int i = is + 1; i <= ie - 1; ++i) {
      sc.denom_x(i, j) = 1. / (1. - dtdx * (ud(i, j, k) - ud(i - 1, j, k)));
      sc.denom_y(i, j) = 1. / (1. - dtdy * (vd(i, j, k) - vd(i, j - 1, k)));
      sc.cx(i, j) = dtdx * ud(i, j, k);
      sc.cy(i, j) = dtdx * vd(i, j, k);
    }
  // uc
  for (int j = js + 3; j <= je - 3; ++j) {
    flux(sc, fxv, row(vort, is + 2, j, is + 2), row(sc.cx, is + 1, j, is + 2), is + 2, ie - 2, PIECEWISE_CONSTANT);
    for (int i = is + 3; i <= ie - 3; ++i) {
      tmp(i, j) = .5 * (vort(i, j) + sc.denom_x(i, j) * (vort(i, j) - rA * (fx(i + 1) - fx(i))));
      lap(i, j) = -2. * vort(i, j) * s->rdx2rdy2 + (vort(i + 1, j) + vort(i - 1, j)) * s->rdx2 +
                  (vort(i, j + 1) + vort(i, j - 1)) * s->rdy2;
    }
  }
  for (int i = is + 7; i <= ie - 7; ++i) {
    flux(sc, fyv, col(tmp, i, js + 5, js + 4), col(sc.cy, i, js + 4, js + 4), js + 4, je - 4, PPM_UNCONSTRAINED);
    for (int j = js + 7; j <= je - 7; ++j)
      uc(i, j, k) = uc(i, j, k) + dt * (vd(i, j, k) * fy(j) + s->vortdamp_ycoeff * (lap(i, j + 1) - lap(i, j))) -
                    dtdx * (ke(i, j) - ke(i - 1, j) - sc.pgfx(i, j));
  }
  // vc
  for (int i = is + 3; i <= ie - 3; ++i) {
    flux(sc, fyv, col(vort, i, js + 2, js + 2), col(sc.cy, i, js + 1, js + 2), js + 2, je - 2, PIECEWISE_CONSTANT);
    for (int j = js + 3; j <= je - 3; ++j)
      tmp(i, j) = .5 * (vort(i, j) + sc.denom_y(i, j) * (vort(i, j) - rA * (fy(j + 1) - fy(j))));
  }
  for (int j = js + 7; j <= je - 7; ++j) {
    flux(sc, fxv, row(tmp, is + 5, j, is + 4), row(sc.cx, is + 4, j, is + 4), is + 4, ie - 4, PPM_UNCONSTRAINED);
    for (int i = is + 7; i <= ie - 7; ++i)
      vc(i, j, k) = vc(i, j, k) - dt * (ud(i, j, k) * fx(i) + s->vortdamp_xcoeff * (lap(i + 1, j) - lap(i, j))) -
                    dtdy * (ke(i, j) - ke(i, j - 1) - sc.pgfy(i, j));
  }
}

// Dynamic-schedule parallel loop over [lo, hi] on std::threads; body(x, t)
// receives the worker index t so that it can use thread-private scratch.
template <class F>
void par_for(int nthreads, int lo, int hi, F&& body) {
  if (nthreads <= 1 || hi - lo < 1) {
    for (int x = lo; x <= hi; ++x) body(x, 0);
    return;
  }
  std::atomic<int> next(lo);
  auto work = [&](int t) {
    for (int x = next.fetch_add(1); x <= hi; x = next.fetch_add(1)) body(x, t);
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; ++t) pool.emplace_back(work, t);
  work(0);
  for (std::thread& th : pool) th.join();
}

template <class R>
std::vector<Scratch<R>> make_scratch(StateT<R>* s) {
  std::vector<Scratch<R>> t((size_t)std::max(1, s->nthreads));
  for (Scratch<R>& x : t) x.alloc(s->is, s->ie, s->js, s->je);
  return t;
}

// mod_sw_dyn.f90:80-416
template <class R>
void cgrid_dynamics_step(StateT<R>* s, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je, L = s->nlay;
  par_for(s->nthreads, js, je, [&](int j, int t) { (void)t;
    for (int k = L; k >= 1; --k)
      for (int i = is; i <= ie; ++i) {
        s->plev(i, j, k) = s->plev(i, j, k + 1) + s->dp(i, j, k);
        s->pkap(i, j, k) = orc_pow_impl(s->plev(i, j, k), KAPPA);
      }
  });
  if (s->nthreads <= 1) {
    for (int k = 1; k <= L; ++k) c_layer1(s, s->sc, k, dt);
  } else {
    std::vector<Scratch<R>> ts = make_scratch(s);
    par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t; c_layer1(s, ts[(size_t)t], k, dt); });
    c_winds(s, s->sc, L);  // the module ua/va keep layer nlay
  }
  par_for(s->nthreads, js + 5, je - 5, [&](int j, int t) { (void)t;
    for (int k = L; k >= 1; --k)
      for (int i = is + 5; i <= ie - 5; ++i) {
        s->plev(i, j, k) = s->plev(i, j, k + 1) + s->dpc(i, j, k);
        s->pkap(i, j, k) = orc_pow_impl(s->plev(i, j, k), KAPPA);
      }
    for (int k = 1; k <= L; ++k)
      for (int i = is + 5; i <= ie - 5; ++i)
        s->gz(i, j, k + 1) = s->gz(i, j, k) + CP_DRY * s->ptc(i, j, k) * (s->pkap(i, j, k) - s->pkap(i, j, k + 1));
  });
  if (s->nthreads <= 1) {
    for (int k = 1; k <= L; ++k) c_layer2(s, s->sc, k, dt, s->sc.ua, s->sc.va);
  } else {
    std::vector<Scratch<R>> ts = make_scratch(s);
    par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t; c_layer2(s, ts[(size_t)t], k, dt, s->sc.ua, s->sc.va); });
  }
}

// ------------------------------------------------------------ D grid ----
template <class R>
void d_winds(StateT<R>* s, Scratch<R>& sc, int k, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  double dtdx = dt * s->rdx, dtdy = dt * s->rdy;
  A3<R> &uc = s->uc, &vc = s->vc;
  for (int j = js + 1; j <= je; ++j)
    for (int i = is + 1; i <= ie; ++i) {
      sc.ub(i, j) = .5 * (uc(i, j, k) + uc(i, j - 1, k));
      sc.vb(i, j) = .5 * (vc(i, j, k) + vc(i - 1, j, k));
    }
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      sc.cx(i, j) = dtdx * uc(i, j, k);
      sc.cy(i, j) = dtdx * vc(i, j, k);
    }
  for (int j = js + 1; j <= je - 1; ++j)
    for (int i = is + 1; i <= ie - 1; ++i) {
      sc.denom_x(i, j) = 1. / (1. - dtdx * (uc(i + 1, j, k) - uc(i, j, k)));
      sc.denom_y(i, j) = 1. / (1. - dtdy * (vc(i, j + 1, k) - vc(i, j, k)));
    }
}

// first layer loop body, mod_sw_dyn.f90:441-598
template <class R>
void d_layer1(StateT<R>* s, Scratch<R>& sc, int k, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  double dtdx = dt * s->rdx, dtdy = dt * s->rdy, rA = s->rA;
  A3<R> &dp = s->dp, &pt = s->pt, &dpc = s->dpc, &ptc = s->ptc, &pkap = s->pkap;
  if (s->poison) { sc.poison(); sc.poison_winds(); }
  d_winds(s, sc, k, dt);
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      s->playkap(i, j, k) = (pkap(i, j, k + 1) - pkap(i, j, k)) / orc_log_impl(pkap(i, j, k + 1) / pkap(i, j, k));
      s->heating_rate(i, j, k) = (s->net_flux(i, j, k + 1) - s->net_flux(i, j, k)) /
                                 (CP_DRY * dpc(i, j, k) / s->gravity) / s->playkap(i, j, k);
    }
  A1<R> &fx = sc.fx, &fy = sc.fy;
  A2<R> &tmp = sc.tmp, &lap = sc.laplacian, &dpfx = sc.dpfx, &dpfy = sc.dpfy;
  V<R> fxv{&fx.v[0], 1, fx.lb}, fyv{&fy.v[0], 1, fy.lb};

  // ---- dp
  for (int i = is + 1; i <= ie - 1; ++i) {
    flux(sc, fyv, col3(dp, i, js, k, js), col(sc.cy, i, js, js), js, je, PIECEWISE_CONSTANT);
    for (int j = js + 1; j <= je - 1; ++j) {
      tmp(i, j) = .5 * (dp(i, j, k) + sc.denom_y(i, j) * (dp(i, j, k) - rA * (fy(j + 1) - fy(j))));
      lap(i, j) = -2. * dp(i, j, k) * s->rdx2rdy2 + (dp(i + 1, j, k) + dp(i - 1, j, k)) * s->rdx2 +
                  (dp(i, j + 1, k) + dp(i, j - 1, k)) * s->rdy2;
    }
  }
  for (int j = js + 4; j <= je - 4; ++j) {
    flux(sc, fxv, row(tmp, is + 1, j, is + 1), row(sc.cx, is + 1, j, is + 1), is + 1, ie - 1, PPM_NONNEGATIVE);
    dpfx(is + 4, j) = fx(is + 4) * sc.cx(is + 4, j);
    for (int i = is + 4; i <= ie - 4; ++i) {
      dpfx(i + 1, j) = fx(i + 1) * sc.cx(i + 1, j);
      dpc(i, j, k) = dp(i, j, k) - (dpfx(i + 1, j) - dpfx(i, j) +
                                    dtdx * s->vortdamp_xcoeff * (lap(i + 1, j) - 2. * lap(i, j) + lap(i - 1, j)));
    }
  }
  for (int j = js + 1; j <= je - 1; ++j) {
    flux(sc, fxv, row3(dp, is, j, k, is), row(sc.cx, is, j, is), is, ie, PIECEWISE_CONSTANT);
    for (int i = is + 1; i <= ie - 1; ++i)
      tmp(i, j) = .5 * (dp(i, j, k) + sc.denom_x(i, j) * (dp(i, j, k) - rA * (fx(i + 1) - fx(i))));
  }
  for (int i = is + 4; i <= ie - 4; ++i) {
    flux(sc, fyv, col(tmp, i, js + 1, js + 1), col(sc.cy, i, js + 1, js + 1), js + 1, je - 1, PPM_NONNEGATIVE);
    dpfy(i, js + 4) = fy(js + 4) * sc.cy(i, js + 4);
    for (int j = js + 4; j <= je - 4; ++j) {
      dpfy(i, j + 1) = fy(j + 1) * sc.cy(i, j + 1);
      dpc(i, j, k) = dpc(i, j, k) - (dpfy(i, j + 1) - dpfy(i, j) +
                                     dtdy * s->vortdamp_ycoeff * (lap(i, j + 1) - 2. * lap(i, j) + lap(i, j - 1)));
    }
  }
  // ---- pt
  for (int i = is + 1; i <= ie - 1; ++i) {
    flux(sc, fyv, col3(pt, i, js, k, js), col(sc.cy, i, js, js), js, je, PIECEWISE_CONSTANT);
    for (int j = js + 1; j <= je - 1; ++j) {
      tmp(i, j) = .5 * (pt(i, j, k) + sc.denom_y(i, j) * (pt(i, j, k) - rA * (fy(j + 1) - fy(j))));
      lap(i, j) = -2. * pt(i, j, k) * s->rdx2rdy2 + (pt(i + 1, j, k) + pt(i - 1, j, k)) * s->rdx2 +
                  (pt(i, j + 1, k) + pt(i, j - 1, k)) * s->rdy2;
    }
  }
  for (int j = js + 4; j <= je - 4; ++j) {
    flux(sc, fxv, row(tmp, is + 1, j, is + 1), row(sc.cx, is + 1, j, is + 1), is + 1, ie - 1, PPM_NONNEGATIVE);
    for (int i = is + 4; i <= ie - 4; ++i)
      ptc(i, j, k) = dp(i, j, k) * pt(i, j, k) -
                     (fx(i + 1) * dpfx(i + 1, j) - fx(i) * dpfx(i, j) +
                      s->vortdamp_xcoeff * ((lap(i + 1, j) - lap(i, j)) * dpfx(i + 1, j) -
                                            (lap(i, j) - lap(i - 1, j)) * dpfx(i, j)));
  }
  for (int j = js + 1; j <= je - 1; ++j) {
    flux(sc, fxv, row3(pt, is, j, k, is), row(sc.cx, is, j, is), is, ie, PIECEWISE_CONSTANT);
    for (int i = is + 1; i <= ie - 1; ++i)
      tmp(i, j) = .5 * (pt(i, j, k) + sc.denom_x(i, j) * (pt(i, j, k) - rA * (fx(i + 1) - fx(i))));
  }
  for (int i = is + 4; i <= ie - 4; ++i) {
    flux(sc, fyv, col(tmp, i, js + 1, js + 1), col(sc.cy, i, js + 1, js + 1), js + 1, je - 1, PPM_NONNEGATIVE);
    for (int j = js + 4; j <= je - 4; ++j)
      ptc(i, j, k) = (ptc(i, j, k) -
                      (fy(j + 1) * dpfy(i, j + 1) - fy(j) * dpfy(i, j) +
                       s->vortdamp_ycoeff * ((lap(i, j + 1) - lap(i, j)) * dpfy(i, j + 1) -
                                             (lap(i, j) - lap(i, j - 1)) * dpfy(i, j))) +
                      dt * dp(i, j, k) * s->heating_rate(i, j, k)) /
                     dpc(i, j, k);
  }
  for (int j = js + 4; j <= je - 4; ++j)
    for (int i = is + 4; i <= ie - 4; ++i) {
      dp(i, j, k) = dpc(i, j, k);
      pt(i, j, k) = ptc(i, j, k);
    }
}

// third layer loop body, mod_sw_dyn.f90:636-769.  ub, vb, cx, cy, denom_x
// and denom_y are the module arrays left by the LAST iteration of the first
// loop (layer nlay): w holds them.
template <class R>
void d_layer3(StateT<R>* s, Scratch<R>& sc, Scratch<R>& w, int k, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je;
  double dtdx = dt * s->rdx, dtdy = dt * s->rdy, rA = s->rA;
  A3<R> &ud = s->ud, &vd = s->vd, &uc = s->uc, &vc = s->vc, &pkapb = s->pkapb, &gzb = s->gzb;
  A1<R> &fx = sc.fx, &fy = sc.fy;
  A2<R> &tmp = sc.tmp, &lap = sc.laplacian, &ke = sc.kinetic_energy, &vort = sc.vorticity, &div = sc.divergence;
  V<R> fxv{&fx.v[0], 1, fx.lb}, fyv{&fy.v[0], 1, fy.lb};
  if (s->poison) sc.poison();

  for (int i = is + 4; i <= ie - 4; ++i) {
    V<R> cv = scaled_temp(sc, dtdy, col(w.vb, i, js + 1, js + 1), js + 1, je - 1);
    flux(sc, fyv, col3(vd, i, js + 1, k, js + 1), cv, js + 1, je - 1, PPM_CONSTRAINED);
    for (int j = js + 4; j <= je - 4; ++j) ke(i, j) = w.vb(i, j) * fy(j);
  }
  for (int j = js + 4; j <= je - 4; ++j) {
    V<R> cv = scaled_temp(sc, dtdx, row(w.ub, is + 1, j, is + 1), is + 1, ie - 1);
    flux(sc, fxv, row3(ud, is + 1, j, k, is + 1), cv, is + 1, ie - 1, PPM_CONSTRAINED);
    for (int i = is + 4; i <= ie - 4; ++i) ke(i, j) = .5 * (ke(i, j) + w.ub(i, j) * fx(i));
  }
  for (int j = js + 1; j <= je - 1; ++j)
    for (int i = is + 1; i <= ie - 1; ++i)
      vort(i, j) = s->coriolis - (ud(i, j + 1, k) - ud(i, j, k)) * s->rdy + (vd(i + 1, j, k) - vd(i, j, k)) * s->rdx;
  for (int j = js + 7; j <= je - 7; ++j)
    for (int i = is + 7; i <= ie - 7; ++i) {
      sc.pgfx(i, j) = ((pkapb(i + 1, j, k) - pkapb(i, j, k + 1)) * (gzb(i, j, k) - gzb(i + 1, j, k + 1)) +
                       (pkapb(i, j, k) - pkapb(i + 1, j, k + 1)) * (gzb(i, j, k + 1) - gzb(i + 1, j, k))) /
                      (pkapb(i + 1, j, k) - pkapb(i, j, k + 1) + pkapb(i, j, k) - pkapb(i + 1, j, k + 1));
      sc.pgfy(i, j) = ((pkapb(i, j + 1, k) - pkapb(i, j, k + 1)) * (gzb(i, j, k) - gzb(i, j + 1, k + 1)) +
                       (pkapb(i, j, k) - pkapb(i, j + 1, k + 1)) * (gzb(i, j, k + 1) - gzb(i, j + 1, k))) /
                      (pkapb(i, j + 1, k) - pkapb(i, j, k + 1) + pkapb(i, j, k) - pkapb(i, j + 1, k + 1));
    }
  for (int j = js + 4; j <= je - 4; ++j)
    for (int i = is + 4; i <= ie - 4; ++i)
      div(i, j) = s->rdx * (ud(i, j, k) - ud(i - 1, j, k)) + s->rdy * (vd(i, j, k) - vd(i, j - 1, k));
  for (int j = js + 5; j <= je - 5; ++j)
    for (int i = is + 5; i <= ie - 5; ++i)
      tmp(i, j) = -2. * div(i, j) * s->rdx2rdy2 + (div(i + 1, j) + div(i - 1, j)) * s->rdx2 +
                  (div(i, j + 1) + div(i, j - 1)) * s->rdy2;
  for (int j = js + 6; j <= je - 6; ++j)
    for (int i = is + 6; i <= ie - 6; ++i)
      div(i, j) = -2. * tmp(i, j) * s->rdx2rdy2 + (tmp(i + 1, j) + tmp(i - 1, j)) * s->rdx2 +
                  (tmp(i, j + 1) + tmp(i, j - 1)) * s->rdy2;
  for (int j = js + 6; j <= je - 6; ++j)
    for (int i = is + 6; i <= ie - 6; ++i) div(i, j) = s->divdamp_coeff * div(i, j);

  // ud
  for (int j = js + 4; j <= je - 4; ++j) {
    flux(sc, fxv, row(vort, is + 1, j, is + 1), row(w.cx, is + 1, j, is + 1), is + 1, ie - 1, PIECEWISE_CONSTANT);
    for (int i = is + 4; i <= ie - 4; ++i) {
      tmp(i, j) = .5 * (vort(i, j) + w.denom_x(i, j) * (vort(i, j) - rA * (fx(i + 1) - fx(i))));
      lap(i, j) = -2. * vort(i, j) * s->rdx2rdy2 + (vort(i + 1, j) + vort(i - 1, j)) * s->rdx2 +
                  (vort(i, j + 1) + vort(i, j - 1)) * s->rdy2;
    }
  }
  for (int i = is + 7; i <= ie - 7; ++i) {
    flux(sc, fyv, col(tmp, i, js + 4, js + 4), col(w.cy, i, js + 4, js + 4), js + 4, je - 4, PPM_CONSTRAINED);
    for (int j = js + 7; j <= je - 7; ++j)
      ud(i, j, k) = ud(i, j, k) + dt * (vc(i, j, k) * fy(j) + s->vortdamp_ycoeff * (lap(i, j) - lap(i, j - 1))) -
                    dtdx * (ke(i + 1, j) - ke(i, j) - div(i + 1, j) + div(i, j) - sc.pgfx(i, j));
  }
  // vd
  for (int i = is + 4; i <= ie - 4; ++i) {
    flux(sc, fyv, col(vort, i, js + 1, js + 1), col(w.cy, i, js + 1, js + 1), js + 1, je - 1, PIECEWISE_CONSTANT);
    for (int j = js + 4; j <= je - 4; ++j)
      tmp(i, j) = .5 * (vort(i, j) + w.denom_y(i, j) * (vort(i, j) - rA * (fy(j + 1) - fy(j))));
  }
  for (int j = js + 7; j <= je - 7; ++j) {
    flux(sc, fxv, row(tmp, is + 4, j, is + 4), row(w.cx, is + 4, j, is + 4), is + 4, ie - 4, PPM_CONSTRAINED);
    for (int i = is + 7; i <= ie - 7; ++i)
      vd(i, j, k) = vd(i, j, k) - dt * (uc(i, j, k) * fx(i) + s->vortdamp_xcoeff * (lap(i, j) - lap(i - 1, j))) -
                    dtdy * (ke(i, j + 1) - ke(i, j) - div(i, j + 1) + div(i, j) - sc.pgfy(i, j));
  }
}

// mod_sw_dyn.f90:424-773
template <class R>
void dgrid_dynamics_step(StateT<R>* s, double dt) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je, L = s->nlay;
  par_for(s->nthreads, js, je, [&](int j, int t) { (void)t;
    for (int k = L; k >= 1; --k)
      for (int i = is; i <= ie; ++i) {
        s->plev(i, j, k) = s->plev(i, j, k + 1) + s->dpc(i, j, k);
        s->pkap(i, j, k) = orc_pow_impl(s->plev(i, j, k), KAPPA);
      }
  });
  if (s->nthreads <= 1) {
    for (int k = 1; k <= L; ++k) d_layer1(s, s->sc, k, dt);
  } else {
    std::vector<Scratch<R>> ts = make_scratch(s);
    par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t; d_layer1(s, ts[(size_t)t], k, dt); });
    d_winds(s, s->sc, L, dt);  // module ub, vb, cx, cy, denom keep layer nlay
  }
  // pressure, pkap, pkapb, gz, gzb on is+4:ie-4 (mod_sw_dyn.f90:606-632)
  par_for(s->nthreads, js + 4, je - 4, [&](int j, int t) { (void)t;
    for (int k = L; k >= 1; --k)
      for (int i = is + 4; i <= ie - 4; ++i) {
        s->plev(i, j, k) = s->plev(i, j, k + 1) + s->dp(i, j, k);
        s->pkap(i, j, k) = orc_pow_impl(s->plev(i, j, k), KAPPA);
      }
  });
  par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t;
    interpolate_to_corners(w3(s->pkapb, is + 4, js + 4, k), w3(s->pkap, is + 4, js + 4, k), is + 4, ie - 4, js + 4, je - 4);
  });
  par_for(s->nthreads, js + 4, je - 4, [&](int j, int t) { (void)t;
    for (int k = 1; k <= L; ++k)
      for (int i = is + 4; i <= ie - 4; ++i)
        s->gz(i, j, k + 1) = s->gz(i, j, k) + CP_DRY * s->pt(i, j, k) * (s->pkap(i, j, k) - s->pkap(i, j, k + 1));
  });
  par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t;
    interpolate_to_corners(w3(s->gzb, is + 4, js + 4, k + 1), w3(s->gz, is + 4, js + 4, k + 1), is + 4, ie - 4, js + 4, je - 4);
  });
  if (s->nthreads <= 1) {
    for (int k = 1; k <= L; ++k) d_layer3(s, s->sc, s->sc, k, dt);
  } else {
    std::vector<Scratch<R>> ts = make_scratch(s);
    par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t; d_layer3(s, ts[(size_t)t], s->sc, k, dt); });
  }
}

// ------------------------------------------------------------- remap ----
template <class R>
struct PPMCol {
  std::vector<R> btm_edge, top_edge, curvature, gam, level_var;
  void alloc(int L) {
    btm_edge.assign((size_t)L + 1, R(NAN));
    top_edge.assign((size_t)L + 1, R(NAN));
    curvature.assign((size_t)L + 1, R(NAN));
    gam.assign((size_t)L + 2, R(NAN));
    level_var.assign((size_t)L + 2, R(NAN));
  }
};

// mod_remap.f90:287-356 (arrays 1-based).  The monotonicity test of the
// last interface reads gam(nlay+1), one past the end of gam; it cannot
// change the result because level_var(nlay) is already clamped to the
// same bounds at :319-320, so it is evaluated with both clamps here.
template <class R>
void vertical_ppm(PPMCol<R>& w, int L, const R* var, const R* coord) {
  R* gam = w.gam.data();
  R* level_var = w.level_var.data();
  R alpha, beta;
  alpha = (coord[L] - coord[L - 1]) / (coord[L + 1] - coord[L]);
  beta = alpha * (.5 + alpha);
  level_var[L + 1] = (2. * alpha * (1. + alpha) * var[L] + var[L - 1]) / beta;
  gam[L] = (1. + alpha * (1.5 + alpha)) / beta;
  for (int k = L; k >= 2; --k) {
    alpha = (coord[k + 1] - coord[k]) / (coord[k] - coord[k - 1]);
    beta = 2. + 2. * alpha - gam[k];
    level_var[k] = (3. * (var[k] + alpha * var[k - 1]) - level_var[k + 1]) / beta;
    gam[k - 1] = alpha / beta;
  }
  beta = 1. + alpha * (1.5 + alpha);
  level_var[1] = (2. * alpha * (1. + alpha) * var[1] + var[2] - beta * level_var[2]) /
                 (alpha * (.5 + alpha) - beta * gam[1]);
  for (int k = 2; k <= L + 1; ++k) level_var[k] = level_var[k] - gam[k - 1] * level_var[k - 1];
  level_var[L] = std::min(level_var[L], std::max(var[L], var[L - 1]));
  level_var[L] = std::max(level_var[L], std::min(var[L], var[L - 1]));
  level_var[2] = std::min(level_var[2], std::max(var[2], var[1]));
  level_var[2] = std::max(level_var[2], std::min(var[2], var[1]));
  for (int k = 2; k <= L - 1; ++k) {
    R lo = std::min(var[k], var[k + 1]), hi = std::max(var[k], var[k + 1]);
    if (k + 2 > L || gam[k + 2] * gam[k] > 0) {
      level_var[k + 1] = std::min(level_var[k + 1], hi);
      level_var[k + 1] = std::max(level_var[k + 1], lo);
    } else if (gam[k + 2] > 0) {
      level_var[k + 1] = std::max(level_var[k + 1], lo);
    } else {
      level_var[k + 1] = std::min(level_var[k + 1], hi);
    }
  }
  R* top_edge = w.top_edge.data();
  R* btm_edge = w.btm_edge.data();
  for (int k = 1; k <= L; ++k) {
    top_edge[k] = level_var[k + 1];
    btm_edge[k] = level_var[k];
  }
  for (int k = 2; k <= L - 1; ++k) {
    R pmp1 = var[k + 1] - 2. * gam[k];
    R lac1 = pmp1 + 1.5 * gam[k - 1];
    top_edge[k + 1] = std::min(std::max(top_edge[k + 1], fmin3(var[k + 1], pmp1, lac1)), fmax3(var[k + 1], pmp1, lac1));
    pmp1 = var[k + 1] + 2. * gam[k + 1];
    lac1 = pmp1 - 1.5 * gam[k];
    btm_edge[k + 1] = std::min(std::max(btm_edge[k + 1], fmin3(var[k + 1], pmp1, lac1)), fmax3(var[k + 1], pmp1, lac1));
  }
  for (int k = 1; k <= L; ++k) w.curvature[k] = 6. * var[k] - 3. * (top_edge[k] + btm_edge[k]);
}

// mod_remap.f90:165-285; the O(nlay^2) pair loop of the reference.
template <class R>
void remap_column(PPMCol<R>& w, int L, const R* src_var, R* dst_var, const R* src_coord,
                  const R* dst_coord, int32_t* trace) {
  for (int m = 1; m <= L; ++m) dst_var[m] = 0.;
  vertical_ppm(w, L, src_var, src_coord);
  const R* btm_edge = w.btm_edge.data();
  const R* top_edge = w.top_edge.data();
  const R* curvature = w.curvature.data();
  if (trace)
    for (int m = 1; m <= L; ++m) {
      int32_t* t = trace + 5 * (m - 1);
      t[0] = t[1] = t[2] = t[3] = -1;
      t[4] = 0;
    }
  for (int k = 1; k <= L; ++k)
    for (int m = 1; m <= L; ++m) {
      R dsrc_coord = src_coord[k + 1] - src_coord[k];
      R s1 = (dst_coord[m] - src_coord[k]) / dsrc_coord;
      R s2 = (dst_coord[m + 1] - src_coord[k]) / dsrc_coord;
      R integral_factor = dsrc_coord / (dst_coord[m + 1] - dst_coord[m]);
      if (src_coord[k + 1] >= dst_coord[m] || src_coord[k] <= dst_coord[m + 1]) continue;
      int which = 0;
      R tmp3 = 2. * s1 * s1;
      if (dst_coord[m + 1] <= src_coord[k + 1] && src_coord[k + 1] < dst_coord[m] && dst_coord[m] < src_coord[k]) {
        R tmp1 = s1 - 1., tmp2 = s1 + 1.;
        dst_var[m] = dst_var[m] + tmp1 / 6. *
                                      (3. * (btm_edge[k] * tmp1 - top_edge[k] * tmp2) + curvature[k] * (tmp3 - tmp2)) *
                                      integral_factor;
        which = 3;
      }
      if (src_coord[k + 1] < dst_coord[m + 1] && dst_coord[m + 1] < src_coord[k] && src_coord[k] <= dst_coord[m]) {
        dst_var[m] = dst_var[m] + (s2 / 2.) *
                                      (btm_edge[k] * (2. - s2) + s2 * (top_edge[k] + curvature[k] * (1. - C2_3 * s2))) *
                                      integral_factor;
        which = which * 10 + 4;
      }
      if (dst_coord[m + 1] <= src_coord[k + 1] && src_coord[k] <= dst_coord[m]) {
        dst_var[m] = dst_var[m] + src_var[k] * integral_factor;
        which = which * 10 + 5;
      }
      if (src_coord[k + 1] < dst_coord[m + 1] && dst_coord[m] < src_coord[k]) {
        R tmp1 = s1 + s2;
        dst_var[m] = dst_var[m] + (s1 - s2) / 6. *
                                      (3. * (btm_edge[k] * (tmp1 - 2.) - top_edge[k] * tmp1) +
                                       curvature[k] * (tmp3 + tmp1 * (2. * s2 - 3.))) *
                                      integral_factor;
        which = which * 10 + 6;
      }
      if (trace) {
        int32_t* t = trace + 5 * (m - 1);
        if (t[0] < 0) { t[0] = k; t[2] = which; }
        else if (t[1] != k - 1) t[4] = -1000000;  // non-contiguous: mark
        t[1] = k;
        t[3] = which;
        if (t[4] >= 0) t[4] += 1;
      }
    }
}

// mod_remap.f90:27-163
template <class R>
void perform_vertical_remapping(StateT<R>* s) {
  int L = s->nlay, isd = s->isd, ied = s->ied, jsd = s->jsd, jed = s->jed;
  int isl = isd - 3, iel = ied + 3, jsl = jsd - 3, jel = jed + 3;
  A3<R> &plev = s->plev, &pkap = s->pkap, &playkap = s->playkap, &gz = s->gz;
  A3<R> &tpl = s->target_plev, &tpk = s->target_pkap, &tplk = s->target_playkap;
  A3<R> &dp = s->dp, &pt = s->pt, &ud = s->ud, &vd = s->vd;

  par_for(s->nthreads, jsl, jel, [&](int j, int t) { (void)t;
    for (int k = L; k >= 1; --k)
      for (int i = isl; i <= iel; ++i) {
        plev(i, j, k) = plev(i, j, k + 1) + dp(i, j, k);
        pkap(i, j, k) = orc_pow_impl(plev(i, j, k), KAPPA);
        R plog = orc_log_impl(pkap(i, j, k + 1) / pkap(i, j, k));
        playkap(i, j, k) = (pkap(i, j, k + 1) - pkap(i, j, k)) / plog;
      }
    for (int k = L; k >= 1; --k)
      for (int i = isl; i <= iel; ++i) {
        tpl(i, j, k) = s->coord_Ak(k) + s->coord_Bk(k) * (plev(i, j, 1) - s->top_pressure);
        tpk(i, j, k) = orc_pow_impl(tpl(i, j, k), KAPPA);
        R plog = orc_log_impl(tpk(i, j, k + 1) / tpk(i, j, k));
        tplk(i, j, k) = (tpk(i, j, k + 1) - tpk(i, j, k)) / plog;
      }
    for (int k = 1; k <= L; ++k)
      for (int i = isl; i <= iel; ++i)
        gz(i, j, k + 1) = gz(i, j, k) + CP_DRY * pt(i, j, k) * (pkap(i, j, k) - pkap(i, j, k + 1));
  });

  int nxr = s->nx + 2, nyr = s->ny + 2;
  auto trace_at = [&](int var, int i, int j) -> int32_t* {
    if (!s->trace) return nullptr;
    return s->trace + (size_t)5 * L * ((size_t)(i - (isd - 1)) + (size_t)nxr * ((size_t)(j - (jsd - 1)) + (size_t)nyr * var));
  };
  if (s->trace)
    for (size_t q = 0; q < (size_t)3 * nyr * nxr * L * 5; ++q) s->trace[q] = -1;

  par_for(s->nthreads, isd - 1, ied + 1, [&](int i, int t) { (void)t;
    PPMCol<R> w;
    w.alloc(L);
    std::vector<R> src_plev(L + 2), dst_plev(L + 2), col(L + 2), out(L + 2);
    for (int j = jsd - 1; j <= jed + 1; ++j) {
      for (int k = 1; k <= L + 1; ++k) {
        src_plev[k] = C7_12 * (plev(i, j, k) + plev(i, j - 1, k)) - C1_12 * (plev(i, j + 1, k) + plev(i, j - 2, k));
        dst_plev[k] = C7_12 * (tpl(i, j, k) + tpl(i, j - 1, k)) - C1_12 * (tpl(i, j + 1, k) + tpl(i, j - 2, k));
      }
      for (int k = 1; k <= L; ++k) col[k] = ud(i, j, k);
      remap_column(w, L, col.data(), out.data(), src_plev.data(), dst_plev.data(), trace_at(0, i, j));
      for (int k = 1; k <= L; ++k) s->u_remap(i, j, k) = out[k];
      for (int k = 1; k <= L + 1; ++k) {
        src_plev[k] = C7_12 * (plev(i, j, k) + plev(i - 1, j, k)) - C1_12 * (plev(i + 1, j, k) + plev(i - 2, j, k));
        dst_plev[k] = C7_12 * (tpl(i, j, k) + tpl(i - 1, j, k)) - C1_12 * (tpl(i + 1, j, k) + tpl(i - 2, j, k));
      }
      for (int k = 1; k <= L; ++k) col[k] = vd(i, j, k);
      remap_column(w, L, col.data(), out.data(), src_plev.data(), dst_plev.data(), trace_at(1, i, j));
      for (int k = 1; k <= L; ++k) s->v_remap(i, j, k) = out[k];
    }
  });

  A3<R> &ur = s->u_remap, &vr = s->v_remap;
  par_for(s->nthreads, isd, ied, [&](int i, int t) { (void)t;
    PPMCol<R> w;
    w.alloc(L);
    std::vector<R> energy(L + 2), energy_remap(L + 2), gz_remap(L + 2), ua(L + 2), va(L + 2);
    std::vector<R> src(L + 2), dst(L + 2);
    for (int j = jsd; j <= jed; ++j) {
      for (int k = 1; k <= L; ++k) {
        ua[k] = (.25 * (ud(i, j, k) + ud(i, j + 1, k)) +
                 .125 * (ud(i - 1, j, k) + ud(i - 1, j + 1, k) + ud(i + 1, j, k) + ud(i + 1, j + 1, k)));
        va[k] = (.25 * (vd(i, j, k) + vd(i + 1, j, k)) +
                 .125 * (vd(i, j - 1, k) + vd(i + 1, j - 1, k) + vd(i, j + 1, k) + vd(i + 1, j + 1, k)));
        energy[k] = CV_DRY * pt(i, j, k) * playkap(i, j, k) +
                    .5 * (gz(i, j, k + 1) + gz(i, j, k) + ua[k] * ua[k] + va[k] * va[k]);
      }
      for (int k = 1; k <= L + 1; ++k) {
        src[k] = plev(i, j, k);
        dst[k] = tpl(i, j, k);
      }
      remap_column(w, L, energy.data(), energy_remap.data(), src.data(), dst.data(), trace_at(2, i, j));
      for (int k = 1; k <= L; ++k) {
        ua[k] = (.25 * (ur(i, j, k) + ur(i, j + 1, k)) +
                 .125 * (ur(i - 1, j, k) + ur(i - 1, j + 1, k) + ur(i + 1, j, k) + ur(i + 1, j + 1, k)));
        va[k] = (.25 * (vr(i, j, k) + vr(i + 1, j, k)) +
                 .125 * (vr(i, j - 1, k) + vr(i + 1, j - 1, k) + vr(i, j + 1, k) + vr(i + 1, j + 1, k)));
      }
      gz_remap[1] = gz(i, j, 1);
      for (int k = 1; k <= L; ++k) {
        s->pt_remap(i, j, k) = (energy_remap[k] - gz_remap[k] - .5 * (ua[k] * ua[k] + va[k] * va[k])) /
                               (CV_DRY * tplk(i, j, k) + .5 * CP_DRY * (tpk(i, j, k) - tpk(i, j, k + 1)));
        gz_remap[k + 1] = gz_remap[k] + CP_DRY * s->pt_remap(i, j, k) * (tpk(i, j, k) - tpk(i, j, k + 1));
      }
    }
  });

  par_for(s->nthreads, 1, L, [&](int k, int t) { (void)t;
    for (int j = jsd; j <= jed; ++j)
      for (int i = isd; i <= ied; ++i) {
        dp(i, j, k) = tpl(i, j, k) - tpl(i, j, k + 1);
        ud(i, j, k) = ur(i, j, k);
        vd(i, j, k) = vr(i, j, k);
        pt(i, j, k) = s->pt_remap(i, j, k);
      }
  });
}

template <class R>
A3<R>* field_ptr(StateT<R>* s, int f) {
  switch (f) {
    case ORC_DP: return &s->dp;
    case ORC_PT: return &s->pt;
    case ORC_UD: return &s->ud;
    case ORC_VD: return &s->vd;
    case ORC_GZ: return &s->gz;
    case ORC_PLEV: return &s->plev;
    case ORC_PKAP: return &s->pkap;
    case ORC_NET_FLUX: return &s->net_flux;
    case ORC_DPC: return &s->dpc;
    case ORC_PTC: return &s->ptc;
    case ORC_UC: return &s->uc;
    case ORC_VC: return &s->vc;
    case ORC_TS: return &s->ts;
    default: return nullptr;
  }
}

}  // namespace

namespace {

template <class R>
bool setup_state(StateT<R>* s, int nx, int ny, int nlay, double dx, double dy, const double* ak, const double* bk,
                 double gravity, double coriolis, double divdamp, double vortdamp) {
  if (nx < HALO || ny < HALO || nlay < 3 || !ak || !bk) return false;
  s->nx = nx; s->ny = ny; s->nlay = nlay; s->dx = dx; s->dy = dy;
  s->isd = 1; s->ied = nx; s->jsd = 1; s->jed = ny;  // mod_tiles.f90:222-241, one image
  s->is = s->isd - HALO; s->ie = s->ied + HALO; s->js = s->jsd - HALO; s->je = s->jed + HALO;
  s->gravity = gravity; s->coriolis = coriolis;
  s->divergence_damping = divdamp; s->vorticity_damping = vortdamp;
  s->coord_Ak.alloc(1, nlay + 1);
  s->coord_Bk.alloc(1, nlay + 1);
  for (int k = 1; k <= nlay + 1; ++k) { s->coord_Ak(k) = ak[k - 1]; s->coord_Bk(k) = bk[k - 1]; }
  int is = s->is, ie = s->ie, js = s->js, je = s->je, L = nlay;
  for (A3<R>* a : {&s->dp, &s->pt, &s->ud, &s->vd, &s->playkap}) a->alloc(is, ie, js, je, 1, L);
  for (A3<R>* a : {&s->plev, &s->pkap, &s->gz}) a->alloc(is, ie, js, je, 1, L + 1);
  s->net_flux.alloc(is, ie, js, je, 1, L + 1, R(0.0));  // radiation is off: zero flux
  for (A3<R>* a : {&s->dpc, &s->ptc, &s->uc, &s->vc, &s->heating_rate}) a->alloc(is, ie, js, je, 1, L);
  for (A3<R>* a : {&s->pkapb, &s->gzb}) a->alloc(is, ie, js, je, 1, L + 1);
  s->sc.alloc(is, ie, js, je);
  // allocate_physics_arrays, mod_physics.f90:193-212; ts, mod_fields.f90:51
  s->ts.alloc(is, ie, js, je, 1, 1);
  s->ts_tend.alloc(s->isd - 2, s->ied + 2, s->jsd - 2, s->jed + 2, 1, 1);
  for (A3<R>* a : {&s->dp_tend, &s->pt_tend, &s->u_tend, &s->v_tend})
    a->alloc(s->isd - 2, s->ied + 2, s->jsd - 2, s->jed + 2, 1, L);
  s->ua.alloc(is, ie, js, je, 1, L);
  s->va.alloc(is, ie, js, je, 1, L);
  s->u_remap.alloc(s->isd - 1, s->ied + 1, s->jsd - 1, s->jed + 1, 1, L);
  s->v_remap.alloc(s->isd - 1, s->ied + 1, s->jsd - 1, s->jed + 1, 1, L);
  s->pt_remap.alloc(s->isd, s->ied, s->jsd, s->jed, 1, L);
  s->target_plev.alloc(s->isd - 3, s->ied + 3, s->jsd - 3, s->jed + 3, 1, L + 1);
  s->target_pkap.alloc(s->isd - 3, s->ied + 3, s->jsd - 3, s->jed + 3, 1, L + 1);
  s->target_playkap.alloc(s->isd - 3, s->ied + 3, s->jsd - 3, s->jed + 3, 1, L);
  size_t nb = (size_t)std::max(nx, ny);
  s->edge_buffer.assign(nb * HALO * (L + 1) * 4 * 5, R(NAN));
  s->corner_buffer.assign((size_t)HALO * HALO * (L + 1) * 4 * 5, R(NAN));
  return true;
}

// copy a field between the state and flat (val, tan) arrays; tan may be NULL
template <class R> inline void put_(R& x, double v, const double* tan, size_t n);
template <> inline void put_<double>(double& x, double v, const double*, size_t) { x = v; }
template <> inline void put_<Dual>(Dual& x, double v, const double* tan, size_t n) { x = Dual(v, tan ? tan[n] : 0.); }
template <class R> inline void get_(const R& x, double* v, double* tan, size_t n);
template <> inline void get_<double>(const double& x, double* v, double*, size_t n) { v[n] = x; }
template <> inline void get_<Dual>(const Dual& x, double* v, double* tan, size_t n) {
  if (v) v[n] = x.v;
  if (tan) tan[n] = x.d;
}

template <class R>
int set_field(StateT<R>* s, int field, const double* a, const double* tan, int with_halo) {
  A3<R>* f = field_ptr(s, field);
  if (!f || !a) return -1;
  if (with_halo) {
    for (size_t n = 0; n < f->v.size(); ++n) put_<R>(f->v[n], a[n], tan, n);
    return 0;
  }
  size_t n = 0;
  for (int k = 1; k <= f->k1; ++k)
    for (int j = s->jsd; j <= s->jed; ++j)
      for (int i = s->isd; i <= s->ied; ++i, ++n) put_<R>((*f)(i, j, k), a[n], tan, n);
  return 0;
}

template <class R>
int get_field(StateT<R>* s, int field, double* a, double* tan, int with_halo) {
  A3<R>* f = field_ptr(s, field);
  if (!f) return -1;
  if (with_halo) {
    for (size_t n = 0; n < f->v.size(); ++n) get_<R>(f->v[n], a, tan, n);
    return 0;
  }
  size_t n = 0;
  for (int k = 1; k <= f->k1; ++k)
    for (int j = s->jsd; j <= s->jed; ++j)
      for (int i = s->isd; i <= s->ied; ++i, ++n) get_<R>((*f)(i, j, k), a, tan, n);
  return 0;
}

template <class R>
void init_state(StateT<R>* s) {
  int is = s->is, ie = s->ie, js = s->js, je = s->je, L = s->nlay;
  double top = s->coord_Ak(1);
  // mod_input.f90:229-231
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) {
      s->plev(i, j, L + 1) = top;
      s->pkap(i, j, L + 1) = orc_pow_impl(top, KAPPA);
    }
  // mod_input.f90:247: halo_exchange(dp, pt, gz, ud, vd) through the
  // 5 x nlay-layer interface, so gz levels 1..nlay are exchanged
  A3<R>* f5[] = {&s->dp, &s->pt, &s->gz, &s->ud, &s->vd};
  halo_exchange(s, f5, 5, L);
  // init_sw_dyn, mod_sw_dyn.f90:958-1023
  s->rdx = 1. / s->dx;
  s->rdx2 = 1. / (s->dx * s->dx);
  s->rdy = 1. / s->dy;
  s->rdy2 = 1. / (s->dy * s->dy);
  s->rdx2rdy2 = s->rdx2 + s->rdy2;
  s->rA = 1. / (s->dx * s->dy);
  for (int j = js; j <= je; ++j)
    for (int i = is; i <= ie; ++i) s->pkapb(i, j, L + 1) = orc_pow_impl(top, KAPPA);
  interpolate_to_corners(w3(s->gzb, is, js, 1), w3(s->gz, is, js, 1), is, ie, js, je);
  double dd = s->divergence_damping * s->dx * s->dy;
  s->divdamp_coeff = dd * dd;
  double vortdamp_coeff = s->vorticity_damping * s->dx * s->dy;
  s->vortdamp_xcoeff = s->dy * s->rdx * vortdamp_coeff;
  s->vortdamp_ycoeff = s->dx * s->rdy * vortdamp_coeff;
  // allocate_remapping_arrays, mod_remap.f90:358-388
  s->top_pressure = top;
  for (int j = s->jsd - 3; j <= s->jed + 3; ++j)
    for (int i = s->isd - 3; i <= s->ied + 3; ++i) {
      s->target_plev(i, j, L + 1) = top;
      s->target_pkap(i, j, L + 1) = orc_pow_impl(top, KAPPA);
    }
}

template <class R>
void cgrid_halo(StateT<R>* s) {
  A3<R>* f4[] = {&s->dpc, &s->ptc, &s->uc, &s->vc};
  halo_exchange(s, f4, 4, s->nlay);
}
template <class R>
void dgrid_halo(StateT<R>* s) {
  A3<R>* f4[] = {&s->dp, &s->pt, &s->ud, &s->vd};
  halo_exchange(s, f4, 4, s->nlay);
}

// ------------------------------------------------------------ physics ----
// calculate_physics_tendencies, src/mod_physics.f90:27-79
template <class R>
void dry_convective_adjustment(StateT<R>* s);
template <class R>
void calculate_physics_tendencies(StateT<R>* s) {
  const int L = s->nlay;
  for (A3<R>* a : {&s->dp_tend, &s->pt_tend, &s->u_tend, &s->v_tend}) std::fill(a->v.begin(), a->v.end(), R(0.));
  // A-grid winds (:39-47)
  for (int j = s->js + 1; j <= s->je - 1; ++j)
    for (int i = s->is + 1; i <= s->ie - 1; ++i)
      for (int k = 1; k <= L; ++k) {
        s->ua(i, j, k) = (.25 * (s->ud(i, j, k) + s->ud(i, j + 1, k)) +
                          .125 * (s->ud(i - 1, j, k) + s->ud(i - 1, j + 1, k) + s->ud(i + 1, j, k) + s->ud(i + 1, j + 1, k)));
        s->va(i, j, k) = (.25 * (s->vd(i, j, k) + s->vd(i + 1, j, k)) +
                          .125 * (s->vd(i, j - 1, k) + s->vd(i + 1, j - 1, k) + s->vd(i, j + 1, k) + s->vd(i + 1, j + 1, k)));
      }
  // levels and pkap (:49-57)
  for (int k = L; k >= 1; --k)
    for (int j = s->js + 1; j <= s->je - 1; ++j)
      for (int i = s->is + 1; i <= s->ie - 1; ++i) {
        s->plev(i, j, k) = s->plev(i, j, k + 1) + s->dp(i, j, k);
        s->pkap(i, j, k) = orc_pow_impl(s->plev(i, j, k), KAPPA);
      }
  // geopotential and layer-mean pkap (:59-71)
  for (int k = 1; k <= L; ++k)
    for (int j = s->js + 1; j <= s->je - 1; ++j)
      for (int i = s->is + 1; i <= s->ie - 1; ++i) {
        s->gz(i, j, k + 1) = s->gz(i, j, k) + CP_DRY * s->pt(i, j, k) * (s->pkap(i, j, k) - s->pkap(i, j, k + 1));
        s->playkap(i, j, k) = (s->pkap(i, j, k + 1) - s->pkap(i, j, k)) /
                              orc_log_impl(s->plev(i, j, k + 1) / s->plev(i, j, k)) / KAPPA;
      }
  dry_convective_adjustment(s);
  // surface_heating (:178-185): heat capacity of 5 m of water, 41680*5 J/m^2/K
  for (int j = s->jsd; j <= s->jed; ++j)
    for (int i = s->isd; i <= s->ied; ++i) s->ts_tend(i, j, 1) = s->net_flux(i, j, 1) / 208400.;
}

// dry_convective_adjustment, src/mod_physics.f90:81-176
template <class R>
void dry_convective_adjustment(StateT<R>* s) {
  const int L = s->nlay;
  const double min_v2 = (double)1e-4f;  // a default-real literal (:86)
  const double critical_richardson_number = .25;
  const double mixing_timescale = 600.;
  std::vector<R> energy(L + 1), u_adj(L + 1), v_adj(L + 1), gz_adj(L + 2), pt_adj(L + 1);
  for (int j = s->jsd - 2; j <= s->jed + 2; ++j)
    for (int i = s->isd - 2; i <= s->ied + 2; ++i) {
      for (int k = 1; k <= L; ++k) {
        energy[k] = CV_DRY * s->pt(i, j, k) * s->playkap(i, j, k) +
                    .5 * (s->gz(i, j, k + 1) + s->gz(i, j, k) + s->ua(i, j, k) * s->ua(i, j, k) +
                          s->va(i, j, k) * s->va(i, j, k));
        u_adj[k] = s->ua(i, j, k);
        v_adj[k] = s->va(i, j, k);
      }
      for (int k = 1; k <= L - 1; ++k) {
        const R du = s->ua(i, j, k + 1) - s->ua(i, j, k), dv = s->va(i, j, k + 1) - s->va(i, j, k);
        const R ri = (s->pt(i, j, k + 1) - s->pt(i, j, k)) *
                     (s->dp(i, j, k) * (s->gz(i, j, k + 1) - s->gz(i, j, k)) +
                      s->dp(i, j, k + 1) * (s->gz(i, j, k + 2) - s->gz(i, j, k + 1))) /
                     ((s->dp(i, j, k) * s->pt(i, j, k) + s->dp(i, j, k + 1) * s->pt(i, j, k + 1)) *
                      (du * du + dv * dv + min_v2));
        if (ri < critical_richardson_number) {
          const R q = ri / critical_richardson_number;
          const R t = 1. - (q > 0. ? q : R(0.));  // max(0.0, q)
          const R mixing_fraction = t * t * s->dp(i, j, k) * s->dp(i, j, k + 1) / (s->dp(i, j, k) + s->dp(i, j, k + 1));
          R exchange = mixing_fraction * (u_adj[k] - u_adj[k + 1]);
          u_adj[k] = u_adj[k] - exchange / s->dp(i, j, k);
          u_adj[k + 1] = u_adj[k + 1] + exchange / s->dp(i, j, k + 1);
          exchange = mixing_fraction * (v_adj[k] - v_adj[k + 1]);
          v_adj[k] = v_adj[k] - exchange / s->dp(i, j, k);
          v_adj[k + 1] = v_adj[k + 1] + exchange / s->dp(i, j, k + 1);
          exchange = mixing_fraction * (energy[k] - energy[k + 1]);
          energy[k] = energy[k] - exchange / s->dp(i, j, k);
          energy[k + 1] = energy[k + 1] + exchange / s->dp(i, j, k + 1);
        }
      }
      for (int k = 1; k <= L; ++k) {
        s->u_tend(i, j, k) = s->u_tend(i, j, k) + (u_adj[k] - s->ua(i, j, k)) / mixing_timescale;
        s->v_tend(i, j, k) = s->v_tend(i, j, k) + (v_adj[k] - s->va(i, j, k)) / mixing_timescale;
      }
      gz_adj[1] = s->gz(i, j, 1);
      for (int k = 1; k <= L; ++k) {
        pt_adj[k] = (energy[k] - gz_adj[k] - .5 * (u_adj[k] * u_adj[k] + v_adj[k] * v_adj[k])) /
                    (CV_DRY * s->playkap(i, j, k) + .5 * CP_DRY * (s->pkap(i, j, k) - s->pkap(i, j, k + 1)));
        gz_adj[k + 1] = gz_adj[k] + CP_DRY * pt_adj[k] * (s->pkap(i, j, k) - s->pkap(i, j, k + 1));
      }
      for (int k = 1; k <= L; ++k)
        s->pt_tend(i, j, k) = s->pt_tend(i, j, k) + (pt_adj[k] - s->pt(i, j, k)) / mixing_timescale;
    }
}

// apply_physics_tendencies, src/mod_physics.f90:187-211
template <class R>
void apply_physics_tendencies(StateT<R>* s, double dt) {
  const int L = s->nlay;
  for (int k = 1; k <= L; ++k)
    for (int j = s->jsd; j <= s->jed; ++j)
      for (int i = s->isd; i <= s->ied; ++i) s->dp(i, j, k) = s->dp(i, j, k) + dt * s->dp_tend(i, j, k);
  for (int k = 1; k <= L; ++k)
    for (int j = s->jsd; j <= s->jed; ++j)
      for (int i = s->isd; i <= s->ied; ++i) s->pt(i, j, k) = s->pt(i, j, k) + dt * s->pt_tend(i, j, k);
  for (int j = s->jsd; j <= s->jed; ++j)
    for (int i = s->isd; i <= s->ied; ++i) s->ts(i, j, 1) = s->ts(i, j, 1) + dt * s->ts_tend(i, j, 1);
  for (int j = s->jsd; j <= s->jed; ++j)
    for (int i = s->isd; i <= s->ied; ++i)
      for (int k = 1; k <= L; ++k) {
        s->ud(i, j, k) = s->ud(i, j, k) + dt * (C7_12 * (s->u_tend(i, j, k) + s->u_tend(i, j - 1, k)) -
                                                C1_12 * (s->u_tend(i, j + 1, k) + s->u_tend(i, j - 2, k)));
        s->vd(i, j, k) = s->vd(i, j, k) + dt * (C7_12 * (s->v_tend(i, j, k) + s->v_tend(i - 1, j, k)) -
                                                C1_12 * (s->v_tend(i + 1, j, k) + s->v_tend(i - 2, j, k)));
      }
}

// physics_halo_exchange, src/mod_physics.f90:213-217 (the 2-D exchange of
// mod_sync.f90:42-52 is the 3-D one on a single level)
template <class R>
void physics_halo(StateT<R>* s) {
  A3<R>* f1[] = {&s->ts};
  halo_exchange(s, f1, 1, 1);
}

}  // namespace

extern "C" {

orc_state* orc_create(int nx, int ny, int nlay, double dx, double dy, const double* ak, const double* bk,
                      double gravity, double coriolis, double divdamp, double vortdamp) {
  orc_state* s = new orc_state();
  if (!setup_state<double>(s, nx, ny, nlay, dx, dy, ak, bk, gravity, coriolis, divdamp, vortdamp)) {
    delete s;
    return nullptr;
  }
  return s;
}
void orc_destroy(orc_state* s) { delete s; }
int orc_field_levels(orc_state* s, int field) {
  A3<double>* a = field_ptr<double>(s, field);
  return a ? a->k1 : -1;
}
int orc_set_field(orc_state* s, int field, const double* a, int with_halo) {
  return set_field<double>(s, field, a, nullptr, with_halo);
}
int orc_get_field(orc_state* s, int field, double* a, int with_halo) {
  return a ? get_field<double>(s, field, a, nullptr, with_halo) : -1;
}
void orc_init(orc_state* s) { init_state<double>(s); }
void orc_cgrid_step(orc_state* s, double dt) { cgrid_dynamics_step<double>(s, dt); }
void orc_cgrid_halo(orc_state* s) { cgrid_halo<double>(s); }
void orc_dgrid_step(orc_state* s, double dt) { dgrid_dynamics_step<double>(s, dt); }
void orc_remap(orc_state* s) { perform_vertical_remapping<double>(s); }
void orc_dgrid_halo(orc_state* s) { dgrid_halo<double>(s); }
void orc_physics_tendencies(orc_state* s) { calculate_physics_tendencies<double>(s); }
void orc_apply_physics(orc_state* s, double dt) { apply_physics_tendencies<double>(s, dt); }
void orc_physics_halo(orc_state* s) { physics_halo<double>(s); }

// mod_fields.f90:69-106
int orc_check_stability(orc_state* s) {
  for (A3<double>* a : {&s->dp, &s->pt, &s->ud, &s->vd})
    for (int k = 1; k <= s->nlay; ++k)
      for (int j = s->jsd; j <= s->jed; ++j)
        for (int i = s->isd; i <= s->ied; ++i)
          if (!std::isfinite((*a)(i, j, k))) return 0;
  return 1;
}

double orc_mass(orc_state* s) {
  double m = 0.;
  for (int k = 1; k <= s->nlay; ++k)
    for (int j = s->jsd; j <= s->jed; ++j)
      for (int i = s->isd; i <= s->ied; ++i) m += s->dp(i, j, k);
  return m;
}

void orc_set_threads(orc_state* s, int n) { s->nthreads = n < 1 ? 1 : n; }
void orc_set_poison(orc_state* s, int on) { s->poison = on != 0; }
void orc_set_remap_trace(orc_state* s, int32_t* buf) { s->trace = buf; }

void orc_pow_array(const double* x, double y, double* out, int n) {
  for (int i = 0; i < n; ++i) out[i] = orc_pow_impl(x[i], y);
}
void orc_log_array(const double* x, double* out, int n) {
  for (int i = 0; i < n; ++i) out[i] = orc_log_impl(x[i]);
}

// ---- tangent-linear model: the same restatement on dual numbers
orc_tlm* tlm_create(int nx, int ny, int nlay, double dx, double dy, const double* ak, const double* bk,
                    double gravity, double coriolis, double divdamp, double vortdamp) {
  orc_tlm* s = new orc_tlm();
  if (!setup_state<Dual>(s, nx, ny, nlay, dx, dy, ak, bk, gravity, coriolis, divdamp, vortdamp)) {
    delete s;
    return nullptr;
  }
  return s;
}
void tlm_destroy(orc_tlm* s) { delete s; }
int tlm_set_field(orc_tlm* s, int field, const double* val, const double* tan, int with_halo) {
  return set_field<Dual>(s, field, val, tan, with_halo);
}
int tlm_get_field(orc_tlm* s, int field, double* val, double* tan, int with_halo) {
  return get_field<Dual>(s, field, val, tan, with_halo);
}
void tlm_init(orc_tlm* s) { init_state<Dual>(s); }
void tlm_cgrid_step(orc_tlm* s, double dt) { cgrid_dynamics_step<Dual>(s, dt); }
void tlm_cgrid_halo(orc_tlm* s) { cgrid_halo<Dual>(s); }
void tlm_dgrid_step(orc_tlm* s, double dt) { dgrid_dynamics_step<Dual>(s, dt); }
void tlm_remap(orc_tlm* s) { perform_vertical_remapping<Dual>(s); }
void tlm_dgrid_halo(orc_tlm* s) { dgrid_halo<Dual>(s); }
void tlm_set_threads(orc_tlm* s, int n) { s->nthreads = n < 1 ? 1 : n; }

}  // extern "C"
