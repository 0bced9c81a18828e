// Per-layer sweep kernels of the B200 dynamical core (one CTA = one
// TX x TY tile of one layer), second generation:
//  * the input tiles plus their stencil halo arrive by TMA (atm_tma.cuh);
//  * every PPM sweep is split into per-cell stages: the monotone slopes
//    dqi_mono (src/mod_sw_dyn.f90:870-875) once per cell, for
//    PPM_CONSTRAINED also the edge values once per cell (:877-911), and
//    then the per-interface flux (:802-838) from those, as the reference's
//    ppm/flux pair does for a whole row.
// Formulas, index shifts and evaluation order are those of the first
// generation (and of the reference), so the FP64 results are unchanged.
#pragma once

#include <type_traits>

#include "atm_kernels.cuh"
#include "atm_tma.cuh"

namespace atm {

// Edge anomalies of a cell from precomputed monotone slopes.  q points at
// the cell (cell spacing sq), mono at its monotone slope (spacing sm).  The
// raw slope dqi of the cell is recomputed from q exactly as slopes() forms it.
template <typename T, int V>
__device__ __forceinline__ void edges_pre(const T* q, int sq, const T* mono, int sm, T& eL, T& eR) {
  const T q0 = q[0];
  eL = (q[-sq] - q0) * T(0.5) + div_const<3>(mono[-sm] - mono[0]);
  eR = (q[sq] - q0) * T(0.5) + div_const<3>(mono[0] - mono[sm]);
  if (V == PPM_CON || V == PPM_NN) {
    const T d0 = (q[sq] - q[-sq]) * T(0.25);
    const T lim = T(2) * fab(d0);
    eL = -cpsign(mn(lim, fab(eL)), d0);
    eR = +cpsign(mn(lim, fab(eR)), d0);
    if (V == PPM_NN) {
      eL = mx(eL, -q0);
      eR = mx(eR, -q0);
      T a = eR - eL;
      T b = T(-3) * (eR + eL);
      if ((fab(a) < -b) && (q0 + a * a / (T(4) * b) + div_const<12>(b) < T(0))) {
        if (eL * eR > T(0)) {
          eL = T(0);
          eR = T(0);
        } else if (eL > eR) {
          eL = T(2) * fab(eR);
        } else {
          eR = T(2) * fab(eL);
        }
      }
    }
  }
}

// Flux at the interface between cells i-1 and i with slopes precomputed
// (PPM_UNCONSTRAINED / PPM_NONNEGATIVE): only the upwind cell's edges.
// q and mono point at cell i.
template <typename T, int V>
__device__ __forceinline__ T flux_pre(const T* q, int sq, const T* mono, int sm, T c) {
  T sa = fab(c);
  T k1 = (T(1) - T(2) * sa) * (T(1) - sa);
  T k2 = sa * (sa - T(1));
  T eL, eR;
  if (c > T(0)) {
    edges_pre<T, V>(q - sq, sq, mono - sm, sm, eL, eR);
    return q[-sq] + k1 * eR + k2 * eL;
  }
  edges_pre<T, V>(q, sq, mono, sm, eL, eR);
  return q[0] + k1 * eL + k2 * eR;
}

// Flux with precomputed edges (PPM_CONSTRAINED): q points at cell i
// (spacing sq), eL and eR at its edges (spacing se).
template <typename T>
__device__ __forceinline__ T flux_con_pre(const T* q, int sq, const T* eL, const T* eR, int se, T c) {
  const T eLm = eL[-se], eRm = eR[-se], eL0 = eL[0], eR0 = eR[0];
  if ((T(3) * fab(eL0 + eR0) > fab(eL0 - eR0)) && (T(3) * fab(eLm + eRm) > fab(eLm - eRm)))
    return (c > T(0)) ? q[-sq] : q[0];
  T sa = fab(c);
  T k1 = (T(1) - T(2) * sa) * (T(1) - sa);
  T k2 = sa * (sa - T(1));
  if (c > T(0)) return q[-sq] + k1 * eRm + k2 * eLm;
  return q[0] + k1 * eL0 + k2 * eR0;
}

// Monotone slope of one cell from its neighbours along s.
template <typename T>
__device__ __forceinline__ T slope_at(const T* q, int s) {
  T mono, dqi;
  slopes(q[-s], q[0], q[s], dqi, mono);
  return mono;
}

// 128-byte aligned start of the dynamic shared memory (TMA destinations)
__device__ __forceinline__ unsigned char* smem_base(unsigned char* raw) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
}

// A shared-memory window of type S read as the sweep type T.
template <typename S, typename T>
struct SmAs {
  Sm<S> s;
  __device__ __forceinline__ T operator()(int x, int y) const { return T(s(x, y)); }
};

// Region loop: body(x, y) for every point of [x0, x0+W) x [y0, y0+Hh).
template <int W, int Hh, typename F>
__device__ __forceinline__ void region(int x0, int y0, F&& body) {
  for (int idx = threadIdx.x; idx < W * Hh; idx += NT) {
    const int y = idx / W;
    const int x = idx - y * W;
    body(x0 + x, y0 + y);
  }
}

// One stage's independent region loops as a single index space: the block's
// threads share the whole stage evenly, where separate region() loops of
// W*H a little above NT points each leave most threads idle in a last
// partial pass.  regions(reg<W1, H1>(x1, y1, body1), reg<W2, H2>(...), ...).
template <int W, int Hh, typename F>
struct Reg {
  static constexpr int N = W * Hh;
  int x0, y0;
  F body;
  __device__ __forceinline__ void at(int idx) const {
    const int y = idx / W;
    body(x0 + idx - y * W, y0 + y);
  }
};
template <int W, int Hh, typename F>
__device__ __forceinline__ Reg<W, Hh, F> reg(int x0, int y0, F body) {
  return Reg<W, Hh, F>{x0, y0, body};
}
template <typename R0, typename... Rs>
__device__ __forceinline__ void reg_dispatch(int idx, const R0& r0, const Rs&... rs) {
  if (idx < R0::N) r0.at(idx);
  else if constexpr (sizeof...(Rs) > 0) reg_dispatch(idx - R0::N, rs...);
}
template <typename R>
__device__ __forceinline__ void reg_loop(const R& r) {
  for (int idx = threadIdx.x; idx < R::N; idx += NT) r.at(idx);
}
// MERGE = false runs the regions one after the other (separate loops), the
// better schedule where the merged dispatch costs more registers than the
// idle threads it saves.
template <bool MERGE = true, typename... Rs>
__device__ __forceinline__ void regions(const Rs&... rs) {
  if constexpr (MERGE) {
    constexpr int N = (Rs::N + ...);
    for (int idx = threadIdx.x; idx < N; idx += NT) reg_dispatch(idx, rs...);
  } else {
    (reg_loop(rs), ...);
  }
}

// Start of a TMA box whose first wanted column is i0, rounded down to a
// 16-byte boundary of the tensor row.
template <typename T>
__device__ __forceinline__ int tma_x0(int i0) {
  constexpr int q = tma_q<T>();
  return ((i0 + H + XOFF) / q) * q - H - XOFF;
}

// ---------------------------------------------------------------- mass ----
// S: element type of the prognostic state (dp, pt, ud, vd), C: of the
// C-grid fields (dpc, ptc, uc, vc), T: the sweep arithmetic.  The FP64 form
// has S = C = T = double; the mixed form keeps the state in double, the
// C-grid fields in float and sweeps in float.
template <typename T, int TX, int TY, bool CGRID, typename S = T, typename C = T>
struct MassL {
  // TMA boxes: dp and pt (state), and the u, v boxes (D winds on the C grid
  // step, C winds on the D grid step)
  using UB = std::conditional_t<CGRID, S, C>;
  static_assert(CGRID || std::is_same_v<C, T>, "the D-grid step sweeps with the C-grid winds' type");
  static constexpr int WD = tma_width<S>(TX + 6), HD = TY + 6;
  static constexpr int WU = tma_width<UB>(CGRID ? TX + 2 : TX + 1), HU = CGRID ? TY + 7 : TY + 6;
  static constexpr int WV = tma_width<UB>(CGRID ? TX + 7 : TX + 6), HV = CGRID ? TY + 2 : TY + 1;
  static constexpr uint32_t tx_bytes =
      (uint32_t)(2 * WD * HD * sizeof(S) + (WU * HU + WV * HV) * sizeof(UB));
  static constexpr size_t boxes = 2 * tma_box_bytes(WD, HD, sizeof(S)) + tma_box_bytes(WU, HU, sizeof(UB)) +
                                  tma_box_bytes(WV, HV, sizeof(UB));
  static constexpr bool NN = !CGRID;
  static constexpr size_t work =
      (CGRID ? box_bytes<T>(TX + 1, TY + 6) + box_bytes<T>(TX + 6, TY + 1) : 0) +  // uc, vc (C grid)
      2 * box_bytes<T>(TX + 6, TY) + 2 * box_bytes<T>(TX, TY + 6) +               // inner sweeps
      2 * box_bytes<T>(TX + 2, TY + 2) +                                         // Laplacians
      2 * box_bytes<T>(TX + 4, TY) + 2 * box_bytes<T>(TX, TY + 4) +               // slopes
      2 * box_bytes<T>(TX + 1, TY) + 2 * box_bytes<T>(TX, TY + 1);                // fluxes
  static constexpr size_t bytes = boxes + work + 128;
  // CTAs per SM the register budget is set for (measured): FP64 C grid 6
  // on 32 x 4 tiles (40 registers), FP64 D grid 5 on 32 x 6 tiles (48
  // registers); the FP32 sweeps keep the compiler's choice
  static constexpr int min_blocks = !std::is_same_v<T, double> ? 1 : CGRID ? 6 : 5;
};

template <typename T, int TX, int TY, bool CGRID, typename S = T, typename C = T>
__global__ void __launch_bounds__(NT, MassL<T, TX, TY, CGRID, S, C>::min_blocks) k_mass2(const __grid_constant__ CUtensorMap m_dp,
                                              const __grid_constant__ CUtensorMap m_pt,
                                              const __grid_constant__ CUtensorMap m_u,
                                              const __grid_constant__ CUtensorMap m_v, Geom g, Consts c,
                                              const double* __restrict__ heat,
                                              std::conditional_t<CGRID, C, S>* __restrict__ dpo,
                                              std::conditional_t<CGRID, C, S>* __restrict__ pto, int lo, int hi,
                                              int* nonfinite, int* timeout) {
  using Lay = MassL<T, TX, TY, CGRID, S, C>;
  using UB = typename Lay::UB;
  using O = std::conditional_t<CGRID, C, S>;
  constexpr int V = CGRID ? PPM_UNC : PPM_NN;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z;
  const int ox = lo + blockIdx.x * TX, oy = lo + blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);

  auto sbox = [&](int i0, int j0, int w, int h) {
    Sm<S> s{reinterpret_cast<S*>(p), tma_x0<S>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(S));
    return s;
  };
  auto ubox = [&](int i0, int j0, int w, int h) {
    Sm<UB> s{reinterpret_cast<UB*>(p), tma_x0<UB>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(UB));
    return s;
  };
  Sm<S> sdp = sbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<S> spt = sbox(ox - 3, oy - 3, Lay::WD, Lay::HD);
  Sm<UB> su = CGRID ? ubox(ox - 1, oy - 3, Lay::WU, Lay::HU) : ubox(ox, oy - 3, Lay::WU, Lay::HU);
  Sm<UB> sv = CGRID ? ubox(ox - 3, oy - 1, Lay::WV, Lay::HV) : ubox(ox - 3, oy, Lay::WV, Lay::HV);
  {
    const TmaBox boxes[4] = {{&m_dp, sdp.p, sdp.x0, sdp.y0, k},
                             {&m_pt, spt.p, spt.x0, spt.y0, k},
                             {&m_u, su.p, su.x0, su.y0, k},
                             {&m_v, sv.p, sv.x0, sv.y0, k}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  // C-grid winds: built from the D-grid winds (C step) or the loaded boxes (D step)
  Sm<T> suc, svc;
  if constexpr (CGRID) {
    suc = carve<T>(p, ox, oy - 3, TX + 1, TY + 6);
    svc = carve<T>(p, ox - 3, oy, TX + 6, TY + 1);
  } else {
    suc = su;
    svc = sv;
  }
  Sm<T> tyd = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> typ = carve<T>(p, ox - 3, oy, TX + 6, TY);
  Sm<T> txd = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> txp = carve<T>(p, ox, oy - 3, TX, TY + 6);
  Sm<T> lpd = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> lpp = carve<T>(p, ox - 1, oy - 1, TX + 2, TY + 2);
  Sm<T> mxd = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> mxp = carve<T>(p, ox - 2, oy, TX + 4, TY);
  Sm<T> myd = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> myp = carve<T>(p, ox, oy - 2, TX, TY + 4);
  Sm<T> fxd = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fxp = carve<T>(p, ox, oy, TX + 1, TY);
  Sm<T> fyd = carve<T>(p, ox, oy, TX, TY + 1);
  Sm<T> fyp = carve<T>(p, ox, oy, TX, TY + 1);

  // merged stage loops measured faster in FP32, slower in FP64
  constexpr bool MG = std::is_same_v<T, float>;
  if constexpr (CGRID) {  // mod_sw_dyn.f90:109-117
    regions<MG>(reg<TX + 1, TY + 6>(ox, oy - 3, [&](int x, int y) {
      T ub = T(.5) * (T(su(x, y)) + T(su(x - 1, y)));
      suc(x, y) = T(.5) * (ub + T(.5) * (T(su(x, y + 1)) + T(su(x - 1, y + 1))));
    }),
            reg<TX + 6, TY + 1>(ox - 3, oy, [&](int x, int y) {
      T vb = T(.5) * (T(sv(x, y)) + T(sv(x, y - 1)));
      svc(x, y) = T(.5) * (vb + T(.5) * (T(sv(x + 1, y)) + T(sv(x + 1, y - 1))));
    }));
    __syncthreads();
  }
  // inner sweeps and Laplacians: mod_sw_dyn.f90:142-155,176-185 (C); 470-482,503-511 (D)
  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  regions<MG>(reg<TX + 6, TY>(ox - 3, oy, [&](int x, int y) {
    T cy0 = dtdx * svc(x, y), cy1 = dtdx * svc(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (svc(x, y + 1) - svc(x, y)));
    const T d0 = T(sdp(x, y)), dm = T(sdp(x, y - 1)), dq = T(sdp(x, y + 1));
    T f0 = (cy0 > T(0)) ? dm : d0;
    T f1 = (cy1 > T(0)) ? d0 : dq;
    tyd(x, y) = T(.5) * (d0 + den * (d0 - rA * (f1 - f0)));
    const T p0 = T(spt(x, y)), pm = T(spt(x, y - 1)), pq = T(spt(x, y + 1));
    f0 = (cy0 > T(0)) ? pm : p0;
    f1 = (cy1 > T(0)) ? p0 : pq;
    typ(x, y) = T(.5) * (p0 + den * (p0 - rA * (f1 - f0)));
  }),
          reg<TX, TY + 6>(ox, oy - 3, [&](int x, int y) {
    T cx0 = dtdx * suc(x, y), cx1 = dtdx * suc(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (suc(x + 1, y) - suc(x, y)));
    const T d0 = T(sdp(x, y)), dm = T(sdp(x - 1, y)), dq = T(sdp(x + 1, y));
    T f0 = (cx0 > T(0)) ? dm : d0;
    T f1 = (cx1 > T(0)) ? d0 : dq;
    txd(x, y) = T(.5) * (d0 + den * (d0 - rA * (f1 - f0)));
    const T p0 = T(spt(x, y)), pm = T(spt(x - 1, y)), pq = T(spt(x + 1, y));
    f0 = (cx0 > T(0)) ? pm : p0;
    f1 = (cx1 > T(0)) ? p0 : pq;
    txp(x, y) = T(.5) * (p0 + den * (p0 - rA * (f1 - f0)));
  }),
          reg<TX + 2, TY + 2>(ox - 1, oy - 1, [&](int x, int y) {
    lpd(x, y) = T(-2.) * T(sdp(x, y)) * rdxy + (T(sdp(x + 1, y)) + T(sdp(x - 1, y))) * rdx2 +
                (T(sdp(x, y + 1)) + T(sdp(x, y - 1))) * rdy2;
    lpp(x, y) = T(-2.) * T(spt(x, y)) * rdxy + (T(spt(x + 1, y)) + T(spt(x - 1, y))) * rdx2 +
                (T(spt(x, y + 1)) + T(spt(x, y - 1))) * rdy2;
  }));
  __syncthreads();
  // monotone slopes of the outer sweeps (ppm, :870-875)
  regions<MG>(reg<TX + 4, TY>(ox - 2, oy, [&](int x, int y) {
    mxd(x, y) = slope_at(tyd.ptr(x, y), 1);
    mxp(x, y) = slope_at(typ.ptr(x, y), 1);
  }),
          reg<TX, TY + 4>(ox, oy - 2, [&](int x, int y) {
    myd(x, y) = slope_at(txd.ptr(x, y), TX);
    myp(x, y) = slope_at(txp.ptr(x, y), TX);
  }));
  __syncthreads();
  // outer sweeps (PPM)
  regions<MG>(reg<TX + 1, TY>(ox, oy, [&](int x, int y) {
    T cx = dtdx * suc(x, y);
    fxd(x, y) = flux_pre<T, V>(tyd.ptr(x, y), 1, mxd.ptr(x, y), 1, cx) * cx;
    fxp(x, y) = flux_pre<T, V>(typ.ptr(x, y), 1, mxp.ptr(x, y), 1, cx);
  }),
          reg<TX, TY + 1>(ox, oy, [&](int x, int y) {
    T cy = dtdx * svc(x, y);
    fyd(x, y) = flux_pre<T, V>(txd.ptr(x, y), TX, myd.ptr(x, y), TX, cy) * cy;
    fyp(x, y) = flux_pre<T, V>(txp.ptr(x, y), TX, myp.ptr(x, y), TX, cy);
  }));
  __syncthreads();

  // updates, mod_sw_dyn.f90:163-172,193-202,230-237,258-267 (C); 490-499,519-528,555-562,582-591 (D)
  const int xhi = g.nx - 1 + hi, yhi = g.ny - 1 + hi;
  const T dxv = dtdx * T(c.vdx), dyv = dtdy * T(c.vdy), vdx = T(c.vdx), vdy = T(c.vdy);
  bool bad = false;
  region<TX, TY>(ox, oy, [&](int x, int y) {
    if (x > xhi || y > yhi) return;
    O vo, qo;
    if constexpr (std::is_same_v<S, T>) {  // the reference's operations, in order
      T d = sdp(x, y);
      T v = d - (fxd(x + 1, y) - fxd(x, y) + dxv * (lpd(x + 1, y) - T(2.) * lpd(x, y) + lpd(x - 1, y)));
      v = v - (fyd(x, y + 1) - fyd(x, y) + dyv * (lpd(x, y + 1) - T(2.) * lpd(x, y) + lpd(x, y - 1)));
      T q = d * spt(x, y) - (fxp(x + 1, y) * fxd(x + 1, y) - fxp(x, y) * fxd(x, y) +
                             vdx * ((lpp(x + 1, y) - lpp(x, y)) * fxd(x + 1, y) - (lpp(x, y) - lpp(x - 1, y)) * fxd(x, y)));
      q = q - (fyp(x, y + 1) * fyd(x, y + 1) - fyp(x, y) * fyd(x, y) +
               vdy * ((lpp(x, y + 1) - lpp(x, y)) * fyd(x, y + 1) - (lpp(x, y) - lpp(x, y - 1)) * fyd(x, y)));
      if (heat) q = q + dt * d * T(heat[g.at(x, y, k)]);
      q = q / v;
      vo = O(v);
      qo = O(q);
    } else {
      // the same update in flux form: interface fluxes (advective plus
      // vorticity-damping) in the sweep type, their differences applied to
      // the state's type, so that mass and dp*pt telescope in S
      auto Fx = [&](int xx) { return fxd(xx, y) + dxv * (lpd(xx, y) - lpd(xx - 1, y)); };
      auto Fy = [&](int yy) { return fyd(x, yy) + dyv * (lpd(x, yy) - lpd(x, yy - 1)); };
      auto Hx = [&](int xx) { return (fxp(xx, y) + vdx * (lpp(xx, y) - lpp(xx - 1, y))) * fxd(xx, y); };
      auto Hy = [&](int yy) { return (fyp(x, yy) + vdy * (lpp(x, yy) - lpp(x, yy - 1))) * fyd(x, yy); };
      const S d = sdp(x, y);
      const S v = d - ((S(Fx(x + 1)) - S(Fx(x))) + (S(Fy(y + 1)) - S(Fy(y))));
      S q = d * spt(x, y) - ((S(Hx(x + 1)) - S(Hx(x))) + (S(Hy(y + 1)) - S(Hy(y))));
      if (heat) q = q + S(c.dt) * d * S(heat[g.at(x, y, k)]);
      q = q / v;
      vo = O(v);
      qo = O(q);
    }
    long long o = g.at(x, y, k);
    dpo[o] = vo;
    pto[o] = qo;
    bool inside = x >= 0 && x < g.nx && y >= 0 && y < g.ny;
    bad = bad || (inside && !(finite_(vo) && finite_(qo)));
  });
  if (nonfinite) flag_nonfinite(nonfinite, bad);
}

// ======================================================== C-grid momentum ==
template <typename T, int TX, int TY, typename S = T>
struct CMomL {
  static constexpr int WU = tma_width<S>(TX + 7), HU = TY + 7;   // ud box x in [ox-4, ox+TX+2]
  static constexpr int WV = tma_width<S>(TX + 7), HV = TY + 7;   // vd box x in [ox-3, ox+TX+3]
  static constexpr int WL = tma_width<S>(TX + 3), HL = TY + 3;   // layer-nlay ud, vd
  static constexpr int WP = tma_width<double>(TX + 1), HP = TY + 1;  // pkap, gz at k and k+1
  // all eight input boxes at once (the adjoint kernel's layout)
  static constexpr uint32_t tx_bytes =
      (uint32_t)((WU * HU + WV * HV + 2 * WL * HL) * sizeof(S) + 4 * WP * HP * sizeof(double));
  static constexpr size_t boxes = tma_box_bytes(WU, HU, sizeof(S)) + tma_box_bytes(WV, HV, sizeof(S)) +
                                  2 * tma_box_bytes(WL, HL, sizeof(S)) + 4 * tma_box_bytes(WP, HP, 8);
  // The forward loads ud, vd and the layer-nlay winds first (tx_main) and
  // the PGF boxes pkap, gz (tx_pgf) after the kinetic-energy stage, three
  // into the ud, vd boxes and one into the layer-nlay ud box, which no later
  // stage reads (the update reads the cell's ud, vd from global memory);
  // the Laplacian of the vorticity is formed a stage later, into the
  // layer-nlay vd box.
  static constexpr uint32_t tx_main = (uint32_t)((WU * HU + WV * HV + 2 * WL * HL) * sizeof(S));
  static constexpr uint32_t tx_pgf = (uint32_t)(4 * WP * HP * sizeof(double));
  static constexpr size_t boxes_main = tma_box_bytes(WU, HU, sizeof(S)) + tma_box_bytes(WV, HV, sizeof(S)) +
                                       2 * tma_box_bytes(WL, HL, sizeof(S));
  static_assert(3 * tma_box_bytes(WP, HP, 8) <= tma_box_bytes(WU, HU, sizeof(S)) + tma_box_bytes(WV, HV, sizeof(S)),
                "three PGF boxes fit where the ud, vd boxes were");
  static_assert(tma_box_bytes(WP, HP, 8) <= tma_box_bytes(WL, HL, sizeof(S)), "one PGF box fits in a layer-nlay box");
  static_assert(box_bytes<T>(TX + 1, TY + 1) <= tma_box_bytes(WL, HL, sizeof(S)), "lap fits in a layer-nlay box");
  // slopes of the KE sweeps, later of the vorticity-flux sweeps (one buffer)
  static constexpr size_t slopes_ke = box_bytes<T>(TX + 1, TY + 4) + box_bytes<T>(TX + 4, TY + 1);
  static constexpr size_t slopes_vf = box_bytes<T>(TX, TY + 3) + box_bytes<T>(TX + 3, TY);
  static constexpr size_t slopes = slopes_ke > slopes_vf ? slopes_ke : slopes_vf;
  static constexpr size_t work = 2 * box_bytes<T>(TX + 6, TY + 6) +                  // uc1, vc1
                                 box_bytes<T>(TX + 5, TY + 5) + box_bytes<T>(TX + 1, TY + 1) +  // vor, ke
                                 box_bytes<T>(TX, TY + 5) + box_bytes<T>(TX + 5, TY) +  // tU, tV
                                 slopes;                                              // slopes
  static constexpr size_t bytes = boxes_main + work + 128;
};

// The layer-nlay A-grid winds at (x, y) from the layer-nlay D-grid winds
// (src/mod_sw_dyn.f90:110-125 at k = nlay), recomputed where they are read.
template <typename T, typename A>
__device__ __forceinline__ void al_winds(const A& udL, const A& vdL, int x, int y, T& ua, T& va) {
  T ub = T(.5) * (udL(x, y) + udL(x - 1, y));
  T ucl = T(.5) * (ub + T(.5) * (udL(x, y + 1) + udL(x - 1, y + 1)));
  ua = T(.5) * (ucl + T(.25) * (udL(x + 1, y) + udL(x, y) + udL(x + 1, y + 1) + udL(x, y + 1)));
  T vb = T(.5) * (vdL(x, y) + vdL(x, y - 1));
  T vcl = T(.5) * (vb + T(.5) * (vdL(x + 1, y) + vdL(x + 1, y - 1)));
  va = T(.5) * (vcl + T(.25) * (vdL(x, y + 1) + vdL(x, y) + vdL(x + 1, y + 1) + vdL(x + 1, y)));
}

template <typename T, int TX, int TY, typename S = T, typename C = T>
__global__ void __launch_bounds__(NT) k_c_mom2(const __grid_constant__ CUtensorMap m_ud,
                                               const __grid_constant__ CUtensorMap m_vd,
                                               const __grid_constant__ CUtensorMap m_udL,
                                               const __grid_constant__ CUtensorMap m_vdL,
                                               const __grid_constant__ CUtensorMap m_pk,
                                               const __grid_constant__ CUtensorMap m_gz, Geom g, Consts c,
                                               const S* __restrict__ ud, const S* __restrict__ vd,
                                               C* __restrict__ uc, C* __restrict__ vc, int* timeout) {
  using Lay = CMomL<T, TX, TY, S>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar, bar_pgf;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy);

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<S> s{reinterpret_cast<S*>(p), tma_x0<S>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(S));
    return s;
  };
  Sm<S> bud = tbox(ox - 4, oy - 3, Lay::WU, Lay::HU);
  Sm<S> bvd = tbox(ox - 3, oy - 4, Lay::WV, Lay::HV);
  Sm<S> budL = tbox(ox - 2, oy - 2, Lay::WL, Lay::HL);
  Sm<S> bvdL = tbox(ox - 2, oy - 2, Lay::WL, Lay::HL);
  const SmAs<S, T> sud{bud}, svd{bvd}, udL{budL}, vdL{bvdL};
  {
    const TmaBox boxes[4] = {{&m_ud, bud.p, bud.x0, bud.y0, k},
                             {&m_vd, bvd.p, bvd.x0, bvd.y0, k},
                             {&m_udL, budL.p, budL.x0, budL.y0, L - 1},
                             {&m_vdL, bvdL.p, bvdL.x0, bvdL.y0, L - 1}};
    if (!tma_fetch(boxes, Lay::tx_main, &bar, timeout, &s_ok)) return;
  }
  // the PGF boxes, loaded after the kinetic energy: three where ud, vd
  // were, one where the layer-nlay ud was
  unsigned char* pq = reinterpret_cast<unsigned char*>(bud.p);
  auto qbox = [&](unsigned char*& q) {
    Sm<double> s{reinterpret_cast<double*>(q), tma_x0<double>(ox - 1), oy - 1, Lay::WP};
    q += tma_box_bytes(Lay::WP, Lay::HP, 8);
    return s;
  };
  const Sm<double> pk0 = qbox(pq);
  const Sm<double> pk1 = qbox(pq);
  const Sm<double> gz0 = qbox(pq);
  unsigned char* pl = reinterpret_cast<unsigned char*>(budL.p);
  const Sm<double> gz1 = qbox(pl);
  // the Laplacian of the vorticity, formed after the kinetic energy, where
  // the layer-nlay vd was
  unsigned char* plap = reinterpret_cast<unsigned char*>(bvdL.p);
  Sm<T> lap = carve<T>(plap, ox, oy, TX + 1, TY + 1);
  Sm<T> uc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> vc1 = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
  Sm<T> vor = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> ke = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  Sm<T> tU = carve<T>(p, ox, oy - 2, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 2, oy, TX + 5, TY);
  // the KE sweeps' slopes are dead before the vorticity-flux sweeps' ones
  // are written (a __syncthreads apart): they share memory
  unsigned char* ps = p;
  Sm<T> mvy = carve<T>(ps, ox - 1, oy - 2, TX + 1, TY + 4);  // slopes of vc1 along y
  Sm<T> mux = carve<T>(ps, ox - 2, oy - 1, TX + 4, TY + 1);  // slopes of uc1 along x
  ps = p;
  Sm<T> mtU = carve<T>(ps, ox, oy - 1, TX, TY + 3);          // slopes of tU along y
  Sm<T> mtV = carve<T>(ps, ox - 1, oy, TX + 3, TY);          // slopes of tV along x
  p += Lay::slopes;

  // C-grid winds of this layer (first-loop values, mod_sw_dyn.f90:110-117)
  region<TX + 6, TY + 6>(ox - 3, oy - 3, [&](int x, int y) {
    T ub = T(.5) * (sud(x, y) + sud(x - 1, y));
    uc1(x, y) = T(.5) * (ub + T(.5) * (sud(x, y + 1) + sud(x - 1, y + 1)));
    T vb = T(.5) * (svd(x, y) + svd(x, y - 1));
    vc1(x, y) = T(.5) * (vb + T(.5) * (svd(x + 1, y) + svd(x + 1, y - 1)));
  });
  __syncthreads();

  const T f = T(c.coriolis);
  // vorticity (mod_sw_dyn.f90:319-323), slopes of the KE sweeps
  regions(reg<TX + 5, TY + 5>(ox - 2, oy - 2, [&](int x, int y) {
    vor(x, y) = f - (uc1(x, y) - uc1(x, y - 1)) * rdy + (vc1(x, y) - vc1(x - 1, y)) * rdx;
  }),
          reg<TX + 1, TY + 4>(ox - 1, oy - 2, [&](int x, int y) { mvy(x, y) = slope_at(vc1.ptr(x, y), TX + 6); }),
          reg<TX + 4, TY + 1>(ox - 2, oy - 1, [&](int x, int y) { mux(x, y) = slope_at(uc1.ptr(x, y), 1); }));
  __syncthreads();

  // kinetic energy (:299-317): q(j) = vc(i, j+1), q(i) = uc(i+1, j); vorticity
  // advection: inner sweeps and Laplacian (:344-367, 388-397)
  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  regions(reg<TX + 1, TY + 1>(ox - 1, oy - 1, [&](int x, int y) {
    T ua, va;  // A-grid winds of layer nlay (mod_sw_dyn.f90:110-125 at k = nlay)
    al_winds<T>(udL, vdL, x, y, ua, va);
    T fy = flux_pre<T, PPM_UNC>(vc1.ptr(x, y + 1), TX + 6, mvy.ptr(x, y + 1), TX + 1, dtdy * va);
    T kv = va * fy;
    T fx = flux_pre<T, PPM_UNC>(uc1.ptr(x + 1, y), 1, mux.ptr(x + 1, y), 1, dtdx * ua);
    ke(x, y) = T(.5) * (kv + ua * fx);
  }),
          reg<TX, TY + 5>(ox, oy - 2, [&](int x, int y) {
    T c0 = dtdx * sud(x - 1, y), c1 = dtdx * sud(x, y);
    T den = T(1) / (T(1) - dtdx * (sud(x, y) - sud(x - 1, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }),
          reg<TX + 5, TY>(ox - 2, oy, [&](int x, int y) {
    T c0 = dtdx * svd(x, y - 1), c1 = dtdx * svd(x, y);
    T den = T(1) / (T(1) - dtdy * (svd(x, y) - svd(x, y - 1)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  }));
  __syncthreads();
  {  // ud, vd and the layer-nlay winds are read no more: the PGF boxes go there
    const TmaBox boxes[4] = {{&m_pk, pk0.p, pk0.x0, pk0.y0, k}, {&m_pk, pk1.p, pk1.x0, pk1.y0, k + 1},
                             {&m_gz, gz0.p, gz0.x0, gz0.y0, k}, {&m_gz, gz1.p, gz1.x0, gz1.y0, k + 1}};
    tma_issue(boxes, Lay::tx_pgf, &bar_pgf);
  }
  regions(reg<TX, TY + 3>(ox, oy - 1, [&](int x, int y) { mtU(x, y) = slope_at(tU.ptr(x, y), TX); }),
          reg<TX + 3, TY>(ox - 1, oy, [&](int x, int y) { mtV(x, y) = slope_at(tV.ptr(x, y), 1); }),
          reg<TX + 1, TY + 1>(ox, oy, [&](int x, int y) {
    lap(x, y) = T(-2.) * vor(x, y) * rdxy + (vor(x + 1, y) + vor(x - 1, y)) * rdx2 +
                (vor(x, y + 1) + vor(x, y - 1)) * rdy2;
  }));
  if (!tma_wait(&bar_pgf, timeout, &s_ok)) return;

  // uc, vc updates (:369-381, 399-411) with the PGF (:325-339)
  const T vdx = T(c.vdx), vdy = T(c.vdy);
  region<TX, TY>(ox, oy, [&](int x, int y) {
    if (x >= g.nx || y >= g.ny) return;
    double pgx = ((pk0(x, y) - pk1(x - 1, y)) * (gz0(x - 1, y) - gz1(x, y)) +
                  (pk0(x - 1, y) - pk1(x, y)) * (gz1(x - 1, y) - gz0(x, y))) /
                 (pk0(x, y) - pk1(x - 1, y) + pk0(x - 1, y) - pk1(x, y));
    double pgy = ((pk0(x, y) - pk1(x, y - 1)) * (gz0(x, y - 1) - gz1(x, y)) +
                  (pk0(x, y - 1) - pk1(x, y)) * (gz1(x, y - 1) - gz0(x, y))) /
                 (pk0(x, y) - pk1(x, y - 1) + pk0(x, y - 1) - pk1(x, y));
    const long long o = g.at(x, y, k);
    const T udx = T(ud[o]), vdx_ = T(vd[o]);  // the cell's ud, vd (their boxes hold the PGF now)
    T fy = flux_pre<T, PPM_UNC>(tU.ptr(x, y + 1), TX, mtU.ptr(x, y + 1), TX, dtdx * vdx_);
    T u = uc1(x, y) + dt * (vdx_ * fy + vdy * (lap(x, y + 1) - lap(x, y))) -
          dtdx * (ke(x, y) - ke(x - 1, y) - T(pgx));
    T fx = flux_pre<T, PPM_UNC>(tV.ptr(x + 1, y), 1, mtV.ptr(x + 1, y), 1, dtdx * udx);
    T v = vc1(x, y) - dt * (udx * fx + vdx * (lap(x + 1, y) - lap(x, y))) -
          dtdy * (ke(x, y) - ke(x, y - 1) - T(pgy));
    uc[o] = C(u);
    vc[o] = C(v);
  });
}

// ======================================================== D-grid momentum ==
template <typename T, int TX, int TY, typename S = T, typename C = T>
struct DMomL {
  static_assert(std::is_same_v<C, T>, "the D-grid step sweeps with the C-grid winds' type");
  static constexpr int WU = tma_width<S>(TX + 6), HU = TY + 6;       // ud, vd: [ox-3, ox+TX+2]^2
  static constexpr int WUL = tma_width<T>(TX + 1), HUL = TY + 5;     // uc layer nlay: x [ox, ox+TX], y [oy-3, oy+TY+1]
  static constexpr int WVL = tma_width<T>(TX + 5), HVL = TY + 1;     // vc layer nlay: x [ox-3, ox+TX+1], y [oy, oy+TY]
  static constexpr int WC = tma_width<T>(TX), HC = TY;               // uc, vc of the layer at the outputs
  static constexpr int WP = tma_width<double>(TX + 1), HP = TY + 1;  // pkapb, gzb
  // all ten input boxes at once (the adjoint kernels' layouts)
  static constexpr uint32_t tx_bytes = (uint32_t)(2 * WU * HU * sizeof(S) +
                                                   (WUL * HUL + WVL * HVL + 2 * WC * HC) * sizeof(T) +
                                                   4 * WP * HP * sizeof(double));
  static constexpr size_t boxes = 2 * tma_box_bytes(WU, HU, sizeof(S)) + tma_box_bytes(WUL, HUL, sizeof(T)) +
                                  tma_box_bytes(WVL, HVL, sizeof(T)) + 2 * tma_box_bytes(WC, HC, sizeof(T)) +
                                  4 * tma_box_bytes(WP, HP, 8);
  // The FP64 forward loads ud, vd and the C-grid winds first (tx_main) and
  // the PGF boxes pkapb, gzb (tx_pgf) later, into the ud, vd boxes, which
  // the stages after the kinetic energy do not read (its update reads the
  // cell's ud, vd from global memory): 34 KB, 6 CTAs per SM instead of 5.
  // The mixed form, at 6 CTAs by its registers already, loads all ten at once.
  static constexpr bool LATE_PGF = std::is_same_v<S, T>;
  static constexpr uint32_t tx_main =
      (uint32_t)(2 * WU * HU * sizeof(S) + (WUL * HUL + WVL * HVL + 2 * WC * HC) * sizeof(T));
  static constexpr uint32_t tx_pgf = (uint32_t)(4 * WP * HP * sizeof(double));
  static constexpr size_t boxes_main = 2 * tma_box_bytes(WU, HU, sizeof(S)) + tma_box_bytes(WUL, HUL, sizeof(T)) +
                                       tma_box_bytes(WVL, HVL, sizeof(T)) + 2 * tma_box_bytes(WC, HC, sizeof(T));
  static_assert(4 * tma_box_bytes(WP, HP, 8) <= 2 * tma_box_bytes(WU, HU, sizeof(S)),
                "the PGF boxes fit where the ud, vd boxes were");
  // the state's ud, vd as sweep-type copies when the types differ
  static constexpr size_t conv = std::is_same_v<S, T> ? 0 : 2 * box_bytes<T>(TX + 6, TY + 6);
  // vor (later ke and dv4), dv0, dv2, tU, tV, lap
  static_assert(2 * box_bytes<T>(TX + 1, TY + 1) <= box_bytes<T>(TX + 5, TY + 5), "ke, dv4 fit where vor was");
  static constexpr size_t work = box_bytes<T>(TX + 5, TY + 5) + box_bytes<T>(TX + 5, TY + 5) +
                                 box_bytes<T>(TX + 3, TY + 3) + box_bytes<T>(TX, TY + 5) + box_bytes<T>(TX + 5, TY) +
                                 box_bytes<T>(TX + 1, TY + 1);
  // slopes of the KE sweeps, later of the vorticity-flux sweeps (one buffer)
  static constexpr size_t slopes_ke = box_bytes<T>(TX + 1, TY + 4) + box_bytes<T>(TX + 4, TY + 1);
  static constexpr size_t slopes_vf = box_bytes<T>(TX, TY + 3) + box_bytes<T>(TX + 3, TY);
  static constexpr size_t slopes = slopes_ke > slopes_vf ? slopes_ke : slopes_vf;
  // edges of the KE sweeps, later of the vorticity-flux sweeps (one buffer)
  static constexpr size_t edges_ke = 2 * box_bytes<T>(TX + 1, TY + 2) + 2 * box_bytes<T>(TX + 2, TY + 1);
  static constexpr size_t edges_vf = 2 * box_bytes<T>(TX, TY + 1) + 2 * box_bytes<T>(TX + 1, TY);
  static constexpr size_t edges = edges_ke > edges_vf ? edges_ke : edges_vf;
  static constexpr size_t bytes = (LATE_PGF ? boxes_main : boxes) + conv + work + slopes + edges + 128;
};

template <typename T, int TX, int TY, typename S = T, typename C = T>
__global__ void __launch_bounds__(NT) k_d_mom2(const __grid_constant__ CUtensorMap m_ud,
                                               const __grid_constant__ CUtensorMap m_vd,
                                               const __grid_constant__ CUtensorMap m_ucL,
                                               const __grid_constant__ CUtensorMap m_vcL,
                                               const __grid_constant__ CUtensorMap m_uc,
                                               const __grid_constant__ CUtensorMap m_vc,
                                               const __grid_constant__ CUtensorMap m_pkb,
                                               const __grid_constant__ CUtensorMap m_gzb, Geom g, Consts c,
                                               const S* __restrict__ ud, const S* __restrict__ vd,
                                               S* __restrict__ udo, S* __restrict__ vdo, int* nonfinite,
                                               int* timeout) {
  using Lay = DMomL<T, TX, TY, S, C>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar, bar_pgf;
  __shared__ int s_ok;
  unsigned char* p = smem_base(smem);
  const int k = blockIdx.z, L = g.L;
  const int ox = blockIdx.x * TX, oy = blockIdx.y * TY;
  const T dt = T(c.dt), dtdx = T(c.dtdx), dtdy = T(c.dtdy), rA = T(c.rA);
  const T rdx = T(c.rdx), rdy = T(c.rdy);

  auto tbox = [&](int i0, int j0, int w, int h) {
    Sm<T> s{reinterpret_cast<T*>(p), tma_x0<T>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(T));
    return s;
  };
  auto sbox = [&](int i0, int j0, int w, int h) {
    Sm<S> s{reinterpret_cast<S*>(p), tma_x0<S>(i0), j0, w};
    p += tma_box_bytes(w, h, sizeof(S));
    return s;
  };
  Sm<S> bud = sbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<S> bvd = sbox(ox - 3, oy - 3, Lay::WU, Lay::HU);
  Sm<T> ucL = tbox(ox, oy - 3, Lay::WUL, Lay::HUL);
  Sm<T> vcL = tbox(ox - 3, oy, Lay::WVL, Lay::HVL);
  Sm<T> suc = tbox(ox, oy, Lay::WC, Lay::HC);
  Sm<T> svc = tbox(ox, oy, Lay::WC, Lay::HC);
  // the PGF boxes: in the ud, vd boxes, loaded later (FP64), or after the
  // C-grid winds and loaded with the rest
  unsigned char* pq = Lay::LATE_PGF ? reinterpret_cast<unsigned char*>(bud.p) : p;
  auto qbox = [&]() {
    Sm<double> s{reinterpret_cast<double*>(pq), tma_x0<double>(ox), oy, Lay::WP};
    pq += tma_box_bytes(Lay::WP, Lay::HP, 8);
    return s;
  };
  const Sm<double> pb0 = qbox();
  const Sm<double> pb1 = qbox();
  const Sm<double> gb0 = qbox();
  const Sm<double> gb1 = qbox();
  if constexpr (Lay::LATE_PGF) {
    const TmaBox boxes[6] = {{&m_ud, bud.p, bud.x0, bud.y0, k},      {&m_vd, bvd.p, bvd.x0, bvd.y0, k},
                             {&m_ucL, ucL.p, ucL.x0, ucL.y0, L - 1}, {&m_vcL, vcL.p, vcL.x0, vcL.y0, L - 1},
                             {&m_uc, suc.p, suc.x0, suc.y0, k},      {&m_vc, svc.p, svc.x0, svc.y0, k}};
    if (!tma_fetch(boxes, Lay::tx_main, &bar, timeout, &s_ok)) return;
  } else {
    p = pq;
    const TmaBox boxes[10] = {
        {&m_ud, bud.p, bud.x0, bud.y0, k},       {&m_vd, bvd.p, bvd.x0, bvd.y0, k},
        {&m_ucL, ucL.p, ucL.x0, ucL.y0, L - 1},  {&m_vcL, vcL.p, vcL.x0, vcL.y0, L - 1},
        {&m_uc, suc.p, suc.x0, suc.y0, k},       {&m_vc, svc.p, svc.x0, svc.y0, k},
        {&m_pkb, pb0.p, pb0.x0, pb0.y0, k},      {&m_pkb, pb1.p, pb1.x0, pb1.y0, k + 1},
        {&m_gzb, gb0.p, gb0.x0, gb0.y0, k},      {&m_gzb, gb1.p, gb1.x0, gb1.y0, k + 1}};
    if (!tma_fetch(boxes, Lay::tx_bytes, &bar, timeout, &s_ok)) return;
  }
  // ud, vd in the sweep type (the boxes themselves when the types agree)
  constexpr int WQ = std::is_same_v<S, T> ? Lay::WU : TX + 6;
  Sm<T> sud, svd;
  if constexpr (std::is_same_v<S, T>) {
    sud = bud;
    svd = bvd;
  } else {
    sud = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
    svd = carve<T>(p, ox - 3, oy - 3, TX + 6, TY + 6);
    region<TX + 6, TY + 6>(ox - 3, oy - 3, [&](int x, int y) {
      sud(x, y) = T(bud(x, y));
      svd(x, y) = T(bvd(x, y));
    });
    __syncthreads();
  }
  Sm<T> vor = carve<T>(p, ox - 3, oy - 3, TX + 5, TY + 5);
  // ke and dv4 are written after the last read of vor (a __syncthreads apart)
  unsigned char* pk = reinterpret_cast<unsigned char*>(vor.p);
  Sm<T> ke = carve<T>(pk, ox, oy, TX + 1, TY + 1);
  Sm<T> dv4 = carve<T>(pk, ox, oy, TX + 1, TY + 1);
  Sm<T> dv0 = carve<T>(p, ox - 2, oy - 2, TX + 5, TY + 5);
  Sm<T> dv2 = carve<T>(p, ox - 1, oy - 1, TX + 3, TY + 3);
  Sm<T> tU = carve<T>(p, ox, oy - 3, TX, TY + 5);
  Sm<T> tV = carve<T>(p, ox - 3, oy, TX + 5, TY);
  Sm<T> lap = carve<T>(p, ox - 1, oy - 1, TX + 1, TY + 1);
  // the KE sweeps' slopes and edges are dead before the vorticity-flux
  // sweeps' ones are written (two __syncthreads apart): they share memory
  unsigned char* ps = p;
  Sm<T> mvy = carve<T>(ps, ox, oy - 2, TX + 1, TY + 4);
  Sm<T> mux = carve<T>(ps, ox - 2, oy, TX + 4, TY + 1);
  ps = p;
  Sm<T> mtU = carve<T>(ps, ox, oy - 2, TX, TY + 3);
  Sm<T> mtV = carve<T>(ps, ox - 2, oy, TX + 3, TY);
  p += Lay::slopes;
  unsigned char* pe = p;
  Sm<T> lvy = carve<T>(pe, ox, oy - 1, TX + 1, TY + 2), rvy = carve<T>(pe, ox, oy - 1, TX + 1, TY + 2);
  Sm<T> lux = carve<T>(pe, ox - 1, oy, TX + 2, TY + 1), rux = carve<T>(pe, ox - 1, oy, TX + 2, TY + 1);
  pe = p;
  Sm<T> ltU = carve<T>(pe, ox, oy - 1, TX, TY + 1), rtU = carve<T>(pe, ox, oy - 1, TX, TY + 1);
  Sm<T> ltV = carve<T>(pe, ox - 1, oy, TX + 1, TY), rtV = carve<T>(pe, ox - 1, oy, TX + 1, TY);
  p += Lay::edges;

  const T f = T(c.coriolis);
  // vorticity (:659-663), divergence (:682-685), slopes of the KE sweeps
  region<TX + 5, TY + 5>(ox - 3, oy - 3, [&](int x, int y) {
    vor(x, y) = f - (sud(x, y + 1) - sud(x, y)) * rdy + (svd(x + 1, y) - svd(x, y)) * rdx;
    int xd = x + 1, yd = y + 1;
    dv0(xd, yd) = rdx * (sud(xd, yd) - sud(xd - 1, yd)) + rdy * (svd(xd, yd) - svd(xd, yd - 1));
  });
  region<TX + 1, TY + 4>(ox, oy - 2, [&](int x, int y) { mvy(x, y) = slope_at(svd.ptr(x, y), WQ); });
  region<TX + 4, TY + 1>(ox - 2, oy, [&](int x, int y) { mux(x, y) = slope_at(sud.ptr(x, y), 1); });
  __syncthreads();

  const T rdx2 = T(c.rdx2), rdy2 = T(c.rdy2), rdxy = T(c.rdx2rdy2);
  // edges of the KE sweeps; del^2 of the divergence (:688-692); inner
  // sweeps of the vorticity with the layer-nlay Courant numbers (:708-722, 744-753)
  region<TX + 1, TY + 2>(ox, oy - 1, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(svd.ptr(x, y), WQ, mvy.ptr(x, y), TX + 1, eL, eR);
    lvy(x, y) = eL;
    rvy(x, y) = eR;
  });
  region<TX + 2, TY + 1>(ox - 1, oy, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(sud.ptr(x, y), 1, mux.ptr(x, y), 1, eL, eR);
    lux(x, y) = eL;
    rux(x, y) = eR;
  });
  region<TX + 3, TY + 3>(ox - 1, oy - 1, [&](int x, int y) {
    dv2(x, y) = T(-2.) * dv0(x, y) * rdxy + (dv0(x + 1, y) + dv0(x - 1, y)) * rdx2 + (dv0(x, y + 1) + dv0(x, y - 1)) * rdy2;
  });
  region<TX, TY + 5>(ox, oy - 3, [&](int x, int y) {
    T c0 = dtdx * ucL(x, y), c1 = dtdx * ucL(x + 1, y);
    T den = T(1) / (T(1) - dtdx * (ucL(x + 1, y) - ucL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x - 1, y) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x + 1, y);
    tU(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  });
  region<TX + 5, TY>(ox - 3, oy, [&](int x, int y) {
    T c0 = dtdx * vcL(x, y), c1 = dtdx * vcL(x, y + 1);
    T den = T(1) / (T(1) - dtdy * (vcL(x, y + 1) - vcL(x, y)));
    T f0 = (c0 > T(0)) ? vor(x, y - 1) : vor(x, y);
    T f1 = (c1 > T(0)) ? vor(x, y) : vor(x, y + 1);
    tV(x, y) = T(.5) * (vor(x, y) + den * (vor(x, y) - rA * (f1 - f0)));
  });
  region<TX + 1, TY + 1>(ox - 1, oy - 1, [&](int x, int y) {
    lap(x, y) = T(-2.) * vor(x, y) * rdxy + (vor(x + 1, y) + vor(x - 1, y)) * rdx2 + (vor(x, y + 1) + vor(x, y - 1)) * rdy2;
  });
  __syncthreads();
  // kinetic energy with PPM_CONSTRAINED (:639-657) and the layer-nlay
  // B-grid winds (:441-444), del^4 (:695-702), slopes of the vorticity-flux sweeps
  region<TX + 1, TY + 1>(ox, oy, [&](int x, int y) {
    const T ubL = T(.5) * (ucL(x, y) + ucL(x, y - 1));
    const T vbL = T(.5) * (vcL(x, y) + vcL(x - 1, y));
    T fy = flux_con_pre<T>(svd.ptr(x, y), WQ, lvy.ptr(x, y), rvy.ptr(x, y), TX + 1, dtdy * vbL);
    T kv = vbL * fy;
    T fx = flux_con_pre<T>(sud.ptr(x, y), 1, lux.ptr(x, y), rux.ptr(x, y), 1, dtdx * ubL);
    ke(x, y) = T(.5) * (kv + ubL * fx);
  });
  const T divdamp = T(c.divdamp);
  region<TX + 1, TY + 1>(ox, oy, [&](int x, int y) {
    T d4 = T(-2.) * dv2(x, y) * rdxy + (dv2(x + 1, y) + dv2(x - 1, y)) * rdx2 + (dv2(x, y + 1) + dv2(x, y - 1)) * rdy2;
    dv4(x, y) = divdamp * d4;
  });
  region<TX, TY + 3>(ox, oy - 2, [&](int x, int y) { mtU(x, y) = slope_at(tU.ptr(x, y), TX); });
  region<TX + 3, TY>(ox - 2, oy, [&](int x, int y) { mtV(x, y) = slope_at(tV.ptr(x, y), 1); });
  __syncthreads();
  if constexpr (Lay::LATE_PGF) {  // the ud, vd boxes are read no more: the PGF boxes go there
    const TmaBox boxes[4] = {{&m_pkb, pb0.p, pb0.x0, pb0.y0, k}, {&m_pkb, pb1.p, pb1.x0, pb1.y0, k + 1},
                             {&m_gzb, gb0.p, gb0.x0, gb0.y0, k}, {&m_gzb, gb1.p, gb1.x0, gb1.y0, k + 1}};
    tma_issue(boxes, Lay::tx_pgf, &bar_pgf);
  }
  region<TX, TY + 1>(ox, oy - 1, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(tU.ptr(x, y), TX, mtU.ptr(x, y), TX, eL, eR);
    ltU(x, y) = eL;
    rtU(x, y) = eR;
  });
  region<TX + 1, TY>(ox - 1, oy, [&](int x, int y) {
    T eL, eR;
    edges_pre<T, PPM_CON>(tV.ptr(x, y), 1, mtV.ptr(x, y), 1, eL, eR);
    ltV(x, y) = eL;
    rtV(x, y) = eR;
  });
  if constexpr (Lay::LATE_PGF) {
    if (!tma_wait(&bar_pgf, timeout, &s_ok)) return;
  } else {
    __syncthreads();
  }

  // ud, vd updates (:724-738, 755-769) with the B-grid PGF (:665-679); the
  // state's ud, vd of the cell from global memory (FP64) or its box
  const T vdx = T(c.vdx), vdy = T(c.vdy);
  bool bad = false;
  region<TX, TY>(ox, oy, [&](int x, int y) {
    if (x >= g.nx || y >= g.ny) return;
    double pgx = ((pb0(x + 1, y) - pb1(x, y)) * (gb0(x, y) - gb1(x + 1, y)) +
                  (pb0(x, y) - pb1(x + 1, y)) * (gb1(x, y) - gb0(x + 1, y))) /
                 (pb0(x + 1, y) - pb1(x, y) + pb0(x, y) - pb1(x + 1, y));
    double pgy = ((pb0(x, y + 1) - pb1(x, y)) * (gb0(x, y) - gb1(x, y + 1)) +
                  (pb0(x, y) - pb1(x, y + 1)) * (gb1(x, y) - gb0(x, y + 1))) /
                 (pb0(x, y + 1) - pb1(x, y) + pb0(x, y) - pb1(x, y + 1));
    T fy = flux_con_pre<T>(tU.ptr(x, y), TX, ltU.ptr(x, y), rtU.ptr(x, y), TX, dtdx * vcL(x, y));
    T fx = flux_con_pre<T>(tV.ptr(x, y), 1, ltV.ptr(x, y), rtV.ptr(x, y), 1, dtdx * ucL(x, y));
    const long long o = g.at(x, y, k);
    S u, v;
    if constexpr (std::is_same_v<S, T>) {  // the reference's operations, in order
      u = ud[o] + dt * (svc(x, y) * fy + vdy * (lap(x, y) - lap(x, y - 1))) -
          dtdx * (ke(x + 1, y) - ke(x, y) - dv4(x + 1, y) + dv4(x, y) - T(pgx));
      v = vd[o] - dt * (suc(x, y) * fx + vdx * (lap(x, y) - lap(x - 1, y))) -
          dtdy * (ke(x, y + 1) - ke(x, y) - dv4(x, y + 1) + dv4(x, y) - T(pgy));
    } else {  // the tendency in the sweep type added to the state's type
      const T du = dt * (svc(x, y) * fy + vdy * (lap(x, y) - lap(x, y - 1))) -
                   dtdx * (ke(x + 1, y) - ke(x, y) - dv4(x + 1, y) + dv4(x, y) - T(pgx));
      const T dv = -dt * (suc(x, y) * fx + vdx * (lap(x, y) - lap(x - 1, y))) -
                   dtdy * (ke(x, y + 1) - ke(x, y) - dv4(x, y + 1) + dv4(x, y) - T(pgy));
      u = bud(x, y) + S(du);
      v = bvd(x, y) + S(dv);
    }
    udo[o] = u;
    vdo[o] = v;
    bad = bad || !(finite_(u) && finite_(v));
  });
  flag_nonfinite(nonfinite, bad);
}

}  // namespace atm
