// C-ABI of the B200 dynamical core (declarations and reference citations in
// include/atmdyn.h).  One context = one single-image domain on one device:
// all fields live in HBM with the reference's 7-wide halo, ping-pong
// buffers hold two time levels of the prognostic state, and every entry
// point enqueues kernels on the context's stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "atmdyn.h"
#include "atm_ensemble.cuh"
#include "atm_ops.h"
#include "atm_physics.h"
#include "atm_radiation.h"

using atm::Geom;
using atm::H;
using atm::XOFF;

namespace {

enum { F_DP = 0, F_PT = 1, F_UD = 2, F_VD = 3 };
enum { C_DPC = 0, C_PTC = 1, C_UC = 2, C_VC = 3 };

// interior <-> contiguous (K, ny, nx) device buffer, with type conversion
template <typename A, typename B>
__global__ void k_interior(Geom g, const A* __restrict__ src, B* __restrict__ dst, int K, int to_field) {
  long long n = (long long)g.nx * g.ny * K;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.nx);
    long long r = q / g.nx;
    int j = (int)(r % g.ny);
    int k = (int)(r / g.ny);
    long long o = g.at(i, j, k);
    if (to_field)
      dst[o] = B(src[q]);
    else
      dst[q] = B(src[o]);
  }
}

// accumulate_output (src/mod_output.f90:94-128): each sum gains dt * value
// with the reference's operations; its compensated_sum never stores the
// compensation, so every update is the plain FP64 add out + val.  The
// winds are the cell-centre averages .5 (ud(j) + ud(j+1)), .5 (vd(i) + vd(i+1)).
template <typename T>
__global__ void k_accumulate(Geom g, const T* __restrict__ dp, const T* __restrict__ pt, const T* __restrict__ ud,
                             const T* __restrict__ vd, const double* __restrict__ nf, const double* __restrict__ ts,
                             double dt, double* acc_dp, double* acc_pt, double* acc_u, double* acc_v, double* acc_nf,
                             double* acc_ts) {
  const long long n = (long long)g.nx * g.ny;
  const long long total = n * (g.L + 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q / n);
    const long long r = q - (long long)k * n;
    const int j = (int)(r / g.nx), i = (int)(r - (long long)j * g.nx);
    const long long o = g.at(i, j, k);
    if (k < g.L) {
      acc_dp[q] = acc_dp[q] + dt * (double)dp[o];
      acc_pt[q] = acc_pt[q] + dt * (double)pt[o];
      acc_u[q] = acc_u[q] + dt * .5 * ((double)ud[o] + (double)ud[o + g.P]);
      acc_v[q] = acc_v[q] + dt * .5 * ((double)vd[o] + (double)vd[o + 1]);
    }
    acc_nf[q] = acc_nf[q] + dt * (nf ? nf[o] : 0.);
    if (k == 0) acc_ts[q] = acc_ts[q] + dt * ts[o];
  }
}

__global__ void k_fill(double* p, long long n, double v) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    p[q] = v;
}

}  // namespace

struct atm_ctx {
  int nx = 0, ny = 0, L = 0, precision = 0, flags = 0;
  double dx = 0, dy = 0;
  std::vector<double> ak, bk;
  Geom geo{};
  atm::Consts cst{};
  const atm::Ops* ops = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  void* st[2][4] = {{nullptr}};
  int cur = 0;
  void* cg[4] = {nullptr};
  double *pkap = nullptr, *gz = nullptr, *pkapb = nullptr, *gzb = nullptr, *stage = nullptr;
  void *urem = nullptr, *vrem = nullptr;
  double *nf = nullptr, *heat = nullptr;
  bool heating = false;
  double *d_ak = nullptr, *d_bk = nullptr, *partial = nullptr, *d_mass = nullptr;
  atm::Status* status = nullptr;
  atm::Status* h_status = nullptr;  // pinned
  double* h_mass = nullptr;         // pinned
  int uploaded = 0;
  bool initialized = false;
  bool flag_valid = false;
  bool remapped = false;
  int32_t* trace_host = nullptr;
  int* trace_fallback = nullptr;
  int* d_trace = nullptr;
  size_t trace_elems = 0;
  // per-stage CUDA-event timing (atm_profile) and the kernel launch counter
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_stage;  // stage of each recorded (start, stop) pair
  size_t ev_used = 0;
  long long launches = 0;
  // adjoint (FP64): two slots of state adjoints (physical index of slot IN
  // is slot_in; the slots swap as steps are reversed), the C-grid adjoints,
  // and the adjoints of pkap, gz, pkapb, gzb and the remapped face winds
  bool adj = false;
  double* lam[2][4] = {{nullptr}};
  double* lam_cg[4] = {nullptr};
  double *lam_pk = nullptr, *lam_gz = nullptr, *lam_pkb = nullptr, *lam_gzb = nullptr;
  double *lam_ur = nullptr, *lam_vr = nullptr;
  int slot_in = 0;
  // output accumulation (src/mod_output.f90:94-142): interior (nx, ny, K)
  // sums of dt * dp, pt, u, v (nlay levels) and net_flux (nlay+1 levels)
  double* acc[6] = {nullptr};
  double acc_time = 0.;
  // column physics (src/mod_physics.f90): surface temperature ts (one
  // level, allocated with the context) and the tendencies of pt, u, v on
  // the A grid and of ts (allocated by the first atm_physics_tendencies)
  double* ts = nullptr;
  double *ph_pt = nullptr, *ph_u = nullptr, *ph_v = nullptr, *ph_ts = nullptr;
  bool phys_ready = false;
  // radiation (src/mod_radiation.f90): the gas-optics tables in one device
  // block (pointers in rad), the distance of each cell centre from the
  // origin (ny, nx) (src/mod_input.f90:233-243)
  double* rad_block = nullptr;
  atm::RadTables rad{};
  double* radius = nullptr;
  std::string err;
};

namespace {

const int MASS_BLOCKS = 296;

int fail(atm_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(atm_ctx* c, const char* what, cudaError_t e) {
  return fail(c, ATM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                               \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail(ctx, #call, e_);   \
  } while (0)

int field_levels(const atm_ctx* c, int f) {
  switch (f) {
    case ATM_DP: case ATM_PT: case ATM_UD: case ATM_VD: return c->L;
    case ATM_DPC: case ATM_PTC: case ATM_UC: case ATM_VC: return c->L;
    case ATM_GZ: case ATM_PLEV: case ATM_PKAP: case ATM_NET_FLUX: return c->L + 1;
    case ATM_TS: return 1;
    default: return -1;
  }
}

size_t level_elems(const atm_ctx* c) { return (size_t)c->geo.S; }

atm::Consts step_consts(const atm_ctx* c, double dt) {
  atm::Consts k = c->cst;
  k.dt = dt;
  k.dtdx = dt * k.rdx;  // mod_sw_dyn.f90:85-86,429-430
  k.dtdy = dt * k.rdy;
  return k;
}

atm::RemapArgs remap_args(const atm_ctx* c) {
  return atm::RemapArgs{c->d_ak, c->d_bk, c->cst.ptop, c->cst.pk_top};
}

void free_all(atm_ctx* c) {
  for (int t = 0; t < 2; ++t)
    for (int f = 0; f < 4; ++f) cudaFree(c->st[t][f]);
  for (int f = 0; f < 4; ++f) cudaFree(c->cg[f]);
  void* ps[] = {c->pkap, c->gz, c->pkapb, c->gzb, c->stage, c->urem, c->vrem, c->nf, c->heat,
                c->d_ak, c->d_bk, c->partial, c->d_mass, c->status, c->d_trace};
  for (void* p : ps) cudaFree(p);
  for (int t = 0; t < 2; ++t)
    for (int f = 0; f < 4; ++f) cudaFree(c->lam[t][f]);
  for (int f = 0; f < 4; ++f) cudaFree(c->lam_cg[f]);
  double* pl[] = {c->lam_pk, c->lam_gz, c->lam_pkb, c->lam_gzb, c->lam_ur, c->lam_vr};
  for (double* p : pl) cudaFree(p);
  for (double* p : c->acc) cudaFree(p);
  double* ph[] = {c->ts, c->ph_pt, c->ph_u, c->ph_v, c->ph_ts, c->rad_block, c->radius};
  for (double* p : ph) cudaFree(p);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->h_mass) cudaFreeHost(c->h_mass);
  if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
}

// host (is:ie, js:je, 1:K) FP64 array <-> pitched FP64 device array
cudaError_t h2d_pitched(atm_ctx* c, double* dev, const double* host, int K) {
  const int wrow = c->nx + 2 * H;
  return cudaMemcpy2DAsync(dev + XOFF, (size_t)c->geo.P * 8, host, (size_t)wrow * 8, (size_t)wrow * 8,
                           (size_t)c->geo.NYP * K, cudaMemcpyHostToDevice, c->stream);
}
cudaError_t d2h_pitched(atm_ctx* c, double* host, const double* dev, int K) {
  const int wrow = c->nx + 2 * H;
  return cudaMemcpy2DAsync(host, (size_t)wrow * 8, dev + XOFF, (size_t)c->geo.P * 8, (size_t)wrow * 8,
                           (size_t)c->geo.NYP * K, cudaMemcpyDeviceToHost, c->stream);
}

const char* const STAGE_NAMES[] = {"c_mass",  "c_column", "c_mom",        "c_halo",      "d_ring",
                                   "d_mass",  "d_column", "d_corners",    "d_mom",       "remap_ring",
                                   "remap_winds", "remap_energy", "d_halo", "heating", "check",
                                   "adj_forward", "adj_remap", "adj_d_mom_ke", "adj_d_column", "adj_d_mass_x",
                                   "adj_c_column", "adj_c_mom", "adj_c_mass", "adj_halo",
                                   "phys_tend", "phys_apply", "phys_halo", "adj_d_mom_vf", "adj_d_mass_y",
                                   "radiation", "radiation_halo"};
constexpr int NSTAGE = 31;
enum { S_CMASS, S_CCOL, S_CMOM, S_CHALO, S_DRING, S_DMASS, S_DCOL, S_DCORN, S_DMOM, S_RRING, S_RWIND, S_RENER,
       S_DHALO, S_HEAT, S_CHECK, S_AFWD, S_ARMP, S_ADMOM, S_ADCOL, S_ADMASS, S_ACCOL, S_ACMOM, S_ACMASS, S_AHALO,
       S_PHYS_TEND, S_PHYS_APPLY, S_PHYS_HALO, S_ADMOM_VF, S_ADMASS_Y, S_RAD, S_RAD_HALO };

// Brackets one stage (one kernel launch unless noted) with CUDA events on
// the context's stream when profiling is on, and counts the launch.
struct Stage {
  atm_ctx* c;
  int id;
  int nlaunch;
  size_t slot;
  Stage(atm_ctx* ctx, int stage, int n = 1) : c(ctx), id(stage), nlaunch(n), slot(0) {
    if (!c->prof) return;
    slot = c->ev_used;
    while (c->ev_pool.size() < slot + 2) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->ev_pool.push_back(e);
    }
    c->ev_used += 2;
    c->ev_stage.push_back(id);
    cudaEventRecord(c->ev_pool[slot], c->stream);
  }
  ~Stage() {
    c->launches += nlaunch;
    if (c->prof) cudaEventRecord(c->ev_pool[slot + 1], c->stream);
  }
};

int require_init(atm_ctx* c) {
  if (!c) return ATM_ERR_ARG;
  if (!c->initialized) return fail(c, ATM_ERR_STATE, "atm_init has not been called");
  return ATM_OK;
}

}  // namespace

extern "C" {

const char* atm_version(void) { return "libatmdyn 0.1 (sm_100a)"; }

const char* atm_last_error(atm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int atm_create(atm_ctx** out, int nx, int ny, int nlay, double dx, double dy, const double* ak, const double* bk,
               double g, double f, double divdamp, double vortdamp, int precision, int flags) {
  if (!out) return ATM_ERR_ARG;
  *out = nullptr;
  if (nx < H || ny < H || nlay < 3 || nlay > atm::MAX_LAYERS || !(dx > 0) || !(dy > 0) || !ak || !bk ||
      (precision != ATM_FP64 && precision != ATM_MIXED))
    return ATM_ERR_ARG;
  atm_ctx* ctx = new atm_ctx();
  ctx->nx = nx; ctx->ny = ny; ctx->L = nlay; ctx->dx = dx; ctx->dy = dy;
  ctx->precision = precision; ctx->flags = flags;
  ctx->ak.assign(ak, ak + nlay + 1);
  ctx->bk.assign(bk, bk + nlay + 1);
  ctx->ops = precision == ATM_FP64 ? &atm::ops_fp64 : &atm::ops_mixed;
  Geom& geo = ctx->geo;
  geo.nx = nx; geo.ny = ny; geo.L = nlay;
  geo.P = ((XOFF + nx + 2 * H) + 31) / 32 * 32;
  geo.NYP = ny + 2 * H;
  geo.S = (long long)geo.P * geo.NYP;
  // init_sw_dyn, src/mod_sw_dyn.f90:961-1021
  atm::Consts& k = ctx->cst;
  k.rdx = 1. / dx;
  k.rdx2 = 1. / (dx * dx);
  k.rdy = 1. / dy;
  k.rdy2 = 1. / (dy * dy);
  k.rdx2rdy2 = k.rdx2 + k.rdy2;
  k.rA = 1. / (dx * dy);
  double dd = divdamp * dx * dy;
  k.divdamp = dd * dd;
  double vortdamp_coeff = vortdamp * dx * dy;
  k.vdx = dy * k.rdx * vortdamp_coeff;
  k.vdy = dx * k.rdy * vortdamp_coeff;
  k.coriolis = f;
  k.gravity = g;
  k.ptop = ak[0];
  k.pk_top = atm_pow(ak[0], atm::KAPPA);

  cudaError_t e;
  if ((e = cudaGetDevice(&ctx->device)) != cudaSuccess) { int r = cuda_fail(ctx, "cudaGetDevice", e); delete ctx; return r; }
  if ((e = ctx->ops->setup()) != cudaSuccess) { int r = cuda_fail(ctx, "kernel set-up", e); delete ctx; return r; }
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    int r = cuda_fail(ctx, "cudaStreamCreate", e); delete ctx; return r;
  }
  const size_t es = (size_t)ctx->ops->elem;
  const size_t lay = level_elems(ctx) * nlay * es;
  const size_t lev = level_elems(ctx) * (nlay + 1) * 8;
  bool ok = true;
  auto alloc = [&](void** p, size_t bytes) {
    if (!ok) return;
    if (cudaMalloc(p, bytes) != cudaSuccess) { ok = false; return; }
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) ok = false;
  };
  for (int t = 0; t < 2; ++t)
    for (int fi = 0; fi < 4; ++fi) alloc(&ctx->st[t][fi], lay);
  const size_t lay_cg = level_elems(ctx) * nlay * (size_t)ctx->ops->cg_elem;
  for (int fi = 0; fi < 4; ++fi) alloc(&ctx->cg[fi], lay_cg);
  alloc(&ctx->urem, lay);
  alloc(&ctx->vrem, lay);
  alloc((void**)&ctx->pkap, lev);
  alloc((void**)&ctx->gz, lev);
  alloc((void**)&ctx->pkapb, lev);
  alloc((void**)&ctx->gzb, lev);
  alloc((void**)&ctx->stage, lev);
  alloc((void**)&ctx->ts, level_elems(ctx) * 8);
  alloc((void**)&ctx->d_ak, (nlay + 1) * 8);
  alloc((void**)&ctx->d_bk, (nlay + 1) * 8);
  alloc((void**)&ctx->partial, MASS_BLOCKS * 8);
  alloc((void**)&ctx->d_mass, 8);
  alloc((void**)&ctx->status, sizeof(atm::Status));
  if (ok && cudaMallocHost((void**)&ctx->h_status, sizeof(atm::Status)) != cudaSuccess) ok = false;
  if (ok && cudaMallocHost((void**)&ctx->h_mass, 8) != cudaSuccess) ok = false;
  if (!ok) {
    cudaGetLastError();
    free_all(ctx);
    delete ctx;
    return ATM_ERR_NOMEM;
  }
  if (cudaMemcpy(ctx->d_ak, ak, (nlay + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(ctx->d_bk, bk, (nlay + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
    free_all(ctx);
    delete ctx;
    return ATM_ERR_CUDA;
  }
  *out = ctx;
  return ATM_OK;
}

int atm_destroy(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return ATM_OK;
}

int atm_set_stream(atm_ctx* ctx, void* stream) {
  if (!ctx) return ATM_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) CK(cudaStreamDestroy(ctx->stream));
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
    ctx->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return ATM_OK;
}

int atm_upload(atm_ctx* ctx, int field, const double* host) {
  if (!ctx || !host) return ATM_ERR_ARG;
  const atm::Ops& ops = *ctx->ops;
  if (field >= ATM_DP && field <= ATM_VD) {
    void* dst = ctx->st[ctx->cur][field];
    if (ops.elem == 8) {
      CK(h2d_pitched(ctx, (double*)dst, host, ctx->L));
    } else {
      CK(h2d_pitched(ctx, ctx->stage, host, ctx->L));
      CK(ops.from_double(ctx->stage, dst, ctx->geo.S * ctx->L, ctx->stream));
    }
  } else if (field == ATM_GZ) {
    CK(h2d_pitched(ctx, ctx->gz, host, 1));  // level 1: surface geopotential
  } else if (field == ATM_NET_FLUX) {
    return atm_set_net_flux(ctx, host);
  } else if (field == ATM_TS) {
    CK(h2d_pitched(ctx, ctx->ts, host, 1));
  } else {
    return fail(ctx, ATM_ERR_ARG, "field cannot be uploaded");
  }
  ctx->uploaded |= 1 << field;
  ctx->flag_valid = false;
  return ATM_OK;
}

int atm_upload_device(atm_ctx* ctx, int field, const void* dev, int dtype_bytes) {
  if (!ctx || !dev || (dtype_bytes != 4 && dtype_bytes != 8)) return ATM_ERR_ARG;
  if (field < ATM_DP || field > ATM_GZ) return fail(ctx, ATM_ERR_ARG, "field cannot be uploaded");
  const int K = field == ATM_GZ ? 1 : ctx->L;
  const bool dbl_field = field == ATM_GZ || ctx->ops->elem == 8;
  void* dst = field == ATM_GZ ? (void*)ctx->gz : ctx->st[ctx->cur][field];
  dim3 grid(1184), block(256);
  if (dbl_field && dtype_bytes == 8) k_interior<double, double><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const double*)dev, (double*)dst, K, 1);
  else if (dbl_field) k_interior<float, double><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const float*)dev, (double*)dst, K, 1);
  else if (dtype_bytes == 8) k_interior<double, float><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const double*)dev, (float*)dst, K, 1);
  else k_interior<float, float><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const float*)dev, (float*)dst, K, 1);
  CK(cudaGetLastError());
  // the halo of a device upload is the periodic image of the interior
  if (field == ATM_GZ) {
    void* f1[1] = {ctx->gz};
    CK(atm::ops_fp64.ring(ctx->geo, f1, nullptr, 1, 1, false, ctx->stream));
  } else {
    void* f1[1] = {dst};
    CK(ctx->ops->ring(ctx->geo, f1, nullptr, 1, ctx->L, false, ctx->stream));
  }
  ctx->uploaded |= 1 << field;
  ctx->flag_valid = false;
  return ATM_OK;
}

int atm_download_device(atm_ctx* ctx, int field, void* dev, int dtype_bytes) {
  if (!ctx || !dev || (dtype_bytes != 4 && dtype_bytes != 8)) return ATM_ERR_ARG;
  if (field < ATM_DP || field > ATM_VD) return fail(ctx, ATM_ERR_ARG, "only prognostic fields");
  const bool dbl_field = ctx->ops->elem == 8;
  const void* src = ctx->st[ctx->cur][field];
  dim3 grid(1184), block(256);
  if (dbl_field && dtype_bytes == 8) k_interior<double, double><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const double*)src, (double*)dev, ctx->L, 0);
  else if (dbl_field) k_interior<double, float><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const double*)src, (float*)dev, ctx->L, 0);
  else if (dtype_bytes == 8) k_interior<float, double><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const float*)src, (double*)dev, ctx->L, 0);
  else k_interior<float, float><<<grid, block, 0, ctx->stream>>>(ctx->geo, (const float*)src, (float*)dev, ctx->L, 0);
  CK(cudaGetLastError());
  return ATM_OK;
}

int atm_download(atm_ctx* ctx, int field, double* host) {
  if (!ctx || !host) return ATM_ERR_ARG;
  const atm::Ops& ops = *ctx->ops;
  const int K = field_levels(ctx, field);
  if (K < 0) return fail(ctx, ATM_ERR_ARG, "unknown field");
  if ((field >= ATM_DP && field <= ATM_VD) || (field >= ATM_DPC && field <= ATM_VC)) {
    const void* src = field <= ATM_VD ? ctx->st[ctx->cur][field] : ctx->cg[field - ATM_DPC];
    if ((field <= ATM_VD ? ops.elem : ops.cg_elem) == 8) {
      CK(d2h_pitched(ctx, host, (const double*)src, K));
    } else {
      CK(ops.to_double(src, ctx->stage, ctx->geo.S * K, ctx->stream));
      CK(d2h_pitched(ctx, host, ctx->stage, K));
    }
  } else if (field == ATM_TS) {
    CK(d2h_pitched(ctx, host, ctx->ts, 1));
  } else if (field == ATM_NET_FLUX) {
    if (ctx->nf) {
      CK(d2h_pitched(ctx, host, ctx->nf, K));
    } else {
      std::memset(host, 0, sizeof(double) * (size_t)(ctx->nx + 2 * H) * (ctx->ny + 2 * H) * K);
      return ATM_OK;
    }
  } else {
    // column diagnostics from the current dp and pt over the whole array
    int r = require_init(ctx);
    if (r) return r;
    atm::Consts k = step_consts(ctx, 0.);
    CK(ops.column(ctx->geo, k, ctx->st[ctx->cur][F_DP], ctx->st[ctx->cur][F_PT], ops.elem, ctx->pkap, ctx->gz, -H, H,
                  ctx->stage, ctx->stream));
    const double* src = field == ATM_PLEV ? ctx->stage : field == ATM_PKAP ? ctx->pkap : ctx->gz;
    CK(d2h_pitched(ctx, host, src, K));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ATM_OK;
}

// net_flux and the heating term it feeds, allocated (zero) on first use
static int ensure_net_flux(atm_ctx* ctx) {
  const size_t lev = level_elems(ctx) * (ctx->L + 1) * 8;
  if (!ctx->nf) {
    CK(cudaMalloc((void**)&ctx->nf, lev));
    CK(cudaMemset(ctx->nf, 0, lev));
  }
  if (!ctx->heat) {
    CK(cudaMalloc((void**)&ctx->heat, lev));
    CK(cudaMemset(ctx->heat, 0, lev));
  }
  return ATM_OK;
}

int atm_set_net_flux(atm_ctx* ctx, const double* host) {
  if (!ctx) return ATM_ERR_ARG;
  if (!host) {
    ctx->heating = false;
    return ATM_OK;
  }
  int r = ensure_net_flux(ctx);
  if (r) return r;
  CK(h2d_pitched(ctx, ctx->nf, host, ctx->L + 1));
  ctx->heating = true;
  return ATM_OK;
}

int atm_init(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  const int need = (1 << ATM_DP) | (1 << ATM_PT) | (1 << ATM_UD) | (1 << ATM_VD) | (1 << ATM_GZ);
  if ((ctx->uploaded & need) != need) return fail(ctx, ATM_ERR_STATE, "upload dp, pt, ud, vd and gz before atm_init");
  const Geom& g = ctx->geo;
  // initial_halo_exchange (src/mod_input.f90:247): dp, pt, ud, vd and the
  // surface geopotential
  CK(ctx->ops->ring(g, ctx->st[ctx->cur], nullptr, 4, ctx->L, false, ctx->stream));
  void* gz1[1] = {ctx->gz};
  CK(atm::ops_fp64.ring(g, gz1, nullptr, 1, 1, false, ctx->stream));
  // and halo_exchange(ts) (src/mod_input.f90:251)
  void* ts1[1] = {ctx->ts};
  CK(atm::ops_fp64.ring(g, ts1, nullptr, 1, 1, false, ctx->stream));
  // model-top constants: pkap(nlay+1) and pkapb(nlay+1) = Ak(1)**kappa
  // (src/mod_input.f90:229-231, src/mod_sw_dyn.f90:991)
  k_fill<<<148, 256, 0, ctx->stream>>>(ctx->pkap + g.S * ctx->L, g.S, ctx->cst.pk_top);
  k_fill<<<148, 256, 0, ctx->stream>>>(ctx->pkapb + g.S * ctx->L, g.S, ctx->cst.pk_top);
  CK(cudaGetLastError());
  // gzb(:,:,1) from the surface geopotential, src/mod_sw_dyn.f90:995-996
  CK(atm::corners(g, ctx->pkap, ctx->gz, ctx->pkapb, ctx->gzb, 0, 0, 1, ctx->stream));
  ctx->initialized = true;
  ctx->flag_valid = false;
  return ATM_OK;
}

int atm_cgrid_step(atm_ctx* ctx, double dt_half) {
  int r = require_init(ctx);
  if (r) return r;
  const atm::Ops& ops = *ctx->ops;
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt_half);
  void* const* s = ctx->st[ctx->cur];
  const double* heat = nullptr;
  if (ctx->heating) {
    Stage t(ctx, S_HEAT);
    CK(ops.heating(g, k, s[F_DP], ops.elem, ctx->nf, ctx->heat, ctx->stream));
    heat = ctx->heat;
  }
  // dpc, ptc on is+5:ie-5 (src/mod_sw_dyn.f90:94-270)
  {
    Stage t(ctx, S_CMASS);
    CK(ops.mass(g, k, s[F_DP], s[F_PT], s[F_UD], s[F_VD], heat, ctx->cg[C_DPC], ctx->cg[C_PTC], -2, 2, nullptr,
                &ctx->status->tma_timeout, true, ctx->stream));
  }
  // plev, pkap, gz (src/mod_sw_dyn.f90:276-292)
  {
    Stage t(ctx, S_CCOL);
    CK(ops.column(g, k, ctx->cg[C_DPC], ctx->cg[C_PTC], ops.cg_elem, ctx->pkap, ctx->gz, -2, 2, nullptr, ctx->stream));
  }
  // uc, vc (src/mod_sw_dyn.f90:294-414)
  {
    Stage t(ctx, S_CMOM);
    CK(ops.c_mom(g, k, s[F_UD], s[F_VD], ctx->pkap, ctx->gz, ctx->cg[C_UC], ctx->cg[C_VC], &ctx->status->tma_timeout,
                 ctx->stream));
  }
  return ATM_OK;
}

int atm_cgrid_halo(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  Stage t(ctx, S_CHALO);
  CK(ctx->ops->ring_cg(ctx->geo, ctx->cg, nullptr, 4, ctx->L, false, ctx->stream));
  return ATM_OK;
}

int atm_dgrid_step(atm_ctx* ctx, double dt) {
  int r = require_init(ctx);
  if (r) return r;
  const atm::Ops& ops = *ctx->ops;
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt);
  const int old = ctx->cur, nxt = 1 - ctx->cur;
  void* const* so = ctx->st[old];
  void* const* sn = ctx->st[nxt];
  const double* heat = nullptr;
  if (ctx->heating) {
    Stage t(ctx, S_HEAT);
    CK(ops.heating(g, k, ctx->cg[C_DPC], ops.cg_elem, ctx->nf, ctx->heat, ctx->stream));  // from dpc, :433-464
    heat = ctx->heat;
  }
  // the new time level keeps the old halo until the D-grid halo exchange
  {
    Stage t(ctx, S_DRING);
    CK(ops.ring(g, ctx->st[nxt], (const void* const*)ctx->st[old], 4, ctx->L, true, ctx->stream));
  }
  CK(cudaMemsetAsync(&ctx->status->nonfinite_step, 0, sizeof(int), ctx->stream));
  // dp, pt on is+4:ie-4 (src/mod_sw_dyn.f90:439-600)
  {
    Stage t(ctx, S_DMASS);
    CK(ops.mass(g, k, so[F_DP], so[F_PT], ctx->cg[C_UC], ctx->cg[C_VC], heat, sn[F_DP], sn[F_PT], -3, 3,
                &ctx->status->nonfinite_step, &ctx->status->tma_timeout, false, ctx->stream));
  }
  // plev, pkap, gz, pkapb, gzb (src/mod_sw_dyn.f90:606-632)
  {
    Stage t(ctx, S_DCOL);
    CK(ops.column(g, k, sn[F_DP], sn[F_PT], ops.elem, ctx->pkap, ctx->gz, -2, 2, nullptr, ctx->stream));
  }
  {
    Stage t(ctx, S_DCORN);
    CK(atm::corners(g, ctx->pkap, ctx->gz, ctx->pkapb, ctx->gzb, 1, 0, ctx->L, ctx->stream));
  }
  // ud, vd on the interior (src/mod_sw_dyn.f90:634-771)
  {
    Stage t(ctx, S_DMOM);
    CK(ops.d_mom(g, k, so[F_UD], so[F_VD], ctx->cg[C_UC], ctx->cg[C_VC], ctx->pkapb, ctx->gzb, sn[F_UD], sn[F_VD],
                 &ctx->status->nonfinite_step, &ctx->status->tma_timeout, ctx->stream));
  }
  ctx->cur = nxt;
  ctx->flag_valid = true;
  ctx->remapped = false;
  return ATM_OK;
}

int atm_remap(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  const atm::Ops& ops = *ctx->ops;
  const Geom& g = ctx->geo;
  const int src = ctx->cur, dst = 1 - ctx->cur;
  void* const* s = ctx->st[src];
  void* const* d = ctx->st[dst];
  // outside the interior the remapped fields keep the arrays' current values
  {
    Stage t(ctx, S_RRING);
    CK(ops.ring(g, ctx->st[dst], (const void* const*)ctx->st[src], 4, ctx->L, true, ctx->stream));
  }
  CK(cudaMemsetAsync(&ctx->status->nonfinite_remap, 0, sizeof(int), ctx->stream));
  CK(cudaMemsetAsync(&ctx->status->fallback_pairs, 0, sizeof(int), ctx->stream));
  int* trace = nullptr;
  if (ctx->trace_host) {
    size_t n = (size_t)3 * (ctx->ny + 2) * (ctx->nx + 2) * ctx->L * 5;
    if (n != ctx->trace_elems) {
      cudaFree(ctx->d_trace);
      ctx->d_trace = nullptr;
      CK(cudaMalloc((void**)&ctx->d_trace, n * 4));
      ctx->trace_elems = n;
    }
    CK(cudaMemsetAsync(ctx->d_trace, 0xff, n * 4, ctx->stream));
    trace = ctx->d_trace;
  }
  atm::RemapArgs ra = remap_args(ctx);
  {
    Stage t(ctx, S_RWIND);
    CK(ops.remap_winds(g, ra, s[F_DP], s[F_UD], s[F_VD], ctx->urem, ctx->vrem, trace, ctx->status, ctx->stream));
  }
  {
    Stage t(ctx, S_RENER);
    CK(ops.remap_energy(g, ra, s[F_DP], s[F_PT], s[F_UD], s[F_VD], ctx->urem, ctx->vrem, ctx->gz, d[F_DP], d[F_PT],
                        d[F_UD], d[F_VD], trace, ctx->status, ctx->stream));
  }
  ctx->cur = dst;
  ctx->remapped = true;
  if (ctx->trace_host) {
    CK(cudaMemcpyAsync(ctx->trace_host, ctx->d_trace, ctx->trace_elems * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_status, ctx->status, sizeof(atm::Status), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->trace_fallback) *ctx->trace_fallback = ctx->h_status->fallback_pairs;
    ctx->trace_host = nullptr;
    ctx->trace_fallback = nullptr;
  }
  return ATM_OK;
}

int atm_dgrid_halo(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  Stage t(ctx, S_DHALO);
  CK(ctx->ops->ring(ctx->geo, ctx->st[ctx->cur], nullptr, 4, ctx->L, false, ctx->stream));
  return ATM_OK;
}

int atm_check_stability(atm_ctx* ctx, int* stable) {
  if (!ctx || !stable) return ATM_ERR_ARG;
  if (!ctx->flag_valid) {
    CK(cudaMemsetAsync(&ctx->status->nonfinite_check, 0, sizeof(int), ctx->stream));
    Stage t(ctx, S_CHECK);
    CK(ctx->ops->check_finite(ctx->geo, (const void* const*)ctx->st[ctx->cur], &ctx->status->nonfinite_check,
                              ctx->stream));
  }
  CK(cudaMemcpyAsync(ctx->h_status, ctx->status, sizeof(atm::Status), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_status->tma_timeout) return fail(ctx, ATM_ERR_CUDA, "a TMA tile load did not complete (wait limit)");
  int bad = !ctx->flag_valid ? ctx->h_status->nonfinite_check
                             : (ctx->remapped ? ctx->h_status->nonfinite_remap : ctx->h_status->nonfinite_step);
  *stable = bad ? 0 : 1;
  return ATM_OK;
}

int atm_mass(atm_ctx* ctx, double* total) {
  if (!ctx || !total) return ATM_ERR_ARG;
  CK(ctx->ops->mass_sum(ctx->geo, ctx->st[ctx->cur][F_DP], ctx->partial, MASS_BLOCKS, ctx->d_mass, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_mass, ctx->d_mass, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *total = *ctx->h_mass;
  return ATM_OK;
}

int atm_step(atm_ctx* ctx, double dt, int do_remap, int* stable) {
  int r;
  if ((r = atm_cgrid_step(ctx, dt / 2.))) return r;  // src/mod_model.f90:147
  if ((r = atm_cgrid_halo(ctx))) return r;
  if ((r = atm_dgrid_step(ctx, dt))) return r;
  if (do_remap && (r = atm_remap(ctx))) return r;
  if ((r = atm_dgrid_halo(ctx))) return r;
  if (stable) return atm_check_stability(ctx, stable);
  return ATM_OK;
}

int atm_sync(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return ATM_OK;
}

int atm_profile(atm_ctx* ctx, int enable) {
  if (!ctx) return ATM_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->prof = enable != 0;
  ctx->ev_used = 0;
  ctx->ev_stage.clear();
  return ATM_OK;
}

int atm_profile_read(atm_ctx* ctx, double* ms, int* count, int nstage) {
  if (!ctx || !ms || !count) return ATM_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < nstage; ++i) { ms[i] = 0.; count[i] = 0; }
  for (size_t p = 0; p < ctx->ev_stage.size(); ++p) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->ev_pool[2 * p], ctx->ev_pool[2 * p + 1]));
    int id = ctx->ev_stage[p];
    if (id < nstage) {
      ms[id] += t;
      count[id] += 1;
    }
  }
  return ATM_OK;
}

const char* atm_profile_stage(int i) { return (i >= 0 && i < NSTAGE) ? STAGE_NAMES[i] : nullptr; }

int atm_launch_count(atm_ctx* ctx, long long* n) {
  if (!ctx || !n) return ATM_ERR_ARG;
  *n = ctx->launches;
  return ATM_OK;
}

int atm_remap_trace(atm_ctx* ctx, int32_t* buf, int* fallback_columns) {
  if (!ctx) return ATM_ERR_ARG;
  ctx->trace_host = buf;
  ctx->trace_fallback = fallback_columns;
  return ATM_OK;
}

int atm_device_div_check(long long n, long long seed, long long* mismatches) {
  if (n <= 0 || !mismatches) return ATM_ERR_ARG;
  unsigned long long* d = nullptr;
  if (cudaMalloc((void**)&d, 8) != cudaSuccess) return ATM_ERR_NOMEM;
  int rc = ATM_OK;
  unsigned long long h = 0;
  if (cudaMemset(d, 0, 8) != cudaSuccess || atm::device_div_check(n, seed, d, 0) != cudaSuccess ||
      cudaMemcpy(&h, d, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = ATM_ERR_CUDA;
  cudaFree(d);
  *mismatches = (long long)h;
  return rc;
}

int atm_device_wait_check(int max_polls, int* timed_out) {
  if (max_polls <= 0 || max_polls > 100000 || !timed_out) return ATM_ERR_ARG;
  int* d = nullptr;
  if (cudaMalloc((void**)&d, 4) != cudaSuccess) return ATM_ERR_NOMEM;
  int rc = ATM_OK;
  int h = -1;
  if (cudaMemset(d, 0xff, 4) != cudaSuccess || atm::device_wait_timeout(max_polls, d, 0) != cudaSuccess ||
      cudaMemcpy(&h, d, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = ATM_ERR_CUDA;
  cudaFree(d);
  *timed_out = h;
  return rc;
}

int atm_device_pow_log(const double* x, double y, double* pow_out, double* log_out, int n) {
  if (n <= 0 || !x || !pow_out || !log_out) return ATM_ERR_ARG;
  double *dx = nullptr, *dp = nullptr, *dl = nullptr;
  size_t b = (size_t)n * 8;
  if (cudaMalloc((void**)&dx, b) != cudaSuccess || cudaMalloc((void**)&dp, b) != cudaSuccess ||
      cudaMalloc((void**)&dl, b) != cudaSuccess) {
    cudaFree(dx); cudaFree(dp); cudaFree(dl);
    return ATM_ERR_NOMEM;
  }
  int rc = ATM_OK;
  if (cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice) != cudaSuccess ||
      atm::device_pow_log(dx, y, dp, dl, n, 0) != cudaSuccess ||
      cudaMemcpy(pow_out, dp, b, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(log_out, dl, b, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = ATM_ERR_CUDA;
  cudaFree(dx); cudaFree(dp); cudaFree(dl);
  return rc;
}

int atm_device_kappa_pow(const double* x, double* out, int n) {
  if (n <= 0 || !x || !out) return ATM_ERR_ARG;
  double *dx = nullptr, *dy = nullptr;
  const size_t b = (size_t)n * 8;
  if (cudaMalloc((void**)&dx, b) != cudaSuccess || cudaMalloc((void**)&dy, b) != cudaSuccess) {
    cudaFree(dx); cudaFree(dy);
    return ATM_ERR_NOMEM;
  }
  int rc = ATM_OK;
  if (cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice) != cudaSuccess || atm::device_kappa_pow(dx, dy, n, 0) != cudaSuccess ||
      cudaMemcpy(out, dy, b, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = ATM_ERR_CUDA;
  cudaFree(dx); cudaFree(dy);
  return rc;
}

}  // extern "C"

// ------------------------------------------------------------- adjoint ----
namespace {

int require_adj(atm_ctx* c) {
  int r = require_init(c);
  if (r) return r;
  if (!c->adj) return fail(c, ATM_ERR_STATE, "atm_adj_enable has not been called");
  if (c->heating) return fail(c, ATM_ERR_UNSUPPORTED, "the adjoint holds the heating term at zero: clear net_flux");
  return ATM_OK;
}

double** slot_fields(atm_ctx* c, int slot) { return c->lam[slot == ATM_ADJ_IN ? c->slot_in : 1 - c->slot_in]; }

cudaError_t zero_fields(atm_ctx* c, double* const* f, int n, int K) {
  for (int i = 0; i < n; ++i) {
    cudaError_t e = cudaMemsetAsync(f[i], 0, (size_t)c->geo.S * K * 8, c->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// forward C step from the state s into cg, pkap, gz (no halo)
int fwd_c(atm_ctx* ctx, double dt_half, void* const* s) {
  const atm::Ops& ops = *ctx->ops;
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt_half);
  CK(ops.mass(g, k, s[F_DP], s[F_PT], s[F_UD], s[F_VD], nullptr, ctx->cg[C_DPC], ctx->cg[C_PTC], -2, 2, nullptr,
              &ctx->status->tma_timeout, true, ctx->stream));
  CK(ops.column(g, k, ctx->cg[C_DPC], ctx->cg[C_PTC], ops.cg_elem, ctx->pkap, ctx->gz, -2, 2, nullptr, ctx->stream));
  CK(ops.c_mom(g, k, s[F_UD], s[F_VD], ctx->pkap, ctx->gz, ctx->cg[C_UC], ctx->cg[C_VC], &ctx->status->tma_timeout,
               ctx->stream));
  ctx->launches += 3;
  return ATM_OK;
}

// forward D step from so (and cg) into sn, without advancing the state
int fwd_d(atm_ctx* ctx, double dt, void* const* so, void* const* sn) {
  const atm::Ops& ops = *ctx->ops;
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt);
  CK(ops.ring(g, sn, (const void* const*)so, 4, ctx->L, true, ctx->stream));
  CK(ops.mass(g, k, so[F_DP], so[F_PT], ctx->cg[C_UC], ctx->cg[C_VC], nullptr, sn[F_DP], sn[F_PT], -3, 3,
              &ctx->status->nonfinite_step, &ctx->status->tma_timeout, false, ctx->stream));
  CK(ops.column(g, k, sn[F_DP], sn[F_PT], ops.elem, ctx->pkap, ctx->gz, -2, 2, nullptr, ctx->stream));
  CK(atm::corners(g, ctx->pkap, ctx->gz, ctx->pkapb, ctx->gzb, 1, 0, ctx->L, ctx->stream));
  CK(ops.d_mom(g, k, so[F_UD], so[F_VD], ctx->cg[C_UC], ctx->cg[C_VC], ctx->pkapb, ctx->gzb, sn[F_UD], sn[F_VD],
               &ctx->status->nonfinite_step, &ctx->status->tma_timeout, ctx->stream));
  ctx->launches += 5;
  return ATM_OK;
}

// lin += (C step)^T lam_cg at the state s; cgf holds the step's dpc, ptc
int adj_c(atm_ctx* ctx, double dt_half, void* const* s, double* const* lin, const void* const* cgf) {
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt_half);
  const double* const* sd = (const double* const*)s;
  const double* const* cg = (const double* const*)cgf;
  {
    Stage t(ctx, S_ACCOL, 2);
    CK(ctx->ops->column(g, k, cg[C_DPC], cg[C_PTC], ctx->ops->cg_elem, ctx->pkap, ctx->gz, -2, 2, nullptr,
                        ctx->stream));
    CK(cudaMemsetAsync(ctx->lam_pk, 0, (size_t)g.S * (ctx->L + 1) * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->lam_gz, 0, (size_t)g.S * (ctx->L + 1) * 8, ctx->stream));
  }
  {
    Stage t(ctx, S_ACMOM);
    CK(atm::adj_c_mom(g, k, sd[F_UD], sd[F_VD], ctx->pkap, ctx->gz, ctx->lam_cg[C_UC], ctx->lam_cg[C_VC], lin[F_UD],
                      lin[F_VD], ctx->lam_pk, ctx->lam_gz, &ctx->status->tma_timeout, ctx->stream));
  }
  {
    Stage t(ctx, S_ACCOL);
    CK(atm::adj_column(g, k, cg[C_DPC], cg[C_PTC], ctx->lam_pk, ctx->lam_gz, ctx->lam_cg[C_DPC], ctx->lam_cg[C_PTC], -2,
                       2, ctx->stream));
  }
  {
    Stage t(ctx, S_ACMASS);
    CK(atm::adj_mass(g, k, sd[F_DP], sd[F_PT], sd[F_UD], sd[F_VD], cg[C_DPC], cg[C_PTC], ctx->lam_cg[C_DPC],
                     ctx->lam_cg[C_PTC], lin[F_DP],
                     lin[F_PT], lin[F_UD], lin[F_VD], -2, 2, &ctx->status->tma_timeout, true, ctx->stream));
  }
  return ATM_OK;
}

// lin, lam_cg += (D step)^T lout at so (with the C-grid fields cgf) -> sn;
// pkapb, gzb must hold the step's values; lout is consumed
int adj_d(atm_ctx* ctx, double dt, const void* const* so, const void* const* sn, double* const* lout,
          double* const* lin, const void* const* cgf) {
  const Geom& g = ctx->geo;
  atm::Consts k = step_consts(ctx, dt);
  const double* const* o = (const double* const*)so;
  const double* const* n = (const double* const*)sn;
  const double* const* cg = (const double* const*)cgf;
  const size_t lev = (size_t)g.S * (ctx->L + 1) * 8;
  CK(cudaMemsetAsync(ctx->lam_pk, 0, lev, ctx->stream));
  CK(cudaMemsetAsync(ctx->lam_gz, 0, lev, ctx->stream));
  CK(cudaMemsetAsync(ctx->lam_pkb, 0, lev, ctx->stream));
  CK(cudaMemsetAsync(ctx->lam_gzb, 0, lev, ctx->stream));
  // the kinetic-energy chain and the rest of the D-momentum reverse, each
  // its own kernel and profiled stage
  for (int part = 1; part <= 2; ++part) {
    Stage t(ctx, part == 1 ? S_ADMOM : S_ADMOM_VF);
    CK(atm::adj_d_mom(g, k, o[F_UD], o[F_VD], cg[C_UC], cg[C_VC], ctx->pkapb, ctx->gzb, lout[F_UD], lout[F_VD],
                      lin[F_UD], lin[F_VD], ctx->lam_cg[C_UC], ctx->lam_cg[C_VC], ctx->lam_pkb, ctx->lam_gzb,
                      &ctx->status->tma_timeout, ctx->stream, part));
  }
  {
    Stage t(ctx, S_ADCOL, 2);
    CK(atm::adj_corners(g, ctx->lam_pkb, ctx->lam_gzb, ctx->lam_pk, ctx->lam_gz, ctx->stream));
    CK(atm::adj_column(g, k, n[F_DP], n[F_PT], ctx->lam_pk, ctx->lam_gz, lout[F_DP], lout[F_PT], -2, 2, ctx->stream));
  }
  // the x and the y branch of the D-grid mass reverse
  for (int part = 1; part <= 2; ++part) {
    Stage t(ctx, part == 1 ? S_ADMASS : S_ADMASS_Y);
    CK(atm::adj_mass(g, k, o[F_DP], o[F_PT], cg[C_UC], cg[C_VC], n[F_DP], n[F_PT], lout[F_DP], lout[F_PT], lin[F_DP],
                     lin[F_PT], ctx->lam_cg[C_UC], ctx->lam_cg[C_VC], -3, 3, &ctx->status->tma_timeout, false,
                     ctx->stream, part));
  }
  {
    Stage t(ctx, S_AHALO);
    CK(atm::adj_ring_copy(g, lout, lin, ctx->L, 3, 0, ctx->stream));
  }
  return ATM_OK;
}

// lin += (remap)^T lout at the pre-remap state s1
int adj_r(atm_ctx* ctx, const void* const* s1, double* const* lout, double* const* lin) {
  const Geom& g = ctx->geo;
  const double* const* s = (const double* const*)s1;
  atm::RemapArgs ra = remap_args(ctx);
  Stage t(ctx, S_ARMP, 4);
  CK(ctx->ops->remap_winds(g, ra, s[F_DP], s[F_UD], s[F_VD], ctx->urem, ctx->vrem, nullptr, ctx->status,
                           ctx->stream));
  CK(cudaMemsetAsync(ctx->lam_ur, 0, (size_t)g.S * ctx->L * 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->lam_vr, 0, (size_t)g.S * ctx->L * 8, ctx->stream));
  CK(atm::adj_remap_energy(g, ra, s[F_DP], s[F_PT], s[F_UD], s[F_VD], (const double*)ctx->urem,
                           (const double*)ctx->vrem, ctx->gz, lout[F_DP], lout[F_PT], lout[F_UD], lout[F_VD], lin[F_DP],
                           lin[F_PT], lin[F_UD], lin[F_VD], ctx->lam_ur, ctx->lam_vr, ctx->stream));
  CK(atm::adj_remap_winds(g, ra, s[F_DP], s[F_UD], s[F_VD], ctx->lam_ur, ctx->lam_vr, lin[F_DP], lin[F_UD], lin[F_VD],
                          ctx->stream));
  // the remapped fields keep the pre-remap ring
  CK(atm::adj_ring_copy(g, lout, lin, ctx->L, 0, 0, ctx->stream));
  return ATM_OK;
}

double* adj_field(atm_ctx* c, int slot, int field) {
  if (field >= ATM_DP && field <= ATM_VD) {
    if (slot != ATM_ADJ_IN && slot != ATM_ADJ_OUT) return nullptr;
    return slot_fields(c, slot)[field];
  }
  if (field >= ATM_DPC && field <= ATM_VC) return c->lam_cg[field - ATM_DPC];
  return nullptr;
}

}  // namespace

extern "C" {

int atm_adj_enable(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  if (ctx->precision != ATM_FP64) return fail(ctx, ATM_ERR_UNSUPPORTED, "the adjoint is defined for the FP64 form");
  if (ctx->adj) return atm_adj_zero(ctx);
  cudaError_t e = atm::adj_setup();
  if (e != cudaSuccess) return cuda_fail(ctx, "adjoint kernel set-up", e);
  const size_t lay = (size_t)ctx->geo.S * ctx->L * 8, lev = (size_t)ctx->geo.S * (ctx->L + 1) * 8;
  bool ok = true;
  auto alloc = [&](double** p, size_t bytes) {
    if (ok && cudaMalloc((void**)p, bytes) != cudaSuccess) ok = false;
  };
  for (int t = 0; t < 2; ++t)
    for (int f = 0; f < 4; ++f) alloc(&ctx->lam[t][f], lay);
  for (int f = 0; f < 4; ++f) alloc(&ctx->lam_cg[f], lay);
  alloc(&ctx->lam_pk, lev);
  alloc(&ctx->lam_gz, lev);
  alloc(&ctx->lam_pkb, lev);
  alloc(&ctx->lam_gzb, lev);
  alloc(&ctx->lam_ur, lay);
  alloc(&ctx->lam_vr, lay);
  if (!ok) {
    cudaGetLastError();
    return fail(ctx, ATM_ERR_NOMEM, "adjoint fields do not fit on the device");
  }
  ctx->adj = true;
  return atm_adj_zero(ctx);
}

int atm_adj_zero(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  if (!ctx->adj) return fail(ctx, ATM_ERR_STATE, "atm_adj_enable has not been called");
  CK(zero_fields(ctx, ctx->lam[0], 4, ctx->L));
  CK(zero_fields(ctx, ctx->lam[1], 4, ctx->L));
  CK(zero_fields(ctx, ctx->lam_cg, 4, ctx->L));
  ctx->slot_in = 0;
  return ATM_OK;
}

int atm_adj_set(atm_ctx* ctx, int slot, int field, const double* host) {
  if (!ctx || !host) return ATM_ERR_ARG;
  if (!ctx->adj) return fail(ctx, ATM_ERR_STATE, "atm_adj_enable has not been called");
  double* f = adj_field(ctx, slot, field);
  if (!f) return fail(ctx, ATM_ERR_ARG, "no such adjoint field");
  CK(h2d_pitched(ctx, f, host, ctx->L));
  return ATM_OK;
}

int atm_adj_get(atm_ctx* ctx, int slot, int field, double* host) {
  if (!ctx || !host) return ATM_ERR_ARG;
  if (!ctx->adj) return fail(ctx, ATM_ERR_STATE, "atm_adj_enable has not been called");
  double* f = adj_field(ctx, slot, field);
  if (!f) return fail(ctx, ATM_ERR_ARG, "no such adjoint field");
  CK(d2h_pitched(ctx, host, f, ctx->L));
  CK(cudaStreamSynchronize(ctx->stream));
  return ATM_OK;
}

int atm_adj_set_device(atm_ctx* ctx, int slot, int field, const double* dev) {
  if (!ctx || !dev) return ATM_ERR_ARG;
  if (!ctx->adj) return fail(ctx, ATM_ERR_STATE, "atm_adj_enable has not been called");
  double* f = adj_field(ctx, slot, field);
  if (!f) return fail(ctx, ATM_ERR_ARG, "no such adjoint field");
  CK(cudaMemsetAsync(f, 0, (size_t)ctx->geo.S * ctx->L * 8, ctx->stream));
  k_interior<double, double><<<1184, 256, 0, ctx->stream>>>(ctx->geo, dev, f, ctx->L, 1);
  CK(cudaGetLastError());
  return ATM_OK;
}

int atm_adj_get_device(atm_ctx* ctx, int slot, int field, double* dev) {
  if (!ctx || !dev) return ATM_ERR_ARG;
  if (!ctx->adj) return fail(ctx, ATM_ERR_STATE, "atm_adj_enable has not been called");
  double* f = adj_field(ctx, slot, field);
  if (!f) return fail(ctx, ATM_ERR_ARG, "no such adjoint field");
  k_interior<double, double><<<1184, 256, 0, ctx->stream>>>(ctx->geo, f, dev, ctx->L, 0);
  CK(cudaGetLastError());
  return ATM_OK;
}

int atm_adj_halo(atm_ctx* ctx, int slot) {
  int r = require_adj(ctx);
  if (r) return r;
  if (slot != ATM_ADJ_IN && slot != ATM_ADJ_OUT) return fail(ctx, ATM_ERR_ARG, "no such adjoint slot");
  Stage t(ctx, S_AHALO);
  CK(atm::adj_ring_fold(ctx->geo, slot_fields(ctx, slot), 4, ctx->L, ctx->stream));
  return ATM_OK;
}

int atm_adj_cgrid_halo(atm_ctx* ctx) {
  int r = require_adj(ctx);
  if (r) return r;
  Stage t(ctx, S_AHALO);
  CK(atm::adj_ring_fold(ctx->geo, ctx->lam_cg, 4, ctx->L, ctx->stream));
  return ATM_OK;
}

int atm_adj_cgrid_step(atm_ctx* ctx, double dt_half) {
  int r = require_adj(ctx);
  if (r) return r;
  void* const* s = ctx->st[ctx->cur];
  {
    Stage t(ctx, S_AFWD, 0);
    if ((r = fwd_c(ctx, dt_half, s))) return r;
  }
  return adj_c(ctx, dt_half, s, slot_fields(ctx, ATM_ADJ_IN), (const void* const*)ctx->cg);
}

int atm_adj_dgrid_step(atm_ctx* ctx, double dt) {
  int r = require_adj(ctx);
  if (r) return r;
  const int cur = ctx->cur;
  {
    Stage t(ctx, S_AFWD, 1);
    if ((r = fwd_c(ctx, dt / 2., ctx->st[cur]))) return r;
    CK(ctx->ops->ring_cg(ctx->geo, ctx->cg, nullptr, 4, ctx->L, false, ctx->stream));
    if ((r = fwd_d(ctx, dt, ctx->st[cur], ctx->st[1 - cur]))) return r;
  }
  return adj_d(ctx, dt, (const void* const*)ctx->st[cur], (const void* const*)ctx->st[1 - cur],
               slot_fields(ctx, ATM_ADJ_OUT), slot_fields(ctx, ATM_ADJ_IN), (const void* const*)ctx->cg);
}

int atm_adj_remap(atm_ctx* ctx) {
  int r = require_adj(ctx);
  if (r) return r;
  return adj_r(ctx, (const void* const*)ctx->st[ctx->cur], slot_fields(ctx, ATM_ADJ_OUT),
               slot_fields(ctx, ATM_ADJ_IN));
}

namespace {

// the reverse of one step given its forward products: s0 = the state before
// the step, cgf = C-grid fields after the C-grid halo, s1 = the state after
// the D-grid step (before the remap); pkapb, gzb must hold the D step's values
int adj_step_given(atm_ctx* ctx, double dt, int do_remap, const void* const* s0, const void* const* cgf,
                   const void* const* s1) {
  const Geom& g = ctx->geo;
  if (do_remap) {
    CK(zero_fields(ctx, slot_fields(ctx, ATM_ADJ_IN), 4, ctx->L));
    int r = adj_r(ctx, s1, slot_fields(ctx, ATM_ADJ_OUT), slot_fields(ctx, ATM_ADJ_IN));
    if (r) return r;
    ctx->slot_in = 1 - ctx->slot_in;
  }
  CK(zero_fields(ctx, slot_fields(ctx, ATM_ADJ_IN), 4, ctx->L));
  CK(zero_fields(ctx, ctx->lam_cg, 4, ctx->L));
  int r = adj_d(ctx, dt, s0, s1, slot_fields(ctx, ATM_ADJ_OUT), slot_fields(ctx, ATM_ADJ_IN), cgf);
  if (r) return r;
  {
    Stage t(ctx, S_AHALO);
    CK(atm::adj_ring_fold(g, ctx->lam_cg, 4, ctx->L, ctx->stream));
  }
  if ((r = adj_c(ctx, dt / 2., const_cast<void* const*>(s0), slot_fields(ctx, ATM_ADJ_IN), cgf))) return r;
  ctx->slot_in = 1 - ctx->slot_in;
  return ATM_OK;
}

size_t field_bytes(const atm_ctx* c) { return (size_t)c->L * c->geo.S * 8; }
size_t level_bytes(const atm_ctx* c) { return (size_t)(c->L + 1) * c->geo.S * 8; }

// Tape of one step: the C-grid fields after their halo (4 fields), the
// state after the D-grid step (4), the state before the step (4), then the
// D step's pkapb and gzb (L + 1 levels each).
constexpr int TAPE_CG = 0, TAPE_S1 = 4, TAPE_S0 = 8, TAPE_FIELDS = 12;

}  // namespace

int atm_adj_step(atm_ctx* ctx, double dt, int do_remap) {
  int r = require_adj(ctx);
  if (r) return r;
  const Geom& g = ctx->geo;
  const int cur = ctx->cur, nxt = 1 - ctx->cur;
  // dgrid_halo_exchange
  {
    Stage t(ctx, S_AHALO);
    CK(atm::adj_ring_fold(g, slot_fields(ctx, ATM_ADJ_OUT), 4, ctx->L, ctx->stream));
  }
  // the forward step from the current state, kept in the other time level
  {
    Stage t(ctx, S_AFWD, 1);
    if ((r = fwd_c(ctx, dt / 2., ctx->st[cur]))) return r;
    CK(ctx->ops->ring_cg(g, ctx->cg, nullptr, 4, ctx->L, false, ctx->stream));
    if ((r = fwd_d(ctx, dt, ctx->st[cur], ctx->st[nxt]))) return r;
  }
  return adj_step_given(ctx, dt, do_remap, (const void* const*)ctx->st[cur], (const void* const*)ctx->cg,
                        (const void* const*)ctx->st[nxt]);
}

int atm_tape_bytes(atm_ctx* ctx, long long* bytes) {
  if (!ctx || !bytes) return ATM_ERR_ARG;
  *bytes = (long long)(TAPE_FIELDS * field_bytes(ctx) + 2 * level_bytes(ctx));
  return ATM_OK;
}

int atm_step_tape(atm_ctx* ctx, double dt, int do_remap, void* tape) {
  int r = require_init(ctx);
  if (r) return r;
  if (ctx->precision != ATM_FP64) return fail(ctx, ATM_ERR_UNSUPPORTED, "tapes are defined for the FP64 form");
  if (!tape) return ATM_ERR_ARG;
  const size_t fb = field_bytes(ctx), lb = level_bytes(ctx);
  char* t = (char*)tape;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(t + (TAPE_S0 + i) * fb, ctx->st[ctx->cur][i], fb, cudaMemcpyDeviceToDevice, ctx->stream));
  if ((r = atm_cgrid_step(ctx, dt / 2.))) return r;
  if ((r = atm_cgrid_halo(ctx))) return r;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(t + (TAPE_CG + i) * fb, ctx->cg[i], fb, cudaMemcpyDeviceToDevice, ctx->stream));
  if ((r = atm_dgrid_step(ctx, dt))) return r;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(t + (TAPE_S1 + i) * fb, ctx->st[ctx->cur][i], fb, cudaMemcpyDeviceToDevice, ctx->stream));
  char* tb = t + TAPE_FIELDS * fb;
  CK(cudaMemcpyAsync(tb, ctx->pkapb, lb, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(tb + lb, ctx->gzb, lb, cudaMemcpyDeviceToDevice, ctx->stream));
  if (do_remap && (r = atm_remap(ctx))) return r;
  return atm_dgrid_halo(ctx);
}

int atm_adj_step_tape(atm_ctx* ctx, double dt, int do_remap, const void* tape) {
  int r = require_adj(ctx);
  if (r) return r;
  if (!tape) return ATM_ERR_ARG;
  const Geom& g = ctx->geo;
  const size_t fb = field_bytes(ctx), lb = level_bytes(ctx);
  const char* t = (const char*)tape;
  const void *cgf[4], *s1[4], *s0[4];
  for (int i = 0; i < 4; ++i) {
    cgf[i] = t + (TAPE_CG + i) * fb;
    s1[i] = t + (TAPE_S1 + i) * fb;
    s0[i] = t + (TAPE_S0 + i) * fb;
  }
  {
    Stage st(ctx, S_AHALO);
    CK(atm::adj_ring_fold(g, slot_fields(ctx, ATM_ADJ_OUT), 4, ctx->L, ctx->stream));
  }
  // the D step's pkapb, gzb are read from the tape for this reverse step
  double* const pkapb = ctx->pkapb;
  double* const gzb = ctx->gzb;
  ctx->pkapb = (double*)(t + TAPE_FIELDS * fb);
  ctx->gzb = (double*)(t + TAPE_FIELDS * fb + lb);
  const int r2 = adj_step_given(ctx, dt, do_remap, s0, cgf, s1);
  ctx->pkapb = pkapb;
  ctx->gzb = gzb;
  return r2;
}

int atm_state_bytes(atm_ctx* ctx, long long* bytes) {
  if (!ctx || !bytes) return ATM_ERR_ARG;
  *bytes = 4LL * ctx->L * ctx->geo.S * ctx->ops->elem;
  return ATM_OK;
}

int atm_state_save(atm_ctx* ctx, void* dev) {
  if (!ctx || !dev) return ATM_ERR_ARG;
  const size_t f = (size_t)ctx->L * ctx->geo.S * ctx->ops->elem;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync((char*)dev + i * f, ctx->st[ctx->cur][i], f, cudaMemcpyDeviceToDevice, ctx->stream));
  return ATM_OK;
}

int atm_state_load(atm_ctx* ctx, const void* dev) {
  if (!ctx || !dev) return ATM_ERR_ARG;
  const size_t f = (size_t)ctx->L * ctx->geo.S * ctx->ops->elem;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(ctx->st[ctx->cur][i], (const char*)dev + i * f, f, cudaMemcpyDeviceToDevice, ctx->stream));
  ctx->flag_valid = false;
  return ATM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ output ----
extern "C" {

namespace {
// levels of an output accumulator: nlay (dp, pt, u, v), nlay + 1 (net
// flux), 1 (ts)
int out_levels(const atm_ctx* c, int which) { return which < ATM_OUT_NFLX ? c->L : which == ATM_OUT_NFLX ? c->L + 1 : 1; }
}  // namespace

int atm_output_enable(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  for (int f = 0; f <= ATM_OUT_TS; ++f) {
    if (!ctx->acc[f]) CK(cudaMalloc((void**)&ctx->acc[f], (size_t)ctx->nx * ctx->ny * out_levels(ctx, f) * 8));
  }
  return atm_output_reset(ctx);
}

int atm_output_reset(atm_ctx* ctx) {
  if (!ctx) return ATM_ERR_ARG;
  if (!ctx->acc[0]) return fail(ctx, ATM_ERR_STATE, "atm_output_enable has not been called");
  for (int f = 0; f <= ATM_OUT_TS; ++f)
    CK(cudaMemsetAsync(ctx->acc[f], 0, (size_t)ctx->nx * ctx->ny * out_levels(ctx, f) * 8, ctx->stream));
  ctx->acc_time = 0.;
  return ATM_OK;
}

int atm_accumulate_output(atm_ctx* ctx, double dt) {
  int r = require_init(ctx);
  if (r) return r;
  if (!ctx->acc[0]) return fail(ctx, ATM_ERR_STATE, "atm_output_enable has not been called");
  void* const* s = ctx->st[ctx->cur];
  const double* nf = ctx->heating ? ctx->nf : nullptr;
  if (ctx->ops->elem == 8)
    k_accumulate<double><<<1184, 256, 0, ctx->stream>>>(ctx->geo, (const double*)s[F_DP], (const double*)s[F_PT],
                                                         (const double*)s[F_UD], (const double*)s[F_VD], nf, ctx->ts,
                                                         dt, ctx->acc[0], ctx->acc[1], ctx->acc[2], ctx->acc[3],
                                                         ctx->acc[4], ctx->acc[5]);
  else
    k_accumulate<float><<<1184, 256, 0, ctx->stream>>>(ctx->geo, (const float*)s[F_DP], (const float*)s[F_PT],
                                                        (const float*)s[F_UD], (const float*)s[F_VD], nf, ctx->ts,
                                                        dt, ctx->acc[0], ctx->acc[1], ctx->acc[2], ctx->acc[3],
                                                        ctx->acc[4], ctx->acc[5]);
  CK(cudaGetLastError());
  ctx->launches += 1;
  ctx->acc_time = ctx->acc_time + dt;
  return ATM_OK;
}

int atm_output_read(atm_ctx* ctx, int which, double* host) {
  if (!ctx || !host || which < 0 || which > ATM_OUT_TS) return ATM_ERR_ARG;
  if (!ctx->acc[0]) return fail(ctx, ATM_ERR_STATE, "atm_output_enable has not been called");
  const size_t n = (size_t)ctx->nx * ctx->ny * out_levels(ctx, which);
  CK(cudaMemcpyAsync(host, ctx->acc[which], n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // write_output (src/mod_output.f90:152): output_field / accumulation_time
  const double t = ctx->acc_time;
  for (size_t q = 0; q < n; ++q) host[q] = host[q] / t;
  return ATM_OK;
}

int atm_output_time(atm_ctx* ctx, double* t) {
  if (!ctx || !t) return ATM_ERR_ARG;
  *t = ctx->acc_time;
  return ATM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ physics ----
extern "C" {

int atm_physics_tendencies(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  if (ctx->ops->elem != 8) return fail(ctx, ATM_ERR_UNSUPPORTED, "the physics needs an FP64 prognostic state");
  if (!ctx->ph_pt) {
    const size_t lay = level_elems(ctx) * ctx->L * 8;
    bool ok = cudaMalloc((void**)&ctx->ph_pt, lay) == cudaSuccess && cudaMalloc((void**)&ctx->ph_u, lay) == cudaSuccess &&
              cudaMalloc((void**)&ctx->ph_v, lay) == cudaSuccess &&
              cudaMalloc((void**)&ctx->ph_ts, level_elems(ctx) * 8) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      double** ph[] = {&ctx->ph_pt, &ctx->ph_u, &ctx->ph_v, &ctx->ph_ts};
      for (double** p : ph) {
        cudaFree(*p);
        *p = nullptr;
      }
      return fail(ctx, ATM_ERR_NOMEM, "physics tendencies");
    }
    CK(cudaMemsetAsync(ctx->ph_ts, 0, level_elems(ctx) * 8, ctx->stream));
  }
  void* const* s = ctx->st[ctx->cur];
  atm::PhysicsArgs a{ctx->cst.ptop, ctx->cst.pk_top, (const double*)s[F_DP], (const double*)s[F_PT],
                     (const double*)s[F_UD], (const double*)s[F_VD], ctx->gz, ctx->heating ? ctx->nf : nullptr,
                     ctx->ph_pt, ctx->ph_u, ctx->ph_v, ctx->ph_ts};
  {
    Stage t(ctx, S_PHYS_TEND);
    CK(atm::physics_tend(ctx->geo, a, ctx->stream));
  }
  ctx->phys_ready = true;
  return ATM_OK;
}

int atm_apply_physics(atm_ctx* ctx, double dt) {
  int r = require_init(ctx);
  if (r) return r;
  if (!ctx->phys_ready) return fail(ctx, ATM_ERR_STATE, "atm_physics_tendencies has not been called");
  void* const* s = ctx->st[ctx->cur];
  atm::PhysicsArgs a{ctx->cst.ptop, ctx->cst.pk_top, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                     ctx->ph_pt, ctx->ph_u, ctx->ph_v, ctx->ph_ts};
  {
    Stage t(ctx, S_PHYS_APPLY);
    CK(atm::physics_apply(ctx->geo, dt, a, (double*)s[F_DP], (double*)s[F_PT], (double*)s[F_UD], (double*)s[F_VD],
                          ctx->ts, ctx->stream));
  }
  ctx->flag_valid = false;
  return ATM_OK;
}

int atm_physics_halo(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  void* ts1[1] = {ctx->ts};
  Stage t(ctx, S_PHYS_HALO);
  CK(atm::ops_fp64.ring(ctx->geo, ts1, nullptr, 1, 1, false, ctx->stream));
  return ATM_OK;
}

int atm_set_gas_optics(atm_ctx* ctx, const atm_gas_optics* t) {
  if (!ctx || !t) return ATM_ERR_ARG;
  if (t->n_g < 1 || t->n_p < 2 || t->n_t < 2 || t->n_planck < 2 || t->n_g > 4096 || t->n_p > 4096 ||
      t->n_t > 255 || t->n_planck > 65536)
    return fail(ctx, ATM_ERR_ARG, "atm_set_gas_optics: table sizes out of range");
  const size_t ng = t->n_g, np = t->n_p, nt = t->n_t, npl = t->n_planck;
  const double* src[8] = {t->pressures,    t->temperatures, t->sw_absorption, t->sw_scattering,
                          t->lw_absorption, t->planck_temperatures, t->planck, t->irradiance_fraction};
  const size_t len[8] = {np, np * nt, ng * np * nt, ng, ng * np * nt, npl, ng * npl, ng};
  for (const double* p : src)
    if (!p) return fail(ctx, ATM_ERR_ARG, "atm_set_gas_optics: null table");
  // the lookups search these axes (mod_gas_optics.f90:4556-4609)
  auto ascending = [](const double* x, size_t n) {
    for (size_t q = 1; q < n; ++q)
      if (!(x[q] > x[q - 1])) return false;
    return true;
  };
  bool ok = ascending(t->pressures, np) && ascending(t->planck_temperatures, npl);
  for (size_t p = 0; p < np && ok; ++p) ok = ascending(t->temperatures + p * nt, nt);
  if (!ok) return fail(ctx, ATM_ERR_ARG, "atm_set_gas_optics: lookup axes must be strictly ascending");
  size_t total = 0;
  for (size_t n : len) total += n;
  std::vector<double> h(total);
  size_t off[8];
  for (int q = 0, at = 0; q < 8; at += (int)len[q], ++q) {
    off[q] = (size_t)at;
    std::memcpy(h.data() + at, src[q], len[q] * 8);
  }
  if (ctx->rad_block) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->rad_block);
    ctx->rad_block = nullptr;
  }
  if (cudaMalloc((void**)&ctx->rad_block, total * 8) != cudaSuccess) {
    cudaGetLastError();
    ctx->rad_block = nullptr;
    return fail(ctx, ATM_ERR_NOMEM, "gas-optics tables");
  }
  CK(cudaMemcpyAsync(ctx->rad_block, h.data(), total * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double* b = ctx->rad_block;
  ctx->rad = atm::RadTables{(int)ng,     (int)np,       (int)nt,       (int)npl,      b + off[0], b + off[1],
                            b + off[2],  b + off[3],    b + off[4],    b + off[5],    b + off[6], b + off[7]};
  return ATM_OK;
}

int atm_set_cell_coordinates(atm_ctx* ctx, const double* xc, const double* yc) {
  if (!ctx || !xc || !yc) return ATM_ERR_ARG;
  const int nx = ctx->nx, ny = ctx->ny;
  // radius = sqrt(xc**2 + yc**2), summed as init_prognostic_fields does (src/mod_input.f90:233-243)
  std::vector<double> r((size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double v = xc[i] * xc[i];
      v = v + yc[j] * yc[j];
      r[(size_t)j * nx + i] = std::sqrt(v);
    }
  if (!ctx->radius && cudaMalloc((void**)&ctx->radius, r.size() * 8) != cudaSuccess) {
    cudaGetLastError();
    ctx->radius = nullptr;
    return fail(ctx, ATM_ERR_NOMEM, "cell radius");
  }
  CK(cudaMemcpyAsync(ctx->radius, r.data(), r.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return ATM_OK;
}

int atm_radiative_heating(atm_ctx* ctx, double time, double solar_zenith_angle, double surface_albedo,
                          double surface_emissivity) {
  (void)time;  // solar_irradiance does not depend on it (src/mod_solar.f90:26-35)
  int r = require_init(ctx);
  if (r) return r;
  if (ctx->ops->elem != 8) return fail(ctx, ATM_ERR_UNSUPPORTED, "the radiation needs an FP64 prognostic state");
  if (!ctx->rad_block) return fail(ctx, ATM_ERR_STATE, "atm_set_gas_optics has not been called");
  if (!ctx->radius) return fail(ctx, ATM_ERR_STATE, "atm_set_cell_coordinates has not been called");
  if ((r = ensure_net_flux(ctx))) return r;
  void* const* s = ctx->st[ctx->cur];
  CK(cudaMemsetAsync(&ctx->status->radiation_range, 0, sizeof(int), ctx->stream));
  atm::RadArgs a{ctx->cst.ptop,
                 ctx->cst.pk_top,
                 ctx->cst.gravity,
                 std::cos(solar_zenith_angle),
                 surface_albedo,
                 surface_emissivity,
                 (const double*)s[F_DP],
                 (const double*)s[F_PT],
                 ctx->ts,
                 ctx->radius,
                 ctx->nf,
                 &ctx->status->radiation_range};
  {
    Stage t(ctx, S_RAD);
    CK(atm::radiative_heating(ctx->geo, ctx->rad, a, ctx->stream));
  }
  ctx->heating = true;
  CK(cudaMemcpyAsync(ctx->h_status, ctx->status, sizeof(atm::Status), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_status->radiation_range)
    return fail(ctx, ATM_ERR_RANGE,
                "radiation: a layer pressure or temperature is outside the gas-optics tables "
                "(the reference stops there: src/mod_gas_optics.f90:4562-4566,4589-4594)");
  return ATM_OK;
}

int atm_radiation_halo(atm_ctx* ctx) {
  int r = require_init(ctx);
  if (r) return r;
  if (!ctx->nf) return fail(ctx, ATM_ERR_STATE, "no net flux to exchange");
  void* nf1[1] = {ctx->nf};
  Stage t(ctx, S_RAD_HALO);
  CK(atm::ops_fp64.ring(ctx->geo, nf1, nullptr, 1, ctx->L + 1, false, ctx->stream));
  return ATM_OK;
}

}  // extern "C"

// ---------------------------------------------------- persistent ensemble --
// Config 5: many members of the mixed form advanced in one cooperative
// launch of the persistent kernel (atm_ensemble.cuh).
struct atm_ens {
  std::vector<atm_ctx*> m;
  std::vector<double> dt;
  std::vector<int> tys;
  atm::EnsMember* d_members = nullptr;
  long long* d_off = nullptr;
  unsigned* d_bar = nullptr;  // arrival count, generation
  int* d_err = nullptr;
  int* h_err = nullptr;  // pinned
  int blocks = 0;
  long long timeout_ns = 2000000000LL;
  cudaStream_t stream = nullptr;
  bool prepared = false;
  int pending_flips = 0;  // time-level swaps of the launches since the last prepare
  unsigned long long* d_stage = nullptr;  // per-stage nanoseconds while profiling
  // dataflow schedule: per-member phase tickets and completion counts, the
  // finished-member count
  int dataflow = 0;
  unsigned long long* d_tk = nullptr;
  unsigned* d_dn = nullptr;
};

namespace {

int ens_free(atm_ens* e) {
  if (!e) return ATM_ERR_ARG;
  cudaFree(e->d_members);
  cudaFree(e->d_off);
  cudaFree(e->d_bar);
  cudaFree(e->d_err);
  cudaFree(e->d_stage);
  cudaFree(e->d_tk);
  cudaFree(e->d_dn);
  if (e->h_err) cudaFreeHost(e->h_err);
  delete e;
  return ATM_OK;
}

// the members' descriptors and the stage work prefix sums, to the device
int ens_upload(atm_ens* e) {
  const int n = (int)e->m.size();
  std::vector<atm::EnsMember> hm(n);
  std::vector<long long> off((size_t)atm::E_NSTAGE * (n + 1), 0);
  for (int i = 0; i < n; ++i) {
    atm_ctx* c = e->m[i];
    atm::EnsMember& d = hm[i];
    d.g = c->geo;
    d.cc = step_consts(c, e->dt[i] / 2.);
    d.cd = step_consts(c, e->dt[i]);
    d.ra = remap_args(c);
    for (int t = 0; t < 2; ++t)
      for (int f = 0; f < 4; ++f) d.st[t][f] = c->st[t][f];
    for (int f = 0; f < 4; ++f) d.cg[f] = c->cg[f];
    d.pkap = c->pkap;
    d.gz = c->gz;
    d.pkapb = c->pkapb;
    d.gzb = c->gzb;
    d.urem = c->urem;
    d.vrem = c->vrem;
    d.status = c->status;
    d.cur0 = c->cur;
    d.tys = e->tys[i];
  }
  for (int s = 0; s < atm::E_NSTAGE; ++s)
    for (int i = 0; i < n; ++i)
      off[(size_t)s * (n + 1) + i + 1] = off[(size_t)s * (n + 1) + i] + atm::ens_items(hm[i].g, s, hm[i].tys);
  if (cudaMemcpy(e->d_members, hm.data(), sizeof(atm::EnsMember) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(e->d_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return ATM_ERR_CUDA;
  return ATM_OK;
}

}  // namespace

extern "C" {

int atm_ensemble_create(atm_ens** out, atm_ctx* const* members, const double* dts, int n) {
  if (!out || !members || !dts || n <= 0) return ATM_ERR_ARG;
  *out = nullptr;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return ATM_ERR_CUDA;
  for (int i = 0; i < n; ++i) {
    atm_ctx* c = members[i];
    // the kernel holds the mixed form's sweeps, remaps at most 64 layers
    // and has no radiative heating term
    if (!c || !c->initialized || c->precision != ATM_MIXED || c->heating || c->L > 64 || c->device != dev ||
        !(dts[i] > 0.))
      return ATM_ERR_ARG;
  }
  atm_ens* e = new atm_ens();
  e->m.assign(members, members + n);
  e->dt.assign(dts, dts + n);
  e->tys.assign(n, 32);
  e->stream = members[0]->stream;
  e->blocks = atm::ensemble_max_blocks();
  const size_t off_bytes = sizeof(long long) * atm::E_NSTAGE * (n + 1);
  if (e->blocks <= 0 || cudaMalloc((void**)&e->d_members, sizeof(atm::EnsMember) * n) != cudaSuccess ||
      cudaMalloc((void**)&e->d_off, off_bytes) != cudaSuccess ||
      cudaMalloc((void**)&e->d_bar, 2 * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc((void**)&e->d_err, sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&e->d_tk, sizeof(unsigned long long) * n) != cudaSuccess ||
      cudaMalloc((void**)&e->d_dn, sizeof(unsigned) * (n + 1)) != cudaSuccess ||
      cudaMallocHost((void**)&e->h_err, sizeof(int)) != cudaSuccess) {
    ens_free(e);
    return ATM_ERR_NOMEM;
  }
  *out = e;
  return ATM_OK;
}

int atm_ensemble_set_strips(atm_ens* e, int member, int rows) {
  if (!e || member < 0 || member >= (int)e->m.size() || (rows != 16 && rows != 32 && rows != 64)) return ATM_ERR_ARG;
  e->tys[member] = rows;
  e->prepared = false;
  return ATM_OK;
}

int atm_ensemble_set_stream(atm_ens* e, void* stream) {
  if (!e) return ATM_ERR_ARG;
  e->stream = (cudaStream_t)stream;
  return ATM_OK;
}

int atm_ensemble_prepare(atm_ens* e) {
  if (!e) return ATM_ERR_ARG;
  for (atm_ctx* c : e->m)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return ATM_ERR_CUDA;
  if (cudaStreamSynchronize(e->stream) != cudaSuccess) return ATM_ERR_CUDA;
  int r = ens_upload(e);
  if (r) return r;
  e->prepared = true;
  e->pending_flips = 0;
  return ATM_OK;
}

int atm_ensemble_run(atm_ens* e, int nsteps, int remap_every) {
  if (!e || nsteps <= 0 || remap_every < 0) return ATM_ERR_ARG;
  if (!e->prepared) return ATM_ERR_STATE;
  // each launch starts from the time levels recorded at prepare: the
  // launches since then must have swapped them an even number of times
  if (e->pending_flips % 2) return ATM_ERR_STATE;
  const int n = (int)e->m.size();
  const int remaps = remap_every > 0 ? nsteps / remap_every : 0;
  if (cudaMemsetAsync(e->d_bar, 0, 2 * sizeof(unsigned), e->stream) != cudaSuccess ||
      cudaMemsetAsync(e->d_err, 0, sizeof(int), e->stream) != cudaSuccess ||
      cudaMemsetAsync(e->d_tk, 0, sizeof(unsigned long long) * n, e->stream) != cudaSuccess ||
      cudaMemsetAsync(e->d_dn, 0, sizeof(unsigned) * (n + 1), e->stream) != cudaSuccess)
    return ATM_ERR_CUDA;
  // per-stage timing needs the stage barriers
  for (atm_ctx* c : e->m)
    if (cudaMemsetAsync(&c->status->nonfinite_step, 0, 2 * sizeof(int), e->stream) != cudaSuccess) return ATM_ERR_CUDA;
  const int dataflow = e->dataflow && !e->d_stage;
  atm::EnsPlan p{e->d_members, e->d_off, n, nsteps, remap_every, e->d_bar, (unsigned)e->blocks, e->d_err,
                 e->timeout_ns, e->d_stage, dataflow, e->d_tk, e->d_dn, e->d_dn + n};
  if (atm::ensemble_launch(p, e->blocks, e->stream) != cudaSuccess) return ATM_ERR_CUDA;
  const int flips = nsteps + remaps;
  e->pending_flips += flips;
  for (atm_ctx* c : e->m) {
    c->cur ^= (flips & 1);
    c->flag_valid = false;  // the stability check reads the state itself
    c->launches += 1;
  }
  return ATM_OK;
}

int atm_ensemble_status(atm_ens* e, int* barrier_timed_out) {
  if (!e || !barrier_timed_out) return ATM_ERR_ARG;
  if (cudaMemcpyAsync(e->h_err, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
      cudaStreamSynchronize(e->stream) != cudaSuccess)
    return ATM_ERR_CUDA;
  *barrier_timed_out = *e->h_err;
  return ATM_OK;
}

int atm_ensemble_set_schedule(atm_ens* e, int dataflow) {
  if (!e || (dataflow != 0 && dataflow != 1)) return ATM_ERR_ARG;
  e->dataflow = dataflow;
  return ATM_OK;
}

int atm_ensemble_profile(atm_ens* e, int enable) {
  if (!e) return ATM_ERR_ARG;
  if (!enable) {
    cudaFree(e->d_stage);
    e->d_stage = nullptr;
    return ATM_OK;
  }
  if (!e->d_stage && cudaMalloc((void**)&e->d_stage, atm::E_NSTAGE * sizeof(unsigned long long)) != cudaSuccess) {
    e->d_stage = nullptr;
    return ATM_ERR_NOMEM;
  }
  return cudaMemsetAsync(e->d_stage, 0, atm::E_NSTAGE * sizeof(unsigned long long), e->stream) == cudaSuccess
             ? ATM_OK
             : ATM_ERR_CUDA;
}

int atm_ensemble_stage_ms(atm_ens* e, double* ms, int n) {
  if (!e || !ms || n < atm::E_NSTAGE) return ATM_ERR_ARG;
  if (!e->d_stage) return ATM_ERR_STATE;
  unsigned long long h[atm::E_NSTAGE];
  if (cudaStreamSynchronize(e->stream) != cudaSuccess ||
      cudaMemcpy(h, e->d_stage, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
    return ATM_ERR_CUDA;
  for (int i = 0; i < atm::E_NSTAGE; ++i) ms[i] = (double)h[i] * 1e-6;
  return ATM_OK;
}

int atm_ensemble_blocks(atm_ens* e, int* blocks) {
  if (!e || !blocks) return ATM_ERR_ARG;
  *blocks = e->blocks;
  return ATM_OK;
}

int atm_ensemble_destroy(atm_ens* e) {
  if (!e) return ATM_ERR_ARG;
  cudaStreamSynchronize(e->stream);
  return ens_free(e);
}

int atm_ensemble_barrier_check(long long timeout_ns, int* timed_out) {
  if (timeout_ns <= 0 || timeout_ns > 2000000000LL || !timed_out) return ATM_ERR_ARG;
  const int blocks = atm::ensemble_max_blocks();
  if (blocks <= 0) return ATM_ERR_CUDA;
  long long* d_off = nullptr;
  unsigned* d_bar = nullptr;
  int* d_err = nullptr;
  int rc = ATM_OK;
  int h = 0;
  if (cudaMalloc((void**)&d_off, sizeof(long long) * atm::E_NSTAGE) != cudaSuccess ||
      cudaMalloc((void**)&d_bar, 2 * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc((void**)&d_err, sizeof(int)) != cudaSuccess) {
    rc = ATM_ERR_NOMEM;
  } else if (cudaMemset(d_off, 0, sizeof(long long) * atm::E_NSTAGE) != cudaSuccess ||
             cudaMemset(d_bar, 0, 2 * sizeof(unsigned)) != cudaSuccess || cudaMemset(d_err, 0, sizeof(int)) != cudaSuccess) {
    rc = ATM_ERR_CUDA;
  } else {
    // no members, one step: the first barrier waits for one block more than
    // the grid holds, so its wait runs out in every block
    atm::EnsPlan p{nullptr, d_off, 0, 1, 0, d_bar, (unsigned)blocks + 1, d_err, timeout_ns, nullptr, 0,
                   nullptr, nullptr, nullptr};
    if (atm::ensemble_launch(p, blocks, 0) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = ATM_ERR_CUDA;
  }
  cudaFree(d_off);
  cudaFree(d_bar);
  cudaFree(d_err);
  *timed_out = h;
  return rc;
}

}  // extern "C"
