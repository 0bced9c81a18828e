// Vertical remap that allocates nothing (atm_remap_noalloc, include/atmdyn.h).
//
// Some callers cannot let the library call cudaMalloc: a host time loop that
// fixes its device-memory budget at start-up (an ensemble driver that splits
// HBM between members, a memory pool shared with other components) or that
// must not meet the device-wide synchronisation cudaMalloc/cudaFree can
// cause in the middle of a step.  For them the remap's only scratch -- the
// remapped face winds of every column, which the potential-temperature
// recovery reads from the neighbouring columns -- lives in one file-scope
// device array of fixed size instead of context memory.  Every GPU that
// loads the library holds this array until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "atmdyn.h"
#include "atm_kernels.cuh"
#include "atm_ops.h"

namespace {

// 8 MiB of FP64 scratch: the status words, the hybrid coefficients and the
// two remapped wind fields, 2 (nx+14)(ny+14) nlay doubles.
constexpr size_t NOALLOC_DOUBLES = size_t(1) << 20;
constexpr size_t HEAD_DOUBLES = 32;  // atm::Status, padded to 256 bytes
static_assert(sizeof(atm::Status) <= HEAD_DOUBLES * sizeof(double), "status words do not fit");

static __device__ __align__(256) double g_remap_scratch[NOALLOC_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
double* g_scratch_addr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device.  The name of
// a __device__ array in host code is only a host-side stand-in, so the
// address is looked up once per device with that device current.
int scratch_address(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return ATM_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_remap_scratch) != cudaSuccess || !p) return ATM_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return ATM_OK;
}

template <int LM>
cudaError_t launch(const atm::Geom& g, const atm::RemapArgs& ra, const double* dp, const double* pt,
                   const double* ud, const double* vd, const double* gzs, double* urem, double* vrem, double* dpo,
                   double* pto, double* udo, double* vdo, atm::Status* st, cudaStream_t s) {
  int nw = (g.nx + 2) * (g.ny + 2);
  atm::k_remap_winds<double, LM><<<dim3((nw + 63) / 64, 2), 64, 0, s>>>(g, ra, dp, ud, vd, urem, vrem, nullptr, st);
  int ne = g.nx * g.ny;
  atm::k_remap_energy<double, LM><<<(ne + 63) / 64, 64, 0, s>>>(g, ra, dp, pt, ud, vd, urem, vrem, gzs, dpo, pto,
                                                                udo, vdo, nullptr, st);
  return cudaGetLastError();
}

}  // namespace

extern "C" int atm_remap_noalloc(int nx, int ny, int nlay, const double* ak, const double* bk, const double* dp,
                                 const double* pt, const double* ud, const double* vd, const double* gzs,
                                 double* dp_out, double* pt_out, double* ud_out, double* vd_out, void* stream,
                                 int* stable, int* fallback_columns) {
  if (nx < atm::H || ny < atm::H || nlay < 3 || nlay > atm::MAX_LAYERS || !ak || !bk || !dp || !pt || !ud || !vd ||
      !gzs || !dp_out || !pt_out || !ud_out || !vd_out)
    return ATM_ERR_ARG;
  const double* ins[] = {dp, pt, ud, vd};
  const double* outs[] = {dp_out, pt_out, ud_out, vd_out};
  for (const double* o : outs)
    for (const double* i : ins)
      if (o == i) return ATM_ERR_ARG;  // the remap reads neighbouring columns: no in-place update
  atm::Geom g;
  g.nx = nx;
  g.ny = ny;
  g.L = nlay;
  g.P = nx + 2 * atm::H;  // the caller's arrays have no row padding
  g.NYP = ny + 2 * atm::H;
  g.S = (long long)g.P * g.NYP;
  const size_t coef = ((size_t)2 * (nlay + 1) + 31) / 32 * 32;
  const size_t need = HEAD_DOUBLES + coef + 2 * (size_t)g.S * nlay;
  if (need > NOALLOC_DOUBLES) return ATM_ERR_TOO_LARGE;

  double* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != ATM_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  atm::Status* st = reinterpret_cast<atm::Status*>(base);
  double* d_ak = base + HEAD_DOUBLES;
  double* d_bk = d_ak + (nlay + 1);
  double* urem = base + HEAD_DOUBLES + coef;
  double* vrem = urem + (size_t)g.S * nlay;
  // the array keeps the previous call's contents: clear the status words and
  // load this call's coefficients
  if (cudaMemsetAsync(st, 0, sizeof(atm::Status), s) != cudaSuccess) return ATM_ERR_CUDA;
  if (cudaMemcpyAsync(d_ak, ak, (nlay + 1) * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_bk, bk, (nlay + 1) * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return ATM_ERR_CUDA;
  atm::RemapArgs ra{d_ak, d_bk, ak[0], atm_pow(ak[0], atm::KAPPA)};
  // Geom::at() includes the row pad of the library's own arrays; shift the
  // caller's unpadded arrays back by that pad so that element (is, js, 1)
  // is the first one accessed
  const int o = atm::XOFF;
  cudaError_t e;
  if (nlay <= 32)
    e = launch<32>(g, ra, dp - o, pt - o, ud - o, vd - o, gzs - o, urem - o, vrem - o, dp_out - o, pt_out - o,
                   ud_out - o, vd_out - o, st, s);
  else if (nlay <= 64)
    e = launch<64>(g, ra, dp - o, pt - o, ud - o, vd - o, gzs - o, urem - o, vrem - o, dp_out - o, pt_out - o,
                   ud_out - o, vd_out - o, st, s);
  else
    e = launch<atm::MAX_LAYERS>(g, ra, dp - o, pt - o, ud - o, vd - o, gzs - o, urem - o, vrem - o, dp_out - o,
                                pt_out - o, ud_out - o, vd_out - o, st, s);
  if (e != cudaSuccess) return ATM_ERR_CUDA;
  if (!stable && !fallback_columns) return ATM_OK;
  // the report: wait for the remap, then read the status words the kernels
  // raised (into a stack copy: nothing is allocated)
  atm::Status h{};
  if (cudaMemcpyAsync(&h, st, sizeof(atm::Status), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ATM_ERR_CUDA;
  if (stable) *stable = h.nonfinite_remap ? 0 : 1;
  if (fallback_columns) *fallback_columns = h.fallback_pairs;
  return ATM_OK;
}
