// Mixed-precision form of the dynamical core: the horizontal sweeps run in
// FP32 (fields and PPM arithmetic), while the column pressure sums, pkap,
// the hydrostatic geopotential feeding the pressure-gradient force, the
// vertical remap and the global mass sum stay in FP64.
#define ATM_FORM_T float
#define ATM_OPS_NAME ops_mixed
#define ATM_MARCH_SWEEPS 1  // the four sweeps as column-marching kernels
#include "atm_launch.cuh"

// ---- the persistent ensemble kernel of the mixed form (atm_ensemble.cuh)
#include "atm_ensemble.cuh"

namespace atm {

int ensemble_max_blocks() {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ensemble<float, double, float>, MW * MWARPS, 0) !=
          cudaSuccess)
    return 0;
  return sms * per_sm;
}

static __global__ void k_kappa_pow(const double* x, double* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = DevicePow::kappa(x[i]);
}

// p**kappa as the mixed form's column and remap kernels evaluate it
cudaError_t device_kappa_pow(const double* x, double* out, int n, cudaStream_t s) {
  k_kappa_pow<<<(n + 255) / 256, 256, 0, s>>>(x, out, n);
  return cudaGetLastError();
}

cudaError_t ensemble_launch(const EnsPlan& plan, int blocks, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(MW * MWARPS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;  // every block resident: the grid barrier can complete
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_ensemble<float, double, float>, plan);
}

}  // namespace atm
