// FP64 form of the dynamical core.  Compiled with --fmad=false: every
// multiply and add is rounded separately, exactly as in the FP64
// restatement of the reference, so the two agree bit for bit.
#define ATM_FORM_T double
#define ATM_OPS_NAME ops_fp64
#include "atm_launch.cuh"

namespace atm {

cudaError_t corners(const Geom& g, const double* pkap, const double* gz, double* pkapb, double* gzb, int with_pkap,
                    int lev0, int nlev, cudaStream_t s) {
  int n = (g.nx + 1) * (g.ny + 1);
  k_corners<<<(n + 255) / 256, 256, 0, s>>>(g, pkap, gz, pkapb, gzb, with_pkap, lev0, nlev);
  return cudaGetLastError();
}

static __global__ void k_pow_log(const double* x, double y, double* p, double* l, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    p[i] = atm_pow(x[i], y);
    l[i] = atm_log(x[i]);
  }
}

cudaError_t device_pow_log(const double* x, double y, double* p, double* l, int n, cudaStream_t s) {
  k_pow_log<<<(n + 255) / 256, 256, 0, s>>>(x, y, p, l, n);
  return cudaGetLastError();
}

}  // namespace atm
