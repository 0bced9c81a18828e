// FP64 form of the dynamical core.  Compiled with --fmad=false: every
// multiply and add is rounded separately, exactly as in the FP64
// restatement of the reference, so the two agree bit for bit.
#define ATM_FORM_T double
#define ATM_OPS_NAME ops_fp64
#include "atm_launch.cuh"

#ifndef ATM_CORNER_CHUNK
#define ATM_CORNER_CHUNK 8
#endif

namespace atm {

cudaError_t corners(const Geom& g, const double* pkap, const double* gz, double* pkapb, double* gzb, int with_pkap,
                    int lev0, int nlev, cudaStream_t s) {
  int n = (g.nx + 1) * (g.ny + 1);
  const int chunk = ATM_CORNER_CHUNK;
  k_corners<<<dim3((n + 255) / 256, (nlev + chunk - 1) / chunk), 256, 0, s>>>(g, pkap, gz, pkapb, gzb, with_pkap,
                                                                             lev0, nlev, chunk);
  return cudaGetLastError();
}

static __global__ void k_pow_log(const double* x, double y, double* p, double* l, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    p[i] = atm_pow(x[i], y);
    l[i] = atm_log(x[i]);
  }
}

// random bit patterns of every exponent, and small integers
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static __global__ void k_div_check(unsigned long long n, unsigned long long seed, unsigned long long* bad) {
  unsigned long long local = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long b = mix64(seed * 0x100000001b3ULL + i);
    double x = __longlong_as_double((long long)b);
    if (i % 7 == 0) x = (double)(long long)(b % 2000001) - 1000000.0;
    bool ok = true;
    double q3 = div_const<3>(x), t3 = x / 3.0;
    double q12 = div_const<12>(x), t12 = x / 12.0;
    ok = ok && (__double_as_longlong(q3) == __double_as_longlong(t3) || (q3 != q3 && t3 != t3));
    ok = ok && (__double_as_longlong(q12) == __double_as_longlong(t12) || (q12 != q12 && t12 != t12));
    if (!ok) ++local;
  }
  if (local) atomicAdd(bad, local);
}

cudaError_t device_div_check(unsigned long long n, unsigned long long seed, unsigned long long* bad, cudaStream_t s) {
  k_div_check<<<1184, 256, 0, s>>>(n, seed, bad);
  return cudaGetLastError();
}

// The bounded wait of the TMA loads, made to run out: one thread arms an
// mbarrier for 16 bytes of transactions that no copy ever brings (no copy
// is issued) and waits on it with mbar_wait's poll limit, as tma_fetch
// does; it must come back with the failure recorded in *flag.
static __global__ void k_wait_timeout(int max_polls, int* flag) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_expect_tx(&bar, 16);
    const bool ok = mbar_wait(&bar, 0, max_polls);
    *flag = ok ? 0 : 1;
  }
}

cudaError_t device_wait_timeout(int max_polls, int* flag, cudaStream_t s) {
  k_wait_timeout<<<1, 32, 0, s>>>(max_polls, flag);
  return cudaGetLastError();
}

cudaError_t device_pow_log(const double* x, double y, double* p, double* l, int n, cudaStream_t s) {
  k_pow_log<<<(n + 255) / 256, 256, 0, s>>>(x, y, p, l, n);
  return cudaGetLastError();
}

}  // namespace atm
