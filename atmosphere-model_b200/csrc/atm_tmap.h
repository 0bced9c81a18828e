// Host side of the TMA tile loads: the driver's tensor-map encoder and a
// cache of one map per (buffer, element size, field shape, box shape).
// Each translation unit that launches TMA kernels gets its own cache.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "atm_common.cuh"

namespace atm {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

using MapKey = std::tuple<const void*, int, int, int, int, int, int>;
std::mutex g_map_mu;
std::map<MapKey, CUtensorMap> g_maps;

// map of a field (K levels of ny+14 rows of pitch P, element size es) for
// boxes of bw x bh elements
cudaError_t tmap(const void* base, int es, const Geom& g, int K, int bw, int bh, CUtensorMap* out) {
  MapKey key{base, es, g.P, g.NYP, K, bw, bh};
  std::lock_guard<std::mutex> lock(g_map_mu);
  auto it = g_maps.find(key);
  if (it != g_maps.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  CUtensorMap m;
  cuuint64_t dims[3] = {(cuuint64_t)g.P, (cuuint64_t)g.NYP, (cuuint64_t)K};
  cuuint64_t strides[2] = {(cuuint64_t)g.P * es, (cuuint64_t)g.S * es};
  cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&m, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                  const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  g_maps.emplace(key, m);
  *out = m;
  return cudaSuccess;
}

}  // namespace
}  // namespace atm
