// Tensor-memory-accelerator (TMA) tile loads for the per-layer kernels.
//
// A field is a 3-D tensor (x: row pitch P, y: ny+14 rows, z: levels) in
// HBM.  One elected thread issues cp.async.bulk.tensor loads of the input
// boxes of a tile into shared memory, all completing on one mbarrier.  Only
// that thread waits on the barrier, with an iteration limit: on a timeout
// it records the failure and the whole block returns after the next
// __syncthreads, so no thread is left spinning.
//
// Box starts are rounded down so that x * element size is a multiple of
// 16 bytes (the rule for tiled TMA); the shared-memory window records the
// rounded start.  Boxes that reach outside the tensor read zeros there,
// which only feed outputs outside the kernel's range.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "atm_common.cuh"

namespace atm {

// bytes of a TMA box of w x h elements of size es, rounded up to 128 bytes
// (the shared-memory alignment the copies use)
__host__ __device__ constexpr size_t tma_box_bytes(int w, int h, int es) {
  return ((size_t)w * h * es + 127) & ~(size_t)127;
}
// x start rounded down to a 16-byte boundary and the width that covers
// [x0, x0 + w) from there, rounded up to whole 16-byte units
template <typename T> __host__ __device__ constexpr int tma_q() { return 16 / (int)sizeof(T); }
template <typename T> __host__ __device__ constexpr int tma_width(int w) {
  // worst case start offset is q-1 elements
  return ((w + tma_q<T>() - 1) + tma_q<T>() - 1) / tma_q<T>() * tma_q<T>();
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// one TMA tile load of a 3-D box whose coordinates are (x, y, z) in elements
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// wait for a phase of the barrier, at most max_iter polls of at most ~1 us
// each; true on success
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int max_iter) {
  uint32_t done = 0;
  for (int it = 0; it < max_iter; ++it) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// A box to load: destination window in shared memory and its start in the
// tensor (interior coordinates i, j of its first element, level k).
struct TmaBox {
  const CUtensorMap* map;
  void* dst;
  int i0, j0, k;
};

// Issue all boxes on one barrier (thread 0 only) and wait (thread 0 only);
// returns false in every thread if the wait timed out.
template <int N>
__device__ __forceinline__ bool tma_fetch(const TmaBox (&boxes)[N], uint32_t bytes, uint64_t* bar, int* timeout_flag,
                                          int* s_ok) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_expect_tx(bar, bytes);
#pragma unroll
    for (int b = 0; b < N; ++b)
      tma_load_3d(boxes[b].dst, boxes[b].map, boxes[b].i0 + H + XOFF, boxes[b].j0 + H, boxes[b].k, bar);
    bool ok = mbar_wait(bar, 0, 1000000);  // about one second at most
    if (!ok) {
      if (timeout_flag) atomicOr(timeout_flag, 1);
      // let copies still in flight land before the block's shared memory is released
      mbar_wait(bar, 0, 1000000);
    }
    *s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  return *s_ok != 0;
}

// The same split in two, for boxes loaded into shared memory that the block
// has finished reading (the caller synchronises the block before the
// issue), so that the copies overlap the block's next stage: tma_issue
// (thread 0 only) initialises bar and issues the boxes; tma_wait waits for
// them as tma_fetch does.
template <int N>
__device__ __forceinline__ void tma_issue(const TmaBox (&boxes)[N], uint32_t bytes, uint64_t* bar) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_init(bar, 1);
    fence_mbar_init();
    mbar_expect_tx(bar, bytes);
#pragma unroll
    for (int b = 0; b < N; ++b)
      tma_load_3d(boxes[b].dst, boxes[b].map, boxes[b].i0 + H + XOFF, boxes[b].j0 + H, boxes[b].k, bar);
  }
}
__device__ __forceinline__ bool tma_wait(uint64_t* bar, int* timeout_flag, int* s_ok) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    bool ok = mbar_wait(bar, 0, 1000000);  // about one second at most
    if (!ok) {
      if (timeout_flag) atomicOr(timeout_flag, 1);
      mbar_wait(bar, 0, 1000000);
    }
    *s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  return *s_ok != 0;
}

}  // namespace atm
