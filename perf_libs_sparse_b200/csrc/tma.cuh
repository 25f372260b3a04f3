// Shared-memory staging helpers for sm_100a kernels: mbarriers, 1-D bulk
// copies and 2-D tensor-map (TMA) copies from this GPU's global memory, and
// bounded waits. No cluster multicast is used anywhere: every copy lands in
// the issuing CTA's own shared memory.
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include <cstdint>

namespace pls {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// One arrival (the issuing thread's expect_tx) completes a phase once the
// expected bytes have landed.
__device__ __forceinline__ void bar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// A barrier whose phase completes after `count` plain arrivals.
__device__ __forceinline__ void bar_init_count(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// One arrival (release: the calling thread's earlier shared-memory accesses
// are ordered before a waiter's later ones).
__device__ __forceinline__ void bar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with `parity`: back-to-back polls first, then
// polls with short sleeps; false after `limit` polls (2^22 is about a
// second).
__device__ __forceinline__ bool bar_wait_bounded(uint64_t *bar, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it) {
    if (bar_try_wait(bar, parity))
      return true;
    if (it >= 1024)
      __nanosleep(256);
  }
  return false;
}

// 1-D bulk copy global -> shared (both addresses 16-byte aligned, bytes a
// multiple of 16), completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// 2-D tiled tensor copy global -> shared of the box at (x, y) (x the inner
// coordinate; x * element size must be a multiple of 16 bytes; y may be
// negative or past the end: those rows read as zeros), completing on `bar`.
// dst 128-byte aligned.
__device__ __forceinline__ void tensor_load_2d(void *dst, const CUtensorMap *map, int32_t x,
                                               int32_t y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
      "r"(smem_addr(bar))
      : "memory");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// to the driver library); null if the driver does not offer it.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

}  // namespace tma
}  // namespace pls
