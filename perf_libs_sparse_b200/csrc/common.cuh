// Device helpers shared by the kernels of libplsparse_b200.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pls {

constexpr int kWarp = 32;

// ---- value loads ----------------------------------------------------------
// Matrix data (values, column indices, SELL offsets) is read once per SpMV,
// so it is loaded with the streaming hint (ld.global.cs: evict-first in L1
// and L2). That keeps the gathered vector x resident in the 126 MB L2.
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16 *p) {
  return __ldcs(p);
}
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) { return __ldcs(p); }
__device__ __forceinline__ uint8_t ld_stream(const uint8_t *p) {
  return (uint8_t)__ldcs((const unsigned char *)p);
}
__device__ __forceinline__ uint16_t ld_stream(const uint16_t *p) {
  return (uint16_t)__ldcs((const unsigned short *)p);
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) {
  return (uint32_t)__ldcs((const unsigned int *)p);
}
__device__ __forceinline__ uint64_t ld_stream(const uint64_t *p) {
  return (uint64_t)__ldcs((const unsigned long long *)p);
}

// Gathered operand (x, rows of B): read-only path, normal L2 residency.
template <class T> __device__ __forceinline__ T ld_ro(const T *p) { return __ldg(p); }

// ---- explicit L2 eviction priorities -----------------------------------
// The matrix stream is read once and marked evict-first; the gathered vector
// is marked evict-last, so the stream cannot push x out of L2 (without this,
// about 40% of random x gathers missed L2 on power-law matrices). sm_100
// takes the priority for scalar loads through a cache-policy operand.
struct L2Policy {
  uint64_t stream, keep;
};
__device__ __forceinline__ L2Policy make_l2_policy() {
  L2Policy p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p.stream));
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p.keep));
  return p;
}
__device__ __forceinline__ double ld_stream(const double *p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float *p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ __nv_bfloat16 ld_stream(const __nv_bfloat16 *p, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return __ushort_as_bfloat16(v);
}
__device__ __forceinline__ int32_t ld_stream(const int32_t *p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int2 ld_stream(const int2 *p, uint64_t pol) {
  int2 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
      : "=r"(v.x), "=r"(v.y)
      : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint16_t ld_stream(const uint16_t *p, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint8_t ld_stream(const uint8_t *p, uint64_t pol) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u8 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
  return (uint8_t)v;
}
__device__ __forceinline__ double ld_keep(const double *p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_keep(const float *p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

// ---- conversions to the accumulator type ------------------------------------
template <class Acc> __device__ __forceinline__ Acc to_acc(double v) { return (Acc)v; }
template <class Acc> __device__ __forceinline__ Acc to_acc(float v) { return (Acc)v; }
template <class Acc> __device__ __forceinline__ Acc to_acc(__nv_bfloat16 v) {
  return (Acc)__bfloat162float(v);
}

template <class T> __device__ __forceinline__ T from_double(double v) { return (T)v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_double<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}

// Accumulator type: FP64 for native double storage, FP32 otherwise.
template <class V, class X> struct AccOf { using type = float; };
template <> struct AccOf<double, double> { using type = double; };

// ---- warp reductions ------------------------------------------------------
template <int W, class T> __device__ __forceinline__ T group_sum(T v, unsigned mask) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1)
    v += __shfl_xor_sync(mask, v, o);
  return v;
}

template <int W> __device__ __forceinline__ unsigned group_mask() {
  if constexpr (W >= 32)
    return 0xffffffffu;
  else
    return ((1u << W) - 1u) << ((threadIdx.x & 31) & ~(W - 1));
}

__host__ __device__ constexpr int64_t div_up(int64_t a, int64_t b) {
  return (a + b - 1) / b;
}

}  // namespace pls
