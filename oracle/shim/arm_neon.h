/*
 * Portable stand-in for <arm_neon.h>, used ONLY to compile the reference
 * library's C++ sources on x86_64 for the CPU oracle (test infrastructure).
 *
 * Every function below is a scalar implementation written from the public
 * Arm C Language Extensions (ACLE) description of the intrinsic's semantics.
 * None of them sits on the sparse x dense execute path: the reference uses
 * them in triangular solves (src/solve_parallel.hpp:56-90), in Gustavson
 * sparse x sparse SpMM (src/matmul_gustavson.cpp:416-497) and in a CSR dot
 * helper (src/compressed_sparse_rows.cpp:1846-1877).
 */
#ifndef PLS_ORACLE_SHIM_ARM_NEON_H
#define PLS_ORACLE_SHIM_ARM_NEON_H

#include <stdint.h>

typedef double float64x2_t __attribute__((vector_size(16)));
typedef double float64x1_t __attribute__((vector_size(8)));
typedef uint8_t uint8x16_t __attribute__((vector_size(16)));
typedef uint16_t uint16x8_t __attribute__((vector_size(16)));
typedef uint32_t uint32x4_t __attribute__((vector_size(16)));
typedef uint64_t uint64x2_t __attribute__((vector_size(16)));

/* Broadcast a scalar to both lanes. */
static inline float64x2_t vdupq_n_f64(double v) {
  float64x2_t r = {v, v};
  return r;
}
/* Load two / one doubles. */
static inline float64x2_t vld1q_f64(const double *p) {
  float64x2_t r = {p[0], p[1]};
  return r;
}
static inline float64x1_t vld1_f64(const double *p) {
  float64x1_t r = {p[0]};
  return r;
}
/* Replace one lane. */
static inline float64x2_t vsetq_lane_f64(double v, float64x2_t a, int lane) {
  a[lane] = v;
  return a;
}
/* Lane-wise fused multiply-add: a + b * c. */
static inline float64x2_t vfmaq_f64(float64x2_t a, float64x2_t b,
                                    float64x2_t c) {
  float64x2_t r = {__builtin_fma(b[0], c[0], a[0]),
                   __builtin_fma(b[1], c[1], a[1])};
  return r;
}
/* a + b * c[lane] (c is a one-lane vector here). */
static inline float64x2_t vfmaq_lane_f64(float64x2_t a, float64x2_t b,
                                         float64x1_t c, int lane) {
  double s = c[lane];
  float64x2_t r = {__builtin_fma(b[0], s, a[0]), __builtin_fma(b[1], s, a[1])};
  return r;
}
static inline float64x2_t vaddq_f64(float64x2_t a, float64x2_t b) {
  return a + b;
}
/* Horizontal add across lanes. */
static inline double vaddvq_f64(float64x2_t a) { return a[0] + a[1]; }
static inline void vst1q_lane_f64(double *p, float64x2_t a, int lane) {
  *p = a[lane];
}

#define PLS_SHIM_LOADS(T, VT, N, SUF)                                          \
  static inline VT vld1q_##SUF(const T *p) {                                  \
    VT r;                                                                      \
    for (int i = 0; i < N; ++i)                                                \
      r[i] = p[i];                                                             \
    return r;                                                                  \
  }                                                                            \
  /* Lane-wise compare-equal: all ones where equal, zero elsewhere. */         \
  static inline VT vceqq_##SUF(VT a, VT b) {                                  \
    VT r;                                                                      \
    for (int i = 0; i < N; ++i)                                                \
      r[i] = (a[i] == b[i]) ? (T)~(T)0 : (T)0;                                 \
    return r;                                                                  \
  }                                                                            \
  /* Horizontal add across lanes, wrapping in the element type. */            \
  static inline T vaddvq_##SUF(VT a) {                                         \
    T s = 0;                                                                   \
    for (int i = 0; i < N; ++i)                                                \
      s = (T)(s + a[i]);                                                       \
    return s;                                                                  \
  }

PLS_SHIM_LOADS(uint8_t, uint8x16_t, 16, u8)
PLS_SHIM_LOADS(uint16_t, uint16x8_t, 8, u16)
PLS_SHIM_LOADS(uint32_t, uint32x4_t, 4, u32)
PLS_SHIM_LOADS(uint64_t, uint64x2_t, 2, u64)

#undef PLS_SHIM_LOADS

#endif
