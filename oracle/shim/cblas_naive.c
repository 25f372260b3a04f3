/*
 * Naive CBLAS routines for the CPU oracle build of the reference library
 * (test infrastructure only). Plain loops following the reference BLAS
 * definitions of scal, axpby, gemv, gemm and trsv. Performance is irrelevant:
 * on the sparse x dense execute path only scal and axpby are reached, on the
 * beta-only scaling and identity edge cases.
 */
#include "cblas.h"

#include <complex.h>

typedef float complex pls_c8;
typedef double complex pls_c16;

static inline float pls_conj_s(float v) { return v; }
static inline double pls_conj_d(double v) { return v; }
static inline pls_c8 pls_conj_c(pls_c8 v) { return conjf(v); }
static inline pls_c16 pls_conj_z(pls_c16 v) { return conj(v); }

/* Element (i, j) of a stored matrix with leading dimension ld. */
#define PLS_AT(A, layout, ld, i, j)                                            \
  ((layout) == CblasRowMajor ? (A)[(i) * (ld) + (j)] : (A)[(j) * (ld) + (i)])

#define PLS_DEFINE(P, T, CONJ)                                                 \
  static void pls_scal_##P(pls_blas_int n, T a, T *x, pls_blas_int incx) {     \
    for (pls_blas_int i = 0; i < n; ++i)                                       \
      x[i * incx] = a * x[i * incx];                                           \
  }                                                                            \
  static void pls_axpby_##P(pls_blas_int n, T a, const T *x,                   \
                            pls_blas_int incx, T b, T *y, pls_blas_int incy) { \
    for (pls_blas_int i = 0; i < n; ++i)                                       \
      y[i * incy] = a * x[i * incx] + b * y[i * incy];                         \
  }                                                                            \
  static void pls_gemv_##P(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t,             \
                           pls_blas_int m, pls_blas_int n, T alpha,            \
                           const T *a, pls_blas_int lda, const T *x,           \
                           pls_blas_int incx, T beta, T *y,                    \
                           pls_blas_int incy) {                                \
    pls_blas_int rows = t == CblasNoTrans ? m : n;                             \
    pls_blas_int cols = t == CblasNoTrans ? n : m;                             \
    for (pls_blas_int i = 0; i < rows; ++i) {                                  \
      T s = 0;                                                                 \
      for (pls_blas_int j = 0; j < cols; ++j) {                                \
        T v = t == CblasNoTrans ? PLS_AT(a, layout, lda, i, j)                 \
                                : PLS_AT(a, layout, lda, j, i);                \
        if (t == CblasConjTrans)                                               \
          v = CONJ(v);                                                         \
        s += v * x[j * incx];                                                  \
      }                                                                        \
      y[i * incy] = alpha * s + (beta == (T)0 ? (T)0 : beta * y[i * incy]);    \
    }                                                                          \
  }                                                                            \
  static void pls_gemm_##P(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta,            \
                           CBLAS_TRANSPOSE tb, pls_blas_int m, pls_blas_int n, \
                           pls_blas_int k, T alpha, const T *a,                \
                           pls_blas_int lda, const T *b, pls_blas_int ldb,     \
                           T beta, T *c, pls_blas_int ldc) {                   \
    for (pls_blas_int i = 0; i < m; ++i) {                                     \
      for (pls_blas_int j = 0; j < n; ++j) {                                   \
        T s = 0;                                                               \
        for (pls_blas_int l = 0; l < k; ++l) {                                 \
          T av = ta == CblasNoTrans ? PLS_AT(a, layout, lda, i, l)             \
                                    : PLS_AT(a, layout, lda, l, i);            \
          T bv = tb == CblasNoTrans ? PLS_AT(b, layout, ldb, l, j)             \
                                    : PLS_AT(b, layout, ldb, j, l);            \
          if (ta == CblasConjTrans)                                            \
            av = CONJ(av);                                                     \
          if (tb == CblasConjTrans)                                            \
            bv = CONJ(bv);                                                     \
          s += av * bv;                                                        \
        }                                                                      \
        T *cij = layout == CblasRowMajor ? &c[i * ldc + j] : &c[j * ldc + i];  \
        *cij = alpha * s + (beta == (T)0 ? (T)0 : beta * *cij);                \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  static void pls_trsv_##P(CBLAS_LAYOUT layout, CBLAS_UPLO uplo,               \
                           CBLAS_TRANSPOSE t, CBLAS_DIAG diag, pls_blas_int n, \
                           const T *a, pls_blas_int lda, T *x,                 \
                           pls_blas_int incx) {                                \
    /* Solve op(A) x = b in place; op(A) is lower iff the stored triangle */   \
    /* is lower and op is identity, or upper and op transposes.          */   \
    int lower = (uplo == CblasLower) == (t == CblasNoTrans);                   \
    for (pls_blas_int s = 0; s < n; ++s) {                                     \
      pls_blas_int i = lower ? s : n - 1 - s;                                  \
      T acc = x[i * incx];                                                     \
      for (pls_blas_int j = 0; j < n; ++j) {                                   \
        if ((lower && j >= i) || (!lower && j <= i))                           \
          continue;                                                            \
        T v = t == CblasNoTrans ? PLS_AT(a, layout, lda, i, j)                 \
                                : PLS_AT(a, layout, lda, j, i);                \
        if (t == CblasConjTrans)                                               \
          v = CONJ(v);                                                         \
        acc -= v * x[j * incx];                                                \
      }                                                                        \
      if (diag == CblasNonUnit) {                                              \
        T d = PLS_AT(a, layout, lda, i, i);                                    \
        if (t == CblasConjTrans)                                               \
          d = CONJ(d);                                                         \
        acc /= d;                                                              \
      }                                                                        \
      x[i * incx] = acc;                                                       \
    }                                                                          \
  }

PLS_DEFINE(s, float, pls_conj_s)
PLS_DEFINE(d, double, pls_conj_d)
PLS_DEFINE(c, pls_c8, pls_conj_c)
PLS_DEFINE(z, pls_c16, pls_conj_z)

void cblas_sscal(pls_blas_int n, float a, float *x, pls_blas_int incx) {
  pls_scal_s(n, a, x, incx);
}
void cblas_dscal(pls_blas_int n, double a, double *x, pls_blas_int incx) {
  pls_scal_d(n, a, x, incx);
}
void cblas_cscal(pls_blas_int n, const void *a, void *x, pls_blas_int incx) {
  pls_scal_c(n, *(const pls_c8 *)a, (pls_c8 *)x, incx);
}
void cblas_zscal(pls_blas_int n, const void *a, void *x, pls_blas_int incx) {
  pls_scal_z(n, *(const pls_c16 *)a, (pls_c16 *)x, incx);
}

void cblas_saxpby(pls_blas_int n, float a, const float *x, pls_blas_int incx,
                  float b, float *y, pls_blas_int incy) {
  pls_axpby_s(n, a, x, incx, b, y, incy);
}
void cblas_daxpby(pls_blas_int n, double a, const double *x, pls_blas_int incx,
                  double b, double *y, pls_blas_int incy) {
  pls_axpby_d(n, a, x, incx, b, y, incy);
}
void cblas_caxpby(pls_blas_int n, const void *a, const void *x,
                  pls_blas_int incx, const void *b, void *y,
                  pls_blas_int incy) {
  pls_axpby_c(n, *(const pls_c8 *)a, (const pls_c8 *)x, incx,
              *(const pls_c8 *)b, (pls_c8 *)y, incy);
}
void cblas_zaxpby(pls_blas_int n, const void *a, const void *x,
                  pls_blas_int incx, const void *b, void *y,
                  pls_blas_int incy) {
  pls_axpby_z(n, *(const pls_c16 *)a, (const pls_c16 *)x, incx,
              *(const pls_c16 *)b, (pls_c16 *)y, incy);
}

void cblas_sgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, float alpha, const float *a, pls_blas_int lda,
                 const float *x, pls_blas_int incx, float beta, float *y,
                 pls_blas_int incy) {
  pls_gemv_s(layout, t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
void cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, double alpha, const double *a,
                 pls_blas_int lda, const double *x, pls_blas_int incx,
                 double beta, double *y, pls_blas_int incy) {
  pls_gemv_d(layout, t, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
void cblas_cgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, const void *alpha, const void *a,
                 pls_blas_int lda, const void *x, pls_blas_int incx,
                 const void *beta, void *y, pls_blas_int incy) {
  pls_gemv_c(layout, t, m, n, *(const pls_c8 *)alpha, (const pls_c8 *)a, lda,
             (const pls_c8 *)x, incx, *(const pls_c8 *)beta, (pls_c8 *)y,
             incy);
}
void cblas_zgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, const void *alpha, const void *a,
                 pls_blas_int lda, const void *x, pls_blas_int incx,
                 const void *beta, void *y, pls_blas_int incy) {
  pls_gemv_z(layout, t, m, n, *(const pls_c16 *)alpha, (const pls_c16 *)a, lda,
             (const pls_c16 *)x, incx, *(const pls_c16 *)beta, (pls_c16 *)y,
             incy);
}

void cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k, float alpha,
                 const float *a, pls_blas_int lda, const float *b,
                 pls_blas_int ldb, float beta, float *c, pls_blas_int ldc) {
  pls_gemm_s(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k, double alpha,
                 const double *a, pls_blas_int lda, const double *b,
                 pls_blas_int ldb, double beta, double *c, pls_blas_int ldc) {
  pls_gemm_d(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
void cblas_cgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k,
                 const void *alpha, const void *a, pls_blas_int lda,
                 const void *b, pls_blas_int ldb, const void *beta, void *c,
                 pls_blas_int ldc) {
  pls_gemm_c(layout, ta, tb, m, n, k, *(const pls_c8 *)alpha,
             (const pls_c8 *)a, lda, (const pls_c8 *)b, ldb,
             *(const pls_c8 *)beta, (pls_c8 *)c, ldc);
}
void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k,
                 const void *alpha, const void *a, pls_blas_int lda,
                 const void *b, pls_blas_int ldb, const void *beta, void *c,
                 pls_blas_int ldc) {
  pls_gemm_z(layout, ta, tb, m, n, k, *(const pls_c16 *)alpha,
             (const pls_c16 *)a, lda, (const pls_c16 *)b, ldb,
             *(const pls_c16 *)beta, (pls_c16 *)c, ldc);
}

void cblas_strsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const float *a,
                 pls_blas_int lda, float *x, pls_blas_int incx) {
  pls_trsv_s(layout, uplo, t, diag, n, a, lda, x, incx);
}
void cblas_dtrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const double *a,
                 pls_blas_int lda, double *x, pls_blas_int incx) {
  pls_trsv_d(layout, uplo, t, diag, n, a, lda, x, incx);
}
void cblas_ctrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const void *a,
                 pls_blas_int lda, void *x, pls_blas_int incx) {
  pls_trsv_c(layout, uplo, t, diag, n, (const pls_c8 *)a, lda, (pls_c8 *)x,
             incx);
}
void cblas_ztrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const void *a,
                 pls_blas_int lda, void *x, pls_blas_int incx) {
  pls_trsv_z(layout, uplo, t, diag, n, (const pls_c16 *)a, lda, (pls_c16 *)x,
             incx);
}
