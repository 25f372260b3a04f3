/*
 * Minimal CBLAS interface for the CPU oracle build of the reference library
 * (test infrastructure only). Declares the routines the reference's
 * src/cblas_wrappers.hpp binds: {s,d,c,z}{scal,axpby,gemv,gemm,trsv}.
 * The implementations in cblas_naive.c are plain loops written from the
 * reference BLAS definitions. On the sparse x dense execute path only
 * scal (src/matvec.cpp:83) and axpby (src/special.cpp:41) are reached.
 */
#ifndef PLS_ORACLE_SHIM_CBLAS_H
#define PLS_ORACLE_SHIM_CBLAS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifdef INTEGER64
typedef int64_t pls_blas_int;
#else
typedef int32_t pls_blas_int;
#endif

typedef enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum CBLAS_TRANSPOSE {
  CblasNoTrans = 111,
  CblasTrans = 112,
  CblasConjTrans = 113
} CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;

void cblas_sscal(pls_blas_int n, float a, float *x, pls_blas_int incx);
void cblas_dscal(pls_blas_int n, double a, double *x, pls_blas_int incx);
void cblas_cscal(pls_blas_int n, const void *a, void *x, pls_blas_int incx);
void cblas_zscal(pls_blas_int n, const void *a, void *x, pls_blas_int incx);

void cblas_saxpby(pls_blas_int n, float a, const float *x, pls_blas_int incx,
                  float b, float *y, pls_blas_int incy);
void cblas_daxpby(pls_blas_int n, double a, const double *x, pls_blas_int incx,
                  double b, double *y, pls_blas_int incy);
void cblas_caxpby(pls_blas_int n, const void *a, const void *x,
                  pls_blas_int incx, const void *b, void *y, pls_blas_int incy);
void cblas_zaxpby(pls_blas_int n, const void *a, const void *x,
                  pls_blas_int incx, const void *b, void *y, pls_blas_int incy);

void cblas_sgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, float alpha, const float *a, pls_blas_int lda,
                 const float *x, pls_blas_int incx, float beta, float *y,
                 pls_blas_int incy);
void cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, double alpha, const double *a,
                 pls_blas_int lda, const double *x, pls_blas_int incx,
                 double beta, double *y, pls_blas_int incy);
void cblas_cgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, const void *alpha, const void *a,
                 pls_blas_int lda, const void *x, pls_blas_int incx,
                 const void *beta, void *y, pls_blas_int incy);
void cblas_zgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE t, pls_blas_int m,
                 pls_blas_int n, const void *alpha, const void *a,
                 pls_blas_int lda, const void *x, pls_blas_int incx,
                 const void *beta, void *y, pls_blas_int incy);

void cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k, float alpha,
                 const float *a, pls_blas_int lda, const float *b,
                 pls_blas_int ldb, float beta, float *c, pls_blas_int ldc);
void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k, double alpha,
                 const double *a, pls_blas_int lda, const double *b,
                 pls_blas_int ldb, double beta, double *c, pls_blas_int ldc);
void cblas_cgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k,
                 const void *alpha, const void *a, pls_blas_int lda,
                 const void *b, pls_blas_int ldb, const void *beta, void *c,
                 pls_blas_int ldc);
void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 pls_blas_int m, pls_blas_int n, pls_blas_int k,
                 const void *alpha, const void *a, pls_blas_int lda,
                 const void *b, pls_blas_int ldb, const void *beta, void *c,
                 pls_blas_int ldc);

void cblas_strsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const float *a,
                 pls_blas_int lda, float *x, pls_blas_int incx);
void cblas_dtrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const double *a,
                 pls_blas_int lda, double *x, pls_blas_int incx);
void cblas_ctrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const void *a,
                 pls_blas_int lda, void *x, pls_blas_int incx);
void cblas_ztrsv(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE t,
                 CBLAS_DIAG diag, pls_blas_int n, const void *a,
                 pls_blas_int lda, void *x, pls_blas_int incx);

#ifdef __cplusplus
}
#endif

#endif
