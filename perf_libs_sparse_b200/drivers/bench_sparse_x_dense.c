/*
 * Sparse x dense benchmark driver with the command line and output of the
 * reference's bench/pl_bench_sparse_x_dense.c (:243-304), running on the
 * B200 library through the drop-in interface:
 *
 *     bench_sparse_x_dense matrix.mtx
 *
 * reads a Matrix Market coordinate file (perflibs_b200_read_mtx), creates
 * the CSR handle A, a row-major dense B of n x 1024 values drawn with
 * srand(1) / rand() in [-1, 1] (the column count shrinks by 8x while n x
 * cols would overflow, as the reference does), a null C, calls
 * perflibs_spmm_optimize and then times 10 perflibs_spmm_exec_d calls with a
 * monotonic clock. Each exec returns when C is complete, as the reference's
 * does, so the wall-clock time covers the device work.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "perflibs_b200.h"
#include "perflibs_sparse.h"

static void die(const char *what) {
  fprintf(stderr, "error: %s\n", what);
  exit(1);
}

static double seconds(void) {
  struct timespec t;
  if (clock_gettime(CLOCK_MONOTONIC, &t) != 0)
    die("clock_gettime failed");
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

int main(int argc, char **argv) {
  const int iters = 10;
  int32_t m = 0, n = 0;
  int64_t nnz = 0;
  int32_t *row_ptr = NULL, *col = NULL;
  double *vals = NULL;
  perflibs_spmat_t A = NULL, B = NULL, C = NULL;
  int32_t cols = 1024;

  if (argc != 2)
    die("usage: bench_sparse_x_dense matrix.mtx");
  if (perflibs_b200_read_mtx(argv[1], &m, &n, &nnz, &row_ptr, &col, &vals) !=
      PERFLIBS_STATUS_SUCCESS)
    die("failed to read the Matrix Market file");

  {
    const uint64_t max_len = (uint64_t)sqrt((double)(SIZE_MAX / sizeof(double)));
    while ((uint64_t)n * (uint64_t)cols > max_len && cols > 1)
      cols = cols / 8 > 0 ? cols / 8 : 1;
  }
  const size_t blen = (size_t)n * (size_t)cols;
  double *bvals = (double *)malloc(sizeof(double) * (blen ? blen : 1));
  if (!bvals)
    die("dense B allocation failed");
  srand(1);
  for (size_t i = 0; i < blen; ++i)
    bvals[i] = 2.0 * rand() / (double)RAND_MAX - 1.0;

  if (perflibs_spmat_create_csr_d(&A, m, n, row_ptr, col, vals, 0) != PERFLIBS_STATUS_SUCCESS)
    die("create A failed");
  if (perflibs_spmat_create_dense_d(&B, PERFLIBS_ROW_MAJOR, n, cols, cols, bvals, 0) !=
      PERFLIBS_STATUS_SUCCESS)
    die("create B failed");
  C = perflibs_spmat_create_null(m, cols);
  if (!C)
    die("create C failed");
  if (perflibs_spmm_optimize(PERFLIBS_SPARSE_OPERATION_NOTRANS, PERFLIBS_SPARSE_OPERATION_NOTRANS,
                             PERFLIBS_SPARSE_SCALAR_ONE, A, B, PERFLIBS_SPARSE_SCALAR_ZERO,
                             C) != PERFLIBS_STATUS_SUCCESS)
    die("optimize failed");

  const double t0 = seconds();
  for (int i = 0; i < iters; ++i)
    if (perflibs_spmm_exec_d(PERFLIBS_SPARSE_OPERATION_NOTRANS, PERFLIBS_SPARSE_OPERATION_NOTRANS,
                             1.0, A, B, 0.0, C) != PERFLIBS_STATUS_SUCCESS)
      die("exec failed");
  const double sec = seconds() - t0;

  printf("A: %lld x %lld nnz=%lld\n", (long long)m, (long long)n, (long long)nnz);
  printf("B: %lld x %lld\n", (long long)n, (long long)cols);
  printf("C: %lld x %lld\n", (long long)m, (long long)cols);
  printf("iters=%d total_s=%.6f avg_s=%.6f\n", iters, sec, sec / iters);

  if (perflibs_spmat_destroy(C) != PERFLIBS_STATUS_SUCCESS ||
      perflibs_spmat_destroy(B) != PERFLIBS_STATUS_SUCCESS ||
      perflibs_spmat_destroy(A) != PERFLIBS_STATUS_SUCCESS)
    die("destroy failed");
  free(bvals);
  free(vals);
  free(col);
  free(row_ptr);
  return 0;
}
