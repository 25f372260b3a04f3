/*
 * Test tap for the reference's unchanged benchmark driver
 * (bench/pl_bench_sparse_x_dense.c): preloaded (LD_PRELOAD) in front of
 * libplsparse_b200.so, it forwards perflibs_spmm_exec_d to the library and,
 * after each successful call, writes C (int32 rows, int32 cols, then the
 * row-major FP64 values) to the file named by PERFLIBS_TAP_C, through the
 * library's own perflibs_spmat_export_dense_d. The driver itself prints
 * only timings; this is how its result reaches the parity check.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>

#include "perflibs_sparse.h"

typedef perflibs_status_t (*spmm_exec_fn)(enum perflibs_sparse_hint_value,
                                          enum perflibs_sparse_hint_value, double,
                                          perflibs_spmat_t, perflibs_spmat_t, double,
                                          perflibs_spmat_t);

perflibs_status_t perflibs_spmm_exec_d(enum perflibs_sparse_hint_value transA,
                                       enum perflibs_sparse_hint_value transB, double alpha,
                                       perflibs_spmat_t A, perflibs_spmat_t B, double beta,
                                       perflibs_spmat_t C) {
  static spmm_exec_fn next = NULL;
  if (!next)
    next = (spmm_exec_fn)dlsym(RTLD_NEXT, "perflibs_spmm_exec_d");
  if (!next)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  const perflibs_status_t st = next(transA, transB, alpha, A, B, beta, C);
  const char *path = getenv("PERFLIBS_TAP_C");
  if (st != PERFLIBS_STATUS_SUCCESS || !path)
    return st;
  perflibs_int_t m = 0, n = 0;
  double *vals = NULL;
  if (perflibs_spmat_export_dense_d(C, PERFLIBS_ROW_MAJOR, &m, &n, &vals) !=
      PERFLIBS_STATUS_SUCCESS)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  FILE *f = fopen(path, "wb");
  if (f) {
    fwrite(&m, sizeof m, 1, f);
    fwrite(&n, sizeof n, 1, f);
    fwrite(vals, sizeof(double), (size_t)m * (size_t)n, f);
    fclose(f);
  }
  free(vals);
  return st;
}
