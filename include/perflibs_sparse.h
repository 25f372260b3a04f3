/*
 * perflibs_sparse.h — drop-in C interface of the B200 sparse x dense execute
 * path (libplsparse_b200.so).
 *
 * This is the subset of the reference library's public header
 * (include/perflibs_sparse.h in perf-libs-sparse) that the sparse x dense
 * execute path needs. Names, enum values, types and argument meanings are
 * kept identical so that existing callers recompile and relink unchanged;
 * each prototype cites the reference declaration it replaces.
 *
 * Provided for input: CSR, BSR, COO and CSC creation (COO and CSC are
 * converted to CSR on the device), dense, null and identity handles.
 * Not provided (outside the execute path): supernodal creation, sparse
 * vectors, SpAdd, SpElMM, SDDMM, SpSV/SpSM, transposition and scaling of a
 * handle, and every complex (_c / _z) entry point. A caller that needs them
 * keeps linking the reference library for those symbols.
 */
#ifndef PERFLIBS_SPARSE_H
#define PERFLIBS_SPARSE_H

#include <stdint.h>

/* include/perflibs_sparse.h:37-42 (reference): 32-bit indices by default,
 * 64-bit under INTEGER64. This library is built for the 32-bit model. */
#ifdef INTEGER64
#error "libplsparse_b200 is built for 32-bit perflibs_int_t"
#endif
typedef int32_t perflibs_int_t;

/* include/perflibs_sparse.h:67-71 and include/perflibs_status.h:17-21 */
#ifndef PERFLIBS_STATUS_DEFINED
#define PERFLIBS_STATUS_DEFINED
typedef enum perflibs_status {
  PERFLIBS_STATUS_SUCCESS = 0,
  PERFLIBS_STATUS_INPUT_PARAMETER_ERROR = 1,
  PERFLIBS_STATUS_EXECUTION_FAILURE = 2,
} perflibs_status_t;
#endif

/* include/perflibs_sparse.h:80-81: opaque handles */
typedef struct perflibs_spmat_top_t *perflibs_spmat_t;
typedef const struct perflibs_spmat_top_t *perflibs_const_spmat_t;

/* include/perflibs_sparse.h:87-101 */
enum perflibs_sparse_hint_type {
  PERFLIBS_SPARSE_HINT_STRUCTURE = 50,
  PERFLIBS_SPARSE_HINT_SPMV_OPERATION = 60,
  PERFLIBS_SPARSE_HINT_SPMM_OPERATION = 61,
  PERFLIBS_SPARSE_HINT_SPADD_OPERATION = 62,
  PERFLIBS_SPARSE_HINT_SPSV_OPERATION = 63,
  PERFLIBS_SPARSE_HINT_SPMM_STRATEGY = 64,
  PERFLIBS_SPARSE_HINT_SPSM_OPERATION = 65,
  PERFLIBS_SPARSE_HINT_SPSV_STRATEGY = 66,
  PERFLIBS_SPARSE_HINT_MEMORY = 70,
  PERFLIBS_SPARSE_HINT_SPMV_INVOCATIONS = 80,
  PERFLIBS_SPARSE_HINT_SPMM_INVOCATIONS = 81,
  PERFLIBS_SPARSE_HINT_SPADD_INVOCATIONS = 82,
  PERFLIBS_SPARSE_HINT_SPSV_INVOCATIONS = 83
};

/* include/perflibs_sparse.h:103 */
enum perflibs_dense_layout { PERFLIBS_COL_MAJOR = 90, PERFLIBS_ROW_MAJOR = 91 };

/* include/perflibs_sparse.h:105-141 */
enum perflibs_sparse_hint_value {
  PERFLIBS_SPARSE_STRUCTURE_DENSE = 100,
  PERFLIBS_SPARSE_STRUCTURE_UNSTRUCTURED = 101,
  PERFLIBS_SPARSE_STRUCTURE_SYMMETRIC = 110,
  PERFLIBS_SPARSE_STRUCTURE_DIAGONAL = 120,
  PERFLIBS_SPARSE_STRUCTURE_BLOCKDIAGONAL = 130,
  PERFLIBS_SPARSE_STRUCTURE_BANDED = 140,
  PERFLIBS_SPARSE_STRUCTURE_TRIANGULAR = 150,
  PERFLIBS_SPARSE_STRUCTURE_BLOCKTRIANGULAR = 160,
  PERFLIBS_SPARSE_STRUCTURE_HERMITIAN = 170,
  PERFLIBS_SPARSE_STRUCTURE_HPCG = 180,
  PERFLIBS_SPARSE_MEMORY_NOALLOCS = 200,
  PERFLIBS_SPARSE_MEMORY_ALLOCS = 201,
  PERFLIBS_SPARSE_OPERATION_NOTRANS = 300,
  PERFLIBS_SPARSE_OPERATION_TRANS = 310,
  PERFLIBS_SPARSE_OPERATION_CONJTRANS = 320,
  PERFLIBS_SPARSE_INVOCATIONS_SINGLE = 400,
  PERFLIBS_SPARSE_INVOCATIONS_FEW = 410,
  PERFLIBS_SPARSE_INVOCATIONS_MANY = 420,
  PERFLIBS_SPARSE_SCALAR_ONE = 500,
  PERFLIBS_SPARSE_SCALAR_ZERO = 501,
  PERFLIBS_SPARSE_SCALAR_ANY = 502,
  PERFLIBS_SPARSE_SPMM_STRAT_UNSET = 600,
  PERFLIBS_SPARSE_SPMM_STRAT_OPT_NO_STRUCT = 601,
  PERFLIBS_SPARSE_SPMM_STRAT_OPT_PART_STRUCT = 602,
  PERFLIBS_SPARSE_SPMM_STRAT_OPT_FULL_STRUCT = 603,
  PERFLIBS_SPARSE_SPSV_STRAT_UNSET = 700,
  PERFLIBS_SPARSE_SPSV_STRAT_SEPARATOR_SPARSE = 701,
  PERFLIBS_SPARSE_SPSV_STRAT_SEPARATOR_DENSE = 702
};

/* include/perflibs_sparse.h:143-146 */
enum perflibs_sparse_norm {
  PERFLIBS_SPARSE_NORM_INF = 1001,
  PERFLIBS_SPARSE_NORM_FRB = 1002
};

/* include/perflibs_sparse.h:149 */
#define PERFLIBS_SPARSE_CREATE_NOCOPY 1

#ifdef __cplusplus
extern "C" {
#endif

/* ---- creation: include/perflibs_sparse.h:157-166 ---- */
perflibs_status_t
perflibs_spmat_create_csr_s(perflibs_spmat_t *A, perflibs_int_t m,
                            perflibs_int_t n, const perflibs_int_t *row_ptr,
                            const perflibs_int_t *col_indx, const float *vals,
                            perflibs_int_t flags);
perflibs_status_t
perflibs_spmat_create_csr_d(perflibs_spmat_t *A, perflibs_int_t m,
                            perflibs_int_t n, const perflibs_int_t *row_ptr,
                            const perflibs_int_t *col_indx, const double *vals,
                            perflibs_int_t flags);

/* include/perflibs_sparse.h:209-216 */
perflibs_status_t perflibs_spmat_create_dense_s(
    perflibs_spmat_t *A, enum perflibs_dense_layout layout, perflibs_int_t m,
    perflibs_int_t n, perflibs_int_t lda, const float *vals,
    perflibs_int_t flags);
perflibs_status_t perflibs_spmat_create_dense_d(
    perflibs_spmat_t *A, enum perflibs_dense_layout layout, perflibs_int_t m,
    perflibs_int_t n, perflibs_int_t lda, const double *vals,
    perflibs_int_t flags);

/* include/perflibs_sparse.h:176-184. The handle is converted to CSR on the
 * device at creation (columns ascending per row). */
perflibs_status_t perflibs_spmat_create_csc_s(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_ptr, const float *vals,
                                              perflibs_int_t flags);
perflibs_status_t perflibs_spmat_create_csc_d(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_ptr, const double *vals,
                                              perflibs_int_t flags);

/* include/perflibs_sparse.h:193-200 (0-based indices). Converted to CSR on
 * the device at creation: entries sorted by (row, column), duplicates kept
 * and added by the kernels. */
perflibs_status_t perflibs_spmat_create_coo_s(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, perflibs_int_t nnz,
                                              const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_indx, const float *vals,
                                              perflibs_int_t flags);
perflibs_status_t perflibs_spmat_create_coo_d(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, perflibs_int_t nnz,
                                              const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_indx, const double *vals,
                                              perflibs_int_t flags);

/* include/perflibs_sparse.h:225-234 */
perflibs_status_t perflibs_spmat_create_bsr_s(
    perflibs_spmat_t *A, enum perflibs_dense_layout block_layout,
    perflibs_int_t m, perflibs_int_t n, perflibs_int_t block_size,
    const perflibs_int_t *row_ptr, const perflibs_int_t *col_indx,
    const float *vals, perflibs_int_t flags);
perflibs_status_t perflibs_spmat_create_bsr_d(
    perflibs_spmat_t *A, enum perflibs_dense_layout block_layout,
    perflibs_int_t m, perflibs_int_t n, perflibs_int_t block_size,
    const perflibs_int_t *row_ptr, const perflibs_int_t *col_indx,
    const double *vals, perflibs_int_t flags);

/* include/perflibs_sparse.h:272-273 (creates a double-precision handle, as
 * the reference does) */
perflibs_spmat_t perflibs_spmat_create_null(perflibs_int_t m, perflibs_int_t n);
perflibs_spmat_t perflibs_spmat_create_identity(perflibs_int_t n);

/* include/perflibs_sparse.h:275-284 */
perflibs_status_t perflibs_spmat_destroy(perflibs_spmat_t A);
perflibs_status_t perflibs_spmat_query(perflibs_spmat_t A,
                                       perflibs_int_t *index_base,
                                       perflibs_int_t *m, perflibs_int_t *n,
                                       perflibs_int_t *nnz);
perflibs_status_t perflibs_spmat_hint(perflibs_spmat_t A,
                                      enum perflibs_sparse_hint_type hint,
                                      enum perflibs_sparse_hint_value value);

/* ---- optimize: include/perflibs_sparse.h:430-436 ---- */
perflibs_status_t perflibs_spmv_optimize(perflibs_spmat_t A);
perflibs_status_t perflibs_spmm_optimize(enum perflibs_sparse_hint_value transA,
                                         enum perflibs_sparse_hint_value transB,
                                         enum perflibs_sparse_hint_value alpha,
                                         perflibs_spmat_t A, perflibs_spmat_t B,
                                         enum perflibs_sparse_hint_value beta,
                                         perflibs_spmat_t C);

/* ---- execute: include/perflibs_sparse.h:464-469, 483-492 ----
 * Host pointers; the call returns when y (or C) holds the result. */
perflibs_status_t perflibs_spmv_exec_s(enum perflibs_sparse_hint_value trans,
                                       float alpha, perflibs_spmat_t A,
                                       const float *x, float beta, float *y);
perflibs_status_t perflibs_spmv_exec_d(enum perflibs_sparse_hint_value trans,
                                       double alpha, perflibs_spmat_t A,
                                       const double *x, double beta, double *y);
perflibs_status_t perflibs_spmm_exec_s(enum perflibs_sparse_hint_value transA,
                                       enum perflibs_sparse_hint_value transB,
                                       float alpha, perflibs_spmat_t A,
                                       perflibs_spmat_t B, float beta,
                                       perflibs_spmat_t C);
perflibs_status_t perflibs_spmm_exec_d(enum perflibs_sparse_hint_value transA,
                                       enum perflibs_sparse_hint_value transB,
                                       double alpha, perflibs_spmat_t A,
                                       perflibs_spmat_t B, double beta,
                                       perflibs_spmat_t C);

/* ---- update: include/perflibs_sparse.h:563-572 ---- */
perflibs_status_t perflibs_spmat_update_s(perflibs_spmat_t A,
                                          perflibs_int_t n_updates,
                                          const perflibs_int_t *row_indx,
                                          const perflibs_int_t *col_indx,
                                          const float *vals);
perflibs_status_t perflibs_spmat_update_d(perflibs_spmat_t A,
                                          perflibs_int_t n_updates,
                                          const perflibs_int_t *row_indx,
                                          const perflibs_int_t *col_indx,
                                          const double *vals);

/* ---- export: include/perflibs_sparse.h:583-591, 640-645 ----
 * Arrays are malloc'ed by the library; the caller frees them. */
perflibs_status_t
perflibs_spmat_export_csr_s(perflibs_const_spmat_t A, perflibs_int_t index_base,
                            perflibs_int_t *m, perflibs_int_t *n,
                            perflibs_int_t **row_ptr, perflibs_int_t **col_indx,
                            float **vals);
perflibs_status_t
perflibs_spmat_export_csr_d(perflibs_const_spmat_t A, perflibs_int_t index_base,
                            perflibs_int_t *m, perflibs_int_t *n,
                            perflibs_int_t **row_ptr, perflibs_int_t **col_indx,
                            double **vals);
perflibs_status_t perflibs_spmat_export_dense_s(
    perflibs_const_spmat_t A, enum perflibs_dense_layout layout,
    perflibs_int_t *m, perflibs_int_t *n, float **vals);
perflibs_status_t perflibs_spmat_export_dense_d(
    perflibs_const_spmat_t A, enum perflibs_dense_layout layout,
    perflibs_int_t *m, perflibs_int_t *n, double **vals);

/* ---- norm: include/perflibs_sparse.h:690-695 ---- */
perflibs_status_t perflibs_spnorm_exec_s(perflibs_spmat_t A,
                                         enum perflibs_sparse_norm nrm,
                                         float *result);
perflibs_status_t perflibs_spnorm_exec_d(perflibs_spmat_t A,
                                         enum perflibs_sparse_norm nrm,
                                         double *result);

/* ---- errors: include/perflibs_sparse.h:769 ---- */
void perflibs_spmat_print_err(perflibs_spmat_t A);

#ifdef __cplusplus
}
#endif

#endif /* PERFLIBS_SPARSE_H */
