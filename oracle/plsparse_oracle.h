/*
 * CPU oracle for the sparse x dense execute path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference library's algorithms on the path
 * (CSR / SELL-C-sigma SpMV, BSR SpMV, CSR SpMM, layout conversions, inf-norm).
 * It is used by tests/ as the parity checker, and by bench.py's CPU-baseline
 * leg when the reference library itself (oracle/_ref) is not available. The
 * shipped B200 library never links, loads or calls it.
 *
 * Parity pinning: this restatement is checked against (a) the reference
 * library compiled from its own sources (oracle/Makefile, target `ref`) on
 * the same inputs, and (b) the golden vectors held by the reference's own
 * tests (test/spmv_basic_d.c, test/bsr_kernel_paths.c,
 * test/matmul_variants_d.c, test/strategy_paths_d.c,
 * test/csr_spmv_omp_paths.c), committed as fixtures under tests/golden/.
 *
 * All matrices use 32-bit indices (the reference's default LP64 build,
 * include/perflibs_sparse.h:37-42). Index base 0 or 1 is taken from
 * row_ptr[0], as the reference does (src/compressed_sparse_rows.cpp:70-79).
 */
#ifndef PLSPARSE_ORACLE_H
#define PLSPARSE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = alpha*A*x + beta*y for CSR A (m rows).
 * mode 0: one accumulator per row, sum += x[col]*val, then
 *         y = y*beta + alpha*sum (beta != 0) or alpha*sum
 *         (src/compressed_sparse_rows.cpp:1114-1138, spmv_csr_vanilla).
 * mode 1: two interleaved accumulators (even / odd positions of the row),
 *         s0 += s1; s0 *= alpha; if beta != 0: s0 += beta*y
 *         (src/compressed_sparse_rows.cpp:1215-1321, the default serial
 *         kernel spmv_csr_notrans_no_parallel_strat). */
void orc_csr_spmv_d(int32_t m, const int32_t *row_ptr, const int32_t *col,
                    const double *vals, const double *x, double *y,
                    double alpha, double beta, int mode);
void orc_csr_spmv_s(int32_t m, const int32_t *row_ptr, const int32_t *col,
                    const float *vals, const float *x, float *y, float alpha,
                    float beta, int mode);

/* y = alpha*A^T*x + beta*y (src/compressed_sparse_rows.cpp:1558-1676):
 * y scaled by beta (or zeroed), then y[col] += alpha*val*x[row] row by row. */
void orc_csr_spmv_trans_d(int32_t m, int32_t n, const int32_t *row_ptr,
                          const int32_t *col, const double *vals,
                          const double *x, double *y, double alpha,
                          double beta);

/* Row-wise magnitude sum_j |a_ij * x_j| (the scale used by the per-row
 * relative-error check of summation-order differences). */
void orc_csr_absdot_d(int32_t m, const int32_t *row_ptr, const int32_t *col,
                      const double *vals, const double *x, double *out);

/* ---- SELL-C-sigma (src/sell_c_sigma.cpp) ---- */

/* Sizes of the layout csr2scs + gen_data_vectors produce for C, sigma (sigma
 * in rows: a multiple of C, or 0 for no sorting). out[0] = nC,
 * out[1] = padded data size cs[nC-1] + cl[nC-1]*C. */
void orc_scs_sizes(int32_t m, const int32_t *row_ptr, int32_t C,
                   int32_t sigma, int64_t *out);

/* Build the full layout, bit for bit what the reference builds
 * (src/sell_c_sigma.cpp:145-336 csr2scs, 584-705 gen_data_vectors):
 *   cs, cl, col_min: nC entries; permd2in, in2permd: nC*C entries (-1 for
 *   padding rows); vals: data size; offsets: data size entries holding the
 *   logical column offset (col - base - col_min[chunk], 0 for padding);
 *   info[0] = col_indx_bytes, info[1] = n_full_chunks, info[2] = ntidyup.
 * Returns 0. */
int orc_scs_build_d(int32_t m, int32_t n, const int32_t *row_ptr,
                    const int32_t *col, const double *vals, int32_t C,
                    int32_t sigma, int64_t *cs, int64_t *cl, int64_t *col_min,
                    int64_t *permd2in, int64_t *in2permd, double *out_vals,
                    int64_t *offsets, int64_t *info);

/* SELL SpMV over a layout built above (src/sell_c_sigma.cpp:719-797,
 * spmv_scs<T,C>): per permuted row, w += v*x[col_min + off] sequentially
 * over the padded chunk width; then y[perm] = alpha*w + beta*y[perm]
 * (beta != 0) or alpha*w. */
void orc_scs_spmv_d(int64_t nC, int32_t C, const int64_t *cs,
                    const int64_t *cl, const int64_t *col_min,
                    const int64_t *permd2in, const double *vals,
                    const int64_t *offsets, const double *x, double *y,
                    double alpha, double beta);

/* SELL beta = nnz / padded nnz actually processed
 * (src/sell_c_sigma.cpp:369-379). */
double orc_scs_beta(int64_t nC, int32_t C, const int64_t *cs,
                    const int64_t *cl, int32_t ntidyup, int64_t nnz);

/* ---- BSR (src/block_sparse_rows.cpp) ---- */

/* y = alpha*A*x + beta*y for BSR A with nrowsb block rows, block size bs,
 * blocks stored row-major (layout 91) or column-major (layout 90).
 * Per block row: y[rows] = beta*y (or 0), then y[row] += alpha*sum over the
 * block row (src/block_sparse_rows.cpp:458-515, 607-742). */
void orc_bsr_spmv_d(int32_t nrowsb, int32_t bs, int32_t layout,
                    const int32_t *row_ptr, const int32_t *col,
                    const double *vals, const double *x, double *y,
                    double alpha, double beta);

/* BSR -> CSR exactly as the reference's bsr2csr
 * (src/compressed_sparse_rows.cpp:966-1056): block rows in order, within a
 * block row scalar row i walks the blocks in stored order and each block's
 * row i left to right; exact zeros are dropped; the index base is kept.
 * Pass NULL outputs first to get out_nnz. Returns the CSR nnz. */
int64_t orc_bsr2csr_d(int32_t nrowsb, int32_t bs, int32_t layout,
                      const int32_t *row_ptr, const int32_t *col,
                      const double *vals, int32_t *out_row_ptr,
                      int32_t *out_col, double *out_vals);

/* CSR -> BSR with block size bs (the reference's csr2bsr only makes bs=1,
 * src/block_sparse_rows.cpp:350-370; this is the general restatement the
 * B200 converter must match bit for bit). m and n must be multiples of bs.
 * Block columns within a block row are ascending; each block is dense bs*bs
 * in `layout` with zeros where A has no entry; index base is kept.
 * Pass NULL outputs first to get the block count. Returns nnzb. */
int64_t orc_csr2bsr_d(int32_t m, int32_t n, int32_t bs, int32_t layout,
                      const int32_t *row_ptr, const int32_t *col,
                      const double *vals, int32_t *out_row_ptr,
                      int32_t *out_col, double *out_vals);

/* ---- SpMM (src/compressed_sparse_rows.cpp:1699-1764) ---- */

/* C = alpha*A*B + beta*C for CSR A (m x kdim), row-major B (ldb) and C (ldc),
 * k right-hand sides. C is assumed already zeroed by the caller when
 * beta == 0 (the reference zeroes it before the kernel,
 * src/matmul.cpp:596-605); per row, C_row *= beta when beta not in {0, 1};
 * then for each nonzero a = alpha*val, C_row += a * B_row(col). */
void orc_csr_spmm_d(int32_t m, const int32_t *row_ptr, const int32_t *col,
                    const double *vals, const double *B, int64_t ldb,
                    double *Cmat, int64_t ldc, int32_t k, double alpha,
                    double beta);
void orc_csr_spmm_s(int32_t m, const int32_t *row_ptr, const int32_t *col,
                    const float *vals, const float *B, int64_t ldb,
                    float *Cmat, int64_t ldc, int32_t k, float alpha,
                    float beta);

/* ---- Norm (src/inf_norm_csr.cpp:12-30) ---- */
/* max_i sum_j |a_ij|, NaN-propagating. */
double orc_csr_inf_norm_d(int32_t m, const int32_t *row_ptr,
                          const double *vals);

/* ---- COO / CSC input (src/compressed_sparse_rows.cpp) ---- */
/* coo2csr (:591-640), 0-based: entries by (row, column), all kept; equal
 * positions in input order (the reference's std::sort leaves them
 * unspecified). row_ptr has m+1 entries, col_out / vals_out nnz. */
void orc_coo2csr_d(int32_t m, int32_t n, int64_t nnz, const int32_t *row,
                   const int32_t *col, const double *vals, int32_t *row_ptr,
                   int32_t *col_out, double *vals_out);
/* csc2csr (:750-800): columns ascending in every row; keeps the base of
 * col_ptr[0]. */
void orc_csc2csr_d(int32_t m, int32_t n, const int32_t *row_indx,
                   const int32_t *col_ptr, const double *vals, int32_t *row_ptr,
                   int32_t *col_out, double *vals_out);

#ifdef __cplusplus
}
#endif

#endif
