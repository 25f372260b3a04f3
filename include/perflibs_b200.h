/*
 * perflibs_b200.h — extensions of libplsparse_b200 beyond the reference
 * interface. None of these has a counterpart in the reference library's
 * include/perflibs_sparse.h unless a comment says so; the drop-in entry
 * points are in perflibs_sparse.h.
 *
 * Device pointers: every *_dev entry point takes device (HBM) pointers and
 * a CUDA stream (a cudaStream_t passed as void*; NULL = the library's own
 * stream for the handle's device). Calls are asynchronous with respect to
 * the host; results are ready when the stream reaches them.
 */
#ifndef PERFLIBS_B200_H
#define PERFLIBS_B200_H

#include <stdint.h>

#include "perflibs_sparse.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- device-pointer execution ----------------------------------------
 * Same semantics as perflibs_spmv_exec_{s,d} (y = alpha*op(A)*x + beta*y),
 * on device arrays, without host copies or synchronisation. */
perflibs_status_t perflibs_b200_spmv_exec_d_dev(
    enum perflibs_sparse_hint_value trans, double alpha, perflibs_spmat_t A,
    const double *x, double beta, double *y, void *stream);
perflibs_status_t perflibs_b200_spmv_exec_s_dev(
    enum perflibs_sparse_hint_value trans, float alpha, perflibs_spmat_t A,
    const float *x, float beta, float *y, void *stream);

/* SpMV that allocates no device memory (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc around their SpMV: code whose
 * device memory is owned by a pool or caching allocator of its own, and
 * latency-critical loops where cudaMalloc / cudaFree (which can synchronise
 * the device) must not run. y = alpha*A*x + beta*y, NOTRANS, on device
 * pointers, asynchronous on `stream` (NULL = the handle's stream).
 *
 * A must already hold its SELL-C-sigma layout (perflibs_spmv_optimize chose
 * SELL, or perflibs_b200_spmat_build_sell / force_config + optimize); other
 * formats return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR. The partial sums of
 * sliced wide chunks and their completion counts go to fixed device arrays
 * (2^21 FP64 elements and 2^18 counts, 17 MiB) that every GPU loading the
 * library holds until exit; a matrix that needs more returns
 * PERFLIBS_STATUS_INPUT_PARAMETER_ERROR with the sizes in the handle's
 * error message. The first call on a device looks the arrays' addresses up
 * (cudaGetSymbolAddress), and so does the first call after the device's
 * context was re-created (cudaDeviceReset); make that first call before any
 * stream capture. All calls share the arrays: calls that overlap on the GPU
 * race, so serialise them (one stream, or events between streams). */
perflibs_status_t perflibs_b200_spmv_exec_d_noalloc(double alpha,
                                                    perflibs_spmat_t A,
                                                    const double *x,
                                                    double beta, double *y,
                                                    void *stream);

/* C = alpha*A*B + beta*C for a sparse A (NOTRANS), row-major dense device
 * B (ldb >= k) and C (ldc >= k) with k columns. beta == 0 overwrites C. */
perflibs_status_t perflibs_b200_spmm_exec_d_dev(double alpha,
                                                perflibs_spmat_t A,
                                                const double *B, int64_t ldb,
                                                int32_t k, double beta,
                                                double *C, int64_t ldc,
                                                void *stream);
perflibs_status_t perflibs_b200_spmm_exec_s_dev(float alpha, perflibs_spmat_t A,
                                                const float *B, int64_t ldb,
                                                int32_t k, float beta,
                                                float *C, int64_t ldc,
                                                void *stream);

/* ---- value storage (opt-in reduced precision) -------------------------
 * NATIVE keeps values in the handle's API type (FP64 for _d handles) and
 * accumulates in it. FP32 / BF16 store values in that type and accumulate
 * in FP32; x, y, B and C keep the API type. Takes effect at the next
 * optimize or exec. */
enum perflibs_b200_storage {
  PERFLIBS_B200_STORAGE_NATIVE = 0,
  PERFLIBS_B200_STORAGE_FP32 = 1,
  PERFLIBS_B200_STORAGE_BF16 = 2
};
perflibs_status_t perflibs_b200_spmat_set_storage(perflibs_spmat_t A,
                                                  int storage);

/* ---- tuning ------------------------------------------------------------
 * How perflibs_spmv_optimize picks the SpMV kernel when the SpMV
 * invocations hint is MANY (the reference's auditioning condition,
 * src/matvec.cpp:624-627):
 *   EXHAUSTIVE: time every candidate (CSR threads-per-row x SELL C x sigma)
 *               with CUDA events and keep the fastest;
 *   SELECTOR:   ask the learned selector attached with
 *               perflibs_b200_spmat_set_selector, and fall back to
 *               EXHAUSTIVE when none is attached;
 *   NONE:       keep the default CSR kernel. */
enum perflibs_b200_tuner {
  PERFLIBS_B200_TUNE_EXHAUSTIVE = 0,
  PERFLIBS_B200_TUNE_SELECTOR = 1,
  PERFLIBS_B200_TUNE_NONE = 2
};
perflibs_status_t perflibs_b200_spmat_set_tuner(perflibs_spmat_t A, int mode);

/* Kernel families. */
enum perflibs_b200_kind {
  PERFLIBS_B200_KIND_CSR = 0,  /* threads-per-row vector CSR */
  PERFLIBS_B200_KIND_SELL = 1, /* SELL-C-sigma, C in {8, 16, 32} */
  PERFLIBS_B200_KIND_CSR_SPLIT = 2 /* CSR with long rows split across CTAs */
};

/* Force a kernel configuration for the next optimize (the role of the
 * reference's internal set_C / set_sigma knobs, src/matrix_state.cpp:
 * 434-457). sigma is in rows: 0 (no sort) or a multiple of C. tpr 0 picks
 * by mean row length. */
perflibs_status_t perflibs_b200_spmat_force_config(perflibs_spmat_t A,
                                                   int kind, int C, int sigma,
                                                   int tpr);

/* The active configuration. */
perflibs_status_t perflibs_b200_spmat_get_config(perflibs_spmat_t A,
                                                 int *kind, int *C, int *sigma,
                                                 int *tpr, int *col_bytes);

/* Launch shape of the active NOTRANS SpMV: kernels launched per call, and
 * for SELL-C-sigma the number of work items and of chunks split into
 * column slices (0 when every chunk is one item). */
perflibs_status_t perflibs_b200_spmat_exec_info(perflibs_spmat_t A,
                                                int32_t *kernels_per_spmv,
                                                int64_t *n_items,
                                                int64_t *n_split);

/* SpMM kernels for a CSR A. The staged kernel copies, for every block of R
 * rows of A, the rows of B the block needs into shared memory (TMA bulk
 * copies) and multiplies from there; the row-group kernel reads B through
 * the caches, its lanes loading a row's entries one group at a time or (the
 * shared-entries variant) a row's lanes loading consecutive entries together
 * and passing them round. The first SpMM of each (k, ldb, value type) times
 * the candidates that apply (the staged kernel needs B rows reused inside
 * row blocks, B 16-byte aligned, ldb and k multiples of 16 bytes) on scratch
 * output and keeps the fastest. The diagonal-form kernel is a candidate
 * when A's entries lie on at most 32 diagonals (the longest row's
 * offsets covering every entry, at least half the diagonal slots filled),
 * its rows are sorted without duplicate columns, and B and C rows are
 * 16-byte vectors (any storage mode): each thread computes 4
 * consecutive rows and loads each row of B once per run of consecutive
 * diagonals. Where the diagonal form applies, a second diagonal-form
 * kernel is a candidate too, with B's rows staged in shared memory by
 * tensor-map (TMA) copies: for diagonals in groups whose centres are evenly
 * spaced (the planes of a 3-D stencil, the lines of a 2-D one) or in one
 * band, each CTA walks a chain of tiles and copies one new window of B per
 * tile; the staged (tiled) kernel is then not timed. set_spmm_path
 * overrides the choice: -1 measured choice (default), 0 row-group kernel,
 * 1 staged kernel whenever it applies, 2 row-group kernel with shared
 * entries whenever the lane shape allows (at least 4 lanes per row of C),
 * 3 diagonal-form kernel whenever it applies, 4 diagonal form with
 * TMA-staged B whenever it applies (else 3 when that applies). */
perflibs_status_t perflibs_b200_spmat_set_spmm_path(perflibs_spmat_t A, int32_t path);

/* Host-buffer SpMV (perflibs_spmv_exec_{s,d}) in row bands: the kernels of
 * band b write rows [r0_b, r1_b) of y, and those rows go back to the host on
 * a second stream while the later bands compute, so the kernels of all but
 * the first band hide under the device-to-host copy. Applies to NOTRANS
 * with CSR or SELL-C-sigma kernels; every row is summed exactly as in one
 * launch. n_bands = 0 (default) splits results of 8 MB and more into bands
 * of at least 4 MB, up to 8; 1 turns banding off; 2..64 asks for that many
 * (SELL bands are whole sort windows, so there may be fewer). */
perflibs_status_t perflibs_b200_spmat_set_host_bands(perflibs_spmat_t A, int32_t n_bands);

/* Bands the handle's last host-buffer SpMV ran in; 0 when it ran as one
 * launch. */
perflibs_status_t perflibs_b200_spmat_host_bands_used(perflibs_spmat_t A, int32_t *n_bands);

/* SpMM plan of the handle: the staged tiles' block height R (0 when none
 * were built: the staged kernel does not apply), the B rows staged per
 * column tile over all blocks and the copy runs; the path the last SpMM
 * took (1 staged, 0 row-group, 2 row-group with shared entries, 3
 * diagonal form, 4 diagonal form with TMA-staged B, -1 none yet); and the
 * two timings of the
 * measured choice in milliseconds (0 when not measured). Any output may be
 * NULL. */
perflibs_status_t perflibs_b200_spmat_spmm_info(perflibs_spmat_t A, int32_t *tile_rows,
                                                int64_t *staged_rows, int64_t *runs,
                                                int32_t *path, float *ms_staged, float *ms_rows);

/* How the handle's active SpMV configuration was chosen: 0 not chosen
 * (default heuristic), 1 timed by the exhaustive tuner, 2 taken from the
 * autotune cache, 3 predicted by the learned selector, 4 forced. */
perflibs_status_t perflibs_b200_spmat_tune_source(perflibs_spmat_t A, int32_t *source);

/* Autotune cache (checkpoint / resume of the exhaustive tuner). Every
 * exhaustive tune is recorded under a key of the GPU model (compute
 * capability and SM count), the matrix's dimensions and nonzero count, the
 * API and storage value types and a 64-bit hash of its sparsity structure
 * (values do not enter: they do not change a kernel's speed). A later
 * exhaustive optimize with the same key applies the recorded configuration
 * and timing table without timing anything (tune_source 2). save writes the
 * process's cache to a text file; load merges a file into it (a malformed
 * or truncated file changes nothing and is an input error); clear empties
 * it; size counts its entries. */
perflibs_status_t perflibs_b200_tune_cache_save(const char *path);
perflibs_status_t perflibs_b200_tune_cache_load(const char *path);
perflibs_status_t perflibs_b200_tune_cache_clear(void);
int64_t perflibs_b200_tune_cache_size(void);

/* Writes past the end of the library's device buffers seen so far in the
 * guard build (libplsparse_b200_guard.so: every buffer followed by a guard
 * of 0xFF bytes, checked when the buffer is freed); -1 in the regular
 * build, which has no guards. */
int64_t perflibs_b200_debug_guard_violations(void);

/* Timings the last exhaustive tune measured: up to `cap` rows of
 * (kind, C, sigma, tpr) in cfg4, milliseconds in ms and the SELL padding
 * efficiency nnz / padded size in beta (1 for CSR rows); any output may be
 * NULL. Returns the count in *count. */
perflibs_status_t perflibs_b200_spmat_tune_table(perflibs_spmat_t A,
                                                 int32_t cap, int32_t *cfg4,
                                                 double *ms, double *beta,
                                                 int32_t *count);

/* The SELL-C-sigma layout held on the device (after optimize picked SELL or
 * after perflibs_b200_spmat_build_sell): info7 = {nC, C, sigma, col_bytes,
 * n_full_chunks, ntidyup, size}; any array pointer may be NULL. Offsets are
 * written with col_bytes bytes each, values in the storage type. */
perflibs_status_t perflibs_b200_spmat_export_sell(
    perflibs_spmat_t A, int64_t *info7, int64_t *cs, int64_t *cl,
    int64_t *col_min, int64_t *permd2in, int64_t *in2permd, void *vals,
    void *offsets);

/* Build (or rebuild) the SELL-C-sigma layout with C and sigma and make it
 * the active SpMV format, without timing anything. */
perflibs_status_t perflibs_b200_spmat_build_sell(perflibs_spmat_t A, int C,
                                                 int sigma);

/* Per-handle CUDA stream for the host-pointer entry points (NULL restores
 * the library stream). */
perflibs_status_t perflibs_b200_spmat_set_stream(perflibs_spmat_t A,
                                                 void *stream);

/* CSR -> BSR on the device for a CSR handle: returns a new BSR handle with
 * block size bs and the given block layout (blocks sorted by block column,
 * zero-filled). m and n must be multiples of bs. */
perflibs_status_t perflibs_b200_spmat_csr_to_bsr(perflibs_spmat_t A,
                                                 int32_t bs, int layout,
                                                 perflibs_spmat_t *out);

/* BSR structure back to host arrays (malloc'ed; the caller frees). */
perflibs_status_t perflibs_b200_spmat_export_bsr_d(
    perflibs_spmat_t A, int32_t *bs, int32_t *nnzb, int32_t **row_ptr,
    int32_t **col_indx, double **vals);

/* ---- creation from device arrays ---------------------------------------
 * A CSR handle whose arrays already live in HBM (0- or 1-based, as
 * row_ptr[0] says; the arrays are copied, the caller keeps ownership).
 * `stream` is the stream the arrays were written on; the copies are ordered
 * after it. With NULL the call first waits for all prior work on the device
 * (the arrays may come from any stream, and the library's own stream does
 * not wait for the legacy default stream). */
perflibs_status_t perflibs_b200_spmat_create_csr_d_dev(
    perflibs_spmat_t *A, int32_t m, int32_t n, const int32_t *row_ptr,
    const int32_t *col_indx, const double *vals, void *stream);

/* ---- structure statistics -----------------------------------------------
 * PERFLIBS_B200_NFEATURES statistics of a CSR handle, computed on the
 * device, in this order:
 *   0 log2(m+1)        1 log2(n+1)        2 log2(nnz+1)
 *   3 mean row length  4 row length std   5 skew    6 excess kurtosis
 *   7 log2(1+min len)  8 log2(1+max len)  9 empty-row fraction
 *  10 log2(1+p50 len) 11 log2(1+p90 len) 12 log2(1+p99 len)
 *  13 log2(max/mean)  14 mean |i-j|/n      15 max |i-j|/n (bandwidth)
 *  16 fraction of nonzeros with |i-j| <= 32
 *  17 block fill at bs 2   18 at bs 4   19 at bs 8   (nnz / (bs^2 * blocks))
 *  20 SELL beta C=8 sigma=0   21 C=32 sigma=0   22 C=32 sigma=1024
 *  23 log2(1+mgmd), mgmd the reference's mean geometric distance between
 *     consecutive nonzeros of a row (src/matrix_statistics.cpp:23-93). */
#define PERFLIBS_B200_NFEATURES 24
perflibs_status_t perflibs_b200_spmat_features(perflibs_spmat_t A,
                                               float *features);

/* ---- learned format / parameter selector ---------------------------------
 * An MLP NFEATURES -> 64 -> 64 -> n_classes (ReLU, softmax), FP32, trained
 * and run by the library's own CUDA kernels. Class c is candidate c of the
 * exhaustive tuner (perflibs_b200_tune_candidates). */
typedef struct perflibs_b200_selector_s *perflibs_b200_selector_t;

/* The tuner's candidate list: cfg4 rows of (kind, C, sigma, tpr). */
perflibs_status_t perflibs_b200_tune_candidates(int32_t cap, int32_t *cfg4,
                                                int32_t *count);

perflibs_status_t perflibs_b200_selector_create(perflibs_b200_selector_t *S,
                                                int32_t n_classes,
                                                uint64_t seed);
perflibs_status_t perflibs_b200_selector_destroy(perflibs_b200_selector_t S);
/* Parameter vector (W1, b1, W2, b2, W3, b3, then the 2*NFEATURES feature
 * normalisation mean / inverse std): count, read, write. */
int64_t perflibs_b200_selector_param_count(perflibs_b200_selector_t S);
perflibs_status_t perflibs_b200_selector_get_params(perflibs_b200_selector_t S,
                                                    float *params);
perflibs_status_t perflibs_b200_selector_set_params(perflibs_b200_selector_t S,
                                                    const float *params);
/* Mean soft-target cross-entropy over n samples (host arrays X[n][NF],
 * T[n][n_classes]) and its gradient w.r.t. the trainable parameters
 * (grad has the trainable-parameter count = param_count - 2*NFEATURES). */
perflibs_status_t perflibs_b200_selector_loss_grad(perflibs_b200_selector_t S,
                                                   const float *X,
                                                   const float *T, int32_t n,
                                                   float *loss, float *grad);
/* Adam training on the device: the feature normalisation is fitted to X
 * first; one epoch = all samples in shuffled mini-batches; each step is a
 * CUDA graph replay. */
perflibs_status_t perflibs_b200_selector_train(perflibs_b200_selector_t S,
                                               const float *X, const float *T,
                                               int32_t n, int32_t epochs,
                                               int32_t batch, float lr,
                                               uint64_t seed,
                                               float *final_loss);
/* Class probabilities (n x n_classes) and argmax classes. */
perflibs_status_t perflibs_b200_selector_predict(perflibs_b200_selector_t S,
                                                 const float *X, int32_t n,
                                                 float *probs, int32_t *cls);
/* Use S when the handle's tuner is PERFLIBS_B200_TUNE_SELECTOR. The selector
 * must outlive the handle's optimize calls. */
perflibs_status_t perflibs_b200_spmat_set_selector(perflibs_spmat_t A,
                                                   perflibs_b200_selector_t S);
/* SpMM kernel selectors (5 classes each: 0 row-group kernel, 1 row group
 * with shared entries, 2 staged, 3 diagonal form, 4 diagonal form with
 * TMA-staged B) for k <= 16, 17..64 and > 64; S may be NULL and entries may
 * be NULL (those k keep the measured choice). With one attached, the first
 * CSR SpMM of a call signature runs the most probable kernel that applies,
 * without timing the candidates. The selectors must outlive the handle's
 * SpMM calls. */
perflibs_status_t perflibs_b200_spmat_set_spmm_selectors(perflibs_spmat_t A,
                                                         const perflibs_b200_selector_t *S);

/* ---- batched uneven SpMM ---------------------------------------------------
 * Many independent products C_i = alpha*A_i*B_i + beta*C_i (FP32 CSR or BSR
 * handles A_i, each with its own row-major device B_i (ldb_i) and C_i
 * (ldc_i) and its own k_i) in ONE persistent kernel launch: a work list of
 * (instance, row tile) items is consumed by a grid sized to the SMs through
 * an atomic counter, so uneven instances balance without waits. exec
 * replays a CUDA graph holding the counter reset and the launch. The batch
 * keeps its own copy of every instance's entries, column index and value
 * side by side (one 8-byte load per entry; BSR instances expanded to scalar
 * rows, blocks in stored order), made at creation: values changed in the
 * handles afterwards (perflibs_spmat_update) are not seen until the batch is
 * created again. The copy takes 8 bytes of device memory per stored scalar
 * entry. */
typedef struct perflibs_b200_batch_s *perflibs_b200_batch_t;
perflibs_status_t perflibs_b200_batch_create(
    perflibs_b200_batch_t *Bt, int32_t count, const perflibs_spmat_t *mats,
    const int32_t *k, const float *const *B, const int64_t *ldb,
    float *const *C, const int64_t *ldc, void *stream);
/* Rows per work item (0 = the autotuned value). */
perflibs_status_t perflibs_b200_batch_set_tile(perflibs_b200_batch_t Bt,
                                               int32_t rows_per_item);
/* Time each candidate tile (rows per item) and keep the fastest;
 * best_tile / best_ms may be NULL. */
perflibs_status_t perflibs_b200_batch_tune(perflibs_b200_batch_t Bt,
                                           int32_t *best_tile,
                                           float *best_ms);
perflibs_status_t perflibs_b200_batch_exec(perflibs_b200_batch_t Bt,
                                           float alpha, float beta);
/* Per-warp work items (the staged items are counted by
 * perflibs_b200_batch_stage_info), kernel launches of one exec, and the
 * rows per item. */
perflibs_status_t perflibs_b200_batch_info(perflibs_b200_batch_t Bt,
                                           int64_t *n_items,
                                           int32_t *launches_per_exec,
                                           int32_t *tile);
/* Staged items: blocks of rows whose entries read a narrow window of B's
 * rows (banded, block-diagonal) are computed by whole CTAs from a copy of
 * that window in shared memory, at most 32 columns of C per item. Which
 * blocks qualify is fixed at creation; the tuner times the batch with and
 * without them and keeps the faster. set_staging(0) sends every row to the
 * per-warp items, set_staging(1) brings the staged items back.
 * staged_items counts the staged items built at creation; on reports
 * whether they run. */
perflibs_status_t perflibs_b200_batch_set_staging(perflibs_b200_batch_t Bt,
                                                  int32_t on);
perflibs_status_t perflibs_b200_batch_stage_info(perflibs_b200_batch_t Bt,
                                                 int64_t *staged_items,
                                                 int32_t *on);
perflibs_status_t perflibs_b200_batch_destroy(perflibs_b200_batch_t Bt);

/* Library / device information: SM count, L2 bytes, device ordinal. */
perflibs_status_t perflibs_b200_device_info(int32_t *sm_count,
                                            int64_t *l2_bytes,
                                            int32_t *device);

/* Version string of the library build. */
const char *perflibs_b200_version(void);

/* ---- Matrix Market input (host only) ----------------------------------
 * Reads a coordinate .mtx file (fields real / integer / pattern; symmetry
 * general / symmetric / skew-symmetric / hermitian, the mirrored entries
 * added as the reference's benchmark driver does,
 * bench/pl_bench_sparse_x_dense.c:124-240) into a 0-based CSR ordered by
 * (row, column), every entry kept. The arrays are malloc'ed; the caller
 * frees them. INPUT_PARAMETER_ERROR for an unreadable or unsupported file. */
perflibs_status_t perflibs_b200_read_mtx(const char *path, int32_t *m, int32_t *n,
                                         int64_t *nnz, int32_t **row_ptr,
                                         int32_t **col_indx, double **vals);

/* ---- failure-path testing ---------------------------------------------
 * For tests of the failure path only. The staged SpMM kernel waits on a
 * shared-memory barrier for its bulk copies with a poll limit; on expiry it
 * flags the failure (reported as EXECUTION_FAILURE by the handle's next
 * SpMM) and stops without touching C. This makes every later staged launch
 * post `shortfall_bytes` (0-4096) more than it copies, so the wait runs out
 * after `wait_polls` polls with no copy in flight. (0, 0) restores the
 * defaults: no shortfall, about a second of polling. */
perflibs_status_t perflibs_b200_testing_stage_fault(int32_t shortfall_bytes, int32_t wait_polls);

/* The handle's error record (what perflibs_spmat_print_err prints): the
 * status of the last failed call (0 when none), the 1-based argument
 * position for input errors, and the message (NUL-terminated, truncated to
 * msg_len - 1 characters). Any pointer may be NULL. */
perflibs_status_t perflibs_b200_spmat_get_error(perflibs_const_spmat_t A, int32_t *type,
                                                int32_t *code, char *msg, int32_t msg_len);

#ifdef __cplusplus
}
#endif

#endif /* PERFLIBS_B200_H */
