// The C interface of libplsparse_b200: handle creation and validation,
// hints, optimize, execute, export, norms and the B200 extensions.
//
// Argument checks, error codes (1-based argument positions) and the
// special-case order follow the reference entry points each function cites,
// so callers see the same statuses. No C++ exception crosses this
// boundary: every entry point converts failures to a status and records the
// message on the handle (printed by perflibs_spmat_print_err).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

std::mutex g_stream_mu;
cudaStream_t g_streams[64] = {};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev)
      cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev)
      cudaSetDevice(prev);
  }
};

__global__ void k_sub_base(int64_t n, int32_t base, int32_t *a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    a[i] -= base;
}

template <class X>
__global__ void k_densify_csr(int32_t m, const int32_t *rp, const int32_t *col,
                              const X *val, X *out, int64_t rs, int64_t cs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  for (int32_t j = rp[i]; j < rp[i + 1]; ++j)
    out[i * rs + (int64_t)col[j] * cs] += val[j];
}

template <class T> constexpr Dt dt_of() {
  return std::is_same_v<T, double> ? Dt::F64 : Dt::F32;
}

Vt native_vt(Dt dt) { return dt == Dt::F64 ? Vt::F64 : Vt::F32; }

int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess)
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "no CUDA device available");
  return d;
}

void set_err(Mat *A, int type, int code, const std::string &msg) {
  if (!A)
    return;
  A->err_type = type;
  A->err_code = code;
  A->err_msg = msg;
}

perflibs_status_t param_error(Mat *A, int code, const std::string &msg = "") {
  set_err(A, PERFLIBS_STATUS_INPUT_PARAMETER_ERROR, code, msg);
  return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
}

template <class F> perflibs_status_t guarded(Mat *A, F &&f) {
  try {
    return f();
  } catch (const Error &e) {
    set_err(A, e.status, 0, e.what());
    return e.status;
  } catch (const std::bad_alloc &) {
    set_err(A, PERFLIBS_STATUS_EXECUTION_FAILURE, 0, "host allocation failed");
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  } catch (const std::exception &e) {
    set_err(A, PERFLIBS_STATUS_EXECUTION_FAILURE, 0, e.what());
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  } catch (...) {
    set_err(A, PERFLIBS_STATUS_EXECUTION_FAILURE, 0, "unknown failure");
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
}

void upload(DevBuf &b, const void *h, size_t bytes, cudaStream_t s) {
  b.reserve(std::max<size_t>(bytes, 16));
  if (bytes)
    PLS_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, s));
}

void upload_index(DevBuf &b, const int32_t *h, int64_t n, int32_t base,
                  cudaStream_t s) {
  upload(b, h, sizeof(int32_t) * n, s);
  if (base != 0 && n > 0) {
    k_sub_base<<<(unsigned)div_up(n, 256), 256, 0, s>>>(n, base, b.as<int32_t>());
    PLS_LAUNCH_CHECK();
  }
}

bool valid_op(int op) {
  return op == PERFLIBS_SPARSE_OPERATION_NOTRANS || op == PERFLIBS_SPARSE_OPERATION_TRANS ||
         op == PERFLIBS_SPARSE_OPERATION_CONJTRANS;
}

bool is_sparse(Fmt f) { return f == Fmt::CSR || f == Fmt::BSR || f == Fmt::SELL; }

Vt target_vt(const Mat *A) {
  switch (A->storage) {
  case PERFLIBS_B200_STORAGE_FP32: return Vt::F32;
  case PERFLIBS_B200_STORAGE_BF16: return Vt::BF16;
  default: return native_vt(A->dt);
  }
}

// Bring the kernels' value copy in line with the requested storage mode.
void prepare_values(Mat *A) {
  const Vt t = target_vt(A);
  cudaStream_t s = stream_of(A);
  if (A->fmt == Fmt::CSR || A->fmt == Fmt::SELL) {
    CsrDev &c = A->csr;
    if (t == c.vt) {
      if (c.lo) {
        c.lo = false;
        c.vals_lo.release();
      }
    } else if (!c.lo || c.vt_lo != t) {
      c.vals_lo.reserve(vt_size(t) * std::max<int64_t>(c.nnz, 1));
      convert_values(c.vals.p, c.vt, c.vals_lo.p, t, c.nnz, s);
      c.vt_lo = t;
      c.lo = true;
    }
    if (A->fmt == Fmt::SELL && A->sell.vt != c.evt())
      apply_config(A, A->cfg);
  } else if (A->fmt == Fmt::BSR) {
    BsrDev &b = A->bsr;
    const int64_t nv = b.nnzb * (int64_t)b.bs * b.bs;
    if (t == b.vt) {
      if (b.lo) {
        b.lo = false;
        b.vals_lo.release();
      }
    } else if (!b.lo || b.vt_lo != t) {
      b.vals_lo.reserve(vt_size(t) * std::max<int64_t>(nv, 1));
      convert_values(b.vals.p, b.vt, b.vals_lo.p, t, nv, s);
      b.vt_lo = t;
      b.lo = true;
      ++b.vals_version;
    }
  }
}

// The reference converts a BSR handle to CSR (dropping exact zeros) for any
// operation its BSR kernels do not cover (src/convert.cpp:139-140,
// src/compressed_sparse_rows.cpp:966-1056).
void bsr_become_csr(Mat *A) {
  if (A->fmt != Fmt::BSR)
    return;
  cudaStream_t s = stream_of(A);
  CsrDev c;
  bsr_to_csr(A->bsr, A->m, true, c, s);
  A->csr = std::move(c);
  A->csr.vt = A->bsr.vt;
  A->nnz = A->csr.nnz;
  A->bsr = BsrDev{};
  A->fmt = Fmt::CSR;
  A->cfg = default_config(A);
  prepare_values(A);
}

Mat *new_mat(Dt dt, Fmt f) {
  auto *A = new Mat;
  A->dt = dt;
  A->fmt = f;
  A->created = f;
  A->device = current_device();
  return A;
}

// ------------------------------------------------------------- creation

template <class T>
perflibs_status_t create_csr(Mat **out, int32_t m, int32_t n, const int32_t *row_ptr,
                             const int32_t *col, const T *vals, int32_t flags) {
  (void)flags;  // the device copy is always private, so NOCOPY changes nothing
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(dt_of<T>(), Fmt::CSR);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/compressed_sparse_rows.cpp:44-68 (check_csr_params)
    if (m < 0)
      return param_error(A, 2);
    if (n < 0)
      return param_error(A, 3);
    if (!row_ptr || (row_ptr[0] != 0 && row_ptr[0] != 1))
      return param_error(A, 4);
    A->m = m;
    A->n = n;
    A->index_base = row_ptr[0];
    A->nnz = (int64_t)row_ptr[m] - A->index_base;
    if (A->nnz < 0)
      return param_error(A, 4, "row_ptr[m] is below row_ptr[0]");
    if (A->nnz > 0 && (!col || !vals))
      return param_error(A, !col ? 5 : 6);
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    CsrDev &c = A->csr;
    c.nnz = A->nnz;
    c.ncols = n;
    c.vt = native_vt(A->dt);
    upload_index(c.row_ptr, row_ptr, (int64_t)m + 1, A->index_base, s);
    upload_index(c.col, col, A->nnz, A->index_base, s);
    upload(c.vals, vals, sizeof(T) * A->nnz, s);
    // Indices are checked before any kernel uses them (the reference reads
    // them as they are).
    const auto bad = check_compressed(m, n, A->nnz, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), s);
    if (bad.first >= 0)
      return param_error(A, 4, "row_ptr decreases or leaves [0, nnz] at row " + std::to_string(bad.first));
    if (bad.second >= 0)
      return param_error(A, 5, "col_indx[" + std::to_string(bad.second) + "] is outside [0, n)");
    A->cfg = default_config(A);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

// COO input (0-based, the C interface's base: src/matrix_api.cpp:95-101),
// converted to CSR on the device at creation; the handle is a CSR handle
// from then on, as the reference's handle becomes one when it is converted
// (src/convert.cpp:112-116).
template <class T>
perflibs_status_t create_coo(Mat **out, int32_t m, int32_t n, int32_t nnz, const int32_t *row,
                             const int32_t *col, const T *vals, int32_t flags) {
  (void)flags;
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(dt_of<T>(), Fmt::CSR);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/coordinate_list.cpp:140-151 checks m and n; a negative nnz and
    // indices out of range are rejected here too (the reference reads them
    // as they are).
    if (m < 0)
      return param_error(A, 2);
    if (n < 0)
      return param_error(A, 3);
    if (nnz < 0)
      return param_error(A, 4);
    if (nnz > 0 && (!row || !col || !vals))
      return param_error(A, !row ? 5 : !col ? 6 : 7);
    A->m = m;
    A->n = n;
    A->index_base = 0;
    A->nnz = nnz;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    DevBuf drow, dcol, dval;
    upload(drow, row, sizeof(int32_t) * (size_t)nnz, s);
    upload(dcol, col, sizeof(int32_t) * (size_t)nnz, s);
    upload(dval, vals, sizeof(T) * (size_t)nnz, s);
    const int64_t bad = coo_to_csr(m, n, nnz, drow.as<int32_t>(), dcol.as<int32_t>(), dval.p,
                                   native_vt(A->dt), A->csr, s);
    if (bad >= 0)
      return param_error(A, row[bad] < 0 || row[bad] >= m ? 5 : 6,
                         "entry " + std::to_string(bad) + " is outside the matrix");
    A->csr.ncols = n;
    A->cfg = default_config(A);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

// CSC input: the CSC arrays are the CSR of A^T, transposed on the device
// into the CSR of A (columns ascending in each row, the order of the
// reference's csc2csr: src/compressed_sparse_rows.cpp:750-800).
template <class T>
perflibs_status_t create_csc(Mat **out, int32_t m, int32_t n, const int32_t *row_indx,
                             const int32_t *col_ptr, const T *vals, int32_t flags) {
  (void)flags;
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(dt_of<T>(), Fmt::CSR);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/compressed_sparse_columns.cpp:162-178
    if (m < 0)
      return param_error(A, 2);
    if (n < 0)
      return param_error(A, 3);
    if (!col_ptr || (col_ptr[0] != 0 && col_ptr[0] != 1))
      return param_error(A, 4);
    A->m = m;
    A->n = n;
    A->index_base = col_ptr[0];
    A->nnz = (int64_t)col_ptr[n] - A->index_base;
    if (A->nnz < 0)
      return param_error(A, 5, "col_ptr[n] is below col_ptr[0]");
    if (A->nnz > 0 && (!row_indx || !vals))
      return param_error(A, !row_indx ? 4 : 6);
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    CsrDev t;  // CSR of A^T: n rows, m columns
    t.nnz = A->nnz;
    t.vt = native_vt(A->dt);
    upload_index(t.row_ptr, col_ptr, (int64_t)n + 1, A->index_base, s);
    upload_index(t.col, row_indx, A->nnz, A->index_base, s);
    upload(t.vals, vals, sizeof(T) * A->nnz, s);
    const auto bad = check_compressed(n, m, A->nnz, t.row_ptr.as<int32_t>(), t.col.as<int32_t>(), s);
    if (bad.first >= 0)
      return param_error(A, 5, "col_ptr decreases or leaves [0, nnz] at column " + std::to_string(bad.first));
    if (bad.second >= 0)
      return param_error(A, 4, "row_indx[" + std::to_string(bad.second) + "] is outside [0, m)");
    build_csr_transpose(t, n, m, A->csr, s);
    A->csr.ncols = n;
    PLS_CUDA(cudaStreamSynchronize(s));
    A->cfg = default_config(A);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

template <class T>
perflibs_status_t create_bsr(Mat **out, int layout, int32_t m, int32_t n, int32_t bs,
                             const int32_t *row_ptr, const int32_t *col, const T *vals,
                             int32_t flags) {
  (void)flags;
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(dt_of<T>(), Fmt::BSR);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/block_sparse_rows.cpp:205-240 (fill_initial_data_bsr)
    if (layout != PERFLIBS_COL_MAJOR && layout != PERFLIBS_ROW_MAJOR)
      return param_error(A, 2);
    if (m < 0)
      return param_error(A, 3);
    if (n < 0)
      return param_error(A, 4);
    if (bs <= 0 || m % bs != 0 || n % bs != 0)
      return param_error(A, 5);
    if (!row_ptr || (row_ptr[0] != 0 && row_ptr[0] != 1))
      return param_error(A, 6);
    A->m = m;
    A->n = n;
    A->index_base = row_ptr[0];
    BsrDev &b = A->bsr;
    b.bs = bs;
    b.layout = layout;
    b.mb = m / bs;
    b.nb = n / bs;
    b.nnzb = (int64_t)row_ptr[b.mb] - A->index_base;
    b.vt = native_vt(A->dt);
    A->nnz = b.nnzb * (int64_t)bs * bs;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    upload_index(b.row_ptr, row_ptr, (int64_t)b.mb + 1, A->index_base, s);
    upload_index(b.col, col, b.nnzb, A->index_base, s);
    upload(b.vals, vals, sizeof(T) * A->nnz, s);
    const auto bad = check_compressed(b.mb, b.nb, b.nnzb, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(), s);
    if (bad.first >= 0)
      return param_error(A, 6, "row_ptr decreases or leaves [0, nnzb] at block row " + std::to_string(bad.first));
    if (bad.second >= 0)
      return param_error(A, 7, "col_indx[" + std::to_string(bad.second) + "] is outside [0, n / bs)");
    return PERFLIBS_STATUS_SUCCESS;
  });
}

template <class T>
perflibs_status_t create_dense(Mat **out, int layout, int32_t m, int32_t n, int32_t lda,
                               const T *vals, int32_t flags) {
  (void)flags;
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(dt_of<T>(), Fmt::DENSE);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/dense.cpp:119-146 (fill_initial_data_dense)
    if (layout != PERFLIBS_COL_MAJOR && layout != PERFLIBS_ROW_MAJOR)
      return param_error(A, 2);
    if (m < 0)
      return param_error(A, 3);
    if (n < 0)
      return param_error(A, 4);
    if ((layout == PERFLIBS_COL_MAJOR && lda < m) || (layout == PERFLIBS_ROW_MAJOR && lda < n))
      return param_error(A, 5);
    A->m = m;
    A->n = n;
    A->nnz = (int64_t)m * n;
    DenseDev &d = A->dense;
    d.layout = layout;
    // The copy is packed (src/dense.hpp:38-56).
    const int64_t outer = layout == PERFLIBS_ROW_MAJOR ? m : n;
    const int64_t inner = layout == PERFLIBS_ROW_MAJOR ? n : m;
    d.lda = std::max<int64_t>(inner, 1);
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    d.vals.reserve(std::max<size_t>(sizeof(T) * outer * inner, 16));
    if (outer * inner > 0)
      PLS_CUDA(cudaMemcpy2DAsync(d.vals.p, sizeof(T) * inner, vals, sizeof(T) * lda,
                                 sizeof(T) * inner, outer, cudaMemcpyHostToDevice, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    return PERFLIBS_STATUS_SUCCESS;
  });
}

// ------------------------------------------------------------------ SpMV

template <class X>
perflibs_status_t spmv_device(int op, X alpha, Mat *A, const X *x, X beta, X *y,
                              cudaStream_t s) {
  const int64_t ylen = op == PERFLIBS_SPARSE_OPERATION_NOTRANS ? A->m : A->n;
  const int64_t xlen = op == PERFLIBS_SPARSE_OPERATION_NOTRANS ? A->n : A->m;
  // src/matvec.cpp:66-88: y = 0 when beta == 0; alpha == 0 or an empty x
  // leaves beta*y.
  if (ylen == 0)
    return PERFLIBS_STATUS_SUCCESS;
  if (xlen == 0 || alpha == X(0)) {
    scal<X>(ylen, beta, y, s);
    return PERFLIBS_STATUS_SUCCESS;
  }
  switch (A->fmt) {
  case Fmt::IDENTITY: {
    // src/special.cpp:17-47: y = alpha*x + beta*y on the diagonal part.
    const int64_t dl = std::min(A->m, A->n);
    axpby<X>(dl, alpha, x, beta, y, s);
    if (ylen > dl)
      scal<X>(ylen - dl, X(0), y + dl, s);
    return PERFLIBS_STATUS_SUCCESS;
  }
  case Fmt::NUL:
    scal<X>(ylen, beta, y, s);  // src/special.cpp:68-79
    return PERFLIBS_STATUS_SUCCESS;
  case Fmt::DENSE:
    spmv_dense<X>(A->dense, A->m, A->n, op != PERFLIBS_SPARSE_OPERATION_NOTRANS, x, y, alpha,
                  beta, s);
    return PERFLIBS_STATUS_SUCCESS;
  default:
    break;
  }
  if (A->fmt == Fmt::BSR && op != PERFLIBS_SPARSE_OPERATION_NOTRANS)
    bsr_become_csr(A);
  run_spmv<X>(A, op, x, y, alpha, beta, s);
  return PERFLIBS_STATUS_SUCCESS;
}

// The reference falls back to CSR when the operation differs from the one
// the handle was optimized for, and records the new operation
// (src/matvec.cpp:110-132).
void align_operation(Mat *A, int op) {
  if (op != A->hint_spmv_op) {
    if (A->fmt == Fmt::SELL) {
      A->fmt = Fmt::CSR;
      A->sell = SellDev{};
    }
    if (A->fmt == Fmt::CSR)
      A->cfg = default_config(A);
    A->hint_spmv_op = op;
    A->tuned = false;
  }
}

template <class X> bool matches(const Mat *A) {
  return A->fmt == Fmt::NUL || A->fmt == Fmt::IDENTITY || A->dt == dt_of<X>();
}

// Host-buffer SpMV in row bands: each band's rows of y go back to the host
// on a second stream while the next bands compute, so only the first band's
// kernels and the copies stay on the critical path. Results of at least
// 2 * kBandBytes are split, into bands of at least kBandBytes of y, at most
// kMaxBands of them. On a 33.5 MB FP64 result (4.2 M rows, SELL-C-sigma) a
// call took 1.56 ms as one launch, 1.35 ms in 4 bands, 1.32 ms in 8 and
// 1.53 ms in 16: smaller bands add more launch and copy overhead than they
// hide.
constexpr int64_t kBandBytes = 4 << 20;
constexpr int kMaxBands = 8;
constexpr int kMaxHostBands = 64;  // bound of an explicit band count

template <class X>
int band_count(const Mat *A, int trans, X alpha, int64_t xlen, int64_t ylen) {
  if (trans != PERFLIBS_SPARSE_OPERATION_NOTRANS || alpha == X(0) || xlen == 0)
    return 1;
  if (A->fmt != Fmt::SELL && A->fmt != Fmt::CSR)
    return 1;
  if (A->host_bands > 0)
    return A->host_bands;
  return (int)std::max<int64_t>(1, std::min<int64_t>(kMaxBands, ylen * (int64_t)sizeof(X) / kBandBytes));
}

// The bands' kernels run in band order on the handle's stream; a band's
// event releases the copy of its rows on the copy stream. All kernels are
// queued before the first copy: with pageable host memory a copy may block
// the host, and the kernels are already queued then. (Bands on several
// streams at once measured slower: the first band then shares the GPU with
// the others and its copy starts later.)
template <class X>
bool spmv_banded(Mat *A, int n_bands, X alpha, X beta, X *y_host, cudaStream_t s) {
  const std::vector<RowBand> *bands;
  if (A->fmt == Fmt::SELL) {
    sell_plan_bands(A->sell, A->m, n_bands);
    bands = &A->sell.bands.bands;
  } else {
    csr_plan_bands(A->csr, A->m, n_bands);
    bands = &A->csr.bands.bands;
  }
  const size_t nb = bands->size();
  if (nb < 2)
    return false;
  BandLanes &L = A->lanes;
  const X *xd = A->xbuf.as<X>();
  X *yd = A->ybuf.as<X>();
  const int tpr = A->cfg.kind == Kind::CSR_SPLIT ? 0
                  : A->cfg.tpr > 0              ? A->cfg.tpr
                                                : default_config(A).tpr;
  for (size_t i = 0; i < nb; ++i) {
    const RowBand &b = (*bands)[i];
    if (A->fmt == Fmt::SELL)
      spmv_sell_band<X>(A->sell, b, xd, yd, alpha, beta, s);
    else
      spmv_csr_band<X>(A->csr, b, tpr, xd, yd, alpha, beta, s);
    PLS_CUDA(cudaEventRecord(L.event(i), s));
  }
  cudaStream_t c = L.copy_stream();
  for (size_t i = 0; i < nb; ++i) {
    const RowBand &b = (*bands)[i];
    PLS_CUDA(cudaStreamWaitEvent(c, L.event(i), 0));
    PLS_CUDA(cudaMemcpyAsync(y_host + b.r0, yd + b.r0, sizeof(X) * (size_t)(b.r1 - b.r0),
                             cudaMemcpyDeviceToHost, c));
  }
  // The copy stream waited for the last band, so once it is idle so is `s`.
  PLS_CUDA(cudaStreamSynchronize(c));
  A->last_host_bands = (int)nb;
  return true;
}

template <class X>
perflibs_status_t spmv_exec_host(int trans, X alpha, Mat *A, const X *x, X beta, X *y) {
  TraceRange trace("perflibs_spmv_exec");
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (!valid_op(trans))
      return param_error(A, 1, "Incorrect transpose option.");
    if (!matches<X>(A))
      return param_error(A, 3, "The matrix handle has a different data type.");
    DeviceGuard g(A->device);
    align_operation(A, trans);
    prepare_values(A);
    A->last_host_bands = 0;
    cudaStream_t s = stream_of(A);
    const int64_t ylen = trans == PERFLIBS_SPARSE_OPERATION_NOTRANS ? A->m : A->n;
    const int64_t xlen = trans == PERFLIBS_SPARSE_OPERATION_NOTRANS ? A->n : A->m;
    if (ylen == 0)
      return PERFLIBS_STATUS_SUCCESS;
    A->xbuf.reserve(sizeof(X) * std::max<int64_t>(xlen, 1));
    A->ybuf.reserve(sizeof(X) * ylen);
    if (xlen > 0)
      PLS_CUDA(cudaMemcpyAsync(A->xbuf.p, x, sizeof(X) * xlen, cudaMemcpyHostToDevice, s));
    // With beta = 0 every kernel writes all of y without reading it (the
    // reference's y = alpha*A*x: old values, NaN included, do not propagate).
    if (beta != X(0))
      PLS_CUDA(cudaMemcpyAsync(A->ybuf.p, y, sizeof(X) * ylen, cudaMemcpyHostToDevice, s));
    const int n_bands = band_count<X>(A, trans, alpha, xlen, ylen);
    if (n_bands > 1 && spmv_banded<X>(A, n_bands, alpha, beta, y, s))
      return PERFLIBS_STATUS_SUCCESS;
    const perflibs_status_t st =
        spmv_device<X>(trans, alpha, A, A->xbuf.as<X>(), beta, A->ybuf.as<X>(), s);
    PLS_CUDA(cudaMemcpyAsync(y, A->ybuf.p, sizeof(X) * ylen, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    return st;
  });
}

template <class X>
perflibs_status_t spmv_exec_dev(int trans, X alpha, Mat *A, const X *x, X beta, X *y,
                                void *stream) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (!valid_op(trans))
      return param_error(A, 1, "Incorrect transpose option.");
    if (!matches<X>(A))
      return param_error(A, 3, "The matrix handle has a different data type.");
    DeviceGuard g(A->device);
    align_operation(A, trans);
    prepare_values(A);
    cudaStream_t s = stream ? (cudaStream_t)stream : stream_of(A);
    // beta = 0: every kernel writes all of y without reading it.
    return spmv_device<X>(trans, alpha, A, x, beta, y, s);
  });
}

// ------------------------------------------------------------------ SpMM

// The reference's repeated-SpMV threshold (src/matmul.cpp:26-28): fewer
// than 5 right-hand sides run as one SpMV per column.
constexpr int kSpmvRhsThreshold = 5;

// The learned SpMM selector's kernel order for k, into the CSR tile state
// (pred_n = 0 when no selector is attached for k's bucket: the candidates
// are then timed). The handle's features are computed on the first
// prediction; a prediction is kept while k stays in its bucket.
void spmm_predict(Mat *A, int k) {
  TileDev &t = A->csr.tiles;
  const int b = spmm_bucket(k);
  perflibs_b200_selector_t S = A->spmm_selector[b];
  if (!S) {
    t.pred_n = 0;
    return;
  }
  if (t.pred_n > 0 && t.pred_bucket == b)
    return;
  if (!A->features_valid) {
    compute_features(A, A->features);
    A->features_valid = true;
  }
  float probs[kSpmmClasses];
  int32_t cls = -1;
  t.pred_n = 0;
  if (selector_classes(S) != kSpmmClasses ||
      perflibs_b200_selector_predict(S, A->features, 1, probs, &cls) != PERFLIBS_STATUS_SUCCESS)
    return;
  int order[kSpmmClasses];
  for (int q = 0; q < kSpmmClasses; ++q)
    order[q] = q;
  std::stable_sort(order, order + kSpmmClasses, [&](int x, int y) { return probs[x] > probs[y]; });
  for (int q = 0; q < kSpmmClasses; ++q)
    t.pred_order[q] = order[q];
  t.pred_n = kSpmmClasses;
  t.pred_bucket = b;
  t.choice_sig = -1;  // decide the kernel again from this order
}

template <class X> void make_dense_zero(Mat *C, Dt dt, int32_t m, int32_t n, int layout) {
  cudaStream_t s = stream_of(C);
  C->dt = dt;
  C->fmt = Fmt::DENSE;
  C->m = m;
  C->n = n;
  C->nnz = (int64_t)m * n;
  C->dense = DenseDev{};
  C->dense.layout = layout;
  C->dense.lda = std::max<int64_t>(layout == PERFLIBS_ROW_MAJOR ? n : m, 1);
  C->dense.vals.reserve(std::max<size_t>(sizeof(X) * (size_t)m * n, 16));
  PLS_CUDA(cudaMemsetAsync(C->dense.vals.p, 0, sizeof(X) * (size_t)m * n, s));
  C->dense.is_zero = true;
}

// Re-lay a dense handle to `layout` in place (the reference replaces B or C
// with a re-laid copy, src/matmul.cpp:513-546, 573-592).
template <class X> void relayout(Mat *D, int layout) {
  if (D->dense.layout == layout)
    return;
  cudaStream_t s = stream_of(D);
  const int64_t rows = D->dense.layout == PERFLIBS_ROW_MAJOR ? D->m : D->n;
  const int64_t cols = D->dense.layout == PERFLIBS_ROW_MAJOR ? D->n : D->m;
  DevBuf nv;
  nv.reserve(std::max<size_t>(sizeof(X) * rows * cols, 16));
  transpose_dense<X>(D->dense.vals.as<X>(), rows, cols, D->dense.lda, nv.as<X>(), rows, s);
  PLS_CUDA(cudaStreamSynchronize(s));
  D->dense.vals = std::move(nv);
  D->dense.layout = layout;
  D->dense.lda = std::max<int64_t>(rows, 1);
}

int spmm_check(int transA, int transB, int alpha_h, Mat *A, Mat *B, int beta_h, Mat *C) {
  // src/matmul.cpp:1197-1311 (spmm_check_params)
  if (!A || !B || !C)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  auto typed = [](const Mat *M) { return M->fmt != Fmt::NUL && M->fmt != Fmt::IDENTITY; };
  if ((typed(A) && typed(B) && A->dt != B->dt) || (typed(A) && typed(C) && A->dt != C->dt) ||
      (typed(B) && typed(C) && B->dt != C->dt))
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (!valid_op(transA) || !valid_op(transB))
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (A->m < 0 || A->n < 0 || B->m < 0 || B->n < 0 || C->m < 0 || C->n < 0)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const bool ta = transA != PERFLIBS_SPARSE_OPERATION_NOTRANS;
  const bool tb = transB != PERFLIBS_SPARSE_OPERATION_NOTRANS;
  const int32_t ak = ta ? A->m : A->n, bk = tb ? B->n : B->m;
  if (ak != bk)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const int32_t cm = ta ? A->n : A->m, cn = tb ? B->m : B->n;
  if (C->m != cm || C->n != cn)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  auto scalar_ok = [](int v) {
    return v == PERFLIBS_SPARSE_SCALAR_ONE || v == PERFLIBS_SPARSE_SCALAR_ZERO ||
           v == PERFLIBS_SPARSE_SCALAR_ANY;
  };
  if (!scalar_ok(alpha_h) || !scalar_ok(beta_h))
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const bool result_dense = A->fmt == Fmt::DENSE || B->fmt == Fmt::DENSE;
  if (beta_h == PERFLIBS_SPARSE_SCALAR_ZERO) {
    if (!(C->fmt == Fmt::NUL || (C->fmt == Fmt::DENSE && result_dense))) {
      set_err(C, PERFLIBS_STATUS_INPUT_PARAMETER_ERROR, 7, "");
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    }
  }
  return PERFLIBS_STATUS_SUCCESS;
}

// C(i, j) = T(j, i) + beta * C(i, j) for an m x n C and an n x m T, any
// layout and leading dimension of either (beta == 0: C is not read).
template <class X>
__global__ void k_add_transposed(int32_t m, int32_t n, const X *__restrict__ T, int64_t ldt,
                                 int t_rowmajor, X *__restrict__ C, int64_t ldc, int c_rowmajor,
                                 X beta, int beta_nz) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * n)
    return;
  // walk C in its storage order
  const int64_t i = c_rowmajor ? idx / n : idx % m;
  const int64_t j = c_rowmajor ? idx % n : idx / m;
  const X t = t_rowmajor ? T[j * ldt + i] : T[i * ldt + j];
  X *c = C + (c_rowmajor ? i * ldc + j : j * ldc + i);
  *c = beta_nz ? t + beta * *c : t;
}

// ---- identity and dense x dense products (not a hot path) ----------------
// Element (i, j) of op(D) for a dense D of leading dimension ld: row-major
// D[i * ld + j], column-major D[j * ld + i]; the transpose swaps i and j.
template <class X>
__device__ __forceinline__ X dense_at(const X *D, int64_t ld, int rowmajor, int trans, int64_t i,
                                      int64_t j) {
  if (trans) {
    const int64_t t = i;
    i = j;
    j = t;
  }
  return rowmajor ? D[i * ld + j] : D[j * ld + i];
}

template <class X>
__device__ __forceinline__ X *dense_ptr(X *C, int64_t ld, int rowmajor, int64_t i, int64_t j) {
  return rowmajor ? C + i * ld + j : C + j * ld + i;
}

// C = alpha * op(A) op(B) + beta * C for dense A (m x k after op) and B
// (k x n): one thread per element of C, products added in the order of the
// inner index (the reference hands this case to cblas_dgemm,
// src/matmul.cpp:383-441).
template <class X>
__global__ void k_dense_gemm(int32_t m, int32_t n, int32_t k, const X *__restrict__ A, int64_t lda,
                             int a_rm, int ta, const X *__restrict__ B, int64_t ldb, int b_rm,
                             int tb, X *__restrict__ C, int64_t ldc, int c_rm, X alpha, X beta,
                             int beta_nz) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * n)
    return;
  const int64_t i = idx / n, j = idx % n;
  X sum = 0;
  for (int64_t l = 0; l < k; ++l)
    sum += dense_at(A, lda, a_rm, ta, i, l) * dense_at(B, ldb, b_rm, tb, l, j);
  X *c = dense_ptr(C, ldc, c_rm, i, j);
  *c = beta_nz ? alpha * sum + beta * *c : alpha * sum;
}

// C = alpha * op(D) + beta * C for a dense D (an identity factor times D).
template <class X>
__global__ void k_dense_axpby(int32_t m, int32_t n, const X *__restrict__ D, int64_t ldd,
                              int d_rm, int td, X *__restrict__ C, int64_t ldc, int c_rm,
                              X alpha, X beta, int beta_nz) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)m * n)
    return;
  const int64_t i = idx / n, j = idx % n;
  X *c = dense_ptr(C, ldc, c_rm, i, j);
  const X d = alpha * dense_at(D, ldd, d_rm, td, i, j);
  *c = beta_nz ? d + beta * *c : d;
}

// C += alpha * op(S) for a CSR S, C already scaled by beta: one thread per
// row i of S, whose entries all land in row i of C (column i when
// transposed), so no two threads write one element and repeated entries of
// a row are added in stored order.
template <class X>
__global__ void k_csr_add_dense(int32_t rows, const int32_t *__restrict__ rp,
                                const int32_t *__restrict__ col, const X *__restrict__ val,
                                X alpha, int trans, X *__restrict__ C, int64_t ldc, int c_rm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows)
    return;
  for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
    const int64_t j = col[p];
    X *c = trans ? dense_ptr(C, ldc, c_rm, j, i) : dense_ptr(C, ldc, c_rm, i, j);
    *c += alpha * val[p];
  }
}

// C += alpha on the diagonal (the identity times the identity).
template <class X>
__global__ void k_add_diag(int32_t n, X alpha, X *__restrict__ C, int64_t ldc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    C[i * ldc + i] += alpha;
}

// The sparse x dense branch of the reference's spmm_exec_checked
// (src/matmul.cpp:343-652), on the device. exec == false is the optimize
// call: it prepares layouts and tunes without computing.
template <class X>
perflibs_status_t spmm_impl(int transA, int transB, X alpha, Mat *A, Mat *B, X beta, Mat *C,
                            bool exec) {
  DeviceGuard g(A->device);
  const bool ta = transA != PERFLIBS_SPARSE_OPERATION_NOTRANS;
  const bool tb = transB != PERFLIBS_SPARSE_OPERATION_NOTRANS;
  const int32_t m = ta ? A->n : A->m;
  const int32_t n = tb ? B->m : B->n;  // right-hand sides
  const int32_t k = ta ? A->m : A->n;
  const Dt dt = dt_of<X>();
  const bool c_null = C->fmt == Fmt::NUL;
  cudaStream_t s = stream_of(A);
  C->stream = C->stream ? C->stream : A->stream;

  // Trivial product (src/matmul.cpp:383-389): AB is the null matrix; then
  // C = beta*C, or C becomes null when beta == 0 (src/matmul.cpp:770-790).
  if (m == 0 || n == 0 || k == 0 || alpha == X(0) || A->fmt == Fmt::NUL || B->fmt == Fmt::NUL) {
    if (!exec)
      return PERFLIBS_STATUS_SUCCESS;
    if (beta == X(0)) {
      C->fmt = Fmt::NUL;
      C->dense = DenseDev{};
      C->nnz = 0;
    } else if (C->fmt == Fmt::DENSE) {
      scal<X>((int64_t)C->m * C->n, beta, C->dense.vals.as<X>(), stream_of(C));
      PLS_CUDA(cudaStreamSynchronize(stream_of(C)));
    }
    return PERFLIBS_STATUS_SUCCESS;
  }
  // Dense x sparse (src/matmul.cpp:654-740): (op(A) op(B))^T = op'(B) op'(A)
  // with each operation flipped, so the sparse x dense path computes
  // T = alpha * op'(B) op'(A) (n x m) and C = T^T + beta * C.
  if (A->fmt == Fmt::DENSE && is_sparse(B->fmt) && (C->fmt == Fmt::DENSE || c_null) && A != C &&
      B != C) {
    if (A->dt != dt || B->dt != dt)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    auto flip = [](int t) {
      return t == PERFLIBS_SPARSE_OPERATION_NOTRANS ? PERFLIBS_SPARSE_OPERATION_TRANS
                                                    : PERFLIBS_SPARSE_OPERATION_NOTRANS;
    };
    std::unique_ptr<Mat> T(new_mat(dt, Fmt::NUL));
    T->m = n;
    T->n = m;
    T->stream = A->stream;
    const perflibs_status_t st =
        spmm_impl<X>(flip(transB), flip(transA), alpha, B, A, X(0), T.get(), exec);
    if (st != PERFLIBS_STATUS_SUCCESS)
      return st;
    if (c_null)
      make_dense_zero<X>(C, dt, m, n, PERFLIBS_ROW_MAJOR);
    if (!exec)
      return PERFLIBS_STATUS_SUCCESS;
    if (T->fmt == Fmt::DENSE) {
      const int64_t total = (int64_t)m * n;
      k_add_transposed<X><<<(unsigned)div_up(total, 256), 256, 0, s>>>(
          m, n, T->dense.vals.as<X>(), T->dense.lda, T->dense.layout == PERFLIBS_ROW_MAJOR,
          C->dense.vals.as<X>(), C->dense.lda, C->dense.layout == PERFLIBS_ROW_MAJOR, beta,
          beta != X(0));
      PLS_LAUNCH_CHECK();
    } else if (beta != X(0)) {  // T is the null matrix: C = beta * C
      scal<X>((int64_t)C->m * C->n, beta, C->dense.vals.as<X>(), s);
    } else {
      PLS_CUDA(cudaMemsetAsync(C->dense.vals.p, 0, sizeof(X) * (size_t)C->m * C->n, s));
    }
    PLS_CUDA(cudaStreamSynchronize(s));
    C->dense.is_zero = false;
    return PERFLIBS_STATUS_SUCCESS;
  }
  // Identity factors (src/matmul.cpp:654-740 dispatch): I op(S) and op(S) I
  // are alpha * op(S) + beta * C for S dense, sparse or the identity; and
  // dense x dense. Simple kernels: these are not the hot path.
  const bool a_id = A->fmt == Fmt::IDENTITY, b_id = B->fmt == Fmt::IDENTITY;
  if ((a_id || b_id || (A->fmt == Fmt::DENSE && B->fmt == Fmt::DENSE)) &&
      (C->fmt == Fmt::DENSE || c_null) && A != C && B != C) {
    if ((!a_id && A->dt != dt) || (!b_id && B->dt != dt))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (c_null)
      make_dense_zero<X>(C, dt, m, n, PERFLIBS_ROW_MAJOR);
    if (!exec)
      return PERFLIBS_STATUS_SUCCESS;
    X *cv = C->dense.vals.as<X>();
    const int64_t ldc = C->dense.lda;
    const int c_rm = C->dense.layout == PERFLIBS_ROW_MAJOR;
    const unsigned blocks = (unsigned)div_up((int64_t)m * n, 256);
    const int bnz = beta != X(0);
    if (!a_id && !b_id) {
      k_dense_gemm<X><<<blocks, 256, 0, s>>>(
          m, n, k, A->dense.vals.as<X>(), A->dense.lda, A->dense.layout == PERFLIBS_ROW_MAJOR, ta,
          B->dense.vals.as<X>(), B->dense.lda, B->dense.layout == PERFLIBS_ROW_MAJOR, tb, cv, ldc,
          c_rm, alpha, beta, bnz);
    } else {
      Mat *S = a_id ? B : A;  // the other factor
      const bool ts = a_id ? tb : ta;
      if (S->fmt == Fmt::DENSE) {
        k_dense_axpby<X><<<blocks, 256, 0, s>>>(m, n, S->dense.vals.as<X>(), S->dense.lda,
                                                S->dense.layout == PERFLIBS_ROW_MAJOR, ts, cv, ldc,
                                                c_rm, alpha, beta, bnz);
      } else {
        scal<X>((int64_t)m * n, beta, cv, s);  // C is packed: m * n elements
        if (S->fmt == Fmt::IDENTITY) {
          k_add_diag<X><<<(unsigned)div_up(std::max<int64_t>(std::min(m, n), 1), 256), 256, 0,
                          s>>>(std::min(m, n), alpha, cv, ldc);
        } else {
          if (S->fmt == Fmt::BSR)
            bsr_become_csr(S);  // as the reference's SpMM does (src/matmul.cpp:616-631)
          k_csr_add_dense<X><<<(unsigned)div_up(std::max<int32_t>(S->m, 1), 256), 256, 0, s>>>(
              S->m, S->csr.row_ptr.as<int32_t>(), S->csr.col.as<int32_t>(), S->csr.vals.as<X>(),
              alpha, ts, cv, ldc, c_rm);
        }
      }
    }
    PLS_LAUNCH_CHECK();
    PLS_CUDA(cudaStreamSynchronize(s));
    C->dense.is_zero = false;
    return PERFLIBS_STATUS_SUCCESS;
  }
  if (!(is_sparse(A->fmt) && B->fmt == Fmt::DENSE && (C->fmt == Fmt::DENSE || c_null) && A != C &&
        B != C))
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                "sparse x sparse products are not provided by the B200 execute path");
  if (A->dt != dt || B->dt != dt)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;

  // Narrow right-hand sides: one SpMV per column (src/matmul.cpp:451-511).
  if (n < kSpmvRhsThreshold) {
    if (c_null)
      make_dense_zero<X>(C, dt, m, n, PERFLIBS_COL_MAJOR);
    if (!exec) {
      align_operation(A, transA);
      A->hint_spmv_inv = A->hint_spmm_inv;
      prepare_values(A);
      if (A->hint_spmv_inv == PERFLIBS_SPARSE_INVOCATIONS_MANY && !A->tuned &&
          (A->fmt == Fmt::CSR) && transA == PERFLIBS_SPARSE_OPERATION_NOTRANS &&
          A->tuner != PERFLIBS_B200_TUNE_NONE) {
        tune_spmv(A);
        A->tuned = true;
        A->tuned_op = transA;
      }
      return PERFLIBS_STATUS_SUCCESS;
    }
    align_operation(A, transA);
    prepare_values(A);
    int64_t b_sr = B->dense.layout == PERFLIBS_ROW_MAJOR ? B->dense.lda : 1;
    int64_t b_sc = B->dense.layout == PERFLIBS_COL_MAJOR ? B->dense.lda : 1;
    if (tb)
      std::swap(b_sr, b_sc);
    const int64_t c_sr = C->dense.layout == PERFLIBS_ROW_MAJOR ? C->dense.lda : 1;
    const int64_t c_sc = C->dense.layout == PERFLIBS_COL_MAJOR ? C->dense.lda : 1;
    DevBuf bw, cw;
    if (b_sr != 1)
      bw.reserve(sizeof(X) * std::max<int64_t>(k, 1));
    if (c_sr != 1)
      cw.reserve(sizeof(X) * std::max<int64_t>(m, 1));
    for (int32_t r = 0; r < n; ++r) {
      const X *bc = B->dense.vals.as<X>() + r * b_sc;
      if (b_sr != 1) {
        strided_copy<X>(bc, b_sr, bw.as<X>(), 1, k, s);
        bc = bw.as<X>();
      }
      X *cc = C->dense.vals.as<X>() + r * c_sc;
      X *cdst = cc;
      if (c_sr != 1) {
        if (beta != X(0))
          strided_copy<X>(cc, c_sr, cw.as<X>(), 1, m, s);
        cc = cw.as<X>();
      }
      spmv_device<X>(transA, alpha, A, bc, beta, cc, s);  // beta = 0: cc written, not read
      if (c_sr != 1)
        strided_copy<X>(cc, 1, cdst, c_sr, m, s);
    }
    PLS_CUDA(cudaStreamSynchronize(s));
    C->dense.is_zero = false;
    return PERFLIBS_STATUS_SUCCESS;
  }

  // B re-laid so that rows of op(B) are contiguous (src/matmul.cpp:513-551).
  if (!tb && B->dense.layout == PERFLIBS_COL_MAJOR)
    relayout<X>(B, PERFLIBS_ROW_MAJOR);
  else if (tb && B->dense.layout == PERFLIBS_ROW_MAJOR)
    relayout<X>(B, PERFLIBS_COL_MAJOR);
  if (c_null)
    make_dense_zero<X>(C, dt, m, n, PERFLIBS_ROW_MAJOR);
  if (C->dense.layout == PERFLIBS_COL_MAJOR)
    relayout<X>(C, PERFLIBS_ROW_MAJOR);

  // A as a row-wise operator: CSR (or BSR, natively) for NOTRANS, the CSR of
  // A^T for TRANS (the reference's CSC view, src/matmul.cpp:616-631).
  prepare_values(A);
  if (ta) {
    bsr_become_csr(A);
    if (!A->has_csrT) {
      build_csr_transpose(A->csr, A->m, A->n, A->csrT, s);
      A->has_csrT = true;
    }
    if (A->csrT.vt != A->csr.evt() || A->csr.lo != A->csrT.lo) {
      A->csrT.lo = false;
      if (A->csr.lo) {
        A->csrT.vals_lo.reserve(vt_size(A->csr.vt_lo) * std::max<int64_t>(A->csrT.nnz, 1));
        convert_values(A->csrT.vals.p, A->csrT.vt, A->csrT.vals_lo.p, A->csr.vt_lo,
                       A->csrT.nnz, s);
        A->csrT.vt_lo = A->csr.vt_lo;
        A->csrT.lo = true;
      }
    }
  }
  if (!exec)
    return PERFLIBS_STATUS_SUCCESS;

  X *Cv = C->dense.vals.as<X>();
  const int64_t ldc = C->dense.lda;
  const X *Bv = B->dense.vals.as<X>();
  const int64_t ldb = B->dense.lda;
  // beta == 0 overwrites C (the reference zeroes it first, src/matmul.cpp:
  // 596-605); the kernels never read C then.
  if (ta)
    spmm_csr<X>(A->csrT, m, Bv, ldb, Cv, ldc, n, alpha, beta, s);
  else if (A->fmt == Fmt::BSR)
    spmm_bsr<X>(A->bsr, Bv, ldb, Cv, ldc, n, alpha, beta, s, A->csr.tiles);
  else
  {
    spmm_predict(A, n);
    spmm_csr<X>(A->csr, m, Bv, ldb, Cv, ldc, n, alpha, beta, s);
  }
  PLS_CUDA(cudaStreamSynchronize(s));
  C->dense.is_zero = false;
  return PERFLIBS_STATUS_SUCCESS;
}

template <class X>
perflibs_status_t spmm_exec_entry(int transA, int transB, X alpha, Mat *A, Mat *B, X beta,
                                  Mat *C) {
  TraceRange trace("perflibs_spmm_exec");
  const int st = spmm_check(transA, transB, PERFLIBS_SPARSE_SCALAR_ANY, A, B,
                            PERFLIBS_SPARSE_SCALAR_ANY, C);
  if (st != PERFLIBS_STATUS_SUCCESS)
    return (perflibs_status_t)st;
  return guarded(A, [&]() { return spmm_impl<X>(transA, transB, alpha, A, B, beta, C, true); });
}

// ---------------------------------------------------------------- export

template <class X>
perflibs_status_t export_csr(const Mat *Ac, int32_t base, int32_t *m, int32_t *n,
                             int32_t **row_ptr, int32_t **col, X **vals) {
  Mat *A = const_cast<Mat *>(Ac);
  if (!A || !m || !n || !row_ptr || !col || !vals)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/export.cpp:41-84 (csr_param_check)
    if (A->m <= 0 || A->n <= 0)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (base != 0 && base != 1)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (!matches<X>(A))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    const CsrDev *src = &A->csr;
    CsrDev tmp;
    // A BSR handle exports through bsr2csr, which drops exact zeros; so
    // does a handle converted to SELL-C-sigma (scs2csr,
    // src/compressed_sparse_rows.cpp:832-936).
    bool drop_zeros = A->fmt == Fmt::SELL;
    if (A->fmt == Fmt::BSR) {
      bsr_to_csr(A->bsr, A->m, true, tmp, s);
      src = &tmp;
    } else if (A->fmt != Fmt::CSR && A->fmt != Fmt::SELL) {
      return PERFLIBS_STATUS_EXECUTION_FAILURE;
    }
    std::vector<int32_t> rp(A->m + 1), c(src->nnz);
    std::vector<X> v(src->nnz);
    PLS_CUDA(cudaMemcpyAsync(rp.data(), src->row_ptr.p, 4 * (A->m + 1), cudaMemcpyDeviceToHost, s));
    if (src->nnz > 0) {
      PLS_CUDA(cudaMemcpyAsync(c.data(), src->col.p, 4 * src->nnz, cudaMemcpyDeviceToHost, s));
      PLS_CUDA(cudaMemcpyAsync(v.data(), src->vals.p, sizeof(X) * src->nnz,
                               cudaMemcpyDeviceToHost, s));
    }
    PLS_CUDA(cudaStreamSynchronize(s));
    int64_t nnz = src->nnz;
    if (drop_zeros) {
      int64_t o = 0;
      std::vector<int32_t> nrp(A->m + 1, 0);
      for (int32_t i = 0; i < A->m; ++i) {
        for (int32_t j = rp[i]; j < rp[i + 1]; ++j)
          if (v[j] != X(0)) {
            c[o] = c[j];
            v[o] = v[j];
            o++;
          }
        nrp[i + 1] = (int32_t)o;
      }
      rp.swap(nrp);
      nnz = o;
    }
    auto *orp = (int32_t *)std::malloc(sizeof(int32_t) * (A->m + 1));
    auto *oc = (int32_t *)std::malloc(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
    auto *ov = (X *)std::malloc(sizeof(X) * std::max<int64_t>(nnz, 1));
    if (!orp || !oc || !ov) {
      std::free(orp);
      std::free(oc);
      std::free(ov);
      return PERFLIBS_STATUS_EXECUTION_FAILURE;
    }
    for (int32_t i = 0; i <= A->m; ++i)
      orp[i] = rp[i] + base;
    for (int64_t j = 0; j < nnz; ++j) {
      oc[j] = c[j] + base;
      ov[j] = v[j];
    }
    *m = A->m;
    *n = A->n;
    *row_ptr = orp;
    *col = oc;
    *vals = ov;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

template <class X>
perflibs_status_t export_dense(const Mat *Ac, int layout, int32_t *m, int32_t *n, X **vals) {
  Mat *A = const_cast<Mat *>(Ac);
  if (!A || !m || !n || !vals)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/export.cpp:442-475 (dense_param_check)
    if (A->m <= 0 || A->n <= 0)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (layout != PERFLIBS_COL_MAJOR && layout != PERFLIBS_ROW_MAJOR)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (!matches<X>(A))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    const int64_t M = A->m, N = A->n;
    DevBuf out;
    out.reserve(sizeof(X) * M * N);
    if (A->fmt == Fmt::DENSE) {
      if (A->dense.layout == layout) {
        PLS_CUDA(cudaMemcpyAsync(out.p, A->dense.vals.p, sizeof(X) * M * N,
                                 cudaMemcpyDeviceToDevice, s));
      } else {
        const int64_t rows = A->dense.layout == PERFLIBS_ROW_MAJOR ? M : N;
        const int64_t cols = A->dense.layout == PERFLIBS_ROW_MAJOR ? N : M;
        transpose_dense<X>(A->dense.vals.as<X>(), rows, cols, A->dense.lda, out.as<X>(), rows, s);
      }
    } else {
      PLS_CUDA(cudaMemsetAsync(out.p, 0, sizeof(X) * M * N, s));
      const CsrDev *src = nullptr;
      CsrDev tmp;
      if (A->fmt == Fmt::CSR || A->fmt == Fmt::SELL) {
        src = &A->csr;
      } else if (A->fmt == Fmt::BSR) {
        bsr_to_csr(A->bsr, A->m, false, tmp, s);
        src = &tmp;
      } else if (A->fmt == Fmt::IDENTITY) {
        std::vector<X> h(M * N, X(0));
        for (int64_t i = 0; i < std::min(M, N); ++i)
          h[i * (layout == PERFLIBS_ROW_MAJOR ? N : M) + i] = X(1);
        PLS_CUDA(cudaMemcpyAsync(out.p, h.data(), sizeof(X) * M * N, cudaMemcpyHostToDevice, s));
      }
      if (src && M > 0) {
        const int64_t rs = layout == PERFLIBS_ROW_MAJOR ? N : 1;
        const int64_t cs = layout == PERFLIBS_ROW_MAJOR ? 1 : M;
        k_densify_csr<X><<<(unsigned)div_up(M, 256), 256, 0, s>>>(
            (int32_t)M, src->row_ptr.as<int32_t>(), src->col.as<int32_t>(), src->vals.as<X>(),
            out.as<X>(), rs, cs);
        PLS_LAUNCH_CHECK();
      }
    }
    X *h = (X *)std::malloc(sizeof(X) * M * N);
    if (!h)
      return PERFLIBS_STATUS_EXECUTION_FAILURE;
    PLS_CUDA(cudaMemcpyAsync(h, out.p, sizeof(X) * M * N, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    *m = (int32_t)M;
    *n = (int32_t)N;
    *vals = h;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

template <class X>
perflibs_status_t spnorm(Mat *A, int nrm, X *result) {
  if (!A || !result)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/norm.cpp:185-211 (spnorm_exec)
    if (nrm != PERFLIBS_SPARSE_NORM_INF && nrm != PERFLIBS_SPARSE_NORM_FRB)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (!matches<X>(A))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (A->nnz == 0 || A->fmt == Fmt::NUL) {
      *result = X(0);
      return PERFLIBS_STATUS_SUCCESS;
    }
    if (A->fmt == Fmt::IDENTITY) {
      *result = nrm == PERFLIBS_SPARSE_NORM_FRB ? (X)std::sqrt((double)A->n) : X(1);
      return PERFLIBS_STATUS_SUCCESS;
    }
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    double r = 0;
    const Vt nv = native_vt(A->dt);
    if (nrm == PERFLIBS_SPARSE_NORM_FRB) {
      if (A->fmt == Fmt::CSR || A->fmt == Fmt::SELL)
        r = frb_norm_values(A->csr.vals.p, nv, A->csr.nnz, s);
      else if (A->fmt == Fmt::BSR)
        r = frb_norm_values(A->bsr.vals.p, nv, A->bsr.nnzb * (int64_t)A->bsr.bs * A->bsr.bs, s);
      else
        r = frb_norm_values(A->dense.vals.p, nv, (int64_t)A->m * A->n, s);
    } else {
      if (A->fmt == Fmt::CSR || A->fmt == Fmt::SELL) {
        CsrDev view;  // authoritative values, not the reduced copy
        r = inf_norm_csr(A->csr, A->m, s);
      } else if (A->fmt == Fmt::BSR) {
        r = inf_norm_bsr(A->bsr, s);
      } else {
        r = inf_norm_dense(A->dense, A->dt, A->m, A->n, s);
      }
    }
    *result = (X)r;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

template <class X>
perflibs_status_t update(Mat *A, int32_t nu, const int32_t *rows, const int32_t *cols,
                         const X *vals) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    // src/matvec.cpp:533-567 (spmat_update)
    if (nu == 0)
      return PERFLIBS_STATUS_SUCCESS;
    if (nu < 0)
      return param_error(A, 1, "The number of updates can not be negative.");
    if (!matches<X>(A))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (A->fmt == Fmt::BSR)
      bsr_become_csr(A);
    if (A->fmt != Fmt::CSR && A->fmt != Fmt::SELL)
      return PERFLIBS_STATUS_EXECUTION_FAILURE;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    // Authoritative values first, then the reduced copy and SELL values.
    const int64_t applied = update_csr_values(A->csr, nullptr, A->m, A->n, nu, rows, cols, vals,
                                              A->dt, A->index_base, s);
    // The cached CSR of A^T holds the old values: the next transposed
    // product builds it again.
    A->has_csrT = false;
    ++A->csr.vals_version;
    if (A->csr.lo || A->fmt == Fmt::SELL) {
      // Re-derive the kernels' copies of the updated entries.
      CsrDev &c = A->csr;
      if (c.lo)
        convert_values(c.vals.p, c.vt, c.vals_lo.p, c.vt_lo, c.nnz, s);
      if (A->fmt == Fmt::SELL) {
        SellDev keep = std::move(A->sell);
        A->sell = SellDev{};
        (void)keep;
        apply_config(A, A->cfg);
      }
      PLS_CUDA(cudaStreamSynchronize(s));
    }
    if (applied < nu) {
      // src/compressed_sparse_rows.cpp:3076-3092: the failing update's
      // position (in the matrix's index base) is the error code.
      return param_error(A, (int)(applied + A->index_base),
                         "An update names an entry that is not stored in the matrix.");
    }
    return PERFLIBS_STATUS_SUCCESS;
  });
}

}  // namespace

cudaStream_t lib_stream(int dev) {
  std::lock_guard<std::mutex> g(g_stream_mu);
  cudaStream_t &s = g_streams[dev & 63];
  if (!s)
    PLS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

cudaStream_t stream_of(const Mat *A) { return A->stream ? A->stream : lib_stream(A->device); }

template <class X>
void run_spmv(Mat *A, int op, const X *x, X *y, X alpha, X beta, cudaStream_t s) {
  if (op == PERFLIBS_SPARSE_OPERATION_NOTRANS) {
    switch (A->fmt) {
    case Fmt::SELL:
      spmv_sell<X>(A->sell, x, y, alpha, beta, s);
      return;
    case Fmt::CSR:
      if (A->cfg.kind == Kind::CSR_SPLIT)
        spmv_csr_split<X>(A->csr, A->m, x, y, alpha, beta, s);
      else
        spmv_csr<X>(A->csr, A->m, A->cfg.tpr > 0 ? A->cfg.tpr : default_config(A).tpr, x, y,
                    alpha, beta, s);
      return;
    case Fmt::BSR:
      spmv_bsr<X>(A->bsr, x, y, alpha, beta, s);
      return;
    default:
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "unsupported format for SpMV");
    }
  }
  if (A->has_csrT && A->csrT.lo == A->csr.lo) {
    const double mean = A->n > 0 ? (double)A->csrT.nnz / A->n : 1;
    int tpr = 1;
    while (tpr * 2 <= mean && tpr < 32)
      tpr *= 2;
    spmv_csr<X>(A->csrT, A->n, tpr, x, y, alpha, beta, s);
  } else {
    spmv_csr_trans<X>(A->csr, A->m, A->n, x, y, alpha, beta, s);
  }
}

template void run_spmv<float>(Mat *, int, const float *, float *, float, float, cudaStream_t);
template void run_spmv<double>(Mat *, int, const double *, double *, double, double,
                               cudaStream_t);

}  // namespace pls

using namespace pls;

// ================================================================ C ABI

extern "C" {

perflibs_status_t perflibs_spmat_create_csr_s(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_ptr,
                                              const perflibs_int_t *col_indx, const float *vals,
                                              perflibs_int_t flags) {
  return create_csr<float>(A, m, n, row_ptr, col_indx, vals, flags);
}
perflibs_status_t perflibs_spmat_create_csr_d(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_ptr,
                                              const perflibs_int_t *col_indx, const double *vals,
                                              perflibs_int_t flags) {
  return create_csr<double>(A, m, n, row_ptr, col_indx, vals, flags);
}
perflibs_status_t perflibs_spmat_create_dense_s(perflibs_spmat_t *A,
                                                enum perflibs_dense_layout layout,
                                                perflibs_int_t m, perflibs_int_t n,
                                                perflibs_int_t lda, const float *vals,
                                                perflibs_int_t flags) {
  return create_dense<float>(A, layout, m, n, lda, vals, flags);
}
perflibs_status_t perflibs_spmat_create_dense_d(perflibs_spmat_t *A,
                                                enum perflibs_dense_layout layout,
                                                perflibs_int_t m, perflibs_int_t n,
                                                perflibs_int_t lda, const double *vals,
                                                perflibs_int_t flags) {
  return create_dense<double>(A, layout, m, n, lda, vals, flags);
}
perflibs_status_t perflibs_spmat_create_bsr_s(perflibs_spmat_t *A,
                                              enum perflibs_dense_layout block_layout,
                                              perflibs_int_t m, perflibs_int_t n,
                                              perflibs_int_t block_size,
                                              const perflibs_int_t *row_ptr,
                                              const perflibs_int_t *col_indx, const float *vals,
                                              perflibs_int_t flags) {
  return create_bsr<float>(A, block_layout, m, n, block_size, row_ptr, col_indx, vals, flags);
}
perflibs_status_t perflibs_spmat_create_bsr_d(perflibs_spmat_t *A,
                                              enum perflibs_dense_layout block_layout,
                                              perflibs_int_t m, perflibs_int_t n,
                                              perflibs_int_t block_size,
                                              const perflibs_int_t *row_ptr,
                                              const perflibs_int_t *col_indx, const double *vals,
                                              perflibs_int_t flags) {
  return create_bsr<double>(A, block_layout, m, n, block_size, row_ptr, col_indx, vals, flags);
}

// include/perflibs_sparse.h:176-208 (reference)
perflibs_status_t perflibs_spmat_create_csc_s(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_ptr, const float *vals,
                                              perflibs_int_t flags) {
  return create_csc<float>(A, m, n, row_indx, col_ptr, vals, flags);
}
perflibs_status_t perflibs_spmat_create_csc_d(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_ptr, const double *vals,
                                              perflibs_int_t flags) {
  return create_csc<double>(A, m, n, row_indx, col_ptr, vals, flags);
}
perflibs_status_t perflibs_spmat_create_coo_s(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, perflibs_int_t nnz,
                                              const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_indx, const float *vals,
                                              perflibs_int_t flags) {
  return create_coo<float>(A, m, n, nnz, row_indx, col_indx, vals, flags);
}
perflibs_status_t perflibs_spmat_create_coo_d(perflibs_spmat_t *A, perflibs_int_t m,
                                              perflibs_int_t n, perflibs_int_t nnz,
                                              const perflibs_int_t *row_indx,
                                              const perflibs_int_t *col_indx, const double *vals,
                                              perflibs_int_t flags) {
  return create_coo<double>(A, m, n, nnz, row_indx, col_indx, vals, flags);
}

// src/matrix_state.cpp:39-58: NULL for negative sizes.
perflibs_spmat_t perflibs_spmat_create_null(perflibs_int_t m, perflibs_int_t n) {
  if (m < 0 || n < 0)
    return nullptr;
  try {
    Mat *A = new_mat(Dt::F64, Fmt::NUL);
    A->m = m;
    A->n = n;
    return A;
  } catch (...) {
    return nullptr;
  }
}

perflibs_spmat_t perflibs_spmat_create_identity(perflibs_int_t n) {
  if (n < 0)
    return nullptr;
  try {
    Mat *A = new_mat(Dt::F64, Fmt::IDENTITY);
    A->m = n;
    A->n = n;
    A->nnz = n;
    return A;
  } catch (...) {
    return nullptr;
  }
}

perflibs_status_t perflibs_spmat_destroy(perflibs_spmat_t A) {
  if (A) {
    DeviceGuard g(A->device);
    delete A;
  }
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_spmat_query(perflibs_spmat_t A, perflibs_int_t *index_base,
                                       perflibs_int_t *m, perflibs_int_t *n,
                                       perflibs_int_t *nnz) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (index_base)
    *index_base = A->index_base;
  if (m)
    *m = A->m;
  if (n)
    *n = A->n;
  if (nnz)
    *nnz = (perflibs_int_t)A->nnz;
  return PERFLIBS_STATUS_SUCCESS;
}

// src/matrix_state.cpp:245-419 (set_hint): each hint accepts exactly the
// reference's value set.
perflibs_status_t perflibs_spmat_hint(perflibs_spmat_t A, enum perflibs_sparse_hint_type hint,
                                      enum perflibs_sparse_hint_value value) {
  if (!A)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  const int v = value;
  auto op_ok = [&] {
    return v == PERFLIBS_SPARSE_OPERATION_NOTRANS || v == PERFLIBS_SPARSE_OPERATION_TRANS ||
           v == PERFLIBS_SPARSE_OPERATION_CONJTRANS;
  };
  auto inv_ok = [&] {
    return v == PERFLIBS_SPARSE_INVOCATIONS_SINGLE || v == PERFLIBS_SPARSE_INVOCATIONS_FEW ||
           v == PERFLIBS_SPARSE_INVOCATIONS_MANY;
  };
  switch ((int)hint) {
  case PERFLIBS_SPARSE_HINT_STRUCTURE:
    if (v == PERFLIBS_SPARSE_STRUCTURE_DENSE || v == PERFLIBS_SPARSE_STRUCTURE_UNSTRUCTURED ||
        v == PERFLIBS_SPARSE_STRUCTURE_SYMMETRIC || v == PERFLIBS_SPARSE_STRUCTURE_DIAGONAL ||
        v == PERFLIBS_SPARSE_STRUCTURE_BLOCKDIAGONAL || v == PERFLIBS_SPARSE_STRUCTURE_BANDED ||
        v == PERFLIBS_SPARSE_STRUCTURE_TRIANGULAR ||
        v == PERFLIBS_SPARSE_STRUCTURE_BLOCKTRIANGULAR ||
        v == PERFLIBS_SPARSE_STRUCTURE_HERMITIAN)
      A->hint_structure = v;
    else if (v == PERFLIBS_SPARSE_STRUCTURE_HPCG)
      A->hint_hpcg = true;
    else
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    break;
  case PERFLIBS_SPARSE_HINT_MEMORY:
    if (v == PERFLIBS_SPARSE_MEMORY_NOALLOCS || v == PERFLIBS_SPARSE_MEMORY_ALLOCS)
      A->hint_memory = v;
    else
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    break;
  case PERFLIBS_SPARSE_HINT_SPMV_OPERATION:
    if (!op_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spmv_op = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPMV_INVOCATIONS:
    if (!inv_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spmv_inv = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPMM_OPERATION:
    if (!op_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spmm_op = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPMM_INVOCATIONS:
    if (!inv_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spmm_inv = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPADD_OPERATION:
    if (!op_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spadd_op = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPADD_INVOCATIONS:
    if (!inv_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spadd_inv = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPMM_STRATEGY:
    if (v == PERFLIBS_SPARSE_SPMM_STRAT_UNSET || v == PERFLIBS_SPARSE_SPMM_STRAT_OPT_NO_STRUCT ||
        v == PERFLIBS_SPARSE_SPMM_STRAT_OPT_PART_STRUCT ||
        v == PERFLIBS_SPARSE_SPMM_STRAT_OPT_FULL_STRUCT)
      A->hint_spmm_strat = v;
    else
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    break;
  case PERFLIBS_SPARSE_HINT_SPSM_OPERATION:
    if (!op_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spsm_op = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPSV_OPERATION:
    if (!op_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spsv_op = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPSV_INVOCATIONS:
    if (!inv_ok())
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    A->hint_spsv_inv = v;
    break;
  case PERFLIBS_SPARSE_HINT_SPSV_STRATEGY:
    if (v == PERFLIBS_SPARSE_SPSV_STRAT_UNSET || v == PERFLIBS_SPARSE_SPSV_STRAT_SEPARATOR_SPARSE ||
        v == PERFLIBS_SPARSE_SPSV_STRAT_SEPARATOR_DENSE)
      A->hint_spsv_strat = v;
    else
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    break;
  default:
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  }
  return PERFLIBS_STATUS_SUCCESS;
}

// src/matvec.cpp:583-630 (spmv_optimize).
perflibs_status_t perflibs_spmv_optimize(perflibs_spmat_t A) {
  TraceRange trace("perflibs_spmv_optimize");
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (A->fmt == Fmt::NUL || A->fmt == Fmt::IDENTITY || A->fmt == Fmt::DENSE)
      return PERFLIBS_STATUS_SUCCESS;
    if (A->nnz == 0)
      return PERFLIBS_STATUS_SUCCESS;
    DeviceGuard g(A->device);
    cudaStream_t s = stream_of(A);
    const int op = A->hint_spmv_op;
    if (A->fmt == Fmt::SELL && A->tuned && A->tuned_op == op && !A->forced)
      return PERFLIBS_STATUS_SUCCESS;
    if (op != PERFLIBS_SPARSE_OPERATION_NOTRANS) {
      // Optimized for the transposed operation: keep the CSR of A^T, the
      // role of the reference's SELL-of-A^T (optimized_op).
      bsr_become_csr(A);
      prepare_values(A);
      if (!A->has_csrT) {
        build_csr_transpose(A->csr, A->m, A->n, A->csrT, s);
        A->has_csrT = true;
      }
      A->tuned = true;
      A->tuned_op = op;
      return PERFLIBS_STATUS_SUCCESS;
    }
    prepare_values(A);
    if (A->forced) {
      bsr_become_csr(A);
      apply_config(A, A->forced_cfg);
      A->tune_source = TuneSource::FORCED;
      A->tuned = true;
      A->tuned_op = op;
      return PERFLIBS_STATUS_SUCCESS;
    }
    if (A->hint_spmv_inv != PERFLIBS_SPARSE_INVOCATIONS_MANY || A->tuner == PERFLIBS_B200_TUNE_NONE)
      return PERFLIBS_STATUS_SUCCESS;
    if (A->fmt == Fmt::BSR)
      return PERFLIBS_STATUS_SUCCESS;  // the BSR kernel is kept, as the reference keeps BSR
    if (A->tuner == PERFLIBS_B200_TUNE_SELECTOR && A->selector) {
      // Learned selector: features on the device, one MLP forward pass,
      // the predicted candidate applied without timing anything.
      float f[PERFLIBS_B200_NFEATURES];
      compute_features(A, f);
      int32_t cls = -1;
      const auto cands = tune_candidates(A);
      if (perflibs_b200_selector_predict(A->selector, f, 1, nullptr, &cls) ==
              PERFLIBS_STATUS_SUCCESS &&
          cls >= 0 && cls < (int32_t)cands.size()) {
        apply_config(A, cands[cls]);
        A->selector_class = cls;
        A->tune_source = TuneSource::SELECTOR;
        A->tuned = true;
        A->tuned_op = op;
        return PERFLIBS_STATUS_SUCCESS;
      }
    }
    tune_spmv(A);
    A->tuned = true;
    A->tuned_op = op;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

// src/matmul.cpp:834-858: optimize is exec without computing, with
// representative scalars.
perflibs_status_t perflibs_spmm_optimize(enum perflibs_sparse_hint_value transA,
                                         enum perflibs_sparse_hint_value transB,
                                         enum perflibs_sparse_hint_value alpha,
                                         perflibs_spmat_t A, perflibs_spmat_t B,
                                         enum perflibs_sparse_hint_value beta,
                                         perflibs_spmat_t C) {
  TraceRange trace("perflibs_spmm_optimize");
  const int st = spmm_check(transA, transB, alpha, A, B, beta, C);
  if (st != PERFLIBS_STATUS_SUCCESS)
    return (perflibs_status_t)st;
  const double a = alpha == PERFLIBS_SPARSE_SCALAR_ZERO ? 0.0
                   : alpha == PERFLIBS_SPARSE_SCALAR_ONE ? 1.0 : 1.5;
  const double b = beta == PERFLIBS_SPARSE_SCALAR_ZERO ? 0.0
                   : beta == PERFLIBS_SPARSE_SCALAR_ONE ? 1.0 : 1.5;
  return guarded(A, [&]() {
    if (A->fmt != Fmt::NUL && A->dt == Dt::F32)
      return spmm_impl<float>(transA, transB, (float)a, A, B, (float)b, C, false);
    return spmm_impl<double>(transA, transB, a, A, B, b, C, false);
  });
}

perflibs_status_t perflibs_spmv_exec_s(enum perflibs_sparse_hint_value trans, float alpha,
                                       perflibs_spmat_t A, const float *x, float beta,
                                       float *y) {
  return spmv_exec_host<float>(trans, alpha, A, x, beta, y);
}
perflibs_status_t perflibs_spmv_exec_d(enum perflibs_sparse_hint_value trans, double alpha,
                                       perflibs_spmat_t A, const double *x, double beta,
                                       double *y) {
  return spmv_exec_host<double>(trans, alpha, A, x, beta, y);
}
perflibs_status_t perflibs_spmm_exec_s(enum perflibs_sparse_hint_value transA,
                                       enum perflibs_sparse_hint_value transB, float alpha,
                                       perflibs_spmat_t A, perflibs_spmat_t B, float beta,
                                       perflibs_spmat_t C) {
  return spmm_exec_entry<float>(transA, transB, alpha, A, B, beta, C);
}
perflibs_status_t perflibs_spmm_exec_d(enum perflibs_sparse_hint_value transA,
                                       enum perflibs_sparse_hint_value transB, double alpha,
                                       perflibs_spmat_t A, perflibs_spmat_t B, double beta,
                                       perflibs_spmat_t C) {
  return spmm_exec_entry<double>(transA, transB, alpha, A, B, beta, C);
}

perflibs_status_t perflibs_spmat_update_s(perflibs_spmat_t A, perflibs_int_t n_updates,
                                          const perflibs_int_t *row_indx,
                                          const perflibs_int_t *col_indx, const float *vals) {
  return update<float>(A, n_updates, row_indx, col_indx, vals);
}
perflibs_status_t perflibs_spmat_update_d(perflibs_spmat_t A, perflibs_int_t n_updates,
                                          const perflibs_int_t *row_indx,
                                          const perflibs_int_t *col_indx, const double *vals) {
  return update<double>(A, n_updates, row_indx, col_indx, vals);
}

perflibs_status_t perflibs_spmat_export_csr_s(perflibs_const_spmat_t A, perflibs_int_t index_base,
                                              perflibs_int_t *m, perflibs_int_t *n,
                                              perflibs_int_t **row_ptr,
                                              perflibs_int_t **col_indx, float **vals) {
  return export_csr<float>(A, index_base, m, n, row_ptr, col_indx, vals);
}
perflibs_status_t perflibs_spmat_export_csr_d(perflibs_const_spmat_t A, perflibs_int_t index_base,
                                              perflibs_int_t *m, perflibs_int_t *n,
                                              perflibs_int_t **row_ptr,
                                              perflibs_int_t **col_indx, double **vals) {
  return export_csr<double>(A, index_base, m, n, row_ptr, col_indx, vals);
}
perflibs_status_t perflibs_spmat_export_dense_s(perflibs_const_spmat_t A,
                                                enum perflibs_dense_layout layout,
                                                perflibs_int_t *m, perflibs_int_t *n,
                                                float **vals) {
  return export_dense<float>(A, layout, m, n, vals);
}
perflibs_status_t perflibs_spmat_export_dense_d(perflibs_const_spmat_t A,
                                                enum perflibs_dense_layout layout,
                                                perflibs_int_t *m, perflibs_int_t *n,
                                                double **vals) {
  return export_dense<double>(A, layout, m, n, vals);
}

perflibs_status_t perflibs_spnorm_exec_s(perflibs_spmat_t A, enum perflibs_sparse_norm nrm,
                                         float *result) {
  return spnorm<float>(A, nrm, result);
}
perflibs_status_t perflibs_spnorm_exec_d(perflibs_spmat_t A, enum perflibs_sparse_norm nrm,
                                         double *result) {
  return spnorm<double>(A, nrm, result);
}

// Error report in the style of the reference's sparse_print_err
// (src/vector_state.cpp:258-282).
void perflibs_spmat_print_err(perflibs_spmat_t A) {
  if (!A)
    return;
  const char *banner = "** libplsparse_b200 ** ";
  if (A->err_type == PERFLIBS_STATUS_EXECUTION_FAILURE) {
    std::fprintf(stderr, "%sExecution failed: %s\n", banner,
                 A->err_msg.empty() ? "unexpected failure" : A->err_msg.c_str());
  } else if (A->err_type == PERFLIBS_STATUS_INPUT_PARAMETER_ERROR) {
    std::fprintf(stderr, "%sParameter error: parameter %d caused an error.\n", banner,
                 A->err_code);
    if (!A->err_msg.empty())
      std::fprintf(stderr, "%s%s\n", banner, A->err_msg.c_str());
  }
}

// ---------------------------------------------------------- extensions

perflibs_status_t perflibs_b200_spmat_set_spmm_path(perflibs_spmat_t A, int32_t path) {
  if (!A || path < -1 || path > 5)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->csr.tiles.forced = path;
  A->csr.tiles.choice_sig = -1;
  A->csr.tiles.last_path = -1;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_set_host_bands(perflibs_spmat_t A, int32_t n_bands) {
  if (!A || n_bands < 0 || n_bands > kMaxHostBands)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->host_bands = n_bands;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_tune_source(perflibs_spmat_t A, int32_t *source) {
  if (!A || !source)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  *source = (int32_t)A->tune_source;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_host_bands_used(perflibs_spmat_t A, int32_t *n_bands) {
  if (!A || !n_bands)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  *n_bands = A->last_host_bands;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_spmm_info(perflibs_spmat_t A, int32_t *tile_rows,
                                                int64_t *staged_rows, int64_t *runs,
                                                int32_t *path, float *ms_staged, float *ms_rows) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const TileDev &t = A->csr.tiles;
  if (tile_rows)
    *tile_rows = t.filled ? t.R : 0;
  if (staged_rows)
    *staged_rows = t.filled ? t.total_uniq : 0;
  if (runs)
    *runs = t.filled ? t.n_runs : 0;
  if (path)
    *path = t.last_path;
  if (ms_staged)
    *ms_staged = t.choice_sig >= 0 ? t.ms_staged : 0.f;
  if (ms_rows)
    *ms_rows = t.choice_sig >= 0 ? t.ms_rows : 0.f;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_get_error(perflibs_const_spmat_t A, int32_t *type,
                                                int32_t *code, char *msg, int32_t msg_len) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (type)
    *type = A->err_type;
  if (code)
    *code = A->err_code;
  if (msg && msg_len > 0) {
    const size_t n = std::min<size_t>(A->err_msg.size(), (size_t)msg_len - 1);
    std::memcpy(msg, A->err_msg.data(), n);
    msg[n] = 0;
  }
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmv_exec_d_dev(enum perflibs_sparse_hint_value trans,
                                                double alpha, perflibs_spmat_t A,
                                                const double *x, double beta, double *y,
                                                void *stream) {
  return spmv_exec_dev<double>(trans, alpha, A, x, beta, y, stream);
}
perflibs_status_t perflibs_b200_spmv_exec_s_dev(enum perflibs_sparse_hint_value trans,
                                                float alpha, perflibs_spmat_t A, const float *x,
                                                float beta, float *y, void *stream) {
  return spmv_exec_dev<float>(trans, alpha, A, x, beta, y, stream);
}

// No device allocation on this path: no staging buffers, no format or
// storage conversion, no tuning — only the SELL kernels, with their
// partial sums in the library's fixed scratch array.
perflibs_status_t perflibs_b200_spmv_exec_d_noalloc(double alpha, perflibs_spmat_t A,
                                                    const double *x, double beta, double *y,
                                                    void *stream) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (A->dt != Dt::F64)
      return param_error(A, 2, "The matrix handle has a different data type.");
    if (A->fmt != Fmt::SELL)
      return param_error(A, 2, "The allocation-free SpMV needs a handle holding its SELL-C-sigma "
                               "layout (optimize it first).");
    if (A->sell.vt != A->csr.evt())
      return param_error(A, 2, "The storage mode changed since optimize; optimize again.");
    if (!x || !y)
      return param_error(A, !x ? 3 : 5);
    DeviceGuard g(A->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : stream_of(A);
    if (alpha == 0.0) {
      scal<double>(A->m, beta, y, s);
      return PERFLIBS_STATUS_SUCCESS;
    }
    spmv_sell_noalloc(A->sell, x, y, alpha, beta, A->device, s);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

}  // extern "C"

template <class X>
static perflibs_status_t spmm_dev(X alpha, Mat *A, const X *B, int64_t ldb, int32_t k, X beta,
                                  X *C, int64_t ldc, void *stream) {
  if (!A || k < 0 || ldb < k || ldc < k)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (!matches<X>(A) || !is_sparse(A->fmt))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    DeviceGuard g(A->device);
    prepare_values(A);
    cudaStream_t s = stream ? (cudaStream_t)stream : stream_of(A);
    if (A->fmt == Fmt::BSR)
      spmm_bsr<X>(A->bsr, B, ldb, C, ldc, k, alpha, beta, s, A->csr.tiles);
    else
    {
      spmm_predict(A, k);
      spmm_csr<X>(A->csr, A->m, B, ldb, C, ldc, k, alpha, beta, s);
    }
    return PERFLIBS_STATUS_SUCCESS;
  });
}

extern "C" {

perflibs_status_t perflibs_b200_spmm_exec_d_dev(double alpha, perflibs_spmat_t A,
                                                const double *B, int64_t ldb, int32_t k,
                                                double beta, double *C, int64_t ldc,
                                                void *stream) {
  return spmm_dev<double>(alpha, A, B, ldb, k, beta, C, ldc, stream);
}
perflibs_status_t perflibs_b200_spmm_exec_s_dev(float alpha, perflibs_spmat_t A, const float *B,
                                                int64_t ldb, int32_t k, float beta, float *C,
                                                int64_t ldc, void *stream) {
  return spmm_dev<float>(alpha, A, B, ldb, k, beta, C, ldc, stream);
}

perflibs_status_t perflibs_b200_spmat_set_storage(perflibs_spmat_t A, int storage) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (storage != PERFLIBS_B200_STORAGE_NATIVE && storage != PERFLIBS_B200_STORAGE_FP32 &&
      storage != PERFLIBS_B200_STORAGE_BF16)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->storage = storage;
  A->tuned = false;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_set_tuner(perflibs_spmat_t A, int mode) {
  if (!A || mode < PERFLIBS_B200_TUNE_EXHAUSTIVE || mode > PERFLIBS_B200_TUNE_NONE)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->tuner = mode;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_force_config(perflibs_spmat_t A, int kind, int C,
                                                   int sigma, int tpr) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  SpmvConfig c;
  if (kind == PERFLIBS_B200_KIND_SELL) {
    if (C != 8 && C != 16 && C != 32)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (sigma < 0 || (sigma != 0 && sigma % C != 0) || sigma > 16384)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    c.kind = Kind::SELL;
    c.C = C;
    c.sigma = sigma;
  } else if (kind == PERFLIBS_B200_KIND_CSR) {
    if (tpr != 0 && tpr != 1 && tpr != 2 && tpr != 4 && tpr != 8 && tpr != 16 && tpr != 32)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    c.kind = Kind::CSR_VECTOR;
    c.tpr = tpr;
  } else if (kind == PERFLIBS_B200_KIND_CSR_SPLIT) {
    c.kind = Kind::CSR_SPLIT;
    c.tpr = tpr > 0 ? tpr : 1024;
  } else {
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  }
  A->forced = true;
  A->forced_cfg = c;
  A->tuned = false;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_get_config(perflibs_spmat_t A, int *kind, int *C,
                                                 int *sigma, int *tpr, int *col_bytes) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const bool sell = A->fmt == Fmt::SELL;
  if (kind)
    *kind = sell ? PERFLIBS_B200_KIND_SELL
                 : (A->cfg.kind == Kind::CSR_SPLIT ? PERFLIBS_B200_KIND_CSR_SPLIT
                                                   : PERFLIBS_B200_KIND_CSR);
  if (C)
    *C = sell ? A->sell.C : 0;
  if (sigma)
    *sigma = sell ? A->sell.sigma : 0;
  if (tpr)
    *tpr = sell ? 0 : A->cfg.tpr;
  if (col_bytes)
    *col_bytes = sell ? A->sell.col_bytes : 4;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_exec_info(perflibs_spmat_t A, int32_t *kernels_per_spmv,
                                                int64_t *n_items, int64_t *n_split) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  int32_t k = 1;
  if (A->fmt == Fmt::CSR && A->cfg.kind == Kind::CSR_SPLIT)
    k = A->csr.n_long > 0 ? 2 : 1;
  if (kernels_per_spmv)
    *kernels_per_spmv = k;
  if (n_items)
    *n_items = A->fmt == Fmt::SELL ? A->sell.n_items : 0;
  if (n_split)
    *n_split = A->fmt == Fmt::SELL ? A->sell.n_split : 0;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_tune_table(perflibs_spmat_t A, int32_t cap, int32_t *cfg4,
                                                 double *ms, double *beta, int32_t *count) {
  if (!A || !count)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const int32_t n = (int32_t)A->tune_table.size();
  for (int32_t i = 0; i < std::min(n, cap); ++i) {
    const auto &t = A->tune_table[i];
    if (cfg4) {
      cfg4[4 * i + 0] = (int)t.cfg.kind;
      cfg4[4 * i + 1] = t.cfg.C;
      cfg4[4 * i + 2] = t.cfg.sigma;
      cfg4[4 * i + 3] = t.cfg.tpr;
    }
    if (ms)
      ms[i] = t.ms;
    if (beta)
      beta[i] = t.beta;
  }
  *count = n;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_build_sell(perflibs_spmat_t A, int C, int sigma) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (C <= 0 || sigma < 0 || (sigma != 0 && sigma % C != 0))
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    DeviceGuard g(A->device);
    bsr_become_csr(A);
    if (A->fmt != Fmt::CSR && A->fmt != Fmt::SELL)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    prepare_values(A);
    A->fmt = Fmt::CSR;
    A->sell = SellDev{};
    SellDev S;
    build_sell(A->csr, A->m, C, sigma, S, stream_of(A));
    A->sell = std::move(S);
    A->fmt = Fmt::SELL;
    A->cfg.kind = Kind::SELL;
    A->cfg.C = C;
    A->cfg.sigma = sigma;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_spmat_export_sell(perflibs_spmat_t A, int64_t *info7, int64_t *cs,
                                                  int64_t *cl, int64_t *col_min,
                                                  int64_t *permd2in, int64_t *in2permd,
                                                  void *vals, void *offsets) {
  if (!A || A->fmt != Fmt::SELL)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    DeviceGuard g(A->device);
    const SellDev &S = A->sell;
    if (info7) {
      info7[0] = S.nC;
      info7[1] = S.C;
      info7[2] = S.sigma;
      info7[3] = S.col_bytes;
      info7[4] = S.n_full_chunks;
      info7[5] = S.ntidyup;
      info7[6] = S.size;
    }
    auto widen32 = [&](const DevBuf &b, int64_t n, int64_t *out) {
      if (!out || n <= 0)
        return;
      std::vector<int32_t> h(n);
      PLS_CUDA(cudaMemcpy(h.data(), b.p, 4 * n, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < n; ++i)
        out[i] = h[i];
    };
    if (cs && S.nC > 0)
      PLS_CUDA(cudaMemcpy(cs, S.cs.p, 8 * S.nC, cudaMemcpyDeviceToHost));
    widen32(S.cl, S.nC, cl);
    widen32(S.col_min, S.nC, col_min);
    widen32(S.permd2in, S.nC * S.C, permd2in);
    if (in2permd) {
      widen32(S.in2permd, A->m, in2permd);
      for (int64_t i = A->m; i < S.nC * S.C; ++i)
        in2permd[i] = -1;
    }
    if (vals && S.size > 0)
      PLS_CUDA(cudaMemcpy(vals, S.vals.p, vt_size(S.vt) * S.size, cudaMemcpyDeviceToHost));
    if (offsets && S.size > 0)
      PLS_CUDA(cudaMemcpy(offsets, S.offsets.p, (size_t)S.col_bytes * S.size,
                          cudaMemcpyDeviceToHost));
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_spmat_set_stream(perflibs_spmat_t A, void *stream) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->stream = (cudaStream_t)stream;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_csr_to_bsr(perflibs_spmat_t A, int32_t bs, int layout,
                                                 perflibs_spmat_t *out) {
  if (!A || !out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    if (A->fmt != Fmt::CSR && A->fmt != Fmt::SELL)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (bs <= 0 || A->m % bs != 0 || A->n % bs != 0)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    if (layout != PERFLIBS_ROW_MAJOR && layout != PERFLIBS_COL_MAJOR)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    DeviceGuard g(A->device);
    std::unique_ptr<Mat> B(new_mat(A->dt, Fmt::BSR));  // freed if the conversion throws
    B->m = A->m;
    B->n = A->n;
    B->index_base = A->index_base;
    B->stream = A->stream;
    csr_to_bsr(A->csr, A->m, A->n, bs, layout, B->bsr, stream_of(A));
    B->bsr.vt = A->csr.vt;
    B->nnz = B->bsr.nnzb * (int64_t)bs * bs;
    *out = B.release();
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_spmat_export_bsr_d(perflibs_spmat_t A, int32_t *bs,
                                                   int32_t *nnzb, int32_t **row_ptr,
                                                   int32_t **col_indx, double **vals) {
  if (!A || A->fmt != Fmt::BSR || A->dt != Dt::F64 || !bs || !nnzb || !row_ptr || !col_indx ||
      !vals)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    DeviceGuard g(A->device);
    const BsrDev &b = A->bsr;
    const int64_t E = (int64_t)b.bs * b.bs;
    auto *rp = (int32_t *)std::malloc(4 * (b.mb + 1));
    auto *c = (int32_t *)std::malloc(4 * std::max<int64_t>(b.nnzb, 1));
    auto *v = (double *)std::malloc(8 * std::max<int64_t>(b.nnzb * E, 1));
    if (!rp || !c || !v) {
      std::free(rp);
      std::free(c);
      std::free(v);
      return PERFLIBS_STATUS_EXECUTION_FAILURE;
    }
    PLS_CUDA(cudaMemcpy(rp, b.row_ptr.p, 4 * (b.mb + 1), cudaMemcpyDeviceToHost));
    if (b.nnzb > 0) {
      PLS_CUDA(cudaMemcpy(c, b.col.p, 4 * b.nnzb, cudaMemcpyDeviceToHost));
      PLS_CUDA(cudaMemcpy(v, b.vals.p, 8 * b.nnzb * E, cudaMemcpyDeviceToHost));
    }
    for (int32_t i = 0; i <= b.mb; ++i)
      rp[i] += A->index_base;
    for (int64_t i = 0; i < b.nnzb; ++i)
      c[i] += A->index_base;
    *bs = b.bs;
    *nnzb = (int32_t)b.nnzb;
    *row_ptr = rp;
    *col_indx = c;
    *vals = v;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_spmat_create_csr_d_dev(perflibs_spmat_t *out, int32_t m,
                                                      int32_t n, const int32_t *row_ptr,
                                                      const int32_t *col_indx, const double *vals,
                                                      void *stream) {
  if (!out)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  Mat *A = nullptr;
  try {
    A = new_mat(Dt::F64, Fmt::CSR);
  } catch (const Error &e) {
    *out = nullptr;
    return e.status;
  } catch (...) {
    *out = nullptr;
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
  *out = A;
  return guarded(A, [&]() -> perflibs_status_t {
    if (m < 0)
      return param_error(A, 2);
    if (n < 0)
      return param_error(A, 3);
    if (!row_ptr)
      return param_error(A, 4);
    // With no stream named, the arrays may still be being written on any
    // stream (the library's own stream does not wait for the legacy default
    // stream), so wait for all prior work on the device first.
    if (!stream)
      PLS_CUDA(cudaDeviceSynchronize());
    cudaStream_t s = stream ? (cudaStream_t)stream : stream_of(A);
    int32_t ends[2] = {0, 0};
    PLS_CUDA(cudaMemcpyAsync(&ends[0], row_ptr, 4, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaMemcpyAsync(&ends[1], row_ptr + m, 4, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    if (ends[0] != 0 && ends[0] != 1)
      return param_error(A, 4);
    A->m = m;
    A->n = n;
    A->index_base = ends[0];
    A->nnz = (int64_t)ends[1] - ends[0];
    if (A->nnz < 0)
      return param_error(A, 4, "row_ptr[m] is below row_ptr[0]");
    CsrDev &c = A->csr;
    c.nnz = A->nnz;
    c.ncols = n;
    c.vt = Vt::F64;
    c.row_ptr.reserve(4 * ((size_t)m + 1));
    c.col.reserve(std::max<size_t>(4 * A->nnz, 16));
    c.vals.reserve(std::max<size_t>(8 * A->nnz, 16));
    PLS_CUDA(cudaMemcpyAsync(c.row_ptr.p, row_ptr, 4 * ((size_t)m + 1), cudaMemcpyDeviceToDevice, s));
    if (A->nnz) {
      PLS_CUDA(cudaMemcpyAsync(c.col.p, col_indx, 4 * A->nnz, cudaMemcpyDeviceToDevice, s));
      PLS_CUDA(cudaMemcpyAsync(c.vals.p, vals, 8 * A->nnz, cudaMemcpyDeviceToDevice, s));
    }
    if (A->index_base) {
      k_sub_base<<<(unsigned)div_up((int64_t)m + 1, 256), 256, 0, s>>>((int64_t)m + 1, 1,
                                                                        c.row_ptr.as<int32_t>());
      if (A->nnz)
        k_sub_base<<<(unsigned)div_up(A->nnz, 256), 256, 0, s>>>(A->nnz, 1, c.col.as<int32_t>());
      PLS_LAUNCH_CHECK();
    }
    const auto bad = check_compressed(m, n, A->nnz, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), s);
    if (bad.first >= 0)
      return param_error(A, 4, "row_ptr decreases or leaves [0, nnz] at row " + std::to_string(bad.first));
    if (bad.second >= 0)
      return param_error(A, 5, "col_indx[" + std::to_string(bad.second) + "] is outside [0, n)");
    A->cfg = default_config(A);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_spmat_features(perflibs_spmat_t A, float *features) {
  if (!A || !features)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return guarded(A, [&]() -> perflibs_status_t {
    DeviceGuard g(A->device);
    bsr_become_csr(A);
    if (A->fmt != Fmt::CSR && A->fmt != Fmt::SELL)
      return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
    compute_features(A, features);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_tune_candidates(int32_t cap, int32_t *cfg4, int32_t *count) {
  if (!count)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  const auto c = tune_candidates(nullptr);
  for (int32_t i = 0; i < std::min<int32_t>(cap, (int32_t)c.size()); ++i) {
    if (cfg4) {
      cfg4[4 * i + 0] = (int)c[i].kind;
      cfg4[4 * i + 1] = c[i].C;
      cfg4[4 * i + 2] = c[i].sigma;
      cfg4[4 * i + 3] = c[i].tpr;
    }
  }
  *count = (int32_t)c.size();
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_set_spmm_selectors(perflibs_spmat_t A,
                                                         const perflibs_b200_selector_t *S) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  for (int b = 0; b < 3; ++b)
    if (S && S[b] && selector_classes(S[b]) != kSpmmClasses)
      return param_error(A, 2, "An SpMM selector must have 5 classes (the SpMM kernels).");
  for (int b = 0; b < 3; ++b)
    A->spmm_selector[b] = S ? S[b] : nullptr;
  A->csr.tiles.pred_n = 0;
  A->csr.tiles.pred_bucket = -1;
  A->csr.tiles.choice_sig = -1;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_spmat_set_selector(perflibs_spmat_t A, perflibs_b200_selector_t S) {
  if (!A)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  A->selector = S;
  A->tuned = false;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_device_info(int32_t *sm_count, int64_t *l2_bytes,
                                            int32_t *device) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  int sms = 0, l2 = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) != cudaSuccess ||
      cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, d) != cudaSuccess)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  if (sm_count)
    *sm_count = sms;
  if (l2_bytes)
    *l2_bytes = l2;
  if (device)
    *device = d;
  return PERFLIBS_STATUS_SUCCESS;
}

const char *perflibs_b200_version(void) { return "libplsparse_b200 0.1 (sm_100a)"; }

}  // extern "C"
