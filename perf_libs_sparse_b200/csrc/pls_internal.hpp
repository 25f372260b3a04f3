// Internal types of libplsparse_b200: the matrix handle, device buffers,
// kernel configurations and the launchers each .cu file provides.
//
// Data layout in HBM (all device arrays are 0-based; the user's index base is
// remembered only for export):
//   CSR   row_ptr int32[m+1], col int32[nnz], vals V[nnz]
//   SELL  cs int64[nC] (chunk start), cl int32[nC] (chunk width),
//         col_min int32[nC], permd2in int32[nC*C] (-1 = padding row),
//         in2permd int32[m], vals V[size], offsets u8/u16/u32/u64[size]
//         (column offset from col_min, width = col_bytes), column-major
//         within each chunk: element (row r, column j) of chunk c sits at
//         cs[c] + j*C + r. This is the reference's SELL-C-sigma layout
//         (src/sell_c_sigma.hpp:43-104) element for element.
//   BSR   row_ptr int32[mb+1], col int32[nnzb], vals V[nnzb*bs*bs] in the
//         user's block layout (row- or column-major blocks)
//   DENSE vals T[m*n] packed (lda = n row-major, lda = m column-major)
// V is the value storage type: the API type (float / double) by default, or
// float / bf16 under the reduced-precision storage modes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "dia_plan.hpp"

#include "../../include/perflibs_b200.h"
#include "../../include/perflibs_sparse.h"

namespace pls {

// ------------------------------------------------------------ errors

struct Error : std::runtime_error {
  perflibs_status_t status;
  Error(perflibs_status_t s, const std::string &m)
      : std::runtime_error(m), status(s) {}
};

// Runs f (which returns a status) so that no exception leaves a C entry
// point: an Error gives its status, anything else (host allocation failure
// included) EXECUTION_FAILURE.
template <class F> perflibs_status_t status_guard(F &&f) noexcept {
  try {
    return f();
  } catch (const Error &e) {
    return e.status;
  } catch (...) {
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  }
}

#define PLS_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      throw ::pls::Error(PERFLIBS_STATUS_EXECUTION_FAILURE,                    \
                         std::string(#call) + ": " + cudaGetErrorString(e_) + \
                             " (" + __FILE__ + ":" + std::to_string(__LINE__) +\
                             ")");                                             \
  } while (0)

#define PLS_LAUNCH_CHECK() PLS_CUDA(cudaGetLastError())

// A pair of timing events, destroyed with the object, also when a timed run
// throws.
struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EventPair() {
    PLS_CUDA(cudaEventCreate(&e0));
    const cudaError_t r = cudaEventCreate(&e1);
    if (r != cudaSuccess) {
      cudaEventDestroy(e0);
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                  std::string("cudaEventCreate: ") + cudaGetErrorString(r));
    }
  }
  EventPair(const EventPair &) = delete;
  EventPair &operator=(const EventPair &) = delete;
  ~EventPair() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
};

// An NVTX range over a library call (optimize, host-pointer exec, SpMM,
// batch tuning), visible in Nsight timelines; free when no tool listens.
// The device-pointer SpMV entry points, the per-iteration hot path, carry
// none, so callers' own ranges around them stay the innermost.
struct TraceRange {
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

// ------------------------------------------------------------ device buffer

#ifdef PLS_DEBUG_GUARDS
// Guard build (libplsparse_b200_guard.so): every device buffer is followed
// by kGuardBytes of 0xFF bytes, NaN as FP64 / FP32 words and -1 as indices.
// A kernel that writes past a buffer's end changes them, and release()
// counts that (perflibs_b200_debug_guard_violations); one that reads past
// the end reads NaN into its result, which the comparison with the oracle
// catches. compute-sanitizer is the tool for this, and it is not available
// on every machine.
constexpr size_t kGuardBytes = 4096;
void guard_arm(void *end);                  // fill the guard (debug.cu)
void guard_check(const void *end) noexcept;  // verify it, count a violation
#endif

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) {
#ifdef PLS_DEBUG_GUARDS
      guard_check(static_cast<char *>(p) + bytes);
#endif
      cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
  }
  // Grow to at least `b` bytes (contents not kept).
  void reserve(size_t b) {
    if (b <= bytes && p)
      return;
    release();
    if (b == 0)
      b = 16;
#ifdef PLS_DEBUG_GUARDS
    PLS_CUDA(cudaMalloc(&p, b + kGuardBytes));
    guard_arm(static_cast<char *>(p) + b);
#else
    PLS_CUDA(cudaMalloc(&p, b));
#endif
    bytes = b;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// ------------------------------------------------------------ enums

enum class Dt : int { F32 = 0, F64 = 1 };
enum class Fmt : int { CSR, BSR, DENSE, NUL, IDENTITY, SELL };
enum class Vt : int { F64 = 0, F32 = 1, BF16 = 2 };  // value storage type

inline size_t vt_size(Vt v) {
  return v == Vt::F64 ? 8 : v == Vt::F32 ? 4 : 2;
}

template <class T> struct Tag { using type = T; };

// Call f(Tag<V>) with the C++ type of a value storage type.
template <class F> void with_vt(Vt vt, F &&f) {
  switch (vt) {
  case Vt::F64: f(Tag<double>{}); break;
  case Vt::F32: f(Tag<float>{}); break;
  case Vt::BF16: f(Tag<__nv_bfloat16>{}); break;
  }
}

// SpMV kernel families the tuner chooses between.
enum class Kind : int { CSR_VECTOR = 0, SELL = 1, CSR_SPLIT = 2 };

struct SpmvConfig {
  Kind kind = Kind::CSR_VECTOR;
  int tpr = 0;   // threads per row (CSR_VECTOR), 0 = pick by mean row length
  int C = 32;    // SELL chunk height
  int sigma = 0; // SELL sort window in rows (0 = no sort)
};

// ------------------------------------------------------------ formats

// Rows [r0, r1) of an SpMV run as one band of a host-buffer call: the band's
// kernels write exactly these rows of y, so the copy of one band's rows to
// the host overlaps the kernels of the next band. For SELL, [c0, c1) are the
// band's chunks (whole sort windows) and [i0, i1) its column slices in the
// plan's arrays; for CSR, [i0, i1) are its long rows.
struct RowBand {
  int64_t r0 = 0, r1 = 0;
  int64_t c0 = 0, c1 = 0;
  int64_t i0 = 0, i1 = 0;
};

// Bands of one layout, built on the first host-buffer call that uses them.
// SELL: `order` holds each band's chunks in the layout's processing order
// (empty when the layout has none); `items` the column slices of the band
// plan's own, finer slicing (chunks wider than split_w), grouped by band,
// with their partial sums in `part` and completion counts in `done`. CSR:
// `order` holds the long rows in increasing order.
struct BandPlan {
  int planned = 0;  // band count asked for when built; 0 = not built
  std::vector<RowBand> bands;
  DevBuf order, items, part, done;
  int32_t split_w = INT32_MAX;
  void clear() {
    planned = 0;
    bands.clear();
    order.release();
    items.release();
    part.release();
    done.release();
    split_w = INT32_MAX;
  }
};

// The copy stream and events of banded host-buffer calls, created on first
// use on the handle's GPU: event i marks the end of band i's kernels on the
// handle's stream, and the copy stream waits for it before copying the
// band's rows of y to the host.
struct BandLanes {
  cudaStream_t copy = nullptr;
  std::vector<cudaEvent_t> ev;
  BandLanes() = default;
  BandLanes(const BandLanes &) = delete;
  BandLanes &operator=(const BandLanes &) = delete;
  ~BandLanes() {
    for (cudaEvent_t e : ev)
      cudaEventDestroy(e);
    if (copy)
      cudaStreamDestroy(copy);
  }
  cudaStream_t copy_stream() {
    if (!copy)
      PLS_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
    return copy;
  }
  cudaEvent_t event(size_t i) {
    while (ev.size() <= i) {
      cudaEvent_t e;
      PLS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev.push_back(e);
    }
    return ev[i];
  }
};

// A 4-byte flag in mapped pinned host memory: kernels write it through the
// device pointer, the host reads it without synchronising.
struct HostFlag {
  int *host = nullptr;
  int *dev = nullptr;
  HostFlag() = default;
  HostFlag(const HostFlag &) = delete;
  HostFlag &operator=(const HostFlag &) = delete;
  HostFlag(HostFlag &&o) noexcept : host(o.host), dev(o.dev) { o.host = o.dev = nullptr; }
  HostFlag &operator=(HostFlag &&o) noexcept {
    if (this != &o) {
      release();
      host = o.host;
      dev = o.dev;
      o.host = o.dev = nullptr;
    }
    return *this;
  }
  ~HostFlag() { release(); }
  void release() {
    if (host)
      cudaFreeHost(host);
    host = dev = nullptr;
  }
  void alloc() {
    if (host)
      return;
    void *h = nullptr, *d = nullptr;
    PLS_CUDA(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
    *(volatile int *)h = 0;
    PLS_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    host = (int *)h;
    dev = (int *)d;
  }
};

// Row-block tiles of the staged SpMM (spmm_tiled.cu): for every block of R
// rows, its distinct columns as runs (c0, len, u0) and every nonzero's row
// in the staged tile.
struct TileDev {
  int R = 0;
  int64_t nblocks = 0;
  int32_t max_uniq = 0, max_bnnz = 0;
  int64_t total_uniq = 0, n_runs = 0;
  bool filled = false;
  // Smallest tile row width (bytes) found unsuitable (INT64_MAX: none).
  int64_t unsuitable_from = INT64_MAX;
  DevBuf nuniq, run_ptr, runs, local;
  HostFlag err;
  // Measured choice between the SpMM kernels for the call signature
  // `choice_sig` (k, ldb, value and API types): 0 row group 64-bit offsets,
  // 2 row group 32-bit, 3 row group with shared entries, 1 staged, 4
  // diagonal form, 5 diagonal form with TMA-staged B, -1 not measured; with
  // the staged and the best row-group timing (ms).
  int64_t choice_sig = -1;
  int choice = -1;
  float ms_staged = 0.f, ms_rows = 0.f;
  // Path forced by perflibs_b200_spmat_set_spmm_path: -1 measured choice,
  // 0 row group, 1 staged (when it applies), 2 row group with shared entries
  // (when the lane shape allows them), 3 diagonal form (when it applies), 4
  // diagonal form with TMA-staged B (when it applies, else 3 when that does).
  int forced = -1;
  // Kernel order predicted by the learned SpMM selector for the current
  // call's k (classes kSpmmClass*, most probable first; pred_n = 0 when no
  // selector is attached): a new call signature takes the first kernel of
  // the order that applies instead of timing the candidates.
  int pred_order[5] = {};
  int pred_n = 0;
  int pred_bucket = -1;
  bool predicted = false;  // the kept choice came from the selector
  // Path of the last SpMM: 1 staged, 0 row group, 2 row group with shared
  // entries, 3 diagonal form, 4 diagonal form with TMA-staged B.
  int last_path = -1;
};

// Diagonal form of a CSR matrix for SpMM (built on the first SpMM that
// measures the kernel choice): every entry (r, c) lies on one of nd
// diagonals c - r = offs[d] (ascending); vals holds, for every block of
// kDiaRows rows and every diagonal, the block's kDiaRows values in the
// kernels' value type (an absent entry is a reserved NaN bit pattern the
// kernel skips). The blocks continue kDiaPadRows rows past the last row,
// all absent, so that a copy of any kDiaPadRows rows starting at a row of
// the matrix stays inside the buffer (kDiaRows, kDiaMax and kDiaPadRows are
// in dia_plan.hpp). state: 0 not examined, 1 built, -1 unsuitable.
struct DiaDev {
  int state = 0;
  int nd = 0;
  int32_t offs[kDiaMax] = {};
  DevBuf vals;
  // Per block of kDiaRows rows (padded like vals): bit d set when every row
  // of the block stores an entry on diagonal d.
  DevBuf full;
  // What was examined: vals_version, type and buffer of the kernels' values
  // (a change of any of them means examining the matrix again).
  uint64_t version = 0;
  Vt vt = Vt::F64;
  const void *src = nullptr;
  // Set (mapped host memory) by the TMA-staged kernel when a copy did not
  // land within its wait limit; reported by the next call.
  HostFlag err;
};

// Bounded waits of the kernels that stage through mbarriers: the poll limit
// (2^22, about a second) and, for failure-path tests only, bytes an mbarrier
// expects beyond what is copied (perflibs_b200_testing_stage_fault).
extern std::atomic<int> g_stage_wait_limit;
extern std::atomic<int> g_stage_shortfall;

struct CsrDev {
  DevBuf row_ptr, col, vals;  // vals in the API type (authoritative)
  int64_t nnz = 0;
  uint64_t vals_version = 0;  // counts value updates (invalidates value copies)
  int32_t ncols = 0;  // columns (bound of col); 0 when not recorded
  Vt vt = Vt::F64;
  // Reduced-precision copy of the values used by the kernels when the
  // handle's storage mode asks for one.
  DevBuf vals_lo;
  Vt vt_lo = Vt::F64;
  bool lo = false;
  const void *ev() const { return lo ? vals_lo.p : vals.p; }
  Vt evt() const { return lo ? vt_lo : vt; }
  // Rows longer than the split threshold, processed by the row-split
  // kernel family (built on demand).
  DevBuf long_rows;
  int n_long = 0;
  int long_threshold = 0;
  // Staged-SpMM tiles (built on the first suitable SpMM).
  TileDev tiles;
  DiaDev dia;
  BandPlan bands;
};

struct SellDev {
  int C = 0, sigma = 0;
  int64_t nC = 0, size = 0;
  int col_bytes = 0;
  int64_t n_full_chunks = 0, ntidyup = 0;
  int32_t max_width = 0;
  DevBuf cs, cl, col_min, permd2in, in2permd, vals, offsets;
  Vt vt = Vt::F64;
  // Column slices (chunk, j0, j1, slot) of the chunks wider than split_w;
  // empty when no chunk is sliced.
  DevBuf items;
  int64_t n_items = 0;
  int slice_w = 0;
  int32_t split_w = INT32_MAX;
  int64_t n_split = 0;  // chunks split into slices
  DevBuf part;          // partial sums of the split chunks' slices (scratch)
  DevBuf done;          // per slot: slices of its chunk finished (0 between launches)
  // Chunk indices by decreasing width (stable); the SpMV kernel takes chunks
  // in this order. Empty when all chunks have the same width.
  DevBuf order;
  BandPlan bands;
};

struct BsrDev {
  int bs = 0;
  int layout = PERFLIBS_ROW_MAJOR;
  int32_t mb = 0, nb = 0;
  int64_t nnzb = 0;
  DevBuf row_ptr, col, vals;
  Vt vt = Vt::F64;
  DevBuf vals_lo;
  Vt vt_lo = Vt::F64;
  bool lo = false;
  uint64_t vals_version = 0;  // counts rebuilds of the kernels' values
  const void *ev() const { return lo ? vals_lo.p : vals.p; }
  Vt evt() const { return lo ? vt_lo : vt; }
  // Tensor-core SpMM (spmm_bsr_tc.cu): the values as FP32 operand blocks
  // (built from ev() at vals_version), its error flag, and the measured
  // choice against the FMA kernel for the call signature tc_sig (0 FMA,
  // 1 tensor cores) with both timings (ms).
  DevBuf tc_vals;
  const void *tc_vals_src = nullptr;
  uint64_t tc_vals_version = ~0ull;
  HostFlag tc_err;
  int64_t tc_sig = -1;
  int tc_choice = 0;
  float ms_tc = 0.f, ms_fma = 0.f;
};

struct DenseDev {
  int layout = PERFLIBS_ROW_MAJOR;
  int64_t lda = 0;
  DevBuf vals;  // API type
  bool is_zero = false;
};

// Per-candidate timing recorded by the tuner.
struct TuneEntry {
  SpmvConfig cfg;
  double ms = 0;
  double beta = 1.0;  // SELL padding efficiency (1 for CSR)
};

// Key of the autotune cache: GPU model, dimensions, value types and a hash
// of the sparsity structure (tune_cache.cu).
struct TuneKey {
  std::string dev;
  int32_t m = 0, n = 0;
  int64_t nnz = 0;
  uint64_t hash = 0;
  int dt = 0, vt = 0;
  bool operator<(const TuneKey &o) const {
    return std::tie(dev, m, n, nnz, hash, dt, vt) <
           std::tie(o.dev, o.m, o.n, o.nnz, o.hash, o.dt, o.vt);
  }
};

// How the active SpMV configuration was chosen (perflibs_b200_spmat_tune_source).
enum class TuneSource : int { NONE = 0, TIMED = 1, CACHE = 2, SELECTOR = 3, FORCED = 4 };

}  // namespace pls

// The opaque handle of the C interface.
struct perflibs_spmat_top_t {
  pls::Dt dt = pls::Dt::F64;
  pls::Fmt fmt = pls::Fmt::CSR;
  // The format the user created (CSR / BSR / DENSE / NUL / IDENTITY);
  // `fmt` may move to SELL after optimize, as in the reference.
  pls::Fmt created = pls::Fmt::CSR;
  int32_t m = 0, n = 0;
  int64_t nnz = 0;
  int32_t index_base = 0;
  int device = 0;

  // Hints (reference defaults: src/types.hpp:40-76).
  int hint_structure = PERFLIBS_SPARSE_STRUCTURE_UNSTRUCTURED;
  int hint_memory = PERFLIBS_SPARSE_MEMORY_ALLOCS;
  int hint_spmv_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  int hint_spmv_inv = PERFLIBS_SPARSE_INVOCATIONS_MANY;
  int hint_spmm_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  int hint_spmm_inv = PERFLIBS_SPARSE_INVOCATIONS_MANY;
  int hint_spadd_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  int hint_spadd_inv = PERFLIBS_SPARSE_INVOCATIONS_MANY;
  int hint_spmm_strat = PERFLIBS_SPARSE_SPMM_STRAT_UNSET;
  int hint_spsm_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  int hint_spsv_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  int hint_spsv_inv = PERFLIBS_SPARSE_INVOCATIONS_MANY;
  int hint_spsv_strat = PERFLIBS_SPARSE_SPSV_STRAT_UNSET;
  bool hint_hpcg = false;

  // Error record (reference sp_error_t, src/util.hpp:294-298).
  int err_type = 0;
  int err_code = 0;
  std::string err_msg;

  // Extension state.
  int storage = PERFLIBS_B200_STORAGE_NATIVE;  // requested value storage
  int tuner = PERFLIBS_B200_TUNE_EXHAUSTIVE;
  perflibs_b200_selector_t selector = nullptr;  // not owned
  int selector_class = -1;                      // last prediction
  // SpMM kernel selectors for k <= 16, 17..64 and > 64 (not owned), and the
  // handle's structure features (computed once, on the first prediction).
  perflibs_b200_selector_t spmm_selector[3] = {nullptr, nullptr, nullptr};
  float features[PERFLIBS_B200_NFEATURES] = {};
  bool features_valid = false;
  bool forced = false;
  pls::SpmvConfig forced_cfg;
  pls::SpmvConfig cfg;  // active SpMV kernel configuration
  bool tuned = false;
  int tuned_op = PERFLIBS_SPARSE_OPERATION_NOTRANS;
  std::vector<pls::TuneEntry> tune_table;
  pls::TuneSource tune_source = pls::TuneSource::NONE;
  cudaStream_t stream = nullptr;  // nullptr = library stream

  pls::CsrDev csr;
  pls::SellDev sell;
  pls::BsrDev bsr;
  pls::DenseDev dense;

  // CSR of A^T (built on demand for transposed operations).
  pls::CsrDev csrT;
  bool has_csrT = false;

  // Staging for host-pointer execution.
  pls::DevBuf xbuf, ybuf;
  pls::BandLanes lanes;
  int host_bands = 0;       // row bands of host-buffer SpMV: 0 = by size, 1 = none
  int last_host_bands = 0;  // bands the last host-buffer SpMV ran in (0 = one launch)
};

namespace pls {

using Mat = perflibs_spmat_top_t;

cudaStream_t lib_stream(int device);
cudaStream_t stream_of(const Mat *A);

// ------------------------------------------------------------ launchers
// SpMV: y = alpha*op(A)*x + beta*y on device pointers. X is float/double.
template <class X>
void spmv_csr(const CsrDev &c, int32_t m, int tpr, const X *x, X *y, X alpha,
              X beta, cudaStream_t s);
template <class X>
void spmv_csr_split(const CsrDev &c, int32_t m, const X *x, X *y, X alpha,
                    X beta, cudaStream_t s);
template <class X>
void spmv_sell(const SellDev &s, const X *x, X *y, X alpha, X beta,
               cudaStream_t st);
template <class X>
void spmv_bsr(const BsrDev &b, const X *x, X *y, X alpha, X beta,
              cudaStream_t s);
// Allocation-free FP64 variant of spmv_sell: the slices' partial sums and
// completion counts in fixed device arrays (see spmv.cu).
void spmv_sell_noalloc(const SellDev &s, const double *x, double *y, double alpha, double beta,
                       int device, cudaStream_t st);
// Row bands for host-buffer SpMV: plan about n_bands bands of equal row
// count (kept when already planned for n_bands), then run one band.
void sell_plan_bands(SellDev &s, int64_t m, int n_bands);
void csr_plan_bands(CsrDev &c, int32_t m, int n_bands);
template <class X>
void spmv_sell_band(const SellDev &s, const RowBand &b, const X *x, X *y, X alpha, X beta,
                    cudaStream_t st);
// tpr = 0 runs the long-row split kernels (threshold c.long_threshold).
template <class X>
void spmv_csr_band(const CsrDev &c, const RowBand &b, int tpr, const X *x, X *y, X alpha,
                   X beta, cudaStream_t s);
template <class X>
void spmv_csr_trans(const CsrDev &c, int32_t m, int32_t n, const X *x, X *y,
                    X alpha, X beta, cudaStream_t s);
template <class X>
void spmv_dense(const DenseDev &d, int32_t m, int32_t n, bool trans,
                const X *x, X *y, X alpha, X beta, cudaStream_t s);
template <class X>
void axpby(int64_t n, X alpha, const X *x, X beta, X *y, cudaStream_t s);
template <class X>
void scal(int64_t n, X beta, X *y, cudaStream_t s);

// SpMM: C = alpha*A*B + beta*C, row-major B (ldb) and C (ldc), k columns.
template <class X>
void spmm_csr(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C,
              int64_t ldc, int k, X alpha, X beta, cudaStream_t s);
// Staged SpMM for matrices whose row blocks reuse B rows; false (nothing
// launched) when the matrix, k or B's layout does not suit it. With
// launch = false it only builds the tiles and says whether it applies.
template <class X>
bool spmm_tiled(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                X alpha, X beta, cudaStream_t s, bool launch = true);
// Diagonal-form SpMM (a few diagonals, rows sorted and free of duplicate
// columns, B and C in 16-byte vectors); false
// (nothing launched) when it does not apply. With launch = false it only
// builds the diagonal form and says whether it applies.
template <class X>
bool spmm_dia(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
              X alpha, X beta, cudaStream_t s, bool launch = true);
// The diagonal form with B's rows staged in shared memory by tensor-map
// copies, for diagonal forms whose diagonals fall into groups with evenly
// spaced centres (planes of a 3-D stencil, lines of a 2-D one) or into one
// band; false (nothing launched) when it does not apply. With launch =
// false it only says whether it applies (building the diagonal form).
template <class X>
bool spmm_dia_tma(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                  X alpha, X beta, cudaStream_t s, bool launch = true);
// BSR SpMM: the FMA kernel, or for bs = 8 with BF16 values and FP32 B / C
// the tensor-core kernel (spmm_bsr_tc.cu). `t` carries the forced path (5:
// tensor cores whenever they apply; -1: the faster of the two, measured on
// the first call of each signature) and receives the path taken (5 tensor
// cores, 6 FMA) and, in ms_staged / ms_rows, the measured tensor-core / FMA
// times.
template <class X>
void spmm_bsr(BsrDev &b, const X *B, int64_t ldb, X *C, int64_t ldc, int k, X alpha, X beta,
              cudaStream_t s, TileDev &t);
// Tensor-core BSR SpMM; false (nothing launched) when it does not apply.
bool spmm_bsr_tc(BsrDev &b, const float *B, int64_t ldb, float *C, int64_t ldc, int k,
                 float alpha, float beta, cudaStream_t s, bool launch);

// Layout helpers.
template <class X>
void transpose_dense(const X *in, int64_t rows, int64_t cols, int64_t ldin,
                     X *out, int64_t ldout, cudaStream_t s);
template <class X>
void strided_copy(const X *in, int64_t stride_in, X *out, int64_t stride_out,
                  int64_t n, cudaStream_t s);

// Conversions.
void convert_values(const void *in, Vt vin, void *out, Vt vout, int64_t n,
                    cudaStream_t s);
void build_sell(const CsrDev &c, int32_t m, int C, int sigma, SellDev &out,
                cudaStream_t s);
void sell_build_work_list(SellDev &s, int slice_w, cudaStream_t st);
void build_csr_transpose(const CsrDev &c, int32_t m, int32_t n, CsrDev &out,
                         cudaStream_t s);
void bsr_to_csr(const BsrDev &b, int32_t m, bool drop_zeros, CsrDev &out,
                cudaStream_t s);
// First bad row (pointers decreasing or outside [0, nnz]) and first bad
// entry (index outside [0, cols)) of 0-based compressed device arrays, -1
// when none.
std::pair<int64_t, int64_t> check_compressed(int32_t rows, int32_t cols, int64_t nnz,
                                             const int32_t *ptr, const int32_t *idx,
                                             cudaStream_t s);
// COO (0-based device arrays, any order, duplicates allowed) -> CSR sorted by
// (row, column), duplicates kept in input order. Returns -1, or the first
// entry whose row or column is out of range (then `out` is untouched).
int64_t coo_to_csr(int32_t m, int32_t n, int64_t nnz, const int32_t *row, const int32_t *col,
                   const void *vals, Vt vt, CsrDev &out, cudaStream_t s);
void csr_to_bsr(const CsrDev &c, int32_t m, int32_t n, int bs, int layout,
                BsrDev &out, cudaStream_t s);
void csr_build_long_rows(CsrDev &c, int32_t m, int threshold, cudaStream_t s);

// Norms (double accumulate on device, result to host).
double inf_norm_csr(const CsrDev &c, int32_t m, cudaStream_t s);
double frb_norm_values(const void *vals, Vt vt, int64_t n, cudaStream_t s);
double inf_norm_bsr(const BsrDev &b, cudaStream_t s);
double inf_norm_dense(const DenseDev &d, Dt dt, int32_t m, int32_t n,
                      cudaStream_t s);

// Updates of existing entries: returns index of the first update that does
// not name a stored entry (or n_updates when all were applied).
int64_t update_csr_values(CsrDev &c, SellDev *sell, int32_t m, int32_t n,
                          int64_t n_updates, const int32_t *rows_host,
                          const int32_t *cols_host, const void *vals_host,
                          Dt dt, int32_t base, cudaStream_t s);

// Classes of the learned SpMM selector: the CSR SpMM kernels.
enum SpmmClass { kSpmmRows = 0, kSpmmShared = 1, kSpmmStaged = 2, kSpmmDia = 3, kSpmmDiaTma = 4,
                 kSpmmClasses = 5 };
// The SpMM selector bucket of k: 0 for k <= 16, 1 for 17..64, 2 above.
inline int spmm_bucket(int k) { return k <= 16 ? 0 : (k <= 64 ? 1 : 2); }
// Classes (outputs) of a selector.
int selector_classes(perflibs_b200_selector_t S);

// Statistics for the learned selector (PERFLIBS_B200_NFEATURES floats).
void compute_features(const Mat *A, float *out);
int64_t count_blocks(const CsrDev &c, int32_t m, int32_t n, int bs, cudaStream_t s);
int64_t sell_padded_size(const CsrDev &c, int32_t m, int C, int sigma, cudaStream_t s);

// Tuning.
// Autotune cache: find computes the matrix's key (one device pass over its
// structure) and looks it up; put records a finished tune under it.
bool tune_cache_find(const Mat *A, SpmvConfig &best, std::vector<TuneEntry> &table,
                     TuneKey &key);
void tune_cache_put(const TuneKey &key, const SpmvConfig &best,
                    const std::vector<TuneEntry> &table);
std::vector<SpmvConfig> tune_candidates(const Mat *A);
void tune_spmv(Mat *A);
SpmvConfig default_config(const Mat *A);
double time_config(Mat *A, const SpmvConfig &cfg, int reps);
void apply_config(Mat *A, const SpmvConfig &cfg);

// Execute a configured SpMV on device pointers.
template <class X>
void run_spmv(Mat *A, int op, const X *x, X *y, X alpha, X beta,
              cudaStream_t s);

}  // namespace pls
