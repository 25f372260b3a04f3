// Diagonal-form SpMM for matrices whose entries lie on a few diagonals
// (stencils on structured grids, narrow-band matrices).
//
// On a 27-point stencil the row-group kernel reads 27 rows of B per row of
// A through L1, although rows r and r + 1 share most of them: the stencil's
// diagonals come in runs of consecutive offsets (o - 1, o, o + 1), and for
// kDiaRows = 4 consecutive rows the 3 diagonals of a run read only 6
// distinct rows of B instead of 12. Here each thread owns kDiaRows
// consecutive rows of C and one 16-byte vector of columns; for every run of
// up to kDiaRun consecutive diagonals it loads those kDiaRows + run - 1 rows
// of B once, with consecutive threads on consecutive column vectors, then
// adds the run's diagonals. The column indices are not read at all.
//
// Layout (DiaDev): for each block of kDiaRows rows and each diagonal d (in
// ascending offset), the kDiaRows values of the block's rows on d, so a
// thread loads them with one or two vector loads. An entry that the matrix
// does not store is a reserved NaN bit pattern and is skipped, so a stored
// row adds
// exactly its own entries, in ascending column order: the order of the
// row-group kernel on rows whose columns are sorted, which the diagonal form
// requires (with no duplicate columns). Results are then bit-identical to
// the row-group kernel (one fma per entry into the same accumulator, the
// same epilogue alpha * acc + beta * C).
//
// The form applies when the longest row's offsets cover every entry, there
// are at most kDiaMax diagonals, at least half of the diagonal slots hold
// entries, and B and C rows are 16-byte vectors. Values are kept in the
// type the kernels use (the API type, or the FP32 / BF16 storage copy, with
// FP32 accumulation as in the row-group kernel). It is built on the first
// SpMM that measures the kernel choice and rebuilt after the values or the
// storage mode change.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "pls_internal.hpp"
#include "spmm_rows.cuh"

namespace pls {

namespace {

constexpr int kDiaRun = 3;  // diagonals per run (longer runs are split)

// Reserved bit patterns for "no entry": signalling NaNs with a payload.
constexpr unsigned long long kAbsentD = 0x7FF0DEAD00000001ull;
constexpr unsigned kAbsentF = 0x7F80DEADu;
constexpr unsigned short kAbsentH = 0x7F81u;  // BF16

__device__ __forceinline__ bool dia_absent(double a) {
  return (unsigned long long)__double_as_longlong(a) == kAbsentD;
}
__device__ __forceinline__ bool dia_absent(float a) { return __float_as_uint(a) == kAbsentF; }
__device__ __forceinline__ bool dia_absent(__nv_bfloat16 a) {
  return __bfloat16_as_ushort(a) == kAbsentH;
}
template <class X> __device__ __forceinline__ X dia_absent_value();
template <> __device__ __forceinline__ double dia_absent_value<double>() {
  return __longlong_as_double((long long)kAbsentD);
}
template <> __device__ __forceinline__ float dia_absent_value<float>() {
  return __uint_as_float(kAbsentF);
}
template <> __device__ __forceinline__ __nv_bfloat16 dia_absent_value<__nv_bfloat16>() {
  return __ushort_as_bfloat16(kAbsentH);
}

struct DiaRuns {
  int n;
  int o0[kDiaMax], len[kDiaMax], d0[kDiaMax];
};

struct DiaOffs {
  int nd;
  int32_t o[kDiaMax];
};

// The longest row (length << 32 | row), by a max over all rows.
__global__ void k_dia_longest(int32_t m, const int32_t *__restrict__ rp,
                              unsigned long long *__restrict__ out) {
  unsigned long long best = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m;
       r += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long len = (unsigned long long)(rp[r + 1] - rp[r]);
    best = max(best, (len << 32) | (unsigned long long)r);
  }
  for (int o = 16; o > 0; o >>= 1)
    best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, best);
}

template <class V>
__global__ void k_dia_fill(int64_t count, V *__restrict__ dv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count)
    dv[i] = dia_absent_value<V>();
}

// One thread per row: put each entry on its diagonal. flag bit 1: columns
// not strictly ascending; 2: an offset outside the diagonals; 4: a value
// equal to the reserved pattern.
template <class V>
__global__ void k_dia_scatter(int32_t m, DiaOffs offs, const int32_t *__restrict__ rp,
                              const int32_t *__restrict__ col, const V *__restrict__ val,
                              V *__restrict__ dv, int *__restrict__ flag) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m)
    return;
  int bad = 0;
  int64_t prev = INT64_MIN;
  for (int32_t p = rp[r]; p < rp[r + 1]; ++p) {
    const int64_t c = col[p];
    if (c <= prev)
      bad |= 1;
    prev = c;
    const int64_t o = c - r;
    int lo = 0, hi = offs.nd;  // first offset >= o
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (offs.o[mid] < o)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo == offs.nd || offs.o[lo] != o) {
      bad |= 2;
      continue;
    }
    const V v = val[p];
    if (dia_absent(v)) {
      bad |= 4;
      continue;
    }
    dv[((r / kDiaRows) * offs.nd + lo) * kDiaRows + r % kDiaRows] = v;
  }
  if (bad)
    atomicOr(flag, bad);
}

// The kDiaRows values of one block of rows on one diagonal (8, 16 or 32
// bytes, aligned to their size).
template <class V>
__device__ __forceinline__ void ld_rows_vals(const V *p, V (&a)[kDiaRows]) {
  constexpr int bytes = kDiaRows * (int)sizeof(V);
  static_assert(bytes == 8 || bytes % 16 == 0, "value blocks load as whole vectors");
  if constexpr (bytes == 8) {
    const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
    memcpy(a, &t, 8);
  } else {
#pragma unroll
    for (int i = 0; i < bytes / 16; ++i) {
      const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p) + i);
      memcpy(reinterpret_cast<char *>(a) + 16 * i, &t, 16);
    }
  }
}

// Threads: (block of kDiaRows rows) x (TK column vectors of VEC); a thread
// loops over C's columns in steps of TK * VEC.
template <class V, class X, int VEC>
__global__ void __launch_bounds__(256, 4)  // 64 registers: 4 blocks per SM
    k_spmm_dia(int32_t m, int32_t n, int nd, DiaRuns runs, const V *__restrict__ dv,
               const X *__restrict__ B, int64_t ldb, X *__restrict__ C, int64_t ldc, int k,
               int lg_tk, X alpha, X beta, int beta_nz) {
  constexpr int RB = kDiaRows;
  using Acc = typename AccOf<V, X>::type;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t rb = g >> lg_tk;
  const int tk = (int)(g & ((1 << lg_tk) - 1));
  const int64_t r0 = rb * RB;
  if (r0 >= m)
    return;
  const V *ab = dv + rb * nd * RB;
  for (int kk = tk * VEC; kk < k; kk += VEC << lg_tk) {
    Acc acc[RB][VEC];
#pragma unroll
    for (int i = 0; i < RB; ++i)
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[i][v] = Acc(0);
    for (int q = 0; q < runs.n; ++q) {
      const int o0 = runs.o0[q], len = runs.len[q], d0 = runs.d0[q];
      X bv[RB + kDiaRun - 1][VEC];
#pragma unroll
      for (int j = 0; j < RB + kDiaRun - 1; ++j) {
        const int64_t br = r0 + o0 + j;
        if (j < RB + len - 1 && br >= 0 && br < n) {
          ld_vec<X, VEC>(B + br * ldb + kk, bv[j]);
        } else {
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            bv[j][v] = X(0);
        }
      }
#pragma unroll
      for (int l = 0; l < kDiaRun; ++l) {
        if (l < len) {
          V a[RB];
          ld_rows_vals<V>(ab + (int64_t)(d0 + l) * RB, a);
#pragma unroll
          for (int i = 0; i < RB; ++i)
            if (!dia_absent(a[i])) {
              const Acc ai = to_acc<Acc>(a[i]);
#pragma unroll
              for (int v = 0; v < VEC; ++v)
                acc[i][v] = fma(ai, to_acc<Acc>(bv[i + l][v]), acc[i][v]);
            }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < RB; ++i) {
      const int64_t r = r0 + i;
      if (r < m) {
        X *cp = C + r * ldc + kk;
        X out[VEC];
        if (beta_nz) {
          X old[VEC];
          ld_vec_plain<X, VEC>(cp, old);
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            out[v] = (X)acc[i][v] * alpha + beta * old[v];
        } else {
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            out[v] = (X)acc[i][v] * alpha;
        }
        st_vec<X, VEC>(cp, out);
      }
    }
  }
}

// Examine the matrix and, when it suits, build its diagonal form from the
// values the kernels use (type V).
template <class V>
void dia_build(CsrDev &c, int32_t m, cudaStream_t s) {
  DiaDev &d = c.dia;
  d.state = -1;
  d.vals.release();
  DevBuf key;
  key.reserve(8);
  PLS_CUDA(cudaMemsetAsync(key.p, 0, 8, s));
  k_dia_longest<<<(unsigned)std::min<int64_t>(div_up(m, 256), 1024), 256, 0, s>>>(
      m, c.row_ptr.as<int32_t>(), key.as<unsigned long long>());
  PLS_LAUNCH_CHECK();
  unsigned long long best = 0;
  PLS_CUDA(cudaMemcpyAsync(&best, key.p, 8, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  const int64_t len = (int64_t)(best >> 32);
  const int32_t row = (int32_t)(best & 0xffffffffull);
  if (len == 0 || len > kDiaMax)
    return;
  int32_t p0 = 0;
  PLS_CUDA(cudaMemcpyAsync(&p0, c.row_ptr.as<int32_t>() + row, 4, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> cols(len);
  PLS_CUDA(cudaMemcpyAsync(cols.data(), c.col.as<int32_t>() + p0, 4 * len,
                           cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  std::vector<int64_t> offs(len);
  for (int64_t i = 0; i < len; ++i)
    offs[i] = (int64_t)cols[i] - row;
  std::sort(offs.begin(), offs.end());
  if (std::adjacent_find(offs.begin(), offs.end()) != offs.end())
    return;
  const int nd = (int)len;
  if ((int64_t)nd * m > 2 * c.nnz)  // fewer than half the diagonal slots hold entries
    return;
  DiaOffs o{};
  o.nd = nd;
  for (int i = 0; i < nd; ++i)
    o.o[i] = (int32_t)offs[i];
  const int64_t count = div_up(m, kDiaRows) * nd * kDiaRows;
  d.vals.reserve(sizeof(V) * count);
  k_dia_fill<V><<<(unsigned)div_up(count, 256), 256, 0, s>>>(count, d.vals.as<V>());
  DevBuf flag;
  flag.reserve(4);
  PLS_CUDA(cudaMemsetAsync(flag.p, 0, 4, s));
  k_dia_scatter<V><<<(unsigned)div_up(m, 256), 256, 0, s>>>(
      m, o, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), static_cast<const V *>(c.ev()),
      d.vals.as<V>(), flag.as<int>());
  PLS_LAUNCH_CHECK();
  int bad = 0;
  PLS_CUDA(cudaMemcpyAsync(&bad, flag.p, 4, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  if (bad) {
    d.vals.release();
    return;
  }
  d.nd = nd;
  for (int i = 0; i < nd; ++i)
    d.offs[i] = o.o[i];
  d.version = c.vals_version;
  d.vt = c.evt();
  d.src = c.ev();
  d.state = 1;
}

template <class V, class X>
void dia_launch(const CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                X alpha, X beta, cudaStream_t s) {
  constexpr int VEC = 16 / (int)sizeof(X);
  const DiaDev &d = c.dia;
  DiaRuns runs{};
  for (int i = 0; i < d.nd;) {
    int len = 1;
    while (i + len < d.nd && len < kDiaRun && d.offs[i + len] == d.offs[i] + len)
      ++len;
    runs.o0[runs.n] = d.offs[i];
    runs.len[runs.n] = len;
    runs.d0[runs.n] = i;
    ++runs.n;
    i += len;
  }
  const int cols = k / VEC;
  int lg_tk = 0;
  while ((1 << lg_tk) < cols && lg_tk < 5)
    ++lg_tk;
  const int64_t threads = div_up(m, kDiaRows) << lg_tk;
  k_spmm_dia<V, X, VEC><<<(unsigned)div_up(threads, 256), 256, 0, s>>>(
      m, c.ncols, d.nd, runs, d.vals.as<V>(), B, ldb, C, ldc, k, lg_tk, alpha, beta,
      beta != X(0));
  PLS_LAUNCH_CHECK();
}

}  // namespace

template <class X>
bool spmm_dia(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
              X alpha, X beta, cudaStream_t s, bool launch) {
  constexpr int VEC = 16 / (int)sizeof(X);
  const Vt api = sizeof(X) == 8 ? Vt::F64 : Vt::F32;
  const Vt vt = c.evt();
  if (m <= 0 || k <= 0 || c.vt != api || c.ncols <= 0 || c.nnz <= 0)
    return false;
  if (vt == Vt::F64 && api != Vt::F64)
    return false;
  if (k % VEC || ldb % VEC || ldc % VEC || (uintptr_t)B % 16 || (uintptr_t)C % 16)
    return false;
  DiaDev &d = c.dia;
  if (d.state != 0 && (d.version != c.vals_version || d.vt != vt || d.src != c.ev()))
    d.state = 0;
  if (d.state == 0) {
    if (vt == Vt::F64)
      dia_build<double>(c, m, s);
    else if (vt == Vt::F32)
      dia_build<float>(c, m, s);
    else
      dia_build<__nv_bfloat16>(c, m, s);
    if (d.state != 1) {  // remember what was examined
      d.version = c.vals_version;
      d.vt = vt;
      d.src = c.ev();
    }
  }
  if (d.state != 1)
    return false;
  if (!launch)
    return true;
  if constexpr (sizeof(X) == 8) {
    if (vt == Vt::F64) {
      dia_launch<double, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
      return true;
    }
  }
  if (vt == Vt::F32)
    dia_launch<float, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else
    dia_launch<__nv_bfloat16, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  return true;
}

template bool spmm_dia<float>(CsrDev &, int32_t, const float *, int64_t, float *, int64_t, int,
                              float, float, cudaStream_t, bool);
template bool spmm_dia<double>(CsrDev &, int32_t, const double *, int64_t, double *, int64_t,
                               int, double, double, cudaStream_t, bool);

}  // namespace pls
