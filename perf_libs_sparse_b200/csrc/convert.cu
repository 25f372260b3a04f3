// Format conversions, norms and in-place value updates on the device.
//
// Optimize-time and export-time work, not the exec path: the sorting steps
// use CUB's device radix sort and scan from the CUDA toolkit headers.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

// Temporary CUB storage, sized on demand.
struct CubTemp {
  DevBuf buf;
  void *get(size_t bytes) {
    buf.reserve(bytes);
    return buf.p;
  }
};

template <class VI, class VO>
__global__ void k_convert(int64_t n, const VI *in, VO *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = from_double<VO>(to_acc<double>(in[i]));
}

__global__ void k_row_of_nnz(int32_t m, const int32_t *__restrict__ rp,
                             int32_t *__restrict__ row_of) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  for (int32_t j = rp[i]; j < rp[i + 1]; ++j)
    row_of[j] = (int32_t)i;
}

__global__ void k_iota(int64_t n, int32_t *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = (int32_t)i;
}

__global__ void k_count_keys(int64_t n, const int32_t *__restrict__ key,
                             int32_t *__restrict__ cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    atomicAdd(cnt + key[i], 1);
}

template <class V>
__global__ void k_gather_transpose(int64_t nnz, const int32_t *__restrict__ perm,
                                   const int32_t *__restrict__ row_of,
                                   const V *__restrict__ val,
                                   int32_t *__restrict__ colT, V *__restrict__ valT) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz)
    return;
  const int32_t p = perm[i];
  colT[i] = row_of[p];
  valT[i] = val[p];
}

// BSR -> CSR, the reference's bsr2csr order (src/compressed_sparse_rows.cpp:
// 966-1056): scalar row i of block row br walks the blocks in stored order
// and each block's row i left to right; exact zeros dropped when asked.
template <class V>
__global__ void k_bsr_row_count(int32_t mb, int bs, int layout, int drop,
                                const int32_t *__restrict__ rp,
                                const V *__restrict__ val,
                                int32_t *__restrict__ cnt) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (int64_t)mb * bs)
    return;
  const int64_t br = r / bs;
  const int i = (int)(r % bs);
  const int64_t E = (int64_t)bs * bs;
  int32_t c = 0;
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b)
    for (int j = 0; j < bs; ++j) {
      const V v = layout == PERFLIBS_ROW_MAJOR ? val[b * E + (int64_t)i * bs + j]
                                               : val[b * E + (int64_t)j * bs + i];
      if (!drop || to_acc<double>(v) != 0.0)
        c++;
    }
  cnt[r] = c;
}

template <class V>
__global__ void k_bsr_row_fill(int32_t mb, int bs, int layout, int drop,
                               const int32_t *__restrict__ rp,
                               const int32_t *__restrict__ col,
                               const V *__restrict__ val,
                               const int32_t *__restrict__ orp,
                               int32_t *__restrict__ ocol, V *__restrict__ oval) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (int64_t)mb * bs)
    return;
  const int64_t br = r / bs;
  const int i = (int)(r % bs);
  const int64_t E = (int64_t)bs * bs;
  int32_t o = orp[r];
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b)
    for (int j = 0; j < bs; ++j) {
      const V v = layout == PERFLIBS_ROW_MAJOR ? val[b * E + (int64_t)i * bs + j]
                                               : val[b * E + (int64_t)j * bs + i];
      if (!drop || to_acc<double>(v) != 0.0) {
        ocol[o] = col[b] * bs + j;
        oval[o] = v;
        o++;
      }
    }
}

__global__ void k_block_keys(int64_t nnz, int bs, int64_t nbc,
                             const int32_t *__restrict__ row_of,
                             const int32_t *__restrict__ col,
                             unsigned long long *__restrict__ key,
                             int32_t *__restrict__ idx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz)
    return;
  key[p] = (unsigned long long)(row_of[p] / bs) * nbc + (col[p] / bs);
  idx[p] = (int32_t)p;
}

__global__ void k_head_flags(int64_t n, const unsigned long long *__restrict__ key,
                             int32_t *__restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// After the inclusive scan, bid[i] - 1 is the block of sorted entry i.
__global__ void k_block_meta(int64_t n, int64_t nbc, const unsigned long long *__restrict__ key,
                             const int32_t *__restrict__ flag,
                             const int32_t *__restrict__ bid,
                             int32_t *__restrict__ bcol, int32_t *__restrict__ rcount) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i])
    return;
  const int64_t b = bid[i] - 1;
  bcol[b] = (int32_t)(key[i] % nbc);
  atomicAdd(rcount + (key[i] / nbc), 1);
}

template <class V>
__global__ void k_block_fill(int64_t n, int bs, int layout,
                             const int32_t *__restrict__ perm,
                             const int32_t *__restrict__ bid,
                             const int32_t *__restrict__ row_of,
                             const int32_t *__restrict__ col,
                             const V *__restrict__ val, V *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int32_t p = perm[i];
  const int64_t b = bid[i] - 1;
  const int li = row_of[p] % bs, lj = col[p] % bs;
  const int64_t at = layout == PERFLIBS_ROW_MAJOR ? (int64_t)li * bs + lj
                                                  : (int64_t)lj * bs + li;
  out[b * bs * bs + at] = val[p];
}

__global__ void k_collect_long(int32_t m, int32_t thr,
                               const int32_t *__restrict__ rp,
                               int32_t *__restrict__ out, int32_t *__restrict__ n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m && rp[i + 1] - rp[i] > thr)
    out[atomicAdd(n, 1)] = (int32_t)i;
}

// ---- norms: non-negative doubles order like their bit patterns.
__device__ __forceinline__ void max_nan(unsigned long long *mx, int *nan, double v) {
  if (v != v)
    atomicExch(nan, 1);
  else
    atomicMax(mx, (unsigned long long)__double_as_longlong(v));
}

template <class V>
__global__ void k_inf_csr(int32_t m, const int32_t *__restrict__ rp,
                          const V *__restrict__ val, unsigned long long *mx,
                          int *nan) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  if (row >= m)
    return;
  const int lane = threadIdx.x & 31;
  double s = 0;
  for (int32_t j = rp[row] + lane; j < rp[row + 1]; j += 32)
    s += fabs(to_acc<double>(val[j]));
  s = group_sum<32>(s, 0xffffffffu);
  if (lane == 0)
    max_nan(mx, nan, s);
}

template <class V>
__global__ void k_inf_bsr(int32_t mb, int bs, int layout,
                          const int32_t *__restrict__ rp,
                          const V *__restrict__ val, unsigned long long *mx,
                          int *nan) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (int64_t)mb * bs)
    return;
  const int64_t br = r / bs;
  const int i = (int)(r % bs);
  const int64_t E = (int64_t)bs * bs;
  double s = 0;
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b)
    for (int j = 0; j < bs; ++j)
      s += fabs(to_acc<double>(layout == PERFLIBS_ROW_MAJOR ? val[b * E + (int64_t)i * bs + j]
                                                             : val[b * E + (int64_t)j * bs + i]));
  max_nan(mx, nan, s);
}

template <class X>
__global__ void k_inf_dense(int64_t m, int64_t n, int64_t rs, int64_t cs,
                            const X *__restrict__ A, unsigned long long *mx,
                            int *nan) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m)
    return;
  double s = 0;
  for (int64_t j = 0; j < n; ++j)
    s += fabs((double)A[r * rs + j * cs]);
  max_nan(mx, nan, s);
}

template <class V>
__global__ void k_absmax(int64_t n, const V *__restrict__ v, unsigned long long *mx,
                         int *nan) {
  double best = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double a = fabs(to_acc<double>(v[i]));
    if (a != a)
      atomicExch(nan, 1);
    else
      best = fmax(best, a);
  }
  atomicMax(mx, (unsigned long long)__double_as_longlong(best));
}

template <class V>
__global__ void k_sumsq_scaled(int64_t n, const V *__restrict__ v, double inv,
                               double *out) {
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double a = to_acc<double>(v[i]) * inv;
    s = fma(a, a, s);
  }
  s = group_sum<32>(s, 0xffffffffu);
  if ((threadIdx.x & 31) == 0)
    atomicAdd(out, s);
}

// ---- updates
__global__ void k_update_find(int64_t nu, int32_t m, int32_t n, int32_t base,
                              const int32_t *__restrict__ ur,
                              const int32_t *__restrict__ uc,
                              const int32_t *__restrict__ rp,
                              const int32_t *__restrict__ col,
                              int64_t *__restrict__ pos) {
  const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu)
    return;
  const int32_t r = ur[u] - base, c = uc[u] - base;
  int64_t p = -1;
  if (r >= 0 && r < m && c >= 0 && c < n)
    for (int32_t j = rp[r]; j < rp[r + 1]; ++j)
      if (col[j] == c) {
        p = j;
        break;
      }
  pos[u] = p;
}

// Applied by one thread in update order, so a repeated entry keeps the last
// value, as the reference's sequential loop does
// (src/compressed_sparse_rows.cpp:3072-3095).
template <class V, class X>
__global__ void k_update_apply(int64_t nu, const int64_t *__restrict__ pos,
                               const int32_t *__restrict__ ur, int32_t base,
                               const X *__restrict__ uv, const int32_t *__restrict__ rp,
                               V *__restrict__ val, const int32_t *__restrict__ in2permd,
                               const int64_t *__restrict__ cs, int C,
                               V *__restrict__ sell_val) {
  for (int64_t u = 0; u < nu; ++u) {
    const int64_t p = pos[u];
    const V v = from_double<V>((double)uv[u]);
    val[p] = v;
    if (sell_val) {
      const int32_t r = ur[u] - base;
      const int64_t j = p - rp[r];
      const int32_t q = in2permd[r];
      sell_val[cs[q / C] + j * C + (q % C)] = v;
    }
  }
}

template <class X>
__global__ void k_transpose(const X *__restrict__ in, int64_t rows, int64_t cols,
                            int64_t ldin, X *__restrict__ out, int64_t ldout) {
  __shared__ X tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols)
      tile[k][threadIdx.x] = in[r * ldin + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols)
      out[c * ldout + r] = tile[threadIdx.x][k];
  }
}

template <class X>
__global__ void k_strided_copy(const X *in, int64_t si, X *out, int64_t so, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i * so] = in[i * si];
}

double finish_norm(DevBuf &acc, cudaStream_t s) {
  unsigned long long h[2];
  PLS_CUDA(cudaMemcpyAsync(h, acc.p, 16, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  int nan;
  std::memcpy(&nan, &h[1], sizeof(int));
  if (nan)
    return std::numeric_limits<double>::quiet_NaN();
  double v;
  std::memcpy(&v, &h[0], sizeof(double));
  return v;
}

}  // namespace

void convert_values(const void *in, Vt vin, void *out, Vt vout, int64_t n,
                    cudaStream_t s) {
  if (n <= 0)
    return;
  if (vin == vout) {
    PLS_CUDA(cudaMemcpyAsync(out, in, vt_size(vin) * n, cudaMemcpyDeviceToDevice, s));
    return;
  }
  with_vt(vin, [&](auto ti) {
    with_vt(vout, [&](auto to) {
      using VI = typename decltype(ti)::type;
      using VO = typename decltype(to)::type;
      k_convert<VI, VO><<<(unsigned)div_up(n, 256), 256, 0, s>>>(
          n, (const VI *)in, (VO *)out);
    });
  });
  PLS_LAUNCH_CHECK();
}

void build_csr_transpose(const CsrDev &c, int32_t m, int32_t n, CsrDev &out,
                         cudaStream_t s) {
  CsrDev T;
  T.vt = c.vt;
  T.nnz = c.nnz;
  T.ncols = m;
  T.row_ptr.reserve(sizeof(int32_t) * (n + 1));
  T.col.reserve(sizeof(int32_t) * std::max<int64_t>(c.nnz, 1));
  T.vals.reserve(vt_size(c.vt) * std::max<int64_t>(c.nnz, 1));
  PLS_CUDA(cudaMemsetAsync(T.row_ptr.p, 0, sizeof(int32_t) * (n + 1), s));
  if (c.nnz > 0) {
    DevBuf row_of, idx, keys_out, idx_out, cnt;
    row_of.reserve(sizeof(int32_t) * c.nnz);
    idx.reserve(sizeof(int32_t) * c.nnz);
    keys_out.reserve(sizeof(int32_t) * c.nnz);
    idx_out.reserve(sizeof(int32_t) * c.nnz);
    cnt.reserve(sizeof(int32_t) * (n + 1));
    PLS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (n + 1), s));
    k_row_of_nnz<<<(unsigned)div_up(m, 256), 256, 0, s>>>(m, c.row_ptr.as<int32_t>(),
                                                           row_of.as<int32_t>());
    // Stable sort of (column, nonzero index): within a column, entries stay
    // in row order, as the reference's csr2csc produces them.
    k_iota<<<(unsigned)div_up(c.nnz, 256), 256, 0, s>>>(c.nnz, idx.as<int32_t>());
    {
      size_t tb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tb, c.col.as<int32_t>(), keys_out.as<int32_t>(),
                                      idx.as<int32_t>(), idx_out.as<int32_t>(), (int)c.nnz, 0,
                                      32, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, c.col.as<int32_t>(),
                                               keys_out.as<int32_t>(), idx.as<int32_t>(),
                                               idx_out.as<int32_t>(), (int)c.nnz, 0, 32, s));
    }
    k_count_keys<<<(unsigned)div_up(c.nnz, 256), 256, 0, s>>>(c.nnz, c.col.as<int32_t>(),
                                                               cnt.as<int32_t>());
    {
      size_t tb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), T.row_ptr.as<int32_t>(),
                                    n + 1, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, cnt.as<int32_t>(),
                                             T.row_ptr.as<int32_t>(), n + 1, s));
    }
    with_vt(c.vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      k_gather_transpose<V><<<(unsigned)div_up(c.nnz, 256), 256, 0, s>>>(
          c.nnz, idx_out.as<int32_t>(), row_of.as<int32_t>(), c.vals.as<V>(),
          T.col.as<int32_t>(), T.vals.as<V>());
    });
    PLS_LAUNCH_CHECK();
    PLS_CUDA(cudaStreamSynchronize(s));
  }
  out = std::move(T);
}

namespace {

// Key row * n + col per entry (the reference's coo2csr ordering key,
// src/compressed_sparse_rows.cpp:591-640) and the entry's index; records
// the first entry with an index out of range.
__global__ void k_coo_keys(int64_t nnz, int32_t m, int32_t n, const int32_t *__restrict__ row,
                           const int32_t *__restrict__ col, unsigned long long *__restrict__ key,
                           int32_t *__restrict__ idx, unsigned long long *__restrict__ bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz)
    return;
  const int32_t r = row[i], c = col[i];
  const bool ok = r >= 0 && r < m && c >= 0 && c < n;
  if (!ok)
    atomicMin(bad, (unsigned long long)i);
  key[i] = ok ? (unsigned long long)r * (unsigned long long)n + (unsigned long long)c : 0ull;
  idx[i] = (int32_t)i;
}

template <class V>
__global__ void k_gather_entries(int64_t nnz, const int32_t *__restrict__ perm,
                                 const int32_t *__restrict__ col, const V *__restrict__ val,
                                 int32_t *__restrict__ ocol, V *__restrict__ oval) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz)
    return;
  const int32_t p = perm[i];
  ocol[i] = col[p];
  oval[i] = val[p];
}

}  // namespace

namespace {

__global__ void k_check_compressed(int32_t rows, int32_t cols, int64_t nnz,
                                   const int32_t *__restrict__ ptr,
                                   const int32_t *__restrict__ idx,
                                   unsigned long long *__restrict__ bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < rows) {
    const int32_t a = ptr[i], b = ptr[i + 1];
    if (a < 0 || b < a || b > nnz)
      atomicMin(bad, (unsigned long long)i);
  }
  if (i < nnz) {
    const int32_t c = idx[i];
    if (c < 0 || c >= cols)
      atomicMin(bad + 1, (unsigned long long)i);
  }
}

}  // namespace

// Structure check of 0-based compressed arrays before any kernel indexes
// with them: the first row whose pointers are decreasing or outside
// [0, nnz], and the first entry whose index is outside [0, cols); -1 each
// when there is none.
std::pair<int64_t, int64_t> check_compressed(int32_t rows, int32_t cols, int64_t nnz,
                                             const int32_t *ptr, const int32_t *idx,
                                             cudaStream_t s) {
  const int64_t work = std::max<int64_t>(rows, nnz);
  if (work == 0)
    return {-1, -1};
  DevBuf bad;
  bad.reserve(16);
  PLS_CUDA(cudaMemsetAsync(bad.p, 0xff, 16, s));
  k_check_compressed<<<(unsigned)div_up(work, 256), 256, 0, s>>>(
      rows, cols, nnz, ptr, idx, bad.as<unsigned long long>());
  PLS_LAUNCH_CHECK();
  unsigned long long h[2];
  PLS_CUDA(cudaMemcpyAsync(h, bad.p, 16, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  return {h[0] == ~0ull ? -1 : (int64_t)h[0], h[1] == ~0ull ? -1 : (int64_t)h[1]};
}

// The entries sorted by (row, column) with a stable radix sort, so equal
// positions keep their input order (the reference's std::sort leaves their
// order unspecified; the values are all kept either way); row_ptr from the
// per-row counts.
int64_t coo_to_csr(int32_t m, int32_t n, int64_t nnz, const int32_t *row, const int32_t *col,
                   const void *vals, Vt vt, CsrDev &out, cudaStream_t s) {
  CsrDev R;
  R.vt = vt;
  R.nnz = nnz;
  R.row_ptr.reserve(sizeof(int32_t) * ((size_t)m + 1));
  R.col.reserve(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  R.vals.reserve(vt_size(vt) * std::max<int64_t>(nnz, 1));
  PLS_CUDA(cudaMemsetAsync(R.row_ptr.p, 0, sizeof(int32_t) * ((size_t)m + 1), s));
  if (nnz > 0) {
    DevBuf key, key_out, idx, idx_out, cnt, bad;
    key.reserve(8 * nnz);
    key_out.reserve(8 * nnz);
    idx.reserve(4 * nnz);
    idx_out.reserve(4 * nnz);
    cnt.reserve(sizeof(int32_t) * ((size_t)m + 1));
    bad.reserve(8);
    PLS_CUDA(cudaMemsetAsync(bad.p, 0xff, 8, s));
    k_coo_keys<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(nnz, m, n, row, col,
                                                           key.as<unsigned long long>(),
                                                           idx.as<int32_t>(),
                                                           bad.as<unsigned long long>());
    PLS_LAUNCH_CHECK();
    unsigned long long first_bad = 0;
    PLS_CUDA(cudaMemcpyAsync(&first_bad, bad.p, 8, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    if (first_bad != ~0ull)
      return (int64_t)first_bad;
    const unsigned long long span = (unsigned long long)m * (unsigned long long)n;
    int end_bit = 1;
    while (end_bit < 64 && (span >> end_bit) != 0)
      ++end_bit;
    {
      size_t tb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<unsigned long long>(),
                                      key_out.as<unsigned long long>(), idx.as<int32_t>(),
                                      idx_out.as<int32_t>(), (int)nnz, 0, end_bit, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, key.as<unsigned long long>(),
                                               key_out.as<unsigned long long>(),
                                               idx.as<int32_t>(), idx_out.as<int32_t>(),
                                               (int)nnz, 0, end_bit, s));
    }
    PLS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * ((size_t)m + 1), s));
    k_count_keys<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(nnz, row, cnt.as<int32_t>());
    {
      size_t tb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), R.row_ptr.as<int32_t>(),
                                    m + 1, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, cnt.as<int32_t>(),
                                             R.row_ptr.as<int32_t>(), m + 1, s));
    }
    with_vt(vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      k_gather_entries<V><<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(
          nnz, idx_out.as<int32_t>(), col, (const V *)vals, R.col.as<int32_t>(), R.vals.as<V>());
    });
    PLS_LAUNCH_CHECK();
  }
  PLS_CUDA(cudaStreamSynchronize(s));
  out = std::move(R);
  return -1;
}

void bsr_to_csr(const BsrDev &b, int32_t m, bool drop_zeros, CsrDev &out,
                cudaStream_t s) {
  CsrDev R;
  R.vt = b.vt;
  R.ncols = b.nb * b.bs;
  R.row_ptr.reserve(sizeof(int32_t) * (m + 1));
  DevBuf cnt;
  cnt.reserve(sizeof(int32_t) * (m + 1));
  PLS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (m + 1), s));
  with_vt(b.vt, [&](auto tag) {
    using V = typename decltype(tag)::type;
    if (m > 0)
      k_bsr_row_count<V><<<(unsigned)div_up(m, 256), 256, 0, s>>>(
          b.mb, b.bs, b.layout, drop_zeros, b.row_ptr.as<int32_t>(), b.vals.as<V>(),
          cnt.as<int32_t>());
  });
  {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), R.row_ptr.as<int32_t>(),
                                  m + 1, s);
    CubTemp tmp;
    PLS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, cnt.as<int32_t>(),
                                           R.row_ptr.as<int32_t>(), m + 1, s));
  }
  int32_t nnz = 0;
  PLS_CUDA(cudaMemcpyAsync(&nnz, R.row_ptr.as<int32_t>() + m, sizeof(int32_t),
                           cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  R.nnz = nnz;
  R.col.reserve(sizeof(int32_t) * std::max(nnz, 1));
  R.vals.reserve(vt_size(b.vt) * std::max(nnz, 1));
  with_vt(b.vt, [&](auto tag) {
    using V = typename decltype(tag)::type;
    if (m > 0)
      k_bsr_row_fill<V><<<(unsigned)div_up(m, 256), 256, 0, s>>>(
          b.mb, b.bs, b.layout, drop_zeros, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(),
          b.vals.as<V>(), R.row_ptr.as<int32_t>(), R.col.as<int32_t>(), R.vals.as<V>());
  });
  PLS_LAUNCH_CHECK();
  PLS_CUDA(cudaStreamSynchronize(s));
  out = std::move(R);
}

void csr_to_bsr(const CsrDev &c, int32_t m, int32_t n, int bs, int layout,
                BsrDev &out, cudaStream_t s) {
  BsrDev B;
  B.bs = bs;
  B.layout = layout;
  B.vt = c.vt;
  B.mb = m / bs;
  B.nb = n / bs;
  const int64_t nbc = std::max<int64_t>(B.nb, 1);
  B.row_ptr.reserve(sizeof(int32_t) * (B.mb + 1));
  DevBuf rcount;
  rcount.reserve(sizeof(int32_t) * (B.mb + 1));
  PLS_CUDA(cudaMemsetAsync(rcount.p, 0, sizeof(int32_t) * (B.mb + 1), s));
  const int64_t nnz = c.nnz;
  DevBuf row_of, key, idx, key2, idx2, flag, bid;
  int64_t nnzb = 0;
  if (nnz > 0) {
    row_of.reserve(sizeof(int32_t) * nnz);
    key.reserve(8 * nnz);
    idx.reserve(4 * nnz);
    key2.reserve(8 * nnz);
    idx2.reserve(4 * nnz);
    flag.reserve(4 * nnz);
    bid.reserve(4 * nnz);
    k_row_of_nnz<<<(unsigned)div_up(m, 256), 256, 0, s>>>(m, c.row_ptr.as<int32_t>(),
                                                           row_of.as<int32_t>());
    k_block_keys<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(
        nnz, bs, nbc, row_of.as<int32_t>(), c.col.as<int32_t>(),
        key.as<unsigned long long>(), idx.as<int32_t>());
    int end_bit = 1;
    while (end_bit < 64 && ((unsigned long long)B.mb * nbc >> end_bit) != 0)
      end_bit++;
    {
      size_t tb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<unsigned long long>(),
                                      key2.as<unsigned long long>(), idx.as<int32_t>(),
                                      idx2.as<int32_t>(), (int)nnz, 0, end_bit, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, key.as<unsigned long long>(),
                                               key2.as<unsigned long long>(), idx.as<int32_t>(),
                                               idx2.as<int32_t>(), (int)nnz, 0, end_bit, s));
    }
    k_head_flags<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(nnz, key2.as<unsigned long long>(),
                                                             flag.as<int32_t>());
    {
      size_t tb = 0;
      cub::DeviceScan::InclusiveSum(nullptr, tb, flag.as<int32_t>(), bid.as<int32_t>(),
                                    (int)nnz, s);
      CubTemp tmp;
      PLS_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(tb), tb, flag.as<int32_t>(),
                                             bid.as<int32_t>(), (int)nnz, s));
    }
    int32_t last = 0;
    PLS_CUDA(cudaMemcpyAsync(&last, bid.as<int32_t>() + nnz - 1, 4, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    nnzb = last;
  }
  B.nnzb = nnzb;
  B.col.reserve(sizeof(int32_t) * std::max<int64_t>(nnzb, 1));
  const int64_t E = (int64_t)bs * bs;
  B.vals.reserve(vt_size(c.vt) * std::max<int64_t>(nnzb * E, 1));
  if (nnzb > 0) {
    PLS_CUDA(cudaMemsetAsync(B.vals.p, 0, vt_size(c.vt) * nnzb * E, s));
    k_block_meta<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(
        nnz, nbc, key2.as<unsigned long long>(), flag.as<int32_t>(), bid.as<int32_t>(),
        B.col.as<int32_t>(), rcount.as<int32_t>());
    with_vt(c.vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      k_block_fill<V><<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(
          nnz, bs, layout, idx2.as<int32_t>(), bid.as<int32_t>(), row_of.as<int32_t>(),
          c.col.as<int32_t>(), c.vals.as<V>(), B.vals.as<V>());
    });
  }
  {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, rcount.as<int32_t>(), B.row_ptr.as<int32_t>(),
                                  B.mb + 1, s);
    CubTemp tmp;
    PLS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, rcount.as<int32_t>(),
                                           B.row_ptr.as<int32_t>(), B.mb + 1, s));
  }
  PLS_LAUNCH_CHECK();
  PLS_CUDA(cudaStreamSynchronize(s));
  out = std::move(B);
}

// Number of distinct bs x bs blocks holding at least one stored entry
// (m and n need not be multiples of bs here).
int64_t count_blocks(const CsrDev &c, int32_t m, int32_t n, int bs, cudaStream_t s) {
  const int64_t nnz = c.nnz;
  if (nnz == 0)
    return 0;
  const int64_t nbc = std::max<int64_t>(div_up(n, bs), 1);
  const int64_t nbr = std::max<int64_t>(div_up(m, bs), 1);
  DevBuf row_of, key, idx, key2, idx2, flag, bid;
  row_of.reserve(4 * nnz);
  key.reserve(8 * nnz);
  idx.reserve(4 * nnz);
  key2.reserve(8 * nnz);
  idx2.reserve(4 * nnz);
  flag.reserve(4 * nnz);
  bid.reserve(4 * nnz);
  k_row_of_nnz<<<(unsigned)div_up(m, 256), 256, 0, s>>>(m, c.row_ptr.as<int32_t>(),
                                                         row_of.as<int32_t>());
  k_block_keys<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(
      nnz, bs, nbc, row_of.as<int32_t>(), c.col.as<int32_t>(), key.as<unsigned long long>(),
      idx.as<int32_t>());
  int end_bit = 1;
  while (end_bit < 64 && ((unsigned long long)nbr * nbc >> end_bit) != 0)
    end_bit++;
  {
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<unsigned long long>(),
                                    key2.as<unsigned long long>(), idx.as<int32_t>(),
                                    idx2.as<int32_t>(), (int)nnz, 0, end_bit, s);
    CubTemp tmp;
    PLS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, key.as<unsigned long long>(),
                                             key2.as<unsigned long long>(), idx.as<int32_t>(),
                                             idx2.as<int32_t>(), (int)nnz, 0, end_bit, s));
  }
  k_head_flags<<<(unsigned)div_up(nnz, 256), 256, 0, s>>>(nnz, key2.as<unsigned long long>(),
                                                           flag.as<int32_t>());
  {
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, flag.as<int32_t>(), bid.as<int32_t>(), (int)nnz, s);
    CubTemp tmp;
    PLS_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(tb), tb, flag.as<int32_t>(), bid.as<int32_t>(),
                                           (int)nnz, s));
  }
  PLS_LAUNCH_CHECK();
  int32_t last = 0;
  PLS_CUDA(cudaMemcpyAsync(&last, bid.as<int32_t>() + nnz - 1, 4, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  return last;
}

void csr_build_long_rows(CsrDev &c, int32_t m, int threshold, cudaStream_t s) {
  c.bands.clear();
  c.long_threshold = threshold;
  c.n_long = 0;
  c.long_rows.reserve(sizeof(int32_t) * std::max(m, 1));
  DevBuf cnt;
  cnt.reserve(4);
  PLS_CUDA(cudaMemsetAsync(cnt.p, 0, 4, s));
  if (m > 0)
    k_collect_long<<<(unsigned)div_up(m, 256), 256, 0, s>>>(
        m, threshold, c.row_ptr.as<int32_t>(), c.long_rows.as<int32_t>(), cnt.as<int32_t>());
  PLS_LAUNCH_CHECK();
  int32_t n = 0;
  PLS_CUDA(cudaMemcpyAsync(&n, cnt.p, 4, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  c.n_long = n;
}

double inf_norm_csr(const CsrDev &c, int32_t m, cudaStream_t s) {
  DevBuf acc;
  acc.reserve(16);
  PLS_CUDA(cudaMemsetAsync(acc.p, 0, 16, s));
  if (m > 0)
    with_vt(c.vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      k_inf_csr<V><<<(unsigned)div_up((int64_t)m * 32, 256), 256, 0, s>>>(
          m, c.row_ptr.as<int32_t>(), c.vals.as<V>(), acc.as<unsigned long long>(),
          (int *)(acc.as<char>() + 8));
    });
  PLS_LAUNCH_CHECK();
  return finish_norm(acc, s);
}

double inf_norm_bsr(const BsrDev &b, cudaStream_t s) {
  DevBuf acc;
  acc.reserve(16);
  PLS_CUDA(cudaMemsetAsync(acc.p, 0, 16, s));
  const int64_t rows = (int64_t)b.mb * b.bs;
  if (rows > 0)
    with_vt(b.vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      k_inf_bsr<V><<<(unsigned)div_up(rows, 256), 256, 0, s>>>(
          b.mb, b.bs, b.layout, b.row_ptr.as<int32_t>(), b.vals.as<V>(),
          acc.as<unsigned long long>(), (int *)(acc.as<char>() + 8));
    });
  PLS_LAUNCH_CHECK();
  return finish_norm(acc, s);
}

double inf_norm_dense(const DenseDev &d, Dt dt, int32_t m, int32_t n,
                      cudaStream_t s) {
  DevBuf acc;
  acc.reserve(16);
  PLS_CUDA(cudaMemsetAsync(acc.p, 0, 16, s));
  const int64_t rs = d.layout == PERFLIBS_ROW_MAJOR ? d.lda : 1;
  const int64_t cs = d.layout == PERFLIBS_ROW_MAJOR ? 1 : d.lda;
  if (m > 0) {
    if (dt == Dt::F64)
      k_inf_dense<double><<<(unsigned)div_up(m, 256), 256, 0, s>>>(
          m, n, rs, cs, d.vals.as<double>(), acc.as<unsigned long long>(),
          (int *)(acc.as<char>() + 8));
    else
      k_inf_dense<float><<<(unsigned)div_up(m, 256), 256, 0, s>>>(
          m, n, rs, cs, d.vals.as<float>(), acc.as<unsigned long long>(),
          (int *)(acc.as<char>() + 8));
  }
  PLS_LAUNCH_CHECK();
  return finish_norm(acc, s);
}

// sqrt(sum v^2) computed as mx * sqrt(sum (v/mx)^2), mx = max |v|: no
// overflow or underflow of the squares (the purpose of the reference's
// three-accumulator scheme, src/norm.cpp:56-138).
double frb_norm_values(const void *vals, Vt vt, int64_t n, cudaStream_t s) {
  if (n <= 0)
    return 0.0;
  DevBuf acc, sum;
  acc.reserve(16);
  sum.reserve(8);
  PLS_CUDA(cudaMemsetAsync(acc.p, 0, 16, s));
  PLS_CUDA(cudaMemsetAsync(sum.p, 0, 8, s));
  const unsigned blocks = (unsigned)std::min<int64_t>(div_up(n, 256), 148 * 8);
  with_vt(vt, [&](auto tag) {
    using V = typename decltype(tag)::type;
    k_absmax<V><<<blocks, 256, 0, s>>>(n, (const V *)vals, acc.as<unsigned long long>(),
                                       (int *)(acc.as<char>() + 8));
  });
  const double mx = finish_norm(acc, s);
  if (mx != mx || mx == 0.0 || mx == INFINITY)
    return mx;
  with_vt(vt, [&](auto tag) {
    using V = typename decltype(tag)::type;
    k_sumsq_scaled<V><<<blocks, 256, 0, s>>>(n, (const V *)vals, 1.0 / mx, sum.as<double>());
  });
  PLS_LAUNCH_CHECK();
  double h = 0;
  PLS_CUDA(cudaMemcpyAsync(&h, sum.p, 8, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  return mx * std::sqrt(h);
}

int64_t update_csr_values(CsrDev &c, SellDev *sell, int32_t m, int32_t n,
                          int64_t nu, const int32_t *rows_host,
                          const int32_t *cols_host, const void *vals_host,
                          Dt dt, int32_t base, cudaStream_t s) {
  if (nu <= 0)
    return nu;
  DevBuf ur, uc, uv, pos;
  ur.reserve(4 * nu);
  uc.reserve(4 * nu);
  const size_t xs = dt == Dt::F64 ? 8 : 4;
  uv.reserve(xs * nu);
  pos.reserve(8 * nu);
  PLS_CUDA(cudaMemcpyAsync(ur.p, rows_host, 4 * nu, cudaMemcpyHostToDevice, s));
  PLS_CUDA(cudaMemcpyAsync(uc.p, cols_host, 4 * nu, cudaMemcpyHostToDevice, s));
  PLS_CUDA(cudaMemcpyAsync(uv.p, vals_host, xs * nu, cudaMemcpyHostToDevice, s));
  k_update_find<<<(unsigned)div_up(nu, 256), 256, 0, s>>>(
      nu, m, n, base, ur.as<int32_t>(), uc.as<int32_t>(), c.row_ptr.as<int32_t>(),
      c.col.as<int32_t>(), pos.as<int64_t>());
  PLS_LAUNCH_CHECK();
  std::vector<int64_t> ph(nu);
  PLS_CUDA(cudaMemcpyAsync(ph.data(), pos.p, 8 * nu, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  int64_t first_bad = nu;
  for (int64_t u = 0; u < nu; ++u)
    if (ph[u] < 0) {
      first_bad = u;
      break;
    }
  if (first_bad > 0) {
    with_vt(c.vt, [&](auto tag) {
      using V = typename decltype(tag)::type;
      const bool use_sell = sell && sell->nC > 0;
      if (dt == Dt::F64)
        k_update_apply<V, double><<<1, 1, 0, s>>>(
            first_bad, pos.as<int64_t>(), ur.as<int32_t>(), base, uv.as<double>(),
            c.row_ptr.as<int32_t>(), c.vals.as<V>(),
            use_sell ? sell->in2permd.as<int32_t>() : nullptr,
            use_sell ? sell->cs.as<int64_t>() : nullptr, use_sell ? sell->C : 1,
            use_sell ? sell->vals.as<V>() : nullptr);
      else
        k_update_apply<V, float><<<1, 1, 0, s>>>(
            first_bad, pos.as<int64_t>(), ur.as<int32_t>(), base, uv.as<float>(),
            c.row_ptr.as<int32_t>(), c.vals.as<V>(),
            use_sell ? sell->in2permd.as<int32_t>() : nullptr,
            use_sell ? sell->cs.as<int64_t>() : nullptr, use_sell ? sell->C : 1,
            use_sell ? sell->vals.as<V>() : nullptr);
    });
    PLS_LAUNCH_CHECK();
    PLS_CUDA(cudaStreamSynchronize(s));
  }
  return first_bad;
}

template <class X>
void transpose_dense(const X *in, int64_t rows, int64_t cols, int64_t ldin,
                     X *out, int64_t ldout, cudaStream_t s) {
  if (rows == 0 || cols == 0)
    return;
  dim3 grid((unsigned)div_up(cols, 32), (unsigned)div_up(rows, 32));
  k_transpose<X><<<grid, dim3(32, 8), 0, s>>>(in, rows, cols, ldin, out, ldout);
  PLS_LAUNCH_CHECK();
}

template <class X>
void strided_copy(const X *in, int64_t si, X *out, int64_t so, int64_t n,
                  cudaStream_t s) {
  if (n <= 0)
    return;
  k_strided_copy<X><<<(unsigned)div_up(n, 256), 256, 0, s>>>(in, si, out, so, n);
  PLS_LAUNCH_CHECK();
}

template void transpose_dense<float>(const float *, int64_t, int64_t, int64_t,
                                     float *, int64_t, cudaStream_t);
template void transpose_dense<double>(const double *, int64_t, int64_t,
                                      int64_t, double *, int64_t, cudaStream_t);
template void strided_copy<float>(const float *, int64_t, float *, int64_t,
                                  int64_t, cudaStream_t);
template void strided_copy<double>(const double *, int64_t, double *, int64_t,
                                   int64_t, cudaStream_t);

}  // namespace pls
