// SpMV kernels of libplsparse_b200 (sm_100a).
//
// All kernels compute y = alpha*op(A)*x + beta*y. The path is HBM-bound
// (about 0.17 flop/byte for FP64 CSR), so the kernels are built around the
// memory system, not the tensor cores:
//   * matrix data is read exactly once with streaming loads; x is gathered
//     through the read-only path and stays resident in L2;
//   * each row's sum runs in one thread or one group of lanes, so a row's
//     result depends only on that row (no atomics on the NOTRANS path);
//   * grids launch one thread group per row / chunk and let the block
//     scheduler balance uneven rows across the 148 SMs.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

template <class X, class Acc>
__device__ __forceinline__ void store_y(X *y, int64_t i, Acc sum, X alpha,
                                        X beta, int beta_nz) {
  // The reference's epilogue: sum*alpha, plus beta*y when beta != 0
  // (src/compressed_sparse_rows.cpp:1289-1298, src/sell_c_sigma.cpp:779-794).
  X s = (X)sum * alpha;
  if (beta_nz)
    s += beta * y[i];
  y[i] = s;
}

// ---------------------------------------------------------------- CSR

// TPR lanes per row; rows longer than skip_len (when > 0) are left to the
// long-row kernel.
template <int TPR, class V, class X>
__global__ void __launch_bounds__(256)
    k_csr_vector(int32_t m, const int32_t *__restrict__ rp,
                 const int32_t *__restrict__ col, const V *__restrict__ val,
                 const X *__restrict__ x, X *__restrict__ y, X alpha, X beta,
                 int beta_nz, int32_t skip_len) {
  using Acc = typename AccOf<V, X>::type;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t row = gid / TPR;
  if (row >= m)
    return;
  const int sub = threadIdx.x & (TPR - 1);
  const int32_t s = __ldg(rp + row), e = __ldg(rp + row + 1);
  if (skip_len > 0 && e - s > skip_len)
    return;  // uniform across the row's lanes
  // Groups of G elements per lane: all value / column loads of a group are
  // issued (predicated past the row end) before the dependent x gathers. One
  // lane per row takes 8, so the short rows that configuration is picked for
  // (stencils) cost one stream round trip and one gather round trip.
  constexpr int G = TPR == 1 ? 8 : 4;
  const L2Policy pol = make_l2_policy();
  Acc sum = 0;
  for (int32_t j = s + sub; j < e; j += G * TPR) {
    V v[G];
    int32_t c[G];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int32_t q = j + u * TPR;
      if (q < e) {
        v[u] = ld_stream(val + q, pol.stream);
        c[u] = ld_stream(col + q, pol.stream);
      } else {
        v[u] = from_double<V>(0.0);
        c[u] = 0;
      }
    }
    Acc xv[G];
#pragma unroll
    for (int u = 0; u < G; ++u)
      xv[u] = j + u * TPR < e ? to_acc<Acc>(ld_keep(x + c[u], pol.keep)) : Acc(0);
#pragma unroll
    for (int u = 0; u < G; ++u)
      if (j + u * TPR < e)
        sum = fma(to_acc<Acc>(v[u]), xv[u], sum);
  }
  if constexpr (TPR > 1)
    sum = group_sum<TPR>(sum, group_mask<TPR>());
  if (sub == 0)
    store_y(y, row, sum, alpha, beta, beta_nz);
}

// One CTA per long row (rows listed in `rows`), block-wide reduction.
template <class V, class X>
__global__ void __launch_bounds__(256)
    k_csr_long(const int32_t *__restrict__ rows, const int32_t *__restrict__ rp,
               const int32_t *__restrict__ col, const V *__restrict__ val,
               const X *__restrict__ x, X *__restrict__ y, X alpha, X beta,
               int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  __shared__ Acc part[8];
  const int32_t row = rows[blockIdx.x];
  const int32_t s = __ldg(rp + row), e = __ldg(rp + row + 1);
  Acc sum = 0;
  for (int32_t j = s + threadIdx.x; j < e; j += blockDim.x)
    sum = fma(to_acc<Acc>(ld_stream(val + j)),
              to_acc<Acc>(ld_ro(x + ld_stream(col + j))), sum);
  sum = group_sum<32>(sum, 0xffffffffu);
  if ((threadIdx.x & 31) == 0)
    part[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    Acc t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      t += part[w];
    store_y(y, row, t, alpha, beta, beta_nz);
  }
}

// Rows [r0, r0 + m): row_ptr holds absolute offsets, so the kernel sees the
// row pointers and y from r0 on.
template <int TPR, class V, class X>
static void launch_csr_vector(const CsrDev &c, int64_t r0, int32_t m, const X *x, X *y,
                              X alpha, X beta, int32_t skip, cudaStream_t s) {
  const int64_t threads = (int64_t)m * TPR;
  const int64_t blocks = div_up(threads, 256);
  k_csr_vector<TPR, V, X><<<(unsigned)blocks, 256, 0, s>>>(
      m, c.row_ptr.as<int32_t>() + r0, c.col.as<int32_t>(), (const V *)c.ev(), x, y + r0,
      alpha, beta, beta != X(0), skip);
}

template <class V, class X>
static void csr_vector_dispatch(const CsrDev &c, int64_t r0, int32_t m, int tpr,
                                const X *x, X *y, X alpha, X beta,
                                int32_t skip, cudaStream_t s) {
  switch (tpr) {
  case 1: launch_csr_vector<1, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  case 2: launch_csr_vector<2, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  case 4: launch_csr_vector<4, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  case 8: launch_csr_vector<8, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  case 16: launch_csr_vector<16, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  default: launch_csr_vector<32, V>(c, r0, m, x, y, alpha, beta, skip, s); break;
  }
}

// Lanes per row of the vector kernel beside the long-row kernel: rows up to
// the threshold take 4 lanes up to 64 entries, then 8, 16 and 32.
static int split_tpr(int32_t threshold) {
  if (threshold <= 64)
    return 4;
  if (threshold <= 256)
    return 8;
  if (threshold <= 1024)
    return 16;
  return 32;
}

template <class X>
void spmv_csr(const CsrDev &c, int32_t m, int tpr, const X *x, X *y, X alpha,
              X beta, cudaStream_t s) {
  if (m == 0)
    return;
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>)
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    else
      csr_vector_dispatch<V, X>(c, 0, m, tpr, x, y, alpha, beta, 0, s);
  });
  PLS_LAUNCH_CHECK();
}

// Vector kernel for rows up to the threshold + one CTA per longer row.
template <class X>
void spmv_csr_split(const CsrDev &c, int32_t m, const X *x, X *y, X alpha,
                    X beta, cudaStream_t s) {
  if (m == 0)
    return;
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      const int32_t thr = c.long_threshold;
      csr_vector_dispatch<V, X>(c, 0, m, split_tpr(thr), x, y, alpha, beta, thr, s);
      if (c.n_long > 0)
        k_csr_long<V, X><<<c.n_long, 256, 0, s>>>(
            c.long_rows.as<int32_t>(), c.row_ptr.as<int32_t>(),
            c.col.as<int32_t>(), (const V *)c.ev(), x, y, alpha, beta,
            beta != X(0));
    }
  });
  PLS_LAUNCH_CHECK();
}

// ---------------------------------------------------------- SELL-C-sigma

// Sum of one SELL row segment: len padded columns starting at vp / op
// (stride C between consecutive columns of the row). Columns are taken in
// groups of kSellGroup: all value and offset loads of a group are issued
// (predicated past len) before any of the group's dependent x gathers, so a
// row costs two memory round trips per group instead of two per column. The
// products are still added one by one in column order j = 0 .. len-1, the
// order of the reference's spmv_scs<T,C> (src/sell_c_sigma.cpp:727-775).
// Groups of 4 hold 40 registers, which lets 12 blocks of 128 threads share
// an SM where groups of 8 (48 registers) let 10: the extra warps keep more
// rows' loads in flight. Measured in alternating runs: C2 339 -> 323 us, a
// 16.7 M-row 5-point Laplacian 319 -> 264 us, the 27-point stencil 113.7 ->
// 112.7 us (C = 32).
constexpr int kSellGroup = 4;
constexpr int kSellBlocksPerSm = 12;
// 128-thread blocks: on power-law layouts a
// block waits for its slowest chunk, and smaller blocks waste less of the
// SM on that wait than 256-thread ones (measured 1.4% on the C2 matrix,
// 3.4% on a 16.7 M-row Laplacian).
constexpr int kSellThreads = 128;

template <int C, class V, class O, class X>
__device__ __forceinline__ typename AccOf<V, X>::type sell_row_sum(const V *vp, const O *op,
                                                                   const X *xb, int32_t len,
                                                                   const L2Policy &pol) {
  using Acc = typename AccOf<V, X>::type;
  Acc acc = 0;
  for (int32_t j = 0; j < len; j += kSellGroup) {
    V v[kSellGroup];
    O o[kSellGroup];
#pragma unroll
    for (int u = 0; u < kSellGroup; ++u) {
      if (j + u < len) {
        v[u] = ld_stream(vp + u * C, pol.stream);
        o[u] = ld_stream(op + u * C, pol.stream);
      } else {
        v[u] = from_double<V>(0.0);
        o[u] = 0;
      }
    }
    Acc xv[kSellGroup];
#pragma unroll
    for (int u = 0; u < kSellGroup; ++u)
      xv[u] = j + u < len ? to_acc<Acc>(ld_keep(xb + o[u], pol.keep)) : Acc(0);
#pragma unroll
    for (int u = 0; u < kSellGroup; ++u)
      if (j + u < len)
        acc = fma(to_acc<Acc>(v[u]), xv[u], acc);
    vp += kSellGroup * C;
    op += kSellGroup * C;
  }
  return acc;
}

// One launch, two kinds of blocks. Blocks [0, slice_blocks) take column
// slices of the few chunks wider than split_w (power-law tails): item =
// (chunk, j0, j1, slot), slices of slice_w columns, the slices of one chunk
// in consecutive slots from first = slot - j0 / slice_w. The remaining
// blocks take one chunk per C lanes (lane r = row r of the chunk, so the C
// lanes read C consecutive values per column: a full 256-byte line for
// C = 32, FP64) and skip the chunks the slices cover; they take the chunks in
// `order` (decreasing width, or c_base onwards when null). Slices come first,
// then the widest chunks, so the longest work starts earliest and the launch
// ends on the narrowest chunks.
//
// A slice writes its partial sums to part[slot*C + r] and counts itself in
// done[first]; the chunk's last slice to finish adds the chunk's partial
// sums in slice order and writes y. The writes are fenced before the count
// and the finisher fences before it reads them through L2, the pattern of
// the CUDA programming guide's last-block reduction. The finisher puts the
// count back to zero, so done[] is all zero between launches.
template <int C, class V, class O, class X>
__global__ void __launch_bounds__(kSellThreads, kSellBlocksPerSm)
    k_sell(int64_t nC, int64_t c_base, int32_t split_w, int32_t slice_w, int64_t n_items,
           int64_t slice_blocks, const int4 *__restrict__ items,
           const int32_t *__restrict__ order, const int64_t *__restrict__ cs,
           const int32_t *__restrict__ cl, const int32_t *__restrict__ cmin,
           const int32_t *__restrict__ perm, const V *__restrict__ vals,
           const O *__restrict__ offs, const X *__restrict__ x, X *__restrict__ y,
           typename AccOf<V, X>::type *__restrict__ part, int32_t *__restrict__ done, X alpha,
           X beta, int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const L2Policy pol = make_l2_policy();
  if (blockIdx.x < slice_blocks) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t it = t / C;
    if (it >= n_items)
      return;  // whole lane groups: C divides 32
    const int r = (int)(t % C);
    Acc v;
    {
      const int4 w = __ldg(items + it);  // chunk, j0, j1, slot
      const int64_t base = __ldg(cs + w.x) + (int64_t)w.y * C + r;
      const X *xb = x + __ldg(cmin + w.x);
      v = sell_row_sum<C, V, O, X>(vals + base, offs + base, xb, w.z - w.y, pol);
    }
    // The item is read again rather than kept in registers over the sum.
    const int4 w = __ldg(items + it);
    const int lane = threadIdx.x & 31;
    const unsigned group = C == 32 ? 0xffffffffu : ((1u << (C & 31)) - 1) << (lane & ~(C - 1));
    __stcg(part + (int64_t)w.w * C + r, v);
    __threadfence();
    __syncwarp(group);
    const int32_t first = w.w - w.y / slice_w;
    const int32_t ns = (__ldg(cl + w.x) + slice_w - 1) / slice_w;
    int last = 0;
    if (r == 0) {
      last = atomicAdd(done + first, 1) == ns - 1;
      if (last)
        done[first] = 0;
    }
    last = __shfl_sync(group, last, lane & ~(C - 1));
    if (!last)
      return;
    __threadfence();
    Acc acc = 0;
    for (int32_t q = 0; q < ns; ++q)
      acc += __ldcg(part + (int64_t)(first + q) * C + r);
    const int32_t dst = __ldg(perm + (int64_t)w.x * C + r);
    if (dst >= 0)
      store_y(y, dst, acc, alpha, beta, beta_nz);
    return;
  }
  const int64_t t = (int64_t)(blockIdx.x - slice_blocks) * blockDim.x + threadIdx.x;
  const int64_t ci = t / C;
  if (ci >= nC)
    return;
  const int64_t c = order ? (int64_t)__ldg(order + ci) : c_base + ci;
  const int r = (int)(t % C);
  const int32_t w = __ldg(cl + c);
  if (w > split_w)
    return;  // sliced chunk: written by its last slice
  const int64_t base = __ldg(cs + c) + r;
  const int32_t cm = __ldg(cmin + c);
  const int32_t dst = __ldg(perm + c * C + r);
  const X *xb = x + (w > 0 ? cm : 0);
  const Acc acc = sell_row_sum<C, V, O, X>(vals + base, offs + base, xb, w, pol);
  if (dst >= 0)
    store_y(y, dst, acc, alpha, beta, beta_nz);
}

// What one k_sell launch covers: n_chunks chunks (order[0, n_chunks), or
// c_base onwards when order is null) and n_items column slices of slice_w
// columns, with their partial sums in `part` and completion counts in `done`
// (one per slot, zero between launches).
struct SellWork {
  int64_t n_chunks = 0, c_base = 0;
  int32_t split_w = INT32_MAX;  // wider chunks are covered by the slices
  int32_t slice_w = 0;
  const int32_t *order = nullptr;
  int64_t n_items = 0;
  const int4 *items = nullptr;
  void *part = nullptr;
  int32_t *done = nullptr;
};

static SellWork whole_work(const SellDev &s) {
  SellWork w;
  w.n_chunks = s.nC;
  w.order = s.order.as<int32_t>();
  if (s.n_items > 0) {
    w.split_w = s.split_w;
    w.slice_w = s.slice_w;
    w.n_items = s.n_items;
    w.items = s.items.as<int4>();
    w.part = s.part.p;
    w.done = s.done.as<int32_t>();
  }
  return w;
}

template <int C, class V, class O, class X>
static void launch_sell(const SellDev &s, const SellWork &w, const X *x, X *y, X alpha,
                        X beta, cudaStream_t st) {
  using Acc = typename AccOf<V, X>::type;
  const int bnz = beta != X(0);
  const int64_t slice_blocks = w.n_items > 0 ? div_up(w.n_items * C, kSellThreads) : 0;
  const int64_t chunk_blocks = div_up(w.n_chunks * C, kSellThreads);
  if (slice_blocks + chunk_blocks == 0)
    return;
  k_sell<C, V, O, X><<<(unsigned)(slice_blocks + chunk_blocks), kSellThreads, 0, st>>>(
      w.n_chunks, w.c_base, w.split_w, w.slice_w, w.n_items, slice_blocks, w.items, w.order,
      s.cs.as<int64_t>(), s.cl.as<int32_t>(), s.col_min.as<int32_t>(), s.permd2in.as<int32_t>(),
      s.vals.as<V>(), s.offsets.as<O>(), x, y, (Acc *)w.part, w.done, alpha, beta, bnz);
}

template <int C, class V, class X>
static void sell_by_width(const SellDev &s, const SellWork &w, const X *x, X *y, X alpha,
                          X beta, cudaStream_t st) {
  switch (s.col_bytes) {
  case 1: launch_sell<C, V, uint8_t, X>(s, w, x, y, alpha, beta, st); break;
  case 2: launch_sell<C, V, uint16_t, X>(s, w, x, y, alpha, beta, st); break;
  case 4: launch_sell<C, V, uint32_t, X>(s, w, x, y, alpha, beta, st); break;
  default:
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "unsupported SELL offset width");
  }
}

template <class X>
static void run_sell(const SellDev &s, const SellWork &w, const X *x, X *y, X alpha, X beta,
                     cudaStream_t st) {
  if (s.nC == 0)
    return;
  with_vt(s.vt, [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      switch (s.C) {
      case 8: sell_by_width<8, V, X>(s, w, x, y, alpha, beta, st); break;
      case 16: sell_by_width<16, V, X>(s, w, x, y, alpha, beta, st); break;
      case 32: sell_by_width<32, V, X>(s, w, x, y, alpha, beta, st); break;
      default:
        throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "SELL chunk height must be 8, 16 or 32");
      }
    }
  });
  PLS_LAUNCH_CHECK();
}

template <class X>
void spmv_sell(const SellDev &s, const X *x, X *y, X alpha, X beta,
               cudaStream_t st) {
  run_sell<X>(s, whole_work(s), x, y, alpha, beta, st);
}

// ------------------------------------------ row bands (host-buffer calls)

template <class T>
static std::vector<T> to_host(const DevBuf &b, int64_t n) {
  std::vector<T> h((size_t)n);
  if (n > 0)
    PLS_CUDA(cudaMemcpy(h.data(), b.p, sizeof(T) * (size_t)n, cudaMemcpyDeviceToHost));
  return h;
}

template <class T>
static void to_device(DevBuf &b, const std::vector<T> &h) {
  b.reserve(sizeof(T) * std::max<size_t>(h.size(), 1));
  if (!h.empty())
    PLS_CUDA(cudaMemcpy(b.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}

// Plans are uploaded with cudaMemcpy / cudaMemset on the legacy stream, which
// the library's non-blocking streams do not wait for (and a copy from
// pageable memory may still be in flight when cudaMemcpy returns): a plan
// ends with a device synchronisation before any kernel reads it.

// Stable grouping of `v` by band: band b's elements keep their order and
// land in [first[b], first[b + 1]).
template <class T, class F>
static std::vector<T> group_by_band(const std::vector<T> &v, size_t n_bands, F band_of,
                                    std::vector<int64_t> &first) {
  first.assign(n_bands + 1, 0);
  for (const T &e : v)
    first[band_of(e) + 1]++;
  for (size_t b = 0; b < n_bands; ++b)
    first[b + 1] += first[b];
  std::vector<int64_t> at(first.begin(), first.end() - 1);
  std::vector<T> out(v.size());
  for (const T &e : v)
    out[(size_t)at[band_of(e)]++] = e;
  return out;
}

// A band is a run of whole sort windows (sigma rows; C rows without
// sorting), so the permutation keeps its rows inside it and its chunks
// [c0, c1) write exactly the rows [c0*C, c1*C) of y. Inside a band the
// chunks keep the layout's processing order (widest first for power-law
// layouts). A band's launch lasts at least as long as one lane group's walk
// along its widest unsliced chunk, a floor that a whole-matrix launch hides
// under other work but a band of a few tens of microseconds does not; so the
// plan slices every chunk wider than 2 * kBandSliceW columns into slices of
// kBandSliceW, widest chunks first within each band.
constexpr int32_t kBandSliceW = 32;

void sell_plan_bands(SellDev &s, int64_t m, int n_bands) {
  if (s.bands.planned == n_bands)
    return;
  s.bands.clear();
  s.bands.planned = n_bands;
  if (s.nC == 0 || n_bands < 1)
    return;
  const int64_t window = (s.sigma > 0 ? s.sigma : s.C) / s.C;  // chunks
  const int64_t per = div_up(div_up(s.nC, window), (int64_t)n_bands) * window;
  std::vector<RowBand> bands;
  for (int64_t c0 = 0; c0 < s.nC; c0 += per) {
    RowBand b;
    b.c0 = c0;
    b.c1 = std::min(s.nC, c0 + per);
    b.r0 = c0 * s.C;
    b.r1 = std::min(m, b.c1 * s.C);
    bands.push_back(b);
  }
  const size_t nb = bands.size();
  const auto band_of = [&](int64_t c) { return (size_t)(c / per); };
  std::vector<int64_t> first;
  if (s.order.p) {
    const auto ord = group_by_band(to_host<int32_t>(s.order, s.nC), nb,
                                   [&](int32_t c) { return band_of(c); }, first);
    to_device(s.bands.order, ord);
  }
  const std::vector<int32_t> cl = to_host<int32_t>(s.cl, s.nC);
  std::vector<int32_t> wide;
  for (int64_t c = 0; c < s.nC; ++c)
    if (cl[c] > 2 * kBandSliceW)
      wide.push_back((int32_t)c);
  if (!wide.empty()) {
    std::stable_sort(wide.begin(), wide.end(),
                     [&](int32_t a, int32_t b) { return cl[a] > cl[b]; });
    wide = group_by_band(wide, nb, [&](int32_t c) { return band_of(c); }, first);
    std::vector<int4> items;
    int32_t slot = 0;
    for (size_t b = 0; b < nb; ++b) {
      bands[b].i0 = (int64_t)items.size();
      for (int64_t k = first[b]; k < first[b + 1]; ++k) {
        const int32_t c = wide[(size_t)k];
        const int32_t ns = (int32_t)div_up(cl[c], kBandSliceW);
        for (int32_t q = 0; q < ns; ++q)
          items.push_back(make_int4(c, q * kBandSliceW,
                                    std::min(cl[c], (q + 1) * kBandSliceW), slot + q));
        slot += ns;
      }
      bands[b].i1 = (int64_t)items.size();
    }
    to_device(s.bands.items, items);
    s.bands.part.reserve(sizeof(double) * (size_t)slot * s.C);  // FP64 covers both accumulators
    s.bands.done.reserve(sizeof(int32_t) * (size_t)slot);
    PLS_CUDA(cudaMemset(s.bands.done.p, 0, sizeof(int32_t) * (size_t)slot));
    s.bands.split_w = 2 * kBandSliceW;
  }
  s.bands.bands = std::move(bands);
  PLS_CUDA(cudaDeviceSynchronize());
}

template <class X>
void spmv_sell_band(const SellDev &s, const RowBand &b, const X *x, X *y, X alpha, X beta,
                    cudaStream_t st) {
  SellWork w;
  w.n_chunks = b.c1 - b.c0;
  w.c_base = b.c0;
  w.split_w = s.bands.split_w;
  w.slice_w = kBandSliceW;
  w.order = s.bands.order.p ? s.bands.order.as<int32_t>() + b.c0 : nullptr;
  w.n_items = b.i1 - b.i0;
  w.items = s.bands.items.p ? s.bands.items.as<int4>() + b.i0 : nullptr;
  w.part = s.bands.part.p;
  w.done = s.bands.done.as<int32_t>();
  run_sell<X>(s, w, x, y, alpha, beta, st);
}

// CSR bands: equal row counts; the long rows (when the split kernels are
// configured) sorted so that each band's are a contiguous run.
void csr_plan_bands(CsrDev &c, int32_t m, int n_bands) {
  if (c.bands.planned == n_bands)
    return;
  c.bands.clear();
  c.bands.planned = n_bands;
  if (m == 0 || n_bands < 1)
    return;
  const int64_t per = div_up((int64_t)m, (int64_t)n_bands);
  std::vector<RowBand> bands;
  for (int64_t r0 = 0; r0 < m; r0 += per) {
    RowBand b;
    b.r0 = r0;
    b.r1 = std::min<int64_t>(m, r0 + per);
    bands.push_back(b);
  }
  if (c.n_long > 0) {
    std::vector<int32_t> rows = to_host<int32_t>(c.long_rows, c.n_long);
    std::sort(rows.begin(), rows.end());
    for (RowBand &b : bands) {
      b.i0 = std::lower_bound(rows.begin(), rows.end(), (int32_t)b.r0) - rows.begin();
      b.i1 = std::lower_bound(rows.begin(), rows.end(), (int32_t)b.r1) - rows.begin();
    }
    to_device(c.bands.order, rows);
  }
  c.bands.bands = std::move(bands);
  PLS_CUDA(cudaDeviceSynchronize());
}

template <class X>
void spmv_csr_band(const CsrDev &c, const RowBand &b, int tpr, const X *x, X *y, X alpha,
                   X beta, cudaStream_t s) {
  const int32_t mb = (int32_t)(b.r1 - b.r0);
  if (mb == 0)
    return;
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else if (tpr > 0) {
      csr_vector_dispatch<V, X>(c, b.r0, mb, tpr, x, y, alpha, beta, 0, s);
    } else {
      const int32_t thr = c.long_threshold;
      csr_vector_dispatch<V, X>(c, b.r0, mb, split_tpr(thr), x, y, alpha, beta, thr, s);
      if (b.i1 > b.i0)
        k_csr_long<V, X><<<(unsigned)(b.i1 - b.i0), 256, 0, s>>>(
            c.bands.order.as<int32_t>() + b.i0, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(),
            (const V *)c.ev(), x, y, alpha, beta, beta != X(0));
    }
  });
  PLS_LAUNCH_CHECK();
}

// -------------------------------------- SELL SpMV without allocation

// Fixed device arrays of the allocation-free SELL entry point, instead of
// per-handle cudaMalloc buffers: the partial sums of the column slices of
// wide chunks (2^21 FP64 elements) and their completion counts (one per
// slot; C >= 8, so 2^18 of them). Every GPU that loads the library holds
// these 17 MiB until the process exits. All calls share them, so calls that
// overlap on the GPU (different streams, or different host threads) race on
// them.
constexpr int64_t kNoAllocScratchElems = int64_t(1) << 21;
constexpr int64_t kNoAllocSlots = kNoAllocScratchElems / 8;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchElems];
static __device__ int32_t g_noalloc_done[kNoAllocSlots];  // zero at load

namespace {
// The arrays' device addresses, per device, with the context they were
// looked up in: after cudaDeviceReset the device's primary context (and the
// module holding the arrays) is created anew, so a lookup is only reused
// while the same context is current.
struct NoAllocAddrs {
  void *ctx = nullptr;
  void *part = nullptr;
  void *count = nullptr;
};
std::mutex g_noalloc_mu;
NoAllocAddrs g_noalloc[64];

// The driver's cuCtxGetCurrent, reached through the runtime (no link to the
// driver library); null if the driver does not offer it.
using CtxGetCurrentFn = int (*)(void **);
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrentFn) nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// The context current on this thread (the caller's DeviceGuard made the
// device current, which binds its primary context); null if unknown.
void *current_context() {
  void *ctx = nullptr;
  const CtxGetCurrentFn fn = ctx_get_current();
  if (!fn || fn(&ctx) != 0)
    return nullptr;
  return ctx;
}

void *symbol_address(const void *sym, const char *what) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, sym);
  if (e != cudaSuccess)
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                std::string("cudaGetSymbolAddress(") + what + "): " + cudaGetErrorString(e));
  return p;
}
}  // namespace

// The SELL SpMV with its slices' partial sums and counts in the fixed
// arrays. Their device addresses come from cudaGetSymbolAddress (in host code
// the arrays' names are only host-side stand-ins), once per device and
// context, with that device current (the caller's DeviceGuard makes it
// current); a call that finds another context current (the device was reset
// since) looks them up again. Every slot a call reads was written earlier in
// the same call, and the counts return to zero by the end of every launch,
// so nothing needs clearing between calls.
void spmv_sell_noalloc(const SellDev &s, const double *x, double *y, double alpha, double beta,
                       int device, cudaStream_t st) {
  if (s.nC == 0)
    return;
  const int64_t slots = s.n_items > 0 ? (int64_t)(s.done.bytes / sizeof(int32_t)) : 0;
  if (slots * s.C > kNoAllocScratchElems)
    throw Error(PERFLIBS_STATUS_INPUT_PARAMETER_ERROR,
                "this matrix needs " + std::to_string(slots * s.C) +
                    " scratch elements; the fixed scratch holds " +
                    std::to_string(kNoAllocScratchElems));
  SellWork w = whole_work(s);
  {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    NoAllocAddrs &a = g_noalloc[device & 63];
    void *ctx = current_context();
    if (!a.part || !ctx || ctx != a.ctx) {
      a.part = symbol_address(g_noalloc_scratch, "scratch");
      a.count = symbol_address(g_noalloc_done, "counts");
      a.ctx = ctx;
    }
    w.part = a.part;
    w.done = static_cast<int32_t *>(a.count);
  }
  run_sell<double>(s, w, x, y, alpha, beta, st);
}

// ------------------------------------------------------------ transpose

// y = alpha*A^T*x + beta*y: y scaled first, then every nonzero scatters
// alpha*val*x[row] into y[col] (the reference's spmv_csr_trans scheme,
// src/compressed_sparse_rows.cpp:1558-1676, with hardware atomics).
template <class V, class X>
__global__ void k_csr_trans_scatter(int32_t m, const int32_t *__restrict__ rp,
                                    const int32_t *__restrict__ col,
                                    const V *__restrict__ val,
                                    const X *__restrict__ x, X *__restrict__ y,
                                    X alpha) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t row = gid / 32;
  if (row >= m)
    return;
  const int lane = threadIdx.x & 31;
  const X xr = alpha * x[row];
  for (int32_t j = rp[row] + lane; j < rp[row + 1]; j += 32)
    atomicAdd(y + col[j], (X)to_acc<double>(val[j]) * xr);
}

template <class X> __global__ void k_scal(int64_t n, X beta, X *y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    y[i] = beta == X(0) ? X(0) : y[i] * beta;
}

template <class X>
__global__ void k_axpby(int64_t n, X alpha, const X *x, X beta, X *y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    y[i] = alpha * x[i] + (beta == X(0) ? X(0) : beta * y[i]);
}

template <class X> void scal(int64_t n, X beta, X *y, cudaStream_t s) {
  if (n <= 0)
    return;
  k_scal<X><<<(unsigned)div_up(n, 256), 256, 0, s>>>(n, beta, y);
  PLS_LAUNCH_CHECK();
}

template <class X>
void axpby(int64_t n, X alpha, const X *x, X beta, X *y, cudaStream_t s) {
  if (n <= 0)
    return;
  k_axpby<X><<<(unsigned)div_up(n, 256), 256, 0, s>>>(n, alpha, x, beta, y);
  PLS_LAUNCH_CHECK();
}

template <class X>
void spmv_csr_trans(const CsrDev &c, int32_t m, int32_t n, const X *x, X *y,
                    X alpha, X beta, cudaStream_t s) {
  scal<X>(n, beta, y, s);
  if (m == 0 || c.nnz == 0)
    return;
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    k_csr_trans_scatter<V, X><<<(unsigned)div_up((int64_t)m * 32, 256), 256, 0, s>>>(
        m, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), (const V *)c.ev(), x, y,
        alpha);
  });
  PLS_LAUNCH_CHECK();
}

// -------------------------------------------------------------- dense

// Output row i of op(A) with element (i, j) at A[i*rs + j*cs]. A warp per
// row when the row is contiguous, a thread per row otherwise.
template <class X>
__global__ void k_gemv_warp(int64_t rows, int64_t cols, const X *A, int64_t rs,
                            const X *x, X *y, X alpha, X beta) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  if (row >= rows)
    return;
  const int lane = threadIdx.x & 31;
  X s = 0;
  for (int64_t j = lane; j < cols; j += 32)
    s = fma(A[row * rs + j], x[j], s);
  s = group_sum<32>(s, 0xffffffffu);
  if (lane == 0)
    y[row] = alpha * s + (beta == X(0) ? X(0) : beta * y[row]);
}

template <class X>
__global__ void k_gemv_thread(int64_t rows, int64_t cols, const X *A,
                              int64_t cs, const X *x, X *y, X alpha, X beta) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows)
    return;
  X s = 0;
  for (int64_t j = 0; j < cols; ++j)
    s = fma(A[row + j * cs], x[j], s);
  y[row] = alpha * s + (beta == X(0) ? X(0) : beta * y[row]);
}

template <class X>
void spmv_dense(const DenseDev &d, int32_t m, int32_t n, bool trans,
                const X *x, X *y, X alpha, X beta, cudaStream_t s) {
  const int64_t rows = trans ? n : m, cols = trans ? m : n;
  if (rows == 0)
    return;
  // Stored element (r, c) at r*lda (row-major) or c*lda (column-major).
  const bool row_contig = (d.layout == PERFLIBS_ROW_MAJOR) != trans;
  const X *A = d.vals.as<X>();
  if (row_contig)
    k_gemv_warp<X><<<(unsigned)div_up(rows * 32, 256), 256, 0, s>>>(
        rows, cols, A, d.lda, x, y, alpha, beta);
  else
    k_gemv_thread<X><<<(unsigned)div_up(rows, 256), 256, 0, s>>>(
        rows, cols, A, d.lda, x, y, alpha, beta);
  PLS_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- BSR

// Block sizes whose bs*bs elements tile a warp (bs = 1, 2, 4): a warp per
// block row; lane l owns element e = l % (bs*bs) of 32/(bs*bs) consecutive
// blocks per step, so every step reads 32 consecutive values. Lanes holding
// the same scalar row are reduced with shuffles at the end.
template <int BS, class V, class X>
__global__ void __launch_bounds__(256)
    k_bsr_small(int32_t mb, int layout, const int32_t *__restrict__ rp,
                const int32_t *__restrict__ col, const V *__restrict__ val,
                const X *__restrict__ x, X *__restrict__ y, X alpha, X beta,
                int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  constexpr int E = BS * BS, PER = 32 / E;
  const int64_t br = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  if (br >= mb)
    return;
  const int lane = threadIdx.x & 31, e = lane % E, slot = lane / E;
  const bool rm = layout == PERFLIBS_ROW_MAJOR;
  const int i = rm ? e / BS : e % BS;
  const int j = rm ? e % BS : e / BS;
  Acc acc = 0;
  for (int32_t b = rp[br] + slot; b < rp[br + 1]; b += PER) {
    const Acc v = to_acc<Acc>(ld_stream(val + (int64_t)b * E + e));
    acc = fma(v, to_acc<Acc>(ld_ro(x + (int64_t)ld_stream(col + b) * BS + j)), acc);
  }
  // Reduce over all lanes with the same i: the j bits and the slot bits.
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int lo = rm ? o : o;  // lane bit o
    const bool is_i_bit = rm ? (o >= BS && o < E) : (o < BS);
    if (!is_i_bit)
      acc += __shfl_xor_sync(0xffffffffu, acc, lo);
  }
  const bool owner = rm ? (j == 0 && slot == 0) : (j == 0 && slot == 0);
  if (owner) {
    const int64_t r = br * BS + i;
    store_y(y, r, acc, alpha, beta, beta_nz);
  }
}

// Any block size: a thread per scalar row.
template <class V, class X>
__global__ void __launch_bounds__(256)
    k_bsr_rows(int32_t mb, int bs, int layout, const int32_t *__restrict__ rp,
               const int32_t *__restrict__ col, const V *__restrict__ val,
               const X *__restrict__ x, X *__restrict__ y, X alpha, X beta,
               int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (int64_t)mb * bs)
    return;
  const int64_t br = r / bs;
  const int i = (int)(r % bs);
  const int64_t E = (int64_t)bs * bs;
  const bool rm = layout == PERFLIBS_ROW_MAJOR;
  Acc acc = 0;
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b) {
    const V *blk = val + (int64_t)b * E;
    const X *xb = x + (int64_t)col[b] * bs;
    for (int j = 0; j < bs; ++j) {
      const V v = rm ? ld_stream(blk + (int64_t)i * bs + j) : ld_stream(blk + (int64_t)j * bs + i);
      acc = fma(to_acc<Acc>(v), to_acc<Acc>(ld_ro(xb + j)), acc);
    }
  }
  store_y(y, r, acc, alpha, beta, beta_nz);
}

template <class X>
void spmv_bsr(const BsrDev &b, const X *x, X *y, X alpha, X beta,
              cudaStream_t s) {
  if (b.mb == 0)
    return;
  const int bnz = beta != X(0);
  with_vt(b.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      const unsigned wblocks = (unsigned)div_up((int64_t)b.mb * 32, 256);
      switch (b.bs) {
      case 1:
        k_bsr_small<1, V, X><<<wblocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), x, y, alpha, beta, bnz);
        break;
      case 2:
        k_bsr_small<2, V, X><<<wblocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), x, y, alpha, beta, bnz);
        break;
      case 4:
        k_bsr_small<4, V, X><<<wblocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), x, y, alpha, beta, bnz);
        break;
      default:
        k_bsr_rows<V, X><<<(unsigned)div_up((int64_t)b.mb * b.bs, 256), 256, 0, s>>>(
            b.mb, b.bs, b.layout, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(),
            (const V *)b.ev(), x, y, alpha, beta, bnz);
      }
    }
  });
  PLS_LAUNCH_CHECK();
}

// ------------------------------------------------------ instantiations
#define PLS_INST(X)                                                            \
  template void spmv_csr<X>(const CsrDev &, int32_t, int, const X *, X *, X,  \
                            X, cudaStream_t);                                  \
  template void spmv_csr_split<X>(const CsrDev &, int32_t, const X *, X *, X, \
                                  X, cudaStream_t);                            \
  template void spmv_sell<X>(const SellDev &, const X *, X *, X, X,           \
                             cudaStream_t);                                    \
  template void spmv_sell_band<X>(const SellDev &, const RowBand &, const X *, \
                                  X *, X, X, cudaStream_t);                    \
  template void spmv_csr_band<X>(const CsrDev &, const RowBand &, int,         \
                                 const X *, X *, X, X, cudaStream_t);          \
  template void spmv_bsr<X>(const BsrDev &, const X *, X *, X, X,             \
                            cudaStream_t);                                     \
  template void spmv_csr_trans<X>(const CsrDev &, int32_t, int32_t,           \
                                  const X *, X *, X, X, cudaStream_t);         \
  template void spmv_dense<X>(const DenseDev &, int32_t, int32_t, bool,       \
                              const X *, X *, X, X, cudaStream_t);             \
  template void axpby<X>(int64_t, X, const X *, X, X *, cudaStream_t);        \
  template void scal<X>(int64_t, X, X *, cudaStream_t);

PLS_INST(float)
PLS_INST(double)

}  // namespace pls
