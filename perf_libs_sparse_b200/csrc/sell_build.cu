// Device CSR -> SELL-C-sigma builder.
//
// Produces, element for element, the layout of the reference's csr2scs +
// gen_data_vectors (src/sell_c_sigma.cpp:145-336, 584-705):
//   1. rows are grouped in windows of sigma rows; inside a window they are
//      ordered by (row length, row index), both descending — the order
//      std::sort with std::greater<> gives std::pair<len, row>
//      (sell_c_sigma.cpp:186-202). The unused tail slots of the last window
//      behave as (0, 0) pairs, exactly like the reference's value-initialised
//      pairs. sigma = 0 means no sorting and a window of C rows.
//   2. chunk c holds sorted positions [c*C, c*C + C); its width cl[c] is the
//      first position's length (sorted) or the chunk maximum (unsorted);
//      cs is the exclusive prefix sum of cl*C (:204-231).
//   3. col_min[c] is the smallest column of the chunk's real rows (INT32_MAX
//      when they are all empty); the offset width in bytes follows from the
//      largest chunk column range: bits(range)/8 + 1, 3 -> 4, > 4 -> 8
//      (:236-320).
//   4. element (r, j) of chunk c is written at cs[c] + j*C + r: the row's
//      j-th value and column offset, or 0 / 0 past the row end and for
//      padding rows (:611-704).
// The window sort is a bitonic sort of 64-bit keys (len << 32 | row) in
// shared memory, one CTA per window; everything else is one thread per row
// or per (chunk, row).
#include <algorithm>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

constexpr int kSortThreads = 1024;
constexpr int kMaxSortWindow = 16384;  // 128 KB of keys in shared memory

// Sort each window of `sigma` rows by key descending; write, per sorted
// position, the row (or -1 past the last row) and its length.
__global__ void __launch_bounds__(kSortThreads)
    k_window_sort(int32_t m, int32_t sigma, int32_t npow2,
                  const int32_t *__restrict__ rp, int32_t *__restrict__ pos_row,
                  int32_t *__restrict__ pos_len) {
  extern __shared__ unsigned long long keys[];
  const int64_t w0 = (int64_t)blockIdx.x * sigma;
  for (int p = threadIdx.x; p < npow2; p += blockDim.x) {
    unsigned long long k = 0ull;  // (0, 0): unused slot
    if (p < sigma && w0 + p < m) {
      const int64_t row = w0 + p;
      const unsigned long long len = (unsigned long long)(rp[row + 1] - rp[row]);
      k = (len << 32) | (unsigned long long)row;
    }
    keys[p] = k;
  }
  __syncthreads();
  // Bitonic sort, descending.
  for (int size = 2; size <= npow2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (npow2 >> 1); t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool desc = ((lo & size) == 0);
        const unsigned long long a = keys[lo], b = keys[hi];
        if ((a < b) == desc) {
          keys[lo] = b;
          keys[hi] = a;
        }
      }
      __syncthreads();
    }
  }
  for (int p = threadIdx.x; p < sigma; p += blockDim.x) {
    const int64_t pos = w0 + p;
    // Positions at or past m are padding (the reference maps only the first
    // min(C, rows - c*C) entries of each chunk).
    const unsigned long long k = keys[p];
    pos_row[pos] = pos < m ? (int32_t)(k & 0xffffffffull) : -1;
    pos_len[pos] = pos < m ? (int32_t)(k >> 32) : 0;
  }
}

// No sorting: position == row.
__global__ void k_identity_positions(int64_t npos, int32_t m,
                                     const int32_t *__restrict__ rp,
                                     int32_t *__restrict__ pos_row,
                                     int32_t *__restrict__ pos_len) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npos)
    return;
  pos_row[p] = p < m ? (int32_t)p : -1;
  pos_len[p] = p < m ? rp[p + 1] - rp[p] : 0;
}

__global__ void k_chunk_width(int64_t nC, int C, int sorted,
                              const int32_t *__restrict__ pos_len,
                              int32_t *__restrict__ cl) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nC)
    return;
  int32_t w = 0;
  if (sorted) {
    w = pos_len[c * C];
  } else {
    for (int r = 0; r < C; ++r)
      w = max(w, pos_len[c * C + r]);
  }
  cl[c] = w;
}

// Exclusive scan of cl[c]*C into cs (one CTA; optimize-time only).
__global__ void __launch_bounds__(1024)
    k_chunk_starts(int64_t nC, int C, const int32_t *__restrict__ cl,
                   int64_t *__restrict__ cs, int64_t *__restrict__ total) {
  __shared__ int64_t part[1024];
  const int64_t per = div_up(nC, blockDim.x);
  const int64_t b = threadIdx.x * per, e = min(nC, b + per);
  int64_t s = 0;
  for (int64_t c = b; c < e; ++c)
    s += (int64_t)cl[c] * C;
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const int64_t v = part[t];
      part[t] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  int64_t run = part[threadIdx.x];
  for (int64_t c = b; c < e; ++c) {
    cs[c] = run;
    run += (int64_t)cl[c] * C;
  }
}

__global__ void k_row_col_range(int32_t m, const int32_t *__restrict__ rp,
                                const int32_t *__restrict__ col,
                                int32_t *__restrict__ rmin,
                                int32_t *__restrict__ rmax) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  int32_t lo = INT32_MAX, hi = 0;
  for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
    const int32_t c = col[j];
    lo = min(lo, c);
    hi = max(hi, c);
  }
  rmin[i] = lo;
  rmax[i] = hi;
}

__global__ void k_chunk_minmax_perm(int64_t nC, int C, int32_t m,
                                    const int32_t *__restrict__ pos_row,
                                    const int32_t *__restrict__ rmin,
                                    const int32_t *__restrict__ rmax,
                                    int32_t *__restrict__ col_min,
                                    int32_t *__restrict__ permd2in,
                                    int32_t *__restrict__ in2permd,
                                    unsigned long long *__restrict__ range) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nC)
    return;
  int32_t lo = INT32_MAX, hi = 0;
  for (int r = 0; r < C; ++r) {
    const int64_t pos = c * C + r;
    const int32_t row = pos < m ? pos_row[pos] : -1;
    permd2in[pos] = row;
    if (row >= 0) {
      in2permd[row] = (int32_t)pos;
      lo = min(lo, rmin[row]);
      hi = max(hi, rmax[row]);
    }
  }
  col_min[c] = lo;
  const int64_t rg = (int64_t)hi - (int64_t)lo;
  if (rg > 0)
    atomicMax(range, (unsigned long long)rg);
}

template <class V, class O>
__global__ void k_fill(int64_t nC, int C, const int64_t *__restrict__ cs,
                       const int32_t *__restrict__ cl,
                       const int32_t *__restrict__ col_min,
                       const int32_t *__restrict__ permd2in,
                       const int32_t *__restrict__ rp,
                       const int32_t *__restrict__ col,
                       const V *__restrict__ val, V *__restrict__ out_v,
                       O *__restrict__ out_o) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t c = t / C;
  if (c >= nC)
    return;
  const int r = (int)(t % C);
  const int32_t row = permd2in[c * C + r];
  int32_t s = 0, len = 0;
  if (row >= 0) {
    s = rp[row];
    len = rp[row + 1] - s;
  }
  const int32_t w = cl[c];
  const int64_t base = cs[c] + r;
  const int32_t cmin = col_min[c];
  for (int32_t j = 0; j < w; ++j) {
    const int64_t o = base + (int64_t)j * C;
    if (j < len) {
      out_v[o] = val[s + j];
      out_o[o] = (O)(col[s + j] - cmin);
    } else {
      out_v[o] = V(0);
      out_o[o] = (O)0;
    }
  }
}

}  // namespace

void build_sell(const CsrDev &c, int32_t m, int C, int sigma, SellDev &out,
                cudaStream_t s) {
  if (C <= 0)
    throw Error(PERFLIBS_STATUS_INPUT_PARAMETER_ERROR, "SELL chunk height must be positive");
  if (sigma != 0 && sigma % C != 0)
    throw Error(PERFLIBS_STATUS_INPUT_PARAMETER_ERROR, "sigma must be 0 or a multiple of C");
  const bool sorted = sigma != 0;
  const int32_t win = sorted ? sigma : C;
  if (sorted && sigma > kMaxSortWindow)
    throw Error(PERFLIBS_STATUS_INPUT_PARAMETER_ERROR, "sigma above 16384 rows is not supported");

  SellDev S;
  S.C = C;
  S.sigma = sigma;
  S.vt = c.evt();  // the kernels' value copy (reduced under FP32 / BF16 storage)
  S.nC = div_up(m, C);
  const int64_t nwin = div_up(m, win);
  const int64_t npos = nwin * win;  // >= nC*C
  const int32_t *rp = c.row_ptr.as<int32_t>();

  DevBuf pos_row, pos_len, rmin, rmax, scratch;
  pos_row.reserve(sizeof(int32_t) * std::max<int64_t>(npos, 1));
  pos_len.reserve(sizeof(int32_t) * std::max<int64_t>(npos, 1));
  if (m > 0) {
    if (sorted) {
      int npow2 = 1;
      while (npow2 < win)
        npow2 <<= 1;
      const size_t smem = sizeof(unsigned long long) * npow2;
      PLS_CUDA(cudaFuncSetAttribute(k_window_sort,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
      k_window_sort<<<(unsigned)nwin, kSortThreads, smem, s>>>(
          m, win, npow2, rp, pos_row.as<int32_t>(), pos_len.as<int32_t>());
    } else {
      k_identity_positions<<<(unsigned)div_up(npos, 256), 256, 0, s>>>(
          npos, m, rp, pos_row.as<int32_t>(), pos_len.as<int32_t>());
    }
    PLS_LAUNCH_CHECK();
  }

  S.cs.reserve(sizeof(int64_t) * std::max<int64_t>(S.nC, 1));
  S.cl.reserve(sizeof(int32_t) * std::max<int64_t>(S.nC, 1));
  S.col_min.reserve(sizeof(int32_t) * std::max<int64_t>(S.nC, 1));
  S.permd2in.reserve(sizeof(int32_t) * std::max<int64_t>(S.nC * C, 1));
  S.in2permd.reserve(sizeof(int32_t) * std::max<int32_t>(m, 1));
  scratch.reserve(16);
  PLS_CUDA(cudaMemsetAsync(scratch.p, 0, 16, s));
  int64_t total = 0;
  unsigned long long range = 0;
  if (S.nC > 0) {
    k_chunk_width<<<(unsigned)div_up(S.nC, 256), 256, 0, s>>>(
        S.nC, C, sorted, pos_len.as<int32_t>(), S.cl.as<int32_t>());
    k_chunk_starts<<<1, 1024, 0, s>>>(S.nC, C, S.cl.as<int32_t>(),
                                      S.cs.as<int64_t>(), scratch.as<int64_t>());
    rmin.reserve(sizeof(int32_t) * m);
    rmax.reserve(sizeof(int32_t) * m);
    k_row_col_range<<<(unsigned)div_up(m, 256), 256, 0, s>>>(
        m, rp, c.col.as<int32_t>(), rmin.as<int32_t>(), rmax.as<int32_t>());
    k_chunk_minmax_perm<<<(unsigned)div_up(S.nC, 256), 256, 0, s>>>(
        S.nC, C, m, pos_row.as<int32_t>(), rmin.as<int32_t>(),
        rmax.as<int32_t>(), S.col_min.as<int32_t>(), S.permd2in.as<int32_t>(),
        S.in2permd.as<int32_t>(),
        (unsigned long long *)(scratch.as<char>() + 8));
    PLS_LAUNCH_CHECK();
    int64_t h2[2];
    PLS_CUDA(cudaMemcpyAsync(h2, scratch.p, 16, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    total = h2[0];
    range = (unsigned long long)h2[1];
    int32_t wmax = 0;
    {
      std::vector<int32_t> clh(S.nC);
      PLS_CUDA(cudaMemcpy(clh.data(), S.cl.p, sizeof(int32_t) * S.nC,
                          cudaMemcpyDeviceToHost));
      int64_t wsum = 0;
      for (auto v : clh) {
        wmax = std::max(wmax, v);
        wsum += v;
      }
      // Longest-first processing order over the whole matrix: the widest
      // chunks start first and the launch ends on the narrowest, and chunks
      // of one block have similar widths, so its warps finish together. It
      // costs one dependent load per chunk, so it is kept for layouts whose
      // widest chunk is more than twice the mean width (power-law rows),
      // where the uneven tail is what it removes.
      if ((int64_t)wmax * S.nC > 2 * wsum) {
        std::vector<int32_t> ord(S.nC);
        for (int64_t i = 0; i < S.nC; ++i)
          ord[i] = (int32_t)i;
        std::stable_sort(ord.begin(), ord.end(),
                         [&](int32_t a, int32_t b) { return clh[a] > clh[b]; });
        S.order.reserve(sizeof(int32_t) * S.nC);
        PLS_CUDA(cudaMemcpy(S.order.p, ord.data(), sizeof(int32_t) * S.nC,
                            cudaMemcpyHostToDevice));
        // The copy runs on the legacy stream, which the library's
        // non-blocking streams do not wait for, and a copy from pageable
        // memory may still be in flight when cudaMemcpy returns.
        PLS_CUDA(cudaDeviceSynchronize());
      }
    }
    S.max_width = wmax;
  }
  S.size = total;

  int bits = 0;
  while (range) {
    range >>= 1;
    bits++;
  }
  int bytes = bits / 8 + 1;
  if (bytes == 3)
    bytes = 4;
  else if (bytes > 4)
    bytes = 8;
  S.col_bytes = bytes;
  const int64_t pad = S.nC * C - m;
  S.n_full_chunks = pad > 0 ? S.nC - 1 : S.nC;
  S.ntidyup = pad == 0 ? 0 : C - pad;

  S.vals.reserve(vt_size(S.vt) * std::max<int64_t>(S.size, 1));
  S.offsets.reserve((size_t)bytes * std::max<int64_t>(S.size, 1));
  if (S.size > 0) {
    const unsigned blocks = (unsigned)div_up(S.nC * C, 256);
    auto fill = [&](auto vtag, auto otag) {
      using V = typename decltype(vtag)::type;
      using O = typename decltype(otag)::type;
      k_fill<V, O><<<blocks, 256, 0, s>>>(
          S.nC, C, S.cs.as<int64_t>(), S.cl.as<int32_t>(),
          S.col_min.as<int32_t>(), S.permd2in.as<int32_t>(), rp,
          c.col.as<int32_t>(), (const V *)c.ev(), S.vals.as<V>(), S.offsets.as<O>());
    };
    auto by_width = [&](auto vtag) {
      switch (bytes) {
      case 1: fill(vtag, Tag<uint8_t>{}); break;
      case 2: fill(vtag, Tag<uint16_t>{}); break;
      case 4: fill(vtag, Tag<uint32_t>{}); break;
      default: fill(vtag, Tag<uint64_t>{}); break;
      }
    };
    switch (S.vt) {
    case Vt::F64: by_width(Tag<double>{}); break;
    case Vt::F32: by_width(Tag<float>{}); break;
    case Vt::BF16: by_width(Tag<__nv_bfloat16>{}); break;
    }
    PLS_LAUNCH_CHECK();
  }
  PLS_CUDA(cudaStreamSynchronize(s));
  out = std::move(S);
}

// Padded size cs[nC-1] + cl[nC-1]*C of the (C, sigma) layout, without
// building it (used for the padding-efficiency statistics).
int64_t sell_padded_size(const CsrDev &c, int32_t m, int C, int sigma, cudaStream_t s) {
  if (m == 0)
    return 0;
  const bool sorted = sigma != 0;
  const int32_t win = sorted ? sigma : C;
  const int64_t nC = div_up(m, C);
  const int64_t nwin = div_up(m, win);
  const int64_t npos = nwin * win;
  DevBuf pos_row, pos_len, cl, cs, total;
  pos_row.reserve(4 * npos);
  pos_len.reserve(4 * npos);
  cl.reserve(4 * nC);
  cs.reserve(8 * nC);
  total.reserve(8);
  const int32_t *rp = c.row_ptr.as<int32_t>();
  if (sorted) {
    int npow2 = 1;
    while (npow2 < win)
      npow2 <<= 1;
    const size_t smem = sizeof(unsigned long long) * npow2;
    PLS_CUDA(cudaFuncSetAttribute(k_window_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    k_window_sort<<<(unsigned)nwin, kSortThreads, smem, s>>>(m, win, npow2, rp, pos_row.as<int32_t>(),
                                                             pos_len.as<int32_t>());
  } else {
    k_identity_positions<<<(unsigned)div_up(npos, 256), 256, 0, s>>>(
        npos, m, rp, pos_row.as<int32_t>(), pos_len.as<int32_t>());
  }
  k_chunk_width<<<(unsigned)div_up(nC, 256), 256, 0, s>>>(nC, C, sorted, pos_len.as<int32_t>(),
                                                          cl.as<int32_t>());
  k_chunk_starts<<<1, 1024, 0, s>>>(nC, C, cl.as<int32_t>(), cs.as<int64_t>(), total.as<int64_t>());
  PLS_LAUNCH_CHECK();
  int64_t t = 0;
  PLS_CUDA(cudaMemcpyAsync(&t, total.p, 8, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  return t;
}

// Slice the chunks wider than 2*slice_w into column slices of slice_w so
// that a few very wide chunks (power-law row lengths) spread over many lane
// groups; the other chunks stay one lane group each. Slices are ordered by
// decreasing chunk width so the longest work starts first.
void sell_build_work_list(SellDev &S, int slice_w, cudaStream_t st) {
  S.bands.clear();
  S.items.release();
  S.part.release();
  S.done.release();
  S.n_items = 0;
  S.n_split = 0;
  S.slice_w = 0;
  S.split_w = INT32_MAX;
  if (S.nC == 0 || slice_w <= 0 || S.max_width <= 2 * slice_w)
    return;
  std::vector<int32_t> cl(S.nC);
  PLS_CUDA(cudaMemcpy(cl.data(), S.cl.p, sizeof(int32_t) * S.nC, cudaMemcpyDeviceToHost));
  std::vector<int64_t> wide;
  for (int64_t c = 0; c < S.nC; ++c)
    if (cl[c] > 2 * slice_w)
      wide.push_back(c);
  std::stable_sort(wide.begin(), wide.end(),
                   [&](int64_t a, int64_t b) { return cl[a] > cl[b]; });
  std::vector<int4> items;
  int32_t slot = 0;
  for (int64_t c : wide) {
    const int32_t w = cl[c];
    const int32_t ns = (int32_t)div_up(w, slice_w);
    for (int32_t q = 0; q < ns; ++q)
      items.push_back(make_int4((int)c, q * slice_w, std::min(w, (q + 1) * slice_w), slot + q));
    slot += ns;
  }
  S.n_items = (int64_t)items.size();
  S.n_split = (int64_t)wide.size();
  S.slice_w = slice_w;
  S.split_w = 2 * slice_w;
  S.items.reserve(sizeof(int4) * items.size());
  PLS_CUDA(cudaMemcpyAsync(S.items.p, items.data(), sizeof(int4) * items.size(),
                           cudaMemcpyHostToDevice, st));
  // Partial sums: one accumulator per (slot, row); FP64 covers both
  // accumulator types. Completion counts: one per slot (the chunk's first
  // slot counts its slices), zero between launches.
  S.part.reserve(sizeof(double) * (size_t)slot * S.C);
  S.done.reserve(sizeof(int32_t) * (size_t)slot);
  PLS_CUDA(cudaMemsetAsync(S.done.p, 0, sizeof(int32_t) * (size_t)slot, st));
  PLS_CUDA(cudaStreamSynchronize(st));
}

}  // namespace pls
