// Sparse x dense SpMM kernels: C = alpha*A*B + beta*C with row-major dense
// B (ldb) and C (ldc), k right-hand sides.
//
// CSR: the row-group loop of spmm_rows.cuh, one group of TK x TN lanes per
// row of A (TK over C's columns with 16-byte vectors when aligned, TN over
// the row's nonzeros, four nonzeros in flight per lane). For the structured
// matrices of this path (stencils, banded) row j of B was read moments
// earlier by a neighbouring row and is served from L1 / L2; the unique rows
// of B are counted once in the algorithmic bytes.
//
// BSR: a warp per block row, lanes over C's columns; each lane keeps bs
// accumulators (one per scalar row of the block row).
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "pls_internal.hpp"
#include "spmm_rows.cuh"

namespace pls {

template <int VEC, int NV, class V, class X, bool OFF32, int ENTRIES>
__device__ __forceinline__ void spmm_csr_rows(int32_t m, int lg_tk, int lg_tn,
                                              const int32_t *__restrict__ rp,
                                              const int32_t *__restrict__ col,
                                              const V *__restrict__ val, const X *__restrict__ B,
                                              int64_t ldb, X *__restrict__ C, int64_t ldc, int k,
                                              X alpha, X beta, int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const L2Policy pol = make_l2_policy();
  const int lg_g = lg_tk + lg_tn;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t row = (warp << (5 - lg_g)) + ((threadIdx.x & 31) >> lg_g);
  const CsrRows<V> A{rp, col, val};
  spmm_row_group<VEC, NV, Acc, X, CsrRows<V>, OFF32, ENTRIES>(
      A, row, row < m, lg_tk, lg_tn, B, ldb, C, ldc, k, alpha, beta, beta_nz, pol);
}

template <int VEC, int NV, class V, class X, bool OFF32, int ENTRIES>
__global__ void __launch_bounds__(256)
    k_spmm_csr(int32_t m, int lg_tk, int lg_tn, const int32_t *__restrict__ rp,
               const int32_t *__restrict__ col, const V *__restrict__ val,
               const X *__restrict__ B, int64_t ldb, X *__restrict__ C, int64_t ldc, int k,
               X alpha, X beta, int beta_nz) {
  spmm_csr_rows<VEC, NV, V, X, OFF32, ENTRIES>(m, lg_tk, lg_tn, rp, col, val, B, ldb, C, ldc, k,
                                               alpha, beta, beta_nz);
}

// Shared entries for FP32 results with one vector per lane, held to 48
// registers (5 blocks of 256 per SM): the shared loads add about 10
// registers, which would cost a resident block. Measured on the 27-point
// stencil (plain row-group kernel / shared uncapped / shared capped): FP32
// k = 32 0.598 / 0.628 / 0.591 ms, k = 128 2.141 / 2.180 / 2.019 ms. FP64
// results spill at the cap and run uncapped (k = 8 0.494 / 0.388 / 0.505,
// k = 32 1.39 / 1.18 / 1.26), as do two vectors per lane (NV = 2).
template <int VEC, class V, class X, bool OFF32>
__global__ void __launch_bounds__(256, 5)
    k_spmm_csr_shared(int32_t m, int lg_tk, int lg_tn, const int32_t *__restrict__ rp,
                      const int32_t *__restrict__ col, const V *__restrict__ val,
                      const X *__restrict__ B, int64_t ldb, X *__restrict__ C, int64_t ldc,
                      int k, X alpha, X beta, int beta_nz) {
  spmm_csr_rows<VEC, 1, V, X, OFF32, kEntriesShared>(m, lg_tk, lg_tn, rp, col, val, B, ldb, C,
                                                     ldc, k, alpha, beta, beta_nz);
}

// 32-bit address arithmetic is possible when every offset into B (rows
// 0 .. ncols-1 of ldb) and C (rows 0 .. m-1 of ldc) fits; ncols 0 means the
// column count was not recorded.
static bool rows_off32_fits(const CsrDev &c, int32_t m, int64_t ldb, int64_t ldc) {
  return c.ncols > 0 && (int64_t)c.ncols * ldb < INT32_MAX && (int64_t)m * ldc < INT32_MAX;
}

// Whether the shared-entries mode applies to this lane shape: one lane group
// per row (TN = 1) of at least 4 lanes, so a shared load covers a group of
// U = 4 entries.
static bool shared_entries_fit(const RowsShape &sh) { return sh.lg_tn == 0 && sh.lg_tk >= 2; }

template <int VEC, class V, class X>
static bool launch_spmm_csr(const CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C,
                            int64_t ldc, int k, X alpha, X beta, bool off32, bool shared,
                            cudaStream_t s) {
  const RowsShape sh = rows_shape(k, VEC, (double)c.nnz / std::max<int32_t>(m, 1));
  const int64_t rows_per_block = (int64_t)8 << (5 - (sh.lg_tk + sh.lg_tn));
  const unsigned blocks = (unsigned)div_up(m, rows_per_block);
  const int bnz = beta != X(0);
  off32 = off32 && rows_off32_fits(c, m, ldb, ldc);
  shared = shared && shared_entries_fit(sh);
  auto go = [&](auto nv_tag, auto off_tag, auto entries_tag) {
    constexpr int NV = decltype(nv_tag)::value;
    constexpr bool OFF = decltype(off_tag)::value;
    constexpr int EM = decltype(entries_tag)::value;
    if constexpr (EM == kEntriesShared && NV == 1 && sizeof(X) == 4)
      k_spmm_csr_shared<VEC, V, X, OFF><<<blocks, 256, 0, s>>>(m, sh.lg_tk, sh.lg_tn,
          c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), (const V *)c.ev(), B, ldb, C, ldc, k,
          alpha, beta, bnz);
    else
      k_spmm_csr<VEC, NV, V, X, OFF, EM><<<blocks, 256, 0, s>>>(m, sh.lg_tk, sh.lg_tn,
          c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), (const V *)c.ev(), B, ldb, C, ldc, k,
          alpha, beta, bnz);
  };
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using T = std::true_type;
  using F = std::false_type;
  auto by_entries = [&](auto nv_tag, auto off_tag) {
    if (shared)
      go(nv_tag, off_tag, std::integral_constant<int, kEntriesShared>{});
    else
      go(nv_tag, off_tag, std::integral_constant<int, kEntriesLane>{});
  };
  if (sh.nv == 2)
    off32 ? by_entries(I2{}, T{}) : by_entries(I2{}, F{});
  else
    off32 ? by_entries(I1{}, T{}) : by_entries(I1{}, F{});
  return shared;
}

// Vector width (columns per load) of the row-group kernel for k columns:
// 16-byte vectors when B and C allow them, else one column. With shared
// entries the width is halved while that leaves fewer than 4 column lanes per
// row (FP32 k = 8: two lanes of 4 columns become four of 2), since the
// shared loads need at least 4 lanes per row.
template <class X>
static int rows_vec(const CsrDev &c, int32_t m, const X *B, int64_t ldb, const X *C,
                    int64_t ldc, int k, bool shared) {
  constexpr int VMAX = 16 / sizeof(X);
  const bool aligned = k >= VMAX && ((uintptr_t)B % 16 == 0) && ((uintptr_t)C % 16 == 0) &&
                       (ldb % VMAX == 0) && (ldc % VMAX == 0);
  int vec = aligned ? VMAX : 1;
  const double mean = (double)c.nnz / std::max<int32_t>(m, 1);
  while (shared && vec > 1 && !shared_entries_fit(rows_shape(k, vec, mean)))
    vec /= 2;
  return vec;
}

// Row-group SpMM (the launch half of spmm_csr), with 32-bit address
// arithmetic when `off32` and the offsets fit, and shared entry loads when
// `shared` and the lane shape allows them (returns whether they ran).
template <class X>
static bool spmm_rows(const CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc,
                      int k, X alpha, X beta, bool off32, bool shared, cudaStream_t s) {
  const int vec = rows_vec<X>(c, m, B, ldb, C, ldc, k, shared);
  bool ran = false;
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      if constexpr (sizeof(X) == 4) {
        if (vec == 4) {
          ran = launch_spmm_csr<4, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, off32, shared, s);
          return;
        }
      }
      if (vec == 2)
        ran = launch_spmm_csr<2, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, off32, shared, s);
      else
        ran = launch_spmm_csr<1, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, off32, shared, s);
    }
  });
  PLS_LAUNCH_CHECK();
  return ran;
}

// Kernel choice for a CSR SpMM, measured once per call signature (k, ldb,
// value and API types): the row-group kernel with 64-bit and, when the
// offsets fit, 32-bit address arithmetic (the better of the two differs
// with k and the value type), the row-group kernel with shared entry loads
// when the lane shape allows them, and the staged kernel when it applies.
// With more than one candidate, the first SpMM of the signature runs each on
// a scratch C (beta = 0, CUDA events, one warm-up and two timed runs) and
// keeps the fastest; later calls use the kept one. choice: 0 row group
// 64-bit, 2 row group 32-bit, 3 row group with shared entries (32-bit
// offsets when they fit), 1 staged, 4 diagonal form, 5 diagonal form with
// TMA-staged B (spmm_dia.cu). Where the diagonal form applies the staged
// kernel is not timed: it stages the same rows of B less compactly.
template <class X>
void spmm_csr(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C,
              int64_t ldc, int k, X alpha, X beta, cudaStream_t s) {
  if (m == 0 || k == 0)
    return;
  const int64_t sig = ((int64_t)k << 32) ^ (ldb << 8) ^ (ldc << 20) ^
                      ((int64_t)sizeof(X) << 4) ^ (int64_t)c.evt();
  TileDev &t = c.tiles;
  const bool fits32 = rows_off32_fits(c, m, ldb, ldc);
  if (t.forced == 0 || t.forced == 2) {
    t.last_path = spmm_rows<X>(c, m, B, ldb, C, ldc, k, alpha, beta, fits32, t.forced == 2, s)
                      ? 2
                      : 0;
    return;
  }
  if (t.forced == 3) {
    const bool dia = spmm_dia<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true);
    if (!dia)
      spmm_rows<X>(c, m, B, ldb, C, ldc, k, alpha, beta, fits32, false, s);
    t.last_path = dia ? 3 : 0;
    return;
  }
  if (t.forced == 4) {
    const bool tma = spmm_dia_tma<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true);
    const bool dia = !tma && spmm_dia<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true);
    if (!tma && !dia)
      spmm_rows<X>(c, m, B, ldb, C, ldc, k, alpha, beta, fits32, false, s);
    t.last_path = tma ? 4 : dia ? 3 : 0;
    return;
  }
  if (t.forced == 1) {
    const bool staged = spmm_tiled<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true);
    if (!staged)
      spmm_rows<X>(c, m, B, ldb, C, ldc, k, alpha, beta, fits32, false, s);
    t.last_path = staged ? 1 : 0;
    return;
  }
  if (t.choice_sig != sig) {
    const bool dia_ok = spmm_dia<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, false);
    const bool tma_ok = dia_ok && spmm_dia_tma<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, false);
    const bool staged_ok = !dia_ok && spmm_tiled<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, false);
    const int vec_s = rows_vec<X>(c, m, B, ldb, C, ldc, k, true);
    const bool shared_ok = shared_entries_fit(
        rows_shape(k, vec_s, (double)c.nnz / std::max<int32_t>(m, 1)));
    t.choice = 0;
    t.ms_rows = t.ms_staged = 0.f;
    t.predicted = false;
    if (t.pred_n > 0) {
      // The learned selector's order: its first kernel that applies, untimed.
      t.choice = fits32 ? 2 : 0;
      for (int q = 0; q < t.pred_n; ++q) {
        const int cls = t.pred_order[q];
        if (cls == kSpmmRows)
          break;
        if (cls == kSpmmShared && shared_ok) {
          t.choice = 3;
          break;
        }
        if (cls == kSpmmStaged && staged_ok) {
          t.choice = 1;
          break;
        }
        if (cls == kSpmmDia && dia_ok) {
          t.choice = 4;
          break;
        }
        if (cls == kSpmmDiaTma && tma_ok) {
          t.choice = 5;
          break;
        }
      }
      t.predicted = true;
    } else if (staged_ok || fits32 || shared_ok || dia_ok || tma_ok) {
      DevBuf scratch;
      scratch.reserve(sizeof(X) * (size_t)m * k);
      X *sc = scratch.as<X>();
      const EventPair ev;
      cudaEvent_t e0 = ev.e0, e1 = ev.e1;
      auto time2 = [&](auto &&run) {
        run();
        PLS_CUDA(cudaEventRecord(e0, s));
        run();
        run();
        PLS_CUDA(cudaEventRecord(e1, s));
        PLS_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PLS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 2;
      };
      const bool sc32 = fits32 && rows_off32_fits(c, m, ldb, k);
      const float ms64 = time2(
          [&] { spmm_rows<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), false, false, s); });
      float best = ms64;
      if (sc32) {
        const float ms32 = time2(
            [&] { spmm_rows<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), true, false, s); });
        if (ms32 < best) {
          best = ms32;
          t.choice = 2;
        }
      }
      if (shared_ok) {
        const float mss = time2(
            [&] { spmm_rows<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), sc32, true, s); });
        if (mss < best) {
          best = mss;
          t.choice = 3;
        }
      }
      t.ms_rows = best;
      if (staged_ok) {
        t.ms_staged =
            time2([&] { spmm_tiled<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), s, true); });
        if (t.ms_staged < best) {
          best = t.ms_staged;
          t.choice = 1;
        }
      }
      if (dia_ok) {
        const float msd =
            time2([&] { spmm_dia<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), s, true); });
        if (msd < best) {
          best = msd;
          t.choice = 4;
        }
      }
      if (tma_ok) {
        const float mst =
            time2([&] { spmm_dia_tma<X>(c, m, B, ldb, sc, (int64_t)k, k, X(1), X(0), s, true); });
        if (mst < best)
          t.choice = 5;
      }
    }
    t.choice_sig = sig;
  }
  if (t.choice == 1 && spmm_tiled<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true)) {
    t.last_path = 1;
    return;
  }
  if (t.choice == 4 && spmm_dia<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true)) {
    t.last_path = 3;
    return;
  }
  if (t.choice == 5 && spmm_dia_tma<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, true)) {
    t.last_path = 4;
    return;
  }
  t.last_path = spmm_rows<X>(c, m, B, ldb, C, ldc, k, alpha, beta,
                             t.choice == 2 || (t.choice == 3 && fits32), t.choice == 3, s)
                    ? 2
                    : 0;
}

// ---------------------------------------------------------------- BSR
template <int BS, class V, class X>
__global__ void __launch_bounds__(256)
    k_spmm_bsr(int32_t mb, int layout, const int32_t *__restrict__ rp,
               const int32_t *__restrict__ col, const V *__restrict__ val,
               const X *__restrict__ B, int64_t ldb, X *__restrict__ C,
               int64_t ldc, int k, X alpha, X beta, int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  __shared__ Acc blk_s[8][BS * BS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t br = (int64_t)blockIdx.x * 8 + warp;
  if (br >= mb)
    return;
  const bool rm = layout == PERFLIBS_ROW_MAJOR;
  for (int j0 = 0; j0 < k; j0 += 32) {
    const int j = j0 + lane;
    Acc acc[BS];
#pragma unroll
    for (int i = 0; i < BS; ++i)
      acc[i] = 0;
    for (int32_t b = rp[br]; b < rp[br + 1]; ++b) {
      for (int e = lane; e < BS * BS; e += 32)
        blk_s[warp][e] = to_acc<Acc>(ld_stream(val + (int64_t)b * BS * BS + e));
      __syncwarp();
      const X *bb = B + (int64_t)__ldg(col + b) * BS * ldb;
      if (j < k) {
#pragma unroll
        for (int jj = 0; jj < BS; ++jj) {
          const Acc bv = to_acc<Acc>(__ldg(bb + (int64_t)jj * ldb + j));
#pragma unroll
          for (int i = 0; i < BS; ++i) {
            const Acc a = rm ? blk_s[warp][i * BS + jj] : blk_s[warp][jj * BS + i];
            acc[i] = fma(a, bv, acc[i]);
          }
        }
      }
      __syncwarp();
    }
    if (j < k) {
#pragma unroll
      for (int i = 0; i < BS; ++i) {
        X *cp = C + (br * BS + i) * ldc + j;
        X o = (X)acc[i] * alpha;
        if (beta_nz)  // an explicit fma: the vector kernel below rounds the same way
          o = fma(beta, *cp, o);
        *cp = o;
      }
    }
  }
}

// bs values of one block row (row-major blocks) or block column
// (column-major blocks), loaded as whole vectors: bs * sizeof(V) bytes, at an
// offset that is a multiple of that size.
template <int BS, class V>
__device__ __forceinline__ void ld_block_line(const V *p, V (&a)[BS]) {
  constexpr int bytes = BS * (int)sizeof(V);
  if constexpr (bytes >= 16) {
#pragma unroll
    for (int h = 0; h < bytes / 16; ++h) {
      const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p) + h);
      memcpy(reinterpret_cast<char *>(a) + 16 * h, &t, 16);
    }
  } else if constexpr (bytes == 8) {
    const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
    memcpy(a, &t, 8);
  } else {
    static_assert(bytes == 4, "block lines of 4, 8 or a multiple of 16 bytes");
    const unsigned t = __ldg(reinterpret_cast<const unsigned *>(p));
    memcpy(a, &t, 4);
  }
}

// Block size 2 / 4 / 8 with 16-byte vectors of B and C: TK = 2^lg_tk lanes
// per block row, each owning one vector of VEC columns per pass, 32 / TK
// block rows per warp. Per block, a lane loads its vector of the block's BS
// rows of B (independent 16-byte loads, issued together) and the block's
// values a line at a time (the same addresses across the block row's
// lanes), then adds, for every row i of the block, a_ij * B_j in ascending
// j: per element of C the order of the scalar kernel above, blocks in stored
// order and columns of a block ascending, so the results are the same bits.
template <int BS, bool RM, class V, class X, int VEC>
__global__ void __launch_bounds__(256)
    k_spmm_bsr_vec(int32_t mb, const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                   const V *__restrict__ val, const X *__restrict__ B, int64_t ldb,
                   X *__restrict__ C, int64_t ldc, int k, int lg_tk, X alpha, X beta,
                   int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t br = g >> lg_tk;
  if (br >= mb)
    return;
  const int tk = (int)(g & ((1 << lg_tk) - 1));
  const int32_t b0 = __ldg(rp + br), b1 = __ldg(rp + br + 1);
  for (int kk = tk * VEC; kk < k; kk += VEC << lg_tk) {
    Acc acc[BS][VEC];
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[i][v] = Acc(0);
    for (int32_t b = b0; b < b1; ++b) {
      const X *bb = B + (int64_t)__ldg(col + b) * BS * ldb + kk;
      X bv[BS][VEC];
#pragma unroll
      for (int j = 0; j < BS; ++j)
        ld_vec<X, VEC>(bb + (int64_t)j * ldb, bv[j]);
      const V *ab = val + (int64_t)b * BS * BS;
      if constexpr (RM) {
#pragma unroll
        for (int i = 0; i < BS; ++i) {
          V a[BS];
          ld_block_line<BS, V>(ab + i * BS, a);
#pragma unroll
          for (int j = 0; j < BS; ++j) {
            const Acc aij = to_acc<Acc>(a[j]);
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              acc[i][v] = fma(aij, to_acc<Acc>(bv[j][v]), acc[i][v]);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < BS; ++j) {
          V a[BS];
          ld_block_line<BS, V>(ab + j * BS, a);
#pragma unroll
          for (int i = 0; i < BS; ++i) {
            const Acc aij = to_acc<Acc>(a[i]);
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              acc[i][v] = fma(aij, to_acc<Acc>(bv[j][v]), acc[i][v]);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < BS; ++i) {
      X *cp = C + (br * BS + i) * ldc + kk;
      X o[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        o[v] = (X)acc[i][v] * alpha;
      if (beta_nz) {  // the scalar kernel's epilogue, element for element
        X old[VEC];
        ld_vec_plain<X, VEC>(cp, old);
#pragma unroll
        for (int v = 0; v < VEC; ++v)
          o[v] = fma(beta, old[v], o[v]);
      }
      st_vec<X, VEC>(cp, o);
    }
  }
}

// Any block size: a thread per (scalar row, column).
template <class V, class X>
__global__ void k_spmm_bsr_generic(int32_t mb, int bs, int layout,
                                   const int32_t *__restrict__ rp,
                                   const int32_t *__restrict__ col,
                                   const V *__restrict__ val,
                                   const X *__restrict__ B, int64_t ldb,
                                   X *__restrict__ C, int64_t ldc, int k,
                                   X alpha, X beta, int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = t / k;
  const int j = (int)(t % k);
  if (r >= (int64_t)mb * bs)
    return;
  const int64_t br = r / bs;
  const int i = (int)(r % bs);
  const int64_t E = (int64_t)bs * bs;
  const bool rm = layout == PERFLIBS_ROW_MAJOR;
  Acc acc = 0;
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b)
    for (int jj = 0; jj < bs; ++jj) {
      const V a = rm ? val[b * E + (int64_t)i * bs + jj] : val[b * E + (int64_t)jj * bs + i];
      acc = fma(to_acc<Acc>(a), to_acc<Acc>(B[((int64_t)col[b] * bs + jj) * ldb + j]), acc);
    }
  X *cp = C + r * ldc + j;
  X o = (X)acc * alpha;
  if (beta_nz)
    o += beta * *cp;
  *cp = o;
}

template <class X>
static void spmm_bsr_fma(const BsrDev &b, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                         X alpha, X beta, cudaStream_t s) {
  if (b.mb == 0 || k == 0)
    return;
  const int bnz = beta != X(0);
  with_vt(b.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      constexpr int VEC = 16 / (int)sizeof(X);
      if ((b.bs == 2 || b.bs == 4 || b.bs == 8) && k % VEC == 0 && ldb % VEC == 0 &&
          ldc % VEC == 0 && (uintptr_t)B % 16 == 0 && (uintptr_t)C % 16 == 0) {
        const int cols = k / VEC;
        int lg_tk = 0;
        while ((1 << lg_tk) < cols && lg_tk < 5)
          ++lg_tk;
        const unsigned grid = (unsigned)div_up((int64_t)b.mb << lg_tk, 256);
        const bool rm = b.layout == PERFLIBS_ROW_MAJOR;
        auto go = [&](auto bs_tag, auto rm_tag) {
          constexpr int BS = decltype(bs_tag)::value;
          constexpr bool RM = decltype(rm_tag)::value;
          k_spmm_bsr_vec<BS, RM, V, X, VEC><<<grid, 256, 0, s>>>(
              b.mb, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(), (const V *)b.ev(), B, ldb, C,
              ldc, k, lg_tk, alpha, beta, bnz);
        };
        using T = std::true_type;
        using F = std::false_type;
        switch (b.bs) {
        case 2: rm ? go(std::integral_constant<int, 2>{}, T{}) : go(std::integral_constant<int, 2>{}, F{}); break;
        case 4: rm ? go(std::integral_constant<int, 4>{}, T{}) : go(std::integral_constant<int, 4>{}, F{}); break;
        default: rm ? go(std::integral_constant<int, 8>{}, T{}) : go(std::integral_constant<int, 8>{}, F{}); break;
        }
        return;
      }
      const unsigned blocks = (unsigned)div_up(b.mb, 8);
      switch (b.bs) {
      case 2:
        k_spmm_bsr<2, V, X><<<blocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), B, ldb, C, ldc, k, alpha, beta, bnz);
        break;
      case 4:
        k_spmm_bsr<4, V, X><<<blocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), B, ldb, C, ldc, k, alpha, beta, bnz);
        break;
      case 8:
        k_spmm_bsr<8, V, X><<<blocks, 256, 0, s>>>(b.mb, b.layout, b.row_ptr.as<int32_t>(),
            b.col.as<int32_t>(), (const V *)b.ev(), B, ldb, C, ldc, k, alpha, beta, bnz);
        break;
      default:
        k_spmm_bsr_generic<V, X><<<(unsigned)div_up((int64_t)b.mb * b.bs * k, 256), 256, 0, s>>>(
            b.mb, b.bs, b.layout, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(),
            (const V *)b.ev(), B, ldb, C, ldc, k, alpha, beta, bnz);
      }
    }
  });
  PLS_LAUNCH_CHECK();
}

// Kernel choice for a BSR SpMM: the tensor-core kernel where it applies
// (bs = 8, BF16 values, FP32 B and C), forced (path 5) or measured against
// the FMA kernel on the first call of each (k, ldb) signature (one warm-up
// and two timed runs of each on a scratch C); the FMA kernel otherwise.
template <class X>
void spmm_bsr(BsrDev &b, const X *B, int64_t ldb, X *C, int64_t ldc, int k, X alpha, X beta,
              cudaStream_t s, TileDev &t) {
  if constexpr (sizeof(X) == 4) {
    if (b.mb > 0 && k > 0 && (t.forced == 5 || t.forced == -1) &&
        spmm_bsr_tc(b, B, ldb, C, ldc, k, alpha, beta, s, false)) {
      bool tc = t.forced == 5;
      if (!tc) {
        const int64_t sig = ((int64_t)k << 32) ^ ldb;
        if (b.tc_sig != sig) {
          DevBuf scratch;
          scratch.reserve(sizeof(float) * (size_t)b.mb * b.bs * k);
          float *sc = scratch.as<float>();
          const EventPair ev;
          cudaEvent_t e0 = ev.e0, e1 = ev.e1;
          auto time2 = [&](auto &&run) {
            run();
            PLS_CUDA(cudaEventRecord(e0, s));
            run();
            run();
            PLS_CUDA(cudaEventRecord(e1, s));
            PLS_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PLS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return ms / 2;
          };
          b.ms_fma = time2([&] { spmm_bsr_fma<float>(b, B, ldb, sc, k, k, 1.f, 0.f, s); });
          b.ms_tc = time2([&] { spmm_bsr_tc(b, B, ldb, sc, k, k, 1.f, 0.f, s, true); });
          b.tc_choice = b.ms_tc < b.ms_fma ? 1 : 0;
          b.tc_sig = sig;
        }
        tc = b.tc_choice == 1;
        t.ms_staged = b.ms_tc;
        t.ms_rows = b.ms_fma;
        t.choice_sig = b.tc_sig | ((int64_t)1 << 62);  // timings valid for spmm_info
      }
      if (tc) {
        spmm_bsr_tc(b, B, ldb, C, ldc, k, alpha, beta, s, true);
        t.last_path = 5;
        return;
      }
    }
  }
  spmm_bsr_fma<X>(b, B, ldb, C, ldc, k, alpha, beta, s);
  t.last_path = 6;
}

template void spmm_csr<float>(CsrDev &, int32_t, const float *, int64_t,
                              float *, int64_t, int, float, float, cudaStream_t);
template void spmm_csr<double>(CsrDev &, int32_t, const double *, int64_t,
                               double *, int64_t, int, double, double,
                               cudaStream_t);
template void spmm_bsr<float>(BsrDev &, const float *, int64_t, float *, int64_t, int, float,
                              float, cudaStream_t, TileDev &);
template void spmm_bsr<double>(BsrDev &, const double *, int64_t, double *, int64_t, int, double,
                               double, cudaStream_t, TileDev &);

}  // namespace pls
