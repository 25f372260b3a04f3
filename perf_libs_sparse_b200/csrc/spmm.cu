// Sparse x dense SpMM kernels: C = alpha*A*B + beta*C with row-major dense
// B (ldb) and C (ldc), k right-hand sides.
//
// CSR: a group of L lanes per row of A, each lane owning VEC consecutive
// columns of C per k-tile (128-bit loads of B and C rows). For every nonzero
// a_ij of the row the group reads row j of B, which for the structured
// matrices of this path (stencils, banded) was read moments earlier by a
// neighbouring row and is served from L2; the unique rows of B are counted
// once in the algorithmic bytes. The per-element sum runs over the row's
// nonzeros in stored order, the order of the reference's row kernel
// (src/compressed_sparse_rows.cpp:1699-1745).
//
// BSR: a warp per block row, lanes over C's columns; each lane keeps bs
// accumulators (one per scalar row of the block row).
#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

template <class X, int VEC> struct VecT;
template <> struct VecT<double, 1> { using T = double; };
template <> struct VecT<double, 2> { using T = double2; };
template <> struct VecT<float, 1> { using T = float; };
template <> struct VecT<float, 2> { using T = float2; };
template <> struct VecT<float, 4> { using T = float4; };

template <class X, int VEC>
__device__ __forceinline__ void ld_vec(const X *p, X (&v)[VEC]) {
  if constexpr (VEC == 1) {
    v[0] = __ldg(p);
  } else {
    using T = typename VecT<X, VEC>::T;
    const T t = __ldg(reinterpret_cast<const T *>(p));
    const X *e = reinterpret_cast<const X *>(&t);
#pragma unroll
    for (int i = 0; i < VEC; ++i)
      v[i] = e[i];
  }
}

template <class X, int VEC>
__device__ __forceinline__ void ld_vec_plain(const X *p, X (&v)[VEC]) {
  if constexpr (VEC == 1) {
    v[0] = *p;
  } else {
    using T = typename VecT<X, VEC>::T;
    const T t = *reinterpret_cast<const T *>(p);
    const X *e = reinterpret_cast<const X *>(&t);
#pragma unroll
    for (int i = 0; i < VEC; ++i)
      v[i] = e[i];
  }
}

template <class X, int VEC>
__device__ __forceinline__ void st_vec(X *p, const X (&v)[VEC]) {
  if constexpr (VEC == 1) {
    *p = v[0];
  } else {
    using T = typename VecT<X, VEC>::T;
    T t;
    X *e = reinterpret_cast<X *>(&t);
#pragma unroll
    for (int i = 0; i < VEC; ++i)
      e[i] = v[i];
    *reinterpret_cast<T *>(p) = t;
  }
}

// L lanes per row, VEC columns per lane per tile; `vec_ok` says whether the
// full-width vector path is aligned for this call (else VEC must be 1).
template <int L, int VEC, class V, class X>
__global__ void __launch_bounds__(256)
    k_spmm_csr(int32_t m, const int32_t *__restrict__ rp,
               const int32_t *__restrict__ col, const V *__restrict__ val,
               const X *__restrict__ B, int64_t ldb, X *__restrict__ C,
               int64_t ldc, int k, X alpha, X beta, int beta_nz) {
  using Acc = typename AccOf<V, X>::type;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t row = gid / L;
  if (row >= m)
    return;
  const int lane = (int)(gid % L);
  const int32_t s = __ldg(rp + row), e = __ldg(rp + row + 1);
  X *crow = C + row * ldc;
  for (int k0 = lane * VEC; k0 < k; k0 += L * VEC) {
    const bool full = k0 + VEC <= k;
    Acc acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v)
      acc[v] = 0;
    int32_t p = s;
    for (; p + 1 < e; p += 2) {
      const Acc a0 = to_acc<Acc>(ld_stream(val + p)), a1 = to_acc<Acc>(ld_stream(val + p + 1));
      const int32_t c0 = ld_stream(col + p), c1 = ld_stream(col + p + 1);
      X b0[VEC], b1[VEC];
      if (full) {
        ld_vec<X, VEC>(B + (int64_t)c0 * ldb + k0, b0);
        ld_vec<X, VEC>(B + (int64_t)c1 * ldb + k0, b1);
      } else {
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
          b0[v] = k0 + v < k ? __ldg(B + (int64_t)c0 * ldb + k0 + v) : X(0);
          b1[v] = k0 + v < k ? __ldg(B + (int64_t)c1 * ldb + k0 + v) : X(0);
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        acc[v] = fma(a0, to_acc<Acc>(b0[v]), acc[v]);
        acc[v] = fma(a1, to_acc<Acc>(b1[v]), acc[v]);
      }
    }
    if (p < e) {
      const Acc a0 = to_acc<Acc>(ld_stream(val + p));
      const int32_t c0 = ld_stream(col + p);
      X b0[VEC];
      if (full) {
        ld_vec<X, VEC>(B + (int64_t)c0 * ldb + k0, b0);
      } else {
#pragma unroll
        for (int v = 0; v < VEC; ++v)
          b0[v] = k0 + v < k ? __ldg(B + (int64_t)c0 * ldb + k0 + v) : X(0);
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[v] = fma(a0, to_acc<Acc>(b0[v]), acc[v]);
    }
    X out[VEC];
    if (beta_nz) {
      X cold[VEC];
      if (full) {
        ld_vec_plain<X, VEC>(crow + k0, cold);
      } else {
#pragma unroll
        for (int v = 0; v < VEC; ++v)
          cold[v] = k0 + v < k ? crow[k0 + v] : X(0);
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        out[v] = (X)acc[v] * alpha + beta * cold[v];
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        out[v] = (X)acc[v] * alpha;
    }
    if (full) {
      st_vec<X, VEC>(crow + k0, out);
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        if (k0 + v < k)
          crow[k0 + v] = out[v];
    }
  }
}

template <int L, int VEC, class V, class X>
static void launch_spmm_csr(const CsrDev &c, int32_t m, const X *B, int64_t ldb,
                            X *C, int64_t ldc, int k, X alpha, X beta,
                            cudaStream_t s) {
  const int64_t blocks = div_up((int64_t)m * L, 256);
  k_spmm_csr<L, VEC, V, X><<<(unsigned)blocks, 256, 0, s>>>(
      m, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(), (const V *)c.ev(), B, ldb, C,
      ldc, k, alpha, beta, beta != X(0));
}

template <int VEC, class V, class X>
static void spmm_csr_lanes(const CsrDev &c, int32_t m, const X *B, int64_t ldb,
                           X *C, int64_t ldc, int k, X alpha, X beta,
                           cudaStream_t s) {
  const int groups = (int)div_up(k, VEC);
  if (groups <= 1)
    launch_spmm_csr<1, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else if (groups <= 2)
    launch_spmm_csr<2, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else if (groups <= 4)
    launch_spmm_csr<4, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else if (groups <= 8)
    launch_spmm_csr<8, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else if (groups <= 16)
    launch_spmm_csr<16, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
  else
    launch_spmm_csr<32, VEC, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
}

template <class X>
void spmm_csr(const CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C,
              int64_t ldc, int k, X alpha, X beta, cudaStream_t s) {
  if (m == 0 || k == 0)
    return;
  constexpr int VMAX = 16 / sizeof(X);
  const bool aligned = ((uintptr_t)B % 16 == 0) && ((uintptr_t)C % 16 == 0) &&
                       (ldb % VMAX == 0) && (ldc % VMAX == 0);
  with_vt(c.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
      if (aligned)
        spmm_csr_lanes<VMAX, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
      else
        spmm_csr_lanes<1, V, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s);
    }
  });
  PLS_LAUNCH_CHECK();
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
        if (beta_nz)
          o += beta * *cp;
        *cp = o;
      }
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
void spmm_bsr(const BsrDev &b, const X *B, int64_t ldb, X *C, int64_t ldc,
              int k, X alpha, X beta, cudaStream_t s) {
  if (b.mb == 0 || k == 0)
    return;
  const int bnz = beta != X(0);
  with_vt(b.evt(), [&](auto tag) {
    using V = typename decltype(tag)::type;
    if constexpr (std::is_same_v<X, float> && std::is_same_v<V, double>) {
      throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE, "FP64 storage with FP32 API");
    } else {
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

template void spmm_csr<float>(const CsrDev &, int32_t, const float *, int64_t,
                              float *, int64_t, int, float, float, cudaStream_t);
template void spmm_csr<double>(const CsrDev &, int32_t, const double *, int64_t,
                               double *, int64_t, int, double, double,
                               cudaStream_t);
template void spmm_bsr<float>(const BsrDev &, const float *, int64_t, float *,
                              int64_t, int, float, float, cudaStream_t);
template void spmm_bsr<double>(const BsrDev &, const double *, int64_t,
                               double *, int64_t, int, double, double,
                               cudaStream_t);

}  // namespace pls
