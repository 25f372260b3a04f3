// Row-group SpMM core: C[row, :] = alpha * A[row, :] * B + beta * C[row, :]
// for one row of A per group of TK x TN lanes (both powers of two, TK * TN
// <= 32, several groups per warp when smaller).
//
//   * TK lanes span C's columns: lane tk owns NV vectors of VEC consecutive
//     columns (16-byte loads of B and C rows when the caller's pointers and
//     leading dimensions allow, VEC = 1 otherwise), so the TK lanes of a group
//     read one contiguous stretch of a B row per nonzero;
//   * TN lanes split the row's nonzeros: lane tn takes entries tn, tn + TN,
//     tn + 2 TN, ... in stored order; the TN partial sums are combined by a
//     shuffle tree at the end;
//   * each lane keeps U nonzeros in flight: the U column / value loads are
//     issued (predicated past the row end), then the U x NV B-row vector
//     loads, then the FMAs, so a row costs a few memory round trips instead
//     of two per nonzero. Short rows on the memory latency were what bounded
//     the one-nonzero-at-a-time form of this loop.
//
// The per-element sum is therefore the TN strided partial sums added in a
// tree: a reordering of the reference's sequential row sum
// (src/compressed_sparse_rows.cpp:1699-1745), within the FP64 tolerance.
#pragma once

#include "common.cuh"

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

// ---- rows of A as the loop reads them -----------------------------------
// range(row) gives the row's entry interval [s, e) and an auxiliary word;
// entry(q, aux) gives entry q's column of B and its value.

template <class Val> struct CsrRows {
  using V = Val;
  const int32_t *rp, *col;
  const V *val;
  __device__ __forceinline__ void range(int64_t r, int32_t &s, int32_t &e, int32_t &aux) const {
    s = __ldg(rp + r);
    e = __ldg(rp + r + 1);
    aux = 0;
  }
  __device__ __forceinline__ void entry(int32_t q, int32_t, int32_t &c, V &a,
                                        const L2Policy &pol) const {
    c = ld_stream(col + q, pol.stream);
    a = ld_stream(val + q, pol.stream);
  }
};

// FP32 CSR with each entry's column and value side by side (int2: column,
// value bits), so one 8-byte load brings both.
struct PackedRows {
  using V = float;
  const int32_t *rp;
  const int2 *cv;
  __device__ __forceinline__ void range(int64_t r, int32_t &s, int32_t &e, int32_t &aux) const {
    s = __ldg(rp + r);
    e = __ldg(rp + r + 1);
    aux = 0;
  }
  __device__ __forceinline__ void entry(int32_t q, int32_t, int32_t &c, float &a,
                                        const L2Policy &pol) const {
    const int2 t = ld_stream(cv + q, pol.stream);
    c = t.x;
    a = __int_as_float(t.y);
  }
};

constexpr int kSpmmInFlight = 4;  // U: nonzeros in flight per lane

// How the lanes of a row get its entries (column, value):
//   kEntriesLane   each lane loads the U entries of its group itself, then
//                  their B rows (two round trips per group);
//   kEntriesAhead  the same, with the next group's entries loaded while
//                  this group's B rows are in flight (one round trip per
//                  group, about 12 more registers). It pays where occupancy
//                  is already bound by other registers (the batched kernel:
//                  3.99 -> 3.85 ms on its 512-instance workload) and costs
//                  where it is not (the single SpMM on a 27-point stencil:
//                  FP64 k = 32 1.32 -> 1.57 ms, 64 instead of 48 registers);
//   kEntriesShared the TK lanes of a row load TK consecutive entries at once
//                  (one coalesced load per array; the next TK are loaded
//                  while these are used) and hand them round with shuffles,
//                  so TK nonzeros cost one entry round trip. Needs TN = 1;
//                  the warp runs to its longest row.
constexpr int kEntriesLane = 0, kEntriesAhead = 1, kEntriesShared = 2;

// One group's row. Every lane of the warp must call this together (the
// reduction shuffles over the whole warp); lanes whose row is past the end
// pass live = false and only take part in the shuffles. TK, TN (as log2)
// and k are uniform across the warp.
// OFF32: every offset into B and C (row * ld + column) fits in 32 bits, so
// the address arithmetic stays 32-bit.
template <int VEC, int NV, class Acc, class X, class Rows, bool OFF32 = false,
          int ENTRIES = kEntriesLane>
__device__ __forceinline__ void spmm_row_group(const Rows &A, int64_t row, bool live, int lg_tk,
                                               int lg_tn, const X *__restrict__ B, int64_t ldb,
                                               X *__restrict__ C, int64_t ldc, int k, X alpha,
                                               X beta, int beta_nz, const L2Policy &pol) {
  constexpr int U = kSpmmInFlight;
  const int lane = threadIdx.x & 31;
  const int TK = 1 << lg_tk, TN = 1 << lg_tn;
  const int tk = lane & (TK - 1);
  const int tn = (lane >> lg_tk) & (TN - 1);
  int32_t s = 0, e = 0, aux = 0;
  if (live)
    A.range(row, s, e, aux);
  int32_t longest = 0;  // kEntriesShared: the warp's longest row
  if constexpr (ENTRIES == kEntriesShared) {
    longest = e - s;
    for (int o = 16; o > 0; o >>= 1)
      longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
  }
  const int tile = TK * VEC * NV;
  for (int k0 = 0; k0 < k; k0 += tile) {
    Acc acc[NV][VEC];
#pragma unroll
    for (int nv = 0; nv < NV; ++nv)
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[nv][v] = Acc(0);
    // Entry q of the row, column -1 past the row end.
    const auto load_entry = [&](int32_t q, int32_t &c, Acc &a) {
      if (q < e) {
        typename Rows::V av;
        A.entry(q, aux, c, av, pol);
        a = to_acc<Acc>(av);
      } else {
        c = -1;
        a = Acc(0);
      }
    };
    // Entries of U nonzeros from position p0 on, TN apart.
    const auto load_entries = [&](int32_t p0, int32_t(&c)[U], Acc(&a)[U]) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        load_entry(p0 + u * TN, c[u], a[u]);
    };
    // The B rows of U entries (column -1: none) and their FMAs.
    const auto consume = [&](const int32_t(&c)[U], const Acc(&a)[U], auto &&in_flight) {
      X b[U][NV][VEC];
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int nv = 0; nv < NV; ++nv) {
          const int kk = k0 + (nv * TK + tk) * VEC;
          const X *bp = OFF32 ? B + ((c[u] < 0 ? 0 : c[u]) * (int32_t)ldb + kk)
                              : B + (int64_t)(c[u] < 0 ? 0 : c[u]) * ldb + kk;
          if (c[u] >= 0 && kk + VEC <= k) {
            ld_vec<X, VEC>(bp, b[u][nv]);
          } else {
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              b[u][nv][v] = (c[u] >= 0 && kk + v < k) ? __ldg(bp + v) : X(0);
          }
        }
      }
      in_flight();  // loads to overlap with the B rows
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int nv = 0; nv < NV; ++nv)
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            acc[nv][v] = fma(a[u], to_acc<Acc>(b[u][nv][v]), acc[nv][v]);
    };
    if constexpr (ENTRIES == kEntriesShared) {
      int32_t cn;
      Acc an;
      load_entry(s + tk, cn, an);
      for (int32_t base = 0; base < longest; base += TK) {
        const int32_t cm = cn;
        const Acc am = an;
        load_entry(s + base + TK + tk, cn, an);
        const int32_t cnt = min(TK, longest - base);
        for (int32_t u0 = 0; u0 < cnt; u0 += U) {
          int32_t c[U];
          Acc a[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int32_t src = u0 + u;
            c[u] = __shfl_sync(0xffffffffu, cm, src & (TK - 1), TK);
            a[u] = __shfl_sync(0xffffffffu, am, src & (TK - 1), TK);
            if (src >= cnt)
              c[u] = -1;
          }
          consume(c, a, [] {});
        }
      }
    } else {
      int32_t cn[U];
      Acc an[U];
      if constexpr (ENTRIES == kEntriesAhead)
        load_entries(s + tn, cn, an);
      for (int32_t p = s + tn; p < e; p += U * TN) {
        int32_t c[U];
        Acc a[U];
        if constexpr (ENTRIES == kEntriesAhead) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            c[u] = cn[u];
            a[u] = an[u];
          }
          consume(c, a, [&] { load_entries(p + U * TN, cn, an); });
        } else {
          load_entries(p, c, a);
          consume(c, a, [] {});
        }
      }
    }
    for (int o = TK; o < TK * TN; o <<= 1)
#pragma unroll
      for (int nv = 0; nv < NV; ++nv)
#pragma unroll
        for (int v = 0; v < VEC; ++v)
          acc[nv][v] += __shfl_xor_sync(0xffffffffu, acc[nv][v], o);
    if (live && tn == 0) {
      X *crow = OFF32 ? C + (int32_t)row * (int32_t)ldc : C + row * ldc;
#pragma unroll
      for (int nv = 0; nv < NV; ++nv) {
        const int kk = k0 + (nv * TK + tk) * VEC;
        X out[VEC];
        if (kk + VEC <= k) {
          if (beta_nz) {
            X old[VEC];
            ld_vec_plain<X, VEC>(crow + kk, old);
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              out[v] = (X)acc[nv][v] * alpha + beta * old[v];
          } else {
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              out[v] = (X)acc[nv][v] * alpha;
          }
          st_vec<X, VEC>(crow + kk, out);
        } else {
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            if (kk + v < k) {
              X o = (X)acc[nv][v] * alpha;
              if (beta_nz)
                o += beta * crow[kk + v];
              crow[kk + v] = o;
            }
        }
      }
    }
  }
}

// Lane shape for k columns and a mean of `mean_len` entries per row:
// (log2 TK, log2 TN, NV) for vectors of VEC columns, NV <= max_nv.
struct RowsShape {
  int lg_tk, lg_tn, nv;
};

inline RowsShape rows_shape(int k, int vec, double mean_len, int max_nv = 2) {
  const int cols = (k + vec - 1) / vec;  // vectors per row of C
  RowsShape sh{0, 0, cols > 32 && max_nv >= 2 ? 2 : 1};
  const int per = (cols + sh.nv - 1) / sh.nv;
  while ((1 << sh.lg_tk) < per && sh.lg_tk < 5)
    ++sh.lg_tk;
  // TN > 1 only when the column lanes alone are one or two: then a row's
  // entries are split like the SpMV lane groups (enough lanes that one pass
  // of U entries per lane covers the mean row). Otherwise each row keeps one
  // lane per column vector and consecutive rows share the warp, so on banded
  // and stencil matrices one load step of the warp reads neighbouring rows
  // of B (contiguous bytes) instead of scattered rows for one row of A.
  if (sh.lg_tk <= 1) {
    const int want = (int)((mean_len + kSpmmInFlight - 1) / kSpmmInFlight);
    while ((1 << sh.lg_tn) < want && sh.lg_tk + sh.lg_tn < 5)
      ++sh.lg_tn;
  }
  return sh;
}

}  // namespace pls
