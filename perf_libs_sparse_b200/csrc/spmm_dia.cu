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
#include "tma.cuh"

namespace pls {

namespace {

// Reserved bit patterns for "no entry": signalling NaNs with a payload.
constexpr unsigned long long kAbsentD = 0x7FF0DEAD00000001ull;
constexpr unsigned kAbsentF = 0x7F80DEADu;
constexpr unsigned short kAbsentH = 0x7F81u;  // BF16

// FP64: the high word alone (one 32-bit compare per entry in the kernels'
// inner loops). Every double with that high word is a NaN, and a matrix that
// stores one is refused by the build (the same test flags it), so the check
// still tells absent entries from stored ones exactly.
__device__ __forceinline__ bool dia_absent(double a) {
  return (unsigned)__double2hiint(a) == (unsigned)(kAbsentD >> 32);
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
// that the absent-entry test takes for the reserved pattern.
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

// One thread per block of kDiaRows rows (including the padding blocks): bit
// d of full[block] is set when every row of the block stores an entry on
// diagonal d.
template <class V>
__global__ void k_dia_full(int64_t nblocks, int nd, const V *__restrict__ dv,
                           uint32_t *__restrict__ full) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks)
    return;
  uint32_t bits = 0;
  for (int d = 0; d < nd; ++d) {
    bool all = true;
#pragma unroll
    for (int i = 0; i < kDiaRows; ++i)
      all = all && !dia_absent(dv[(b * nd + d) * kDiaRows + i]);
    if (all)
      bits |= 1u << d;
  }
  full[b] = bits;
}

// The RB values of a thread's rows on one diagonal (RB * sizeof(V) bytes:
// 4, 8 or a multiple of 16, aligned to their size).
template <int RB, class V>
__device__ __forceinline__ void ld_rows_vals(const V *p, V (&a)[RB]) {
  constexpr int bytes = RB * (int)sizeof(V);
  if constexpr (bytes == 4) {
    const unsigned t = __ldg(reinterpret_cast<const unsigned *>(p));
    memcpy(a, &t, 4);
  } else if constexpr (bytes == 8) {
    const uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
    memcpy(a, &t, 8);
  } else {
    static_assert(bytes % 16 == 0, "value lines load as whole vectors");
#pragma unroll
    for (int i = 0; i < bytes / 16; ++i) {
      const uint4 t = __ldg(reinterpret_cast<const uint4 *>(p) + i);
      memcpy(reinterpret_cast<char *>(a) + 16 * i, &t, 16);
    }
  }
}

// One run of len consecutive diagonals for a thread's RB rows: B's rows
// br0 + j, j = 0 .. RB + len - 2, at bp + j * ldb (columns of the thread's
// vector); the values of the run's diagonal l at ab + l * kDiaRows (the
// thread's RB of its block's kDiaRows values).
// INSIDE: len == kDiaRun and the rows all lie inside B, so the loads are
// neither checked nor predicated (otherwise rows outside [0, n) read as
// zeros). CHECK: absent entries are skipped (without it the block must store
// every diagonal). Either way each stored entry is one fma in ascending
// diagonal order.
template <bool INSIDE, bool CHECK, int RB, class V, class X, class Acc, int VEC>
__device__ __forceinline__ void dia_run(const X *bp, int64_t ldb, int64_t br0, int64_t n,
                                        int len, const V *ab, Acc (&acc)[RB][VEC]) {
  constexpr bool FAST = INSIDE;
  X bv[RB + kDiaRun - 1][VEC];
#pragma unroll
  for (int j = 0; j < RB + kDiaRun - 1; ++j) {
    if (FAST || (j < RB + len - 1 && br0 + j >= 0 && br0 + j < n)) {
      ld_vec<X, VEC>(bp + j * ldb, bv[j]);
    } else {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        bv[j][v] = X(0);
    }
  }
#pragma unroll
  for (int l = 0; l < kDiaRun; ++l) {
    if (FAST || l < len) {
      V a[RB];
      ld_rows_vals<RB, V>(ab + l * kDiaRows, a);
#pragma unroll
      for (int i = 0; i < RB; ++i)
        if (!CHECK || !dia_absent(a[i])) {
          const Acc ai = to_acc<Acc>(a[i]);
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            acc[i][v] = fma(ai, to_acc<Acc>(bv[i + l][v]), acc[i][v]);
        }
    }
  }
}

// Line patches: dia_patch_plan / dia_patch_unit in dia_plan.hpp.

// Rows per thread. Each thread owns kDiaThreadRows consecutive rows of one
// block of kDiaRows (a unit) and one 16-byte vector of C's columns.
constexpr int kDiaThreadRows = 4;

// Threads: (unit of RB rows) x (TK column vectors of VEC); a thread loops
// over C's columns in steps of TK * VEC. MASK (threads that make more than
// one pass over the columns): the block's full-diagonal mask is loaded first
// and blocks that store every diagonal skip the absent checks; with one pass
// that load's latency costs more than the checks (C3, FP64: 0.233 against
// 0.331 ms at k = 8, 0.725 against 0.849 ms at k = 32; at k = 128, two
// passes, 2.21 against 2.43 ms). A thread's unit comes from the line-patch
// plan (dia_patch_unit).
template <class V, class X, int VEC, bool MASK, int RB>
__global__ void __launch_bounds__(256, RB == kDiaRows ? 4 : 6)
    k_spmm_dia(int32_t m, int32_t n, int nd, DiaRuns runs, const V *__restrict__ dv,
               const uint32_t *__restrict__ dfull, uint32_t full_mask,
               const X *__restrict__ B, int64_t ldb, X *__restrict__ C, int64_t ldc, int k,
               int lg_tk, DiaPatchPlan patch, X alpha, X beta, int beta_nz) {
  static_assert(kDiaRows % RB == 0, "a thread's rows lie in one block");
  constexpr int SUB = kDiaRows / RB;  // units per block
  using Acc = typename AccOf<V, X>::type;
  const int64_t u = dia_patch_unit(blockIdx.x, (int)threadIdx.x, lg_tk, patch);
  const int tk = (int)(threadIdx.x & ((1 << lg_tk) - 1));
  const int64_t r0 = u * RB;
  if (r0 >= m)
    return;
  const int64_t rb = u / SUB;  // the unit's block
  const V *ab = dv + rb * nd * kDiaRows + (u % SUB) * RB;
  const bool full = MASK && (__ldg(dfull + rb) & full_mask) == full_mask;
  for (int kk = tk * VEC; kk < k; kk += VEC << lg_tk) {
    Acc acc[RB][VEC];
#pragma unroll
    for (int i = 0; i < RB; ++i)
#pragma unroll
      for (int v = 0; v < VEC; ++v)
        acc[i][v] = Acc(0);
    for (int q = 0; q < runs.n; ++q) {
      const int o0 = runs.o0[q], len = runs.len[q];
      const int64_t br0 = r0 + o0;
      const X *bp = B + br0 * ldb + kk;
      const V *aq = ab + runs.d0[q] * kDiaRows;
      if (len == kDiaRun && br0 >= 0 && br0 + RB + kDiaRun - 2 < n) {
        if (MASK && full)
          dia_run<true, false, RB, V, X, Acc, VEC>(bp, ldb, br0, n, len, aq, acc);
        else
          dia_run<true, true, RB, V, X, Acc, VEC>(bp, ldb, br0, n, len, aq, acc);
      } else {
        dia_run<false, true, RB, V, X, Acc, VEC>(bp, ldb, br0, n, len, aq, acc);
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
  d.full.release();
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
  const int64_t count = div_up((int64_t)m + kDiaPadRows, kDiaRows) * nd * kDiaRows;
  // 16 bytes of slack: the staged kernel's copies end on a 16-byte boundary.
  d.vals.reserve(sizeof(V) * count + 16);
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
  const int64_t nblocks = div_up((int64_t)m + kDiaPadRows, kDiaRows);
  d.full.reserve(sizeof(uint32_t) * nblocks + 16);  // slack as for vals
  k_dia_full<V><<<(unsigned)div_up(nblocks, 256), 256, 0, s>>>(nblocks, nd, d.vals.as<V>(),
                                                              d.full.as<uint32_t>());
  PLS_LAUNCH_CHECK();
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
  const DiaRuns runs = dia_runs(d.offs, d.nd);
  const int cols = k / VEC;
  int lg_tk = 0;
  while ((1 << lg_tk) < cols && lg_tk < 5)
    ++lg_tk;
  constexpr int RB = kDiaThreadRows;
  const int64_t nunits = div_up(m, RB);
  const int64_t threads = nunits << lg_tk;
  const uint32_t full_mask = d.nd >= 32 ? 0xffffffffu : (1u << d.nd) - 1u;
  const bool passes = cols > (1 << lg_tk);
  const DiaPatchPlan patch = dia_patch_plan(runs, RB, nunits, lg_tk);
  auto kern = passes ? k_spmm_dia<V, X, VEC, true, RB> : k_spmm_dia<V, X, VEC, false, RB>;
  kern<<<(unsigned)div_up(threads, 256), 256, 0, s>>>(
      m, c.ncols, d.nd, runs, d.vals.as<V>(), d.full.as<uint32_t>(), full_mask, B, ldb, C, ldc,
      k, lg_tk, patch, alpha, beta, beta != X(0));
  PLS_LAUNCH_CHECK();
}


// ------------------------------------------- diagonal form, B staged by TMA
//
// The kernel above reads B through L1 from L2: on the 27-point stencil each
// run of 3 diagonals loads its 6 rows of B once per 4 rows of C, so every
// row of B crosses from L2 about 13 times per SpMM. Here B's rows are staged
// in shared memory by tensor-map (TMA) copies and each crosses about 3
// times.
//
// Groups and windows. The sorted diagonal offsets fall into G groups with
// centres c_g = c_0 + g P, P rows apart (G = 3 planes of a 3-D stencil,
// P = the plane size; lines of a 2-D stencil), each within h of its centre.
// A tile is L consecutive rows of C starting at R, and a KS-column slice of
// B and C; for group g it needs B's rows [R + c_g - h, R + c_g + L + h),
// the window PW(t + g) of the chain of tiles R = b + t P. Consecutive tiles
// of a chain share windows, so a CTA walks a chain: at tile t it holds
// PW(t) .. PW(t + G - 1) in G shared-memory slots, and as soon as group 0
// is done with PW(t) it issues the copy of PW(t + G) into that slot, which
// lands while groups 1 .. G - 1 compute. One group (a band) is a chain of
// consecutive tiles (P = L) with two slots, the next tile's window loading
// while the current one computes.
//
// Values. The tile's L x nd values (the diagonal form's blocks of 4 rows,
// contiguous for consecutive rows) arrive by one 1-D bulk copy into one of
// two slabs, the next tile's while the current one computes.
//
// Threads. 256 consumer threads: NV column lanes of one 16-byte vector each
// (KS = NV * VEC columns) x 256 / NV row groups of kDiaRows rows, so
// L = 1024 / NV; and one producer warp that issues the copies. Per run of consecutive diagonals a thread reads its 4 + run
// - 1 window rows once from shared memory. Entries are added per row in
// ascending offset, one fma each, with the epilogue alpha * acc + beta * C:
// the order and arithmetic of k_spmm_dia, so the results are the same bits.
//
// Work items are (segment of Z tiles of one chain, column slice), column
// slice fastest so that the slices of a tile run together and its values
// come from L2 after the first. Waits are bounded; a wait that runs out
// sets the mapped error flag and stops the warp (the producer stops when a
// slot is not released in time, then waits, bounded, for the copies in
// flight before the CTA ends), leaving part of C unwritten; the host
// reports it on the next call.

// Shared-memory loads by 32-bit shared address (a constant part of the
// address folds into the instruction's offset).
__device__ __forceinline__ void lds16(uint32_t a, double (&v)[2]) {
  asm("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "r"(a));
}
__device__ __forceinline__ void lds16(uint32_t a, float (&v)[4]) {
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
      : "r"(a));
}
// The RB values of a thread's rows on one diagonal (RB * sizeof(V) bytes,
// aligned to their size).
template <class V, int RB>
__device__ __forceinline__ void lds_vals(uint32_t a, V (&v)[RB]) {
  constexpr int bytes = RB * (int)sizeof(V);
  if constexpr (bytes == 4) {
    uint32_t u;
    asm("ld.shared.b32 %0, [%1];" : "=r"(u) : "r"(a));
    memcpy(v, &u, 4);
  } else if constexpr (bytes == 8) {
    uint32_t u[2];
    asm("ld.shared.v2.b32 {%0, %1}, [%2];" : "=r"(u[0]), "=r"(u[1]) : "r"(a));
    memcpy(v, u, 8);
  } else {
#pragma unroll
    for (int h = 0; h < bytes / 16; ++h) {
      uint32_t u[4];
      asm("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];"
          : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3])
          : "r"(a + 16 * h));
      memcpy(reinterpret_cast<char *>(v) + 16 * h, u, 16);
    }
  }
}

// The products of one run of len diagonals for a thread's RB rows: window
// rows j = 0 .. RB + len - 2 at wa + j * ROW (shared addresses), values of
// the run's diagonal l at va + l * kDiaRows * sizeof(V). CHECK: skip absent
// entries.
template <bool CHECK, int LEN, class V, class X, class Acc, int VEC, int ROW, int RB>
__device__ __forceinline__ void dia_tma_run(uint32_t wa, uint32_t va, int len,
                                            Acc (&acc)[RB][VEC]) {
  X bv[RB + kDiaRun - 1][VEC];
#pragma unroll
  for (int j = 0; j < RB + kDiaRun - 1; ++j)
    if (j < RB + (LEN ? LEN : len) - 1)
      lds16(wa + j * ROW, bv[j]);
#pragma unroll
  for (int l = 0; l < kDiaRun; ++l) {
    if (l < (LEN ? LEN : len)) {
      V av[RB];
      lds_vals<V, RB>(va + l * kDiaRows * (int)sizeof(V), av);
#pragma unroll
      for (int i = 0; i < RB; ++i)
        if (!CHECK || !dia_absent(av[i])) {
          const Acc ai = to_acc<Acc>(av[i]);
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            acc[i][v] = fma(ai, to_acc<Acc>(bv[i + l][v]), acc[i][v]);
        }
    }
  }
}

// One group's runs for a thread's RB rows: the thread's first window row at
// shared address wrow (rows of ROW bytes), its values of diagonal 0 at
// vrow. Full runs of kDiaRun diagonals take the unpredicated body.
template <bool CHECK, class V, class X, class Acc, int VEC, int ROW, int RB>
__device__ __forceinline__ void dia_tma_group(const DiaTmaArgs &a, int g, uint32_t wrow,
                                              uint32_t vrow, Acc (&acc)[RB][VEC]) {
  for (int r = a.grp_run0[g]; r < a.grp_run0[g + 1]; ++r) {
    const int len = a.run_len[r];
    const uint32_t wa = wrow + (uint32_t)a.run_q0[r] * ROW;
    const uint32_t va = vrow + (uint32_t)a.run_d0[r] * (kDiaRows * (int)sizeof(V));
    if (len == kDiaRun)
      dia_tma_run<CHECK, kDiaRun, V, X, Acc, VEC, ROW, RB>(wa, va, len, acc);
    else
      dia_tma_run<CHECK, 0, V, X, Acc, VEC, ROW, RB>(wa, va, len, acc);
  }
}

// Slab of one tile: its values, copied from the 16-byte boundary at or
// below their first byte, then (from the next 16-byte boundary on) its
// blocks' full-diagonal masks, copied the same way.
struct DiaSlab {
  int64_t v_lo, v_bytes, f_lo, f_bytes;
  int v_skew, f_skew;  // bytes from the copies' starts to the tile's first value / mask
  int64_t f_at;        // offset of the masks in the slab
};

template <class V>
__device__ __forceinline__ DiaSlab dia_slab(int64_t R, int L, int nd) {
  DiaSlab sl;
  const int64_t v0 = R * nd * (int64_t)sizeof(V);
  sl.v_lo = v0 & ~(int64_t)15;
  sl.v_bytes = ((v0 + (int64_t)L * nd * (int64_t)sizeof(V) + 15) & ~(int64_t)15) - sl.v_lo;
  sl.v_skew = (int)(v0 - sl.v_lo);
  const int64_t f0 = (R / kDiaRows) * (int64_t)sizeof(uint32_t);
  sl.f_lo = f0 & ~(int64_t)15;
  sl.f_bytes = ((f0 + (int64_t)(L / kDiaRows) * 4 + 15) & ~(int64_t)15) - sl.f_lo;
  sl.f_skew = (int)(f0 - sl.f_lo);
  sl.f_at = ((int64_t)L * nd * (int64_t)sizeof(V) + 15) / 16 * 16 + 16;
  return sl;
}

// Warp roles. NT = kDiaRows * kDiaTmaThreads / RB consumer threads
// compute; one more warp issues the copies (its lane 0). Each window slot
// has a full barrier (its copy landed) and an empty barrier (every consumer
// warp is done with the window it holds), and so has each values slab. A
// consumer warp waits only for the copies it reads and releases each window
// after its last use, so the warps of a CTA never meet at a CTA-wide
// barrier while they work; the producer refills a slot as soon as it is
// released.
template <class V, class X, int NV, int RB>
__global__ void __launch_bounds__(kDiaRows * kDiaTmaThreads / RB + 32, 1)
    k_spmm_dia_tma(const __grid_constant__ CUtensorMap tmB, const DiaTmaArgs a,
                   const V *__restrict__ dv, const uint32_t *__restrict__ dfull,
                   X *__restrict__ C, int64_t ldc, X alpha, X beta, int beta_nz,
                   int *__restrict__ err) {
  constexpr int VEC = 16 / (int)sizeof(X);
  constexpr int KS = NV * VEC;
  constexpr int NT = kDiaRows * kDiaTmaThreads / RB;
  constexpr int NCW = NT / 32;  // consumer warps
  constexpr int L = NT / NV * RB;
  static_assert(L == kDiaTmaThreads / NV * kDiaRows, "the tile of the launch plan");
  static_assert(kDiaRows % RB == 0, "a thread's rows lie in one block");
  static_assert(NT % 32 == 0, "whole consumer warps");
  using Acc = typename AccOf<V, X>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t wfull[kDiaTmaMaxSlots], wempty[kDiaTmaMaxSlots];
  __shared__ __align__(8) uint64_t vfull[2], vempty[2];
  // Tensor copies land on 128-byte boundaries: the launch adds 128 bytes so
  // that the slots can start at the first such boundary.
  unsigned char *smem = smem_raw + ((128u - (tma::smem_addr(smem_raw) & 127u)) & 127u);
  const int tid = threadIdx.x;
  unsigned char *vbase = smem + (size_t)a.S * a.slot_bytes;
  if (tid == 0) {
    for (int s = 0; s < a.S; ++s) {
      tma::bar_init(&wfull[s]);
      tma::bar_init_count(&wempty[s], NCW);
    }
    for (int s = 0; s < 2; ++s) {
      tma::bar_init(&vfull[s]);
      tma::bar_init_count(&vempty[s], NCW);
    }
    tma::bar_init_fence();
  }
  __syncthreads();

  // Position of work item `item`: column slice k0, chain start b, rows of a
  // tile inside the chain's period, tiles [t0, t1). False when empty.
  struct Pos {
    int k0, rows_tile, t0, t1;
    int64_t b;
  };
  const auto item_pos = [&](int64_t item, Pos &p) {
    const int slice = (int)(item % a.n_slices);
    const int64_t rest = item / a.n_slices;
    const int chain = (int)(rest % a.n_chains);
    const int seg = (int)(rest / a.n_chains);
    p.k0 = slice * KS;
    p.b = (int64_t)chain * L;
    p.rows_tile = (int)min((int64_t)L, (int64_t)a.P - p.b);
    const int64_t tiles = p.b < a.m ? ((int64_t)a.m - p.b + a.P - 1) / a.P : 0;
    p.t0 = (int)((int64_t)seg * a.Z);
    p.t1 = (int)min((int64_t)p.t0 + a.Z, tiles);
    return p.t0 < p.t1;
  };

  if (tid >= NT) {
    // ---- producer (lane 0 of the last warp) ----
    if (tid == NT) {
      int nw[kDiaTmaMaxSlots], nv[2] = {0, 0};  // copies issued into each slot / slab
      for (int s = 0; s < kDiaTmaMaxSlots; ++s)
        nw[s] = 0;
      bool ok = true;
      for (int64_t item = blockIdx.x; ok && item < a.n_items; item += gridDim.x) {
        Pos p;
        if (!item_pos(item, p))
          continue;
        const auto issue_window = [&](int w) {
          const int s = w % a.S;
          if (nw[s] > 0 && !tma::bar_wait_bounded(&wempty[s], (uint32_t)(nw[s] - 1) & 1u, a.wait_limit))
            return false;
          ++nw[s];
          const int64_t row0 = p.b + (int64_t)w * a.P + a.win0;
          tma::bar_expect_tx(&wfull[s], (uint32_t)(a.slot_bytes + a.tx_extra));
          for (int j = 0; j < a.NB; ++j)
            tma::tensor_load_2d(smem + (size_t)s * a.slot_bytes + (size_t)j * a.BR * KS * sizeof(X),
                                &tmB, p.k0, (int32_t)(row0 + (int64_t)j * a.BR), &wfull[s]);
          return true;
        };
        const auto issue_vals = [&](int t) {
          const int s = t & 1;
          if (nv[s] > 0 && !tma::bar_wait_bounded(&vempty[s], (uint32_t)(nv[s] - 1) & 1u, a.wait_limit))
            return false;
          ++nv[s];
          const DiaSlab sl = dia_slab<V>(p.b + (int64_t)t * a.P, L, a.nd);
          unsigned char *slab = vbase + (size_t)s * a.vslab_bytes;
          tma::bar_expect_tx(&vfull[s], (uint32_t)(sl.v_bytes + sl.f_bytes));
          tma::bulk_load(slab, reinterpret_cast<const char *>(dv) + sl.v_lo, (uint32_t)sl.v_bytes,
                         &vfull[s]);
          tma::bulk_load(slab + sl.f_at, reinterpret_cast<const char *>(dfull) + sl.f_lo,
                         (uint32_t)sl.f_bytes, &vfull[s]);
          return true;
        };
        // Tile t reads values(t) and windows t .. t + G - 1, in that order
        // of need; window w's slot held window w - S, released by tile w - S.
        ok = issue_vals(p.t0);
        for (int g = 0; ok && g < a.G; ++g)
          ok = issue_window(p.t0 + g);
        for (int t = p.t0 + 1; ok && t < p.t1; ++t) {
          ok = issue_vals(t);
          if (ok)
            ok = issue_window(t + a.G - 1);
        }
      }
      if (!ok) {
        // A slot was not released in time: record it and give the copies
        // in flight a bounded wait (the shared memory must outlive them).
        *(volatile int *)err = 1;
        __threadfence_system();
      }
      for (int s = 0; s < a.S; ++s)
        if (nw[s] > 0)
          tma::bar_wait_bounded(&wfull[s], (uint32_t)(nw[s] - 1) & 1u, a.wait_limit);
      for (int s = 0; s < 2; ++s)
        if (nv[s] > 0)
          tma::bar_wait_bounded(&vfull[s], (uint32_t)(nv[s] - 1) & 1u, a.wait_limit);
    }
  } else {
    // ---- consumers ----
    const int lane = tid & 31;
    const int cl = tid % NV;
    const int i0 = (tid / NV) * RB;
    const uint32_t full_mask = a.nd >= 32 ? 0xffffffffu : (1u << a.nd) - 1u;
    uint32_t wph = 0, vph = 0;  // parity of the next phase of each full barrier
    bool ok = true;
    // A warp-wide bounded wait (the whole warp takes the same decision).
    const auto wait = [&](uint64_t *bar, uint32_t parity) {
      return __all_sync(0xffffffffu, tma::bar_wait_bounded(bar, parity, a.wait_limit)) != 0;
    };
    const auto release = [&](uint64_t *bar) {
      __syncwarp();
      if (lane == 0)
        tma::bar_arrive(bar);
    };
    for (int64_t item = blockIdx.x; ok && item < a.n_items; item += gridDim.x) {
      Pos p;
      if (!item_pos(item, p))
        continue;
      for (int t = p.t0; t < p.t1; ++t) {
        const int64_t R = p.b + (int64_t)t * a.P;
        const int vs = t & 1;
        if (!(ok = wait(&vfull[vs], (vph >> vs) & 1u)))
          break;
        vph ^= 1u << vs;
        Acc acc[RB][VEC];
#pragma unroll
        for (int i = 0; i < RB; ++i)
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            acc[i][v] = Acc(0);
        const DiaSlab sl = dia_slab<V>(R, L, a.nd);
        const unsigned char *slab = vbase + (size_t)vs * a.vslab_bytes;
        const uint32_t vrow =
            tma::smem_addr(slab + sl.v_skew) +
            (uint32_t)(((i0 / kDiaRows) * a.nd * kDiaRows + i0 % kDiaRows) * (int)sizeof(V));
        const uint32_t blk_full =
            reinterpret_cast<const uint32_t *>(slab + sl.f_at + sl.f_skew)[i0 / kDiaRows];
        const bool checked = (blk_full & full_mask) != full_mask;
        for (int g = 0; g < a.G; ++g) {
          const int s = (t + g) % a.S;
          if (t == p.t0 || g == a.G - 1) {  // the window's first use in this item
            if (!(ok = wait(&wfull[s], (wph >> s) & 1u)))
              break;
            wph ^= 1u << s;
          }
          constexpr int ROW = KS * (int)sizeof(X);
          const uint32_t wrow = tma::smem_addr(smem + (size_t)s * a.slot_bytes) +
                                (uint32_t)(i0 * ROW + cl * 16);
          if (checked)
            dia_tma_group<true, V, X, Acc, VEC, ROW, RB>(a, g, wrow, vrow, acc);
          else
            dia_tma_group<false, V, X, Acc, VEC, ROW, RB>(a, g, wrow, vrow, acc);
          // Window t ends its use with group 0 of tile t; on the item's last
          // tile every window it holds ends its use.
          if (g == 0 || t == p.t1 - 1)
            release(&wempty[s]);
        }
        if (!ok)
          break;
        release(&vempty[vs]);
        const int col = p.k0 + cl * VEC;
        if (col < a.k) {
#pragma unroll
          for (int i = 0; i < RB; ++i) {
            const int64_t row = R + i0 + i;
            if (i0 + i < p.rows_tile && row < a.m) {
              X *cp = C + row * ldc + col;
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
    }
    if (!ok && lane == 0) {
      // A copy did not land in time: record it; this warp stops (the
      // producer drains the copies in flight before the CTA ends).
      *(volatile int *)err = 1;
      __threadfence_system();
    }
  }
  __syncthreads();
}

template <class V, class X, int NV>
void dia_tma_run(const DiaDev &d, const DiaTmaShape &sh, const CUtensorMap &map, X *C,
                 int64_t ldc, X alpha, X beta, int sms, cudaStream_t s) {
  constexpr int RB = kDiaTmaThreadRows;
  constexpr int NT = kDiaRows * kDiaTmaThreads / RB + 32;  // consumers + the producer warp
  auto kern = k_spmm_dia_tma<V, X, NV, RB>;
  const size_t smem = sh.smem + 128;  // room to align the slots (see the kernel)
  PLS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  PLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  const unsigned grid =
      (unsigned)std::min<int64_t>(sh.a.n_items, (int64_t)sms * std::max(per_sm, 1));
  kern<<<grid, NT, smem, s>>>(map, sh.a, d.vals.as<V>(), d.full.as<uint32_t>(), C, ldc, alpha,
                              beta, beta != X(0), d.err.dev);
  PLS_LAUNCH_CHECK();
}

template <class V, class X>
bool dia_tma_launch(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                    X alpha, X beta, cudaStream_t s, bool launch) {
  DiaDev &d = c.dia;
  int dev = 0, sms = 0;
  PLS_CUDA(cudaGetDevice(&dev));
  PLS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DiaTmaShape sh = dia_tma_shape(d.offs, d.nd, m, k, (int)sizeof(X), (int)sizeof(V), sms);
  const tma::EncodeTiledFn enc = tma::encode_tiled();
  if (!sh.ok || !enc || c.ncols <= 0 || (uintptr_t)d.vals.p % 16)
    return false;
  // B as a 2-D tensor (k columns innermost, ncols rows of ldb elements),
  // copied in boxes of KS columns x BR rows; rows outside [0, ncols) and
  // columns past k read as zeros. A shape the driver refuses is not used.
  constexpr int VEC = 16 / (int)sizeof(X);
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)c.ncols};
  const cuuint64_t strides[1] = {(cuuint64_t)ldb * sizeof(X)};
  const cuuint32_t box[2] = {(cuuint32_t)(sh.NV * VEC), (cuuint32_t)sh.a.BR};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&map, sizeof(X) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, const_cast<X *>(B), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return false;
  if (!launch)
    return true;
  if (!d.err.host)
    d.err.alloc();
  sh.a.tx_extra = g_stage_shortfall.load();
  sh.a.wait_limit = g_stage_wait_limit.load();
  switch (sh.NV) {
  case 8: dia_tma_run<V, X, 8>(d, sh, map, C, ldc, alpha, beta, sms, s); break;
  case 4: dia_tma_run<V, X, 4>(d, sh, map, C, ldc, alpha, beta, sms, s); break;
  default: dia_tma_run<V, X, 2>(d, sh, map, C, ldc, alpha, beta, sms, s); break;
  }
  return true;
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


template <class X>
bool spmm_dia_tma(CsrDev &c, int32_t m, const X *B, int64_t ldb, X *C, int64_t ldc, int k,
                  X alpha, X beta, cudaStream_t s, bool launch) {
  DiaDev &d = c.dia;
  if (d.err.host && *(volatile int *)d.err.host) {
    *(volatile int *)d.err.host = 0;
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                "diagonal-form SpMM: a staged copy did not complete (reported by an earlier call)");
  }
  // The diagonal form itself (built or examined here) and its conditions.
  if (!spmm_dia<X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, false))
    return false;
  const Vt vt = c.evt();
  if constexpr (sizeof(X) == 8) {
    if (vt == Vt::F64)
      return dia_tma_launch<double, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, launch);
  }
  if (vt == Vt::F32)
    return dia_tma_launch<float, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, launch);
  if (vt == Vt::BF16)
    return dia_tma_launch<__nv_bfloat16, X>(c, m, B, ldb, C, ldc, k, alpha, beta, s, launch);
  return false;
}

template bool spmm_dia_tma<float>(CsrDev &, int32_t, const float *, int64_t, float *, int64_t,
                                  int, float, float, cudaStream_t, bool);
template bool spmm_dia_tma<double>(CsrDev &, int32_t, const double *, int64_t, double *, int64_t,
                                   int, double, double, cudaStream_t, bool);

}  // namespace pls
