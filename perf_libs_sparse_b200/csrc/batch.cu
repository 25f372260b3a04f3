// Batched uneven SpMM in one persistent launch.
//
// Instances are FP32 CSR or BSR handles, each with its own dense row-major
// B_i / C_i and k_i. The work is cut into items of R rows (R block-aligned
// for BSR), sorted by estimated work (rows x nonzeros per row x k, largest
// first), and consumed by a grid of (SMs x resident blocks) CTAs: each warp
// takes the next item from a global atomic counter until the list is empty.
// Nothing ever waits on another warp, so there is no spin and no deadlock
// whatever the scheduling; the counter is reset by a memset node in the same
// CUDA graph that holds the launch.
//
// Inside an item, rows go through the row-group loop of spmm_rows.cuh with
// the instance's own lane shape (TK lanes over C's columns, 16-byte vectors
// when its B and C allow, TN lanes over a row's entries). Every instance is
// read from the batch's own copy of its entries, (column, value) side by
// side; a BSR instance is expanded at creation into scalar rows whose
// entries are its blocks' rows in stored order.
//
// Staged items come first. Where a block of rows reads only a narrow window
// of B's rows (banded matrices: a block of 128 rows with half-bandwidth 64
// reads 256 rows of B, each of them up to 129 times; BSR block diagonals:
// each row of B bs times), a whole CTA takes the block: it copies the
// window's rows of B, up to 32 columns at a time, into shared memory once
// and computes every row of the block from there, so each B element comes
// from L2 once per block instead of once per nonzero that reads it. The CTA
// takes the next staged item from a second counter; when none are left its
// warps go on to the per-warp items. Which blocks are staged is decided at
// creation from each block's column window; the tuner times the batch with
// and without them.
#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "pls_internal.hpp"
#include "spmm_rows.cuh"

namespace pls {

namespace {

struct InstDesc {
  const int32_t *rp;   // row pointers of the scalar rows (a BSR instance's: the batch's)
  const int32_t *col;  // the handle's arrays, read once at creation
  const float *val;
  const int2 *cv;      // the batch's packed (column, value) copy the kernel reads
  const float *B;
  float *C;
  int64_t ldb, ldc;
  int32_t m, k, bs, layout, is_bsr;  // bs / is_bsr: block-aligned items for BSR
  int32_t lg_tk, lg_tn, path;  // path: 0 = VEC 4, 1 = VEC 1 x 1, 2 = VEC 1 x 2, 3 = BSR blocks
  const int32_t *brp;  // BSR: the handle's block row pointers (path 3 reads the blocks)
  // CSR with every row's columns consecutive (bands): the values alone, a
  // copy made at creation; staged rows read them instead of the packed
  // entries (null otherwise)
  const float *band_val;
};

struct Item {
  int32_t inst, row0, row1, pad;
};

// A staged item: rows [row0, row1) of instance `inst`, whose entries all
// have columns in [lo, lo + w), for C's columns [c0, c0 + ks) (ks <= 32).
// The window sits in shared memory as w rows of 4 * tk floats (ks rounded
// up to whole float4s, zero past ks).
struct SItem {
  int32_t inst, row0, row1, lo;
  int32_t w, c0, ks, tk;
};

constexpr int kBatchThreads = 256;
constexpr int kStageFloats = 8192;  // 32 KB of shared memory per CTA
constexpr int kStageCols = 32;      // widest column slice of a staged item

// One item's rows with the instance's vector shape.
template <class Rows, bool OFF32>
__device__ __forceinline__ void batch_rows(const Rows &A, const InstDesc &d, const Item &w,
                                           int lane, float alpha, float beta, int beta_nz,
                                           const L2Policy &pol) {
  const int lg_g = d.lg_tk + d.lg_tn;
  for (int32_t r0 = w.row0; r0 < w.row1; r0 += (32 >> lg_g)) {
    const int32_t row = r0 + (lane >> lg_g);
    const bool live = row < w.row1;
    if (d.path == 0)
      spmm_row_group<4, 1, float, float, Rows, OFF32, kEntriesAhead>(
          A, row, live, d.lg_tk, d.lg_tn, d.B, d.ldb, d.C, d.ldc, d.k, alpha, beta, beta_nz, pol);
    else if (d.path == 1)
      spmm_row_group<1, 1, float, float, Rows, OFF32, kEntriesAhead>(
          A, row, live, d.lg_tk, d.lg_tn, d.B, d.ldb, d.C, d.ldc, d.k, alpha, beta, beta_nz, pol);
    else
      spmm_row_group<1, 2, float, float, Rows, OFF32, kEntriesAhead>(
          A, row, live, d.lg_tk, d.lg_tn, d.B, d.ldb, d.C, d.ldc, d.k, alpha, beta, beta_nz, pol);
  }
}

// bs values of one block column of the column-major copy: bs * 4 bytes at
// a multiple of that size.
template <int BS>
__device__ __forceinline__ void ld_block_line_f(const float *p, float (&a)[BS]) {
  if constexpr (BS == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
    a[0] = t.x, a[1] = t.y;
  } else {
#pragma unroll
    for (int h = 0; h < BS / 4; ++h) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(p) + h);
      a[4 * h] = t.x, a[4 * h + 1] = t.y, a[4 * h + 2] = t.z, a[4 * h + 3] = t.w;
    }
  }
}

// A BSR instance's rows [w.row0, w.row1) (whole block rows) read as blocks:
// TK = 2^lg_tk lanes per block row, one column of C each per pass, 32 / TK
// block rows per warp. d.val is the batch's column-major copy of the blocks
// (column j of block b at b * bs * bs + j * bs). Per block a lane takes the
// block's columns j in order: its element of B's row col * bs + j
// (coalesced across the lanes), the block's column j (the same addresses
// across the block row's lanes), and one fma per row of the block. Per
// element of C that is the order of the scalar rows the other paths read
// (blocks in stored order, then the block's columns). B's rows are read once
// per block instead of once per scalar row.
template <int BS>
__device__ __forceinline__ void batch_bsr_rows(const InstDesc &d, const Item &w, int lane,
                                               float alpha, float beta, int beta_nz) {
  const int TK = 1 << d.lg_tk, per = 32 >> d.lg_tk;
  const int t = lane & (TK - 1);
  const int32_t br1 = w.row1 / BS;
  for (int32_t br = w.row0 / BS + (lane >> d.lg_tk); br < br1; br += per) {
    const int32_t b0 = __ldg(d.brp + br), b1 = __ldg(d.brp + br + 1);
    for (int kk = t; kk < d.k; kk += TK) {
      float acc[BS];
#pragma unroll
      for (int i = 0; i < BS; ++i)
        acc[i] = 0.f;
      for (int32_t b = b0; b < b1; ++b) {
        const float *bp = d.B + (int64_t)__ldg(d.col + b) * BS * d.ldb + kk;
        const float *ab = d.val + (int64_t)b * BS * BS;
#pragma unroll
        for (int j = 0; j < BS; ++j) {
          const float bj = __ldg(bp + (int64_t)j * d.ldb);
          float a[BS];
          ld_block_line_f<BS>(ab + j * BS, a);
#pragma unroll
          for (int i = 0; i < BS; ++i)
            acc[i] = fmaf(a[i], bj, acc[i]);
        }
      }
#pragma unroll
      for (int i = 0; i < BS; ++i) {
        float *cp = d.C + ((int64_t)br * BS + i) * d.ldc + kk;
        *cp = beta_nz ? acc[i] * alpha + beta * *cp : acc[i] * alpha;
      }
    }
  }
}

// One staged item, by the whole CTA. The window of B (rows lo .. lo + w - 1,
// columns c0 .. c0 + ks - 1) is copied into `stage` (row stride 4 tk
// floats); then tk lanes per row own 4 columns each, and every row of the
// item adds its entries in stored order from the staged rows. Each entry's
// column lies in the window (the item was built from the minimum and
// maximum column of its entries), so the stage reads stay inside
// w * 4 tk floats.
__device__ __forceinline__ void staged_item(const SItem &w, const InstDesc &d,
                                            float *__restrict__ stage, float alpha, float beta,
                                            int beta_nz) {
  constexpr int warps = kBatchThreads / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int TK = w.tk, KSP = 4 * w.tk;
  if ((d.ldb & 3) == 0 && ((uintptr_t)d.B & 15) == 0) {
    // TK lanes per window row, a float4 each (c0 is a multiple of 32, so
    // every row segment starts on 16 bytes)
    const int per = 32 / TK;
    const int rs = lane / TK, c4 = lane - rs * TK, c = 4 * c4;
    if (rs < per) {
      const float *src = d.B + (int64_t)w.lo * d.ldb + w.c0 + c;
      float4 *dst = reinterpret_cast<float4 *>(stage) + c4;
#pragma unroll 4
      for (int r = warp * per + rs; r < w.w; r += warps * per) {
        const float *p = src + (int64_t)r * d.ldb;
        float4 v;
        if (c + 4 <= w.ks) {
          v = __ldg(reinterpret_cast<const float4 *>(p));
        } else {
          v.x = c < w.ks ? __ldg(p) : 0.f;
          v.y = c + 1 < w.ks ? __ldg(p + 1) : 0.f;
          v.z = c + 2 < w.ks ? __ldg(p + 2) : 0.f;
          v.w = 0.f;  // c + 3 >= ks here
        }
        dst[r * TK] = v;
      }
    }
  } else {
    // 32 / KSP window rows per warp pass, a lane per column
    const int per = 32 / KSP;
    const int rs = lane / KSP, c = lane - rs * KSP;
    if (rs < per) {
      const bool in = c < w.ks;
      const float *src = d.B + (int64_t)w.lo * d.ldb + w.c0 + (in ? c : 0);
#pragma unroll 4
      for (int r = warp * per + rs; r < w.w; r += warps * per)
        stage[r * KSP + c] = in ? __ldg(src + (int64_t)r * d.ldb) : 0.f;
    }
  }
  __syncthreads();
  const float4 *st4 = reinterpret_cast<const float4 *>(stage);
  const int per = 32 / TK;  // rows per warp
  const int rs = lane / TK, tk = lane - rs * TK;
  if (rs >= per)
    return;
  const int kk = w.c0 + 4 * tk;  // this lane's first column of C
  const int kend = w.c0 + w.ks;
  const bool vec = d.path == 0 && kk + 4 <= kend;
  for (int32_t row = w.row0 + warp * per + rs; row < w.row1; row += warps * per) {
    const int32_t s = __ldg(d.rp + row), e = __ldg(d.rp + row + 1);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const auto add = [&](int2 t) {
      const float4 b = st4[(t.x - w.lo) * TK + tk];
      const float a = __int_as_float(t.y);
      acc.x = fmaf(a, b.x, acc.x);
      acc.y = fmaf(a, b.y, acc.y);
      acc.z = fmaf(a, b.z, acc.z);
      acc.w = fmaf(a, b.w, acc.w);
    };
    if (d.band_val) {
      // consecutive columns: the row's first column, then its values alone
      // (4 bytes per entry), in stored order
      if (s < e) {
        const float4 *sp = st4 + (__ldg(d.cv + s).x - w.lo) * TK + tk;
        const auto addv = [&](float a, const float4 b) {
          acc.x = fmaf(a, b.x, acc.x);
          acc.y = fmaf(a, b.y, acc.y);
          acc.z = fmaf(a, b.z, acc.z);
          acc.w = fmaf(a, b.w, acc.w);
        };
        int32_t q = s;
        for (; q + 4 <= e; q += 4) {
          float a[4];
#pragma unroll
          for (int u = 0; u < 4; ++u)
            a[u] = __ldg(d.band_val + q + u);
#pragma unroll
          for (int u = 0; u < 4; ++u)
            addv(a[u], sp[(q - s + u) * TK]);
        }
        for (; q < e; ++q)
          addv(__ldg(d.band_val + q), sp[(q - s) * TK]);
      }
    } else {
      int32_t q = s;
      for (; q + 4 <= e; q += 4) {
        int2 t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          t[u] = __ldg(d.cv + q + u);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          add(t[u]);
      }
      for (; q < e; ++q)
        add(__ldg(d.cv + q));
    }
    float *crow = d.C + (int64_t)row * d.ldc + kk;
    const float sum[4] = {acc.x, acc.y, acc.z, acc.w};
    if (vec) {
      float out[4];
      if (beta_nz) {
        const float4 old = *reinterpret_cast<const float4 *>(crow);
        const float o[4] = {old.x, old.y, old.z, old.w};
#pragma unroll
        for (int v = 0; v < 4; ++v)
          out[v] = sum[v] * alpha + beta * o[v];
      } else {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          out[v] = sum[v] * alpha;
      }
      *reinterpret_cast<float4 *>(crow) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (kk + v < kend) {
          float o = sum[v] * alpha;
          if (beta_nz)
            o += beta * crow[v];
          crow[v] = o;
        }
    }
  }
}

// counters[0] hands out the per-warp items, counters[1] the staged ones.
// The dynamic shared memory (kStageFloats floats) is needed only when there
// are staged items.
template <bool OFF32>
__global__ void __launch_bounds__(kBatchThreads, 4)  // 64 registers: 4 blocks per SM
    k_batch_spmm(const InstDesc *__restrict__ inst, const Item *__restrict__ items,
                 int64_t n_items, const SItem *__restrict__ sitems, int64_t n_sitems,
                 unsigned long long *__restrict__ counters, float alpha, float beta,
                 int beta_nz) {
  extern __shared__ float4 stage4[];
  __shared__ unsigned long long s_ticket;
  if (n_sitems > 0) {
    for (;;) {
      if (threadIdx.x == 0)
        s_ticket = atomicAdd(counters + 1, 1ull);
      __syncthreads();
      const unsigned long long t = s_ticket;
      if (t >= (unsigned long long)n_sitems)
        break;  // every thread read the same ticket: the whole CTA leaves
      const SItem w = sitems[t];
      staged_item(w, inst[w.inst], reinterpret_cast<float *>(stage4), alpha, beta, beta_nz);
      __syncthreads();  // the stage and s_ticket are reused by the next item
    }
  }
  const L2Policy pol = make_l2_policy();
  const int lane = threadIdx.x & 31;
  unsigned long long it = 0;
  if (lane == 0)
    it = atomicAdd(counters, 1ull);
  it = __shfl_sync(0xffffffffu, it, 0);
  while (it < (unsigned long long)n_items) {
    // Take the next ticket now; its round trip overlaps this item's loads.
    unsigned long long next = 0;
    if (lane == 0)
      next = atomicAdd(counters, 1ull);
    const Item w = items[it];
    const InstDesc d = inst[w.inst];
    if (d.path == 3) {
      if (d.bs == 8)
        batch_bsr_rows<8>(d, w, lane, alpha, beta, beta_nz);
      else if (d.bs == 4)
        batch_bsr_rows<4>(d, w, lane, alpha, beta, beta_nz);
      else
        batch_bsr_rows<2>(d, w, lane, alpha, beta, beta_nz);
    } else {
      const PackedRows A{d.rp, d.cv};
      batch_rows<PackedRows, OFF32>(A, d, w, lane, alpha, beta, beta_nz, pol);
    }
    it = __shfl_sync(0xffffffffu, next, 0);
  }
}

// The column window of each block of rs rows of one instance: x = smallest
// column, y = largest (INT32_MAX / INT32_MIN for a block without entries),
// z = the block's entries. One CTA of 256 threads per block.
__global__ void __launch_bounds__(256)
    k_block_window(int32_t m, int32_t rs, const int32_t *__restrict__ rp,
                   const int2 *__restrict__ cv, int4 *__restrict__ out) {
  __shared__ int s_lo[8], s_hi[8];
  const int64_t r0 = (int64_t)blockIdx.x * rs;
  const int64_t r1 = r0 + rs < (int64_t)m ? r0 + rs : (int64_t)m;
  const int32_t p0 = rp[r0], p1 = rp[r1];
  int lo = INT32_MAX, hi = INT32_MIN;
  for (int32_t p = p0 + (int32_t)threadIdx.x; p < p1; p += 256) {
    const int c = cv[p].x;
    lo = min(lo, c);
    hi = max(hi, c);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    s_lo[threadIdx.x >> 5] = lo;
    s_hi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < 8; ++i) {
      lo = min(lo, s_lo[i]);
      hi = max(hi, s_hi[i]);
    }
    out[blockIdx.x] = make_int4(lo, hi, p1 - p0, 0);
  }
}

// Clears *flag when some row's columns are not consecutive.
__global__ void k_rows_consecutive(int32_t m, const int32_t *__restrict__ rp,
                                   const int32_t *__restrict__ col, int *__restrict__ flag) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m)
    return;
  for (int32_t p = rp[r] + 1; p < rp[r + 1]; ++p)
    if (col[p] != col[p - 1] + 1) {
      atomicAnd(flag, 0);
      return;
    }
}

// The blocks of a BSR instance, column-major (element (i, j) of block p at
// p * bs * bs + j * bs + i), from either block layout.
__global__ void k_bsr_colmajor(int64_t nnzb, int32_t bs, int rowmajor,
                               const float *__restrict__ val, float *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t E = (int64_t)bs * bs;
  if (e >= nnzb * E)
    return;
  const int64_t p = e / E;
  const int32_t r = (int32_t)(e % E), j = r / bs, i = r % bs;
  out[e] = val[p * E + (rowmajor ? (int64_t)i * bs + j : r)];
}

__global__ void k_pack_cv(int64_t nnz, const int32_t *__restrict__ col,
                          const float *__restrict__ val, int2 *__restrict__ cv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nnz)
    cv[i] = make_int2(col[i], __float_as_int(val[i]));
}

// A BSR instance as scalar CSR rows. Row i of block row br holds, block by
// block in stored order, the bs entries of the block's row i: it starts
// after the br block rows before it (bs * bs entries per block) and the i
// rows of br before it (bs entries per block of br).
__global__ void k_bsr_scalar_rp(int32_t mb, int32_t bs, const int32_t *__restrict__ rp,
                                int32_t *__restrict__ srp) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r > (int64_t)mb * bs)
    return;
  if (r == (int64_t)mb * bs) {
    srp[r] = rp[mb] * bs * bs;
    return;
  }
  const int32_t br = (int32_t)(r / bs), i = (int32_t)(r % bs);
  srp[r] = rp[br] * bs * bs + i * bs * (rp[br + 1] - rp[br]);
}

// The entries of scalar row r: (column, value) for every block of its block
// row and every column jj of the block, in that order (the order the BSR
// kernels add them in); blocks are row-major (value i*bs + jj) or
// column-major (jj*bs + i).
__global__ void k_bsr_pack(int32_t mb, int32_t bs, int rowmajor, const int32_t *__restrict__ rp,
                           const int32_t *__restrict__ col, const float *__restrict__ val,
                           const int32_t *__restrict__ srp, int2 *__restrict__ cv) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (int64_t)mb * bs)
    return;
  const int32_t br = (int32_t)(r / bs), i = (int32_t)(r % bs);
  int64_t pos = srp[r];
  for (int32_t b = rp[br]; b < rp[br + 1]; ++b)
    for (int32_t jj = 0; jj < bs; ++jj) {
      const float v = val[(int64_t)b * bs * bs + (rowmajor ? i * bs + jj : jj * bs + i)];
      cv[pos++] = make_int2(col[b] * bs + jj, __float_as_int(v));
    }
}

}  // namespace

}  // namespace pls

struct perflibs_b200_batch_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<pls::InstDesc> host;
  std::vector<double> work_per_row;  // nonzeros per row x k (for ordering)
  pls::DevBuf inst, items, counter;
  pls::DevBuf packed;  // every instance's (column, value) pairs, packed at creation
  pls::DevBuf scalar_rp;  // row pointers of the BSR instances' scalar rows
  pls::DevBuf bsr_cm;     // column-major copies of the blocks read as blocks (path 3)
  pls::DevBuf band_vals;  // the values of the band instances (consecutive columns)
  pls::DevBuf sitems;     // staged items, largest first
  // Per instance, the row ranges left to the per-warp items when staged
  // items are on (the blocks that were not staged).
  std::vector<std::vector<std::pair<int32_t, int32_t>>> warp_ranges;
  int64_t n_items = 0;
  int64_t n_sitems = 0;  // staged items built at creation
  bool staging = true;   // run them (else every row goes to per-warp items)
  int32_t tile = 0;
  int grid = 0;
  cudaGraphExec_t graph = nullptr;
  float g_alpha = 0.f, g_beta = 0.f;
  bool graph_valid = false;
  bool own_stream = false;
  bool off32 = true;  // every B / C offset of every instance fits in 32 bits
  ~perflibs_b200_batch_s() {
    if (graph)
      cudaGraphExecDestroy(graph);
    if (own_stream && stream)
      cudaStreamDestroy(stream);
  }
};

namespace pls {

using Batch = perflibs_b200_batch_s;

namespace {

// The per-warp items: the rows not in staged items (all rows when staging
// is off), cut into items of `tile` rows.
void build_items(Batch *B, int32_t tile) {
  std::vector<std::pair<double, Item>> v;
  for (int32_t i = 0; i < (int32_t)B->host.size(); ++i) {
    const InstDesc &d = B->host[i];
    int32_t R = tile;
    if (d.is_bsr)
      R = std::max<int32_t>(d.bs, (tile / d.bs) * d.bs);
    const std::vector<std::pair<int32_t, int32_t>> all{{0, d.m}};
    for (const auto &rg : B->staging ? B->warp_ranges[i] : all)
      for (int32_t r0 = rg.first; r0 < rg.second; r0 += R) {
        Item it{i, r0, std::min(rg.second, r0 + R), 0};
        v.push_back({B->work_per_row[i] * (it.row1 - it.row0), it});
      }
  }
  std::stable_sort(v.begin(), v.end(), [](auto &a, auto &b) { return a.first > b.first; });
  std::vector<Item> items(v.size());
  for (size_t j = 0; j < v.size(); ++j)
    items[j] = v[j].second;
  B->n_items = (int64_t)items.size();
  B->items.reserve(sizeof(Item) * std::max<size_t>(items.size(), 1));
  if (!items.empty())
    PLS_CUDA(cudaMemcpyAsync(B->items.p, items.data(), sizeof(Item) * items.size(),
                             cudaMemcpyHostToDevice, B->stream));
  PLS_CUDA(cudaStreamSynchronize(B->stream));
  B->tile = tile;
  B->graph_valid = false;
}

// The staged items, once at creation (the packed entries must be in
// place). Each instance with k >= 1 is cut into blocks of rs rows, rs half
// the window rows its widest column slice (min(k, 32) columns, rounded up
// to float4s) leaves in kStageFloats. A block is staged when its entries'
// column window fits in the stage and holds at most half as many rows of B
// as the block has entries (each staged B row read at least twice on
// average); it then gives one item per column slice of 32. The other rows
// go to the per-warp items.
void build_staged(Batch *B) {
  const int32_t count = (int32_t)B->host.size();
  B->warp_ranges.assign(count, {});
  std::vector<std::pair<double, SItem>> v;
  DevBuf win;
  std::vector<int4> hw;
  for (int32_t i = 0; i < count; ++i) {
    const InstDesc &d = B->host[i];
    auto &ranges = B->warp_ranges[i];
    const auto to_warps = [&](int32_t r0, int32_t r1) {
      if (!ranges.empty() && ranges.back().second == r0)
        ranges.back().second = r1;
      else
        ranges.push_back({r0, r1});
    };
    if (d.m == 0)
      continue;
    if (d.k < 1 || d.path == 3) {  // BSR read as blocks: per-warp items only
      to_warps(0, d.m);
      continue;
    }
    const int32_t ksp0 = 4 * (int32_t)div_up(std::min(d.k, kStageCols), 4);
    const int32_t wmax = kStageFloats / ksp0;
    const int32_t rs = wmax / 2;
    const int64_t nblk = div_up((int64_t)d.m, (int64_t)rs);
    win.reserve(sizeof(int4) * nblk);
    k_block_window<<<(unsigned)nblk, 256, 0, B->stream>>>(d.m, rs, d.rp, d.cv, win.as<int4>());
    PLS_LAUNCH_CHECK();
    hw.resize(nblk);
    PLS_CUDA(cudaMemcpyAsync(hw.data(), win.p, sizeof(int4) * nblk, cudaMemcpyDeviceToHost,
                             B->stream));
    PLS_CUDA(cudaStreamSynchronize(B->stream));
    for (int64_t j = 0; j < nblk; ++j) {
      const int32_t r0 = (int32_t)(j * rs), r1 = (int32_t)std::min<int64_t>(d.m, r0 + (int64_t)rs);
      const int4 b = hw[j];
      const int64_t w = (int64_t)b.y - b.x + 1;
      if (b.z == 0 || w > wmax || (int64_t)b.z < 2 * w) {
        to_warps(r0, r1);
        continue;
      }
      for (int32_t c0 = 0; c0 < d.k; c0 += kStageCols) {
        const int32_t ks = std::min(kStageCols, d.k - c0);
        const SItem it{i, r0, r1, b.x, (int32_t)w, c0, ks, (int32_t)div_up(ks, 4)};
        v.push_back({(double)b.z * it.tk + (double)w * it.tk, it});
      }
    }
  }
  std::stable_sort(v.begin(), v.end(), [](auto &a, auto &b) { return a.first > b.first; });
  std::vector<SItem> items(v.size());
  for (size_t j = 0; j < v.size(); ++j)
    items[j] = v[j].second;
  B->n_sitems = (int64_t)items.size();
  B->sitems.reserve(sizeof(SItem) * std::max<size_t>(items.size(), 1));
  if (!items.empty())
    PLS_CUDA(cudaMemcpyAsync(B->sitems.p, items.data(), sizeof(SItem) * items.size(),
                             cudaMemcpyHostToDevice, B->stream));
  PLS_CUDA(cudaStreamSynchronize(B->stream));
}

void capture(Batch *B, float alpha, float beta) {
  if (B->graph) {
    cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
  }
  cudaGraph_t g;
  cudaStream_t s = B->stream;
  PLS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(B->counter.p, 0, 16, s);
  const int64_t n_s = B->staging ? B->n_sitems : 0;
  // A launch refused during capture invalidates the capture: end it, take
  // the launch's error (so that it does not surface in a later call) and
  // report it.
  cudaError_t launch = cudaSuccess;
  if (B->n_items > 0 || n_s > 0) {
    auto kern = B->off32 ? k_batch_spmm<true> : k_batch_spmm<false>;
    const size_t smem = n_s > 0 ? sizeof(float) * kStageFloats : 0;
    kern<<<B->grid, kBatchThreads, smem, s>>>(
        B->inst.as<InstDesc>(), B->items.as<Item>(), B->n_items, B->sitems.as<SItem>(), n_s,
        B->counter.as<unsigned long long>(), alpha, beta, beta != 0.f);
    launch = cudaGetLastError();
  }
  const cudaError_t ended = cudaStreamEndCapture(s, &g);
  if (launch != cudaSuccess || ended != cudaSuccess) {
    if (ended == cudaSuccess)
      cudaGraphDestroy(g);
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                std::string("batch capture: ") +
                    cudaGetErrorString(launch != cudaSuccess ? launch : ended));
  }
  PLS_CUDA(cudaGraphInstantiate(&B->graph, g, 0));
  cudaGraphDestroy(g);
  B->g_alpha = alpha;
  B->g_beta = beta;
  B->graph_valid = true;
}

void run(Batch *B, float alpha, float beta) {
  if (!B->graph_valid || alpha != B->g_alpha || beta != B->g_beta)
    capture(B, alpha, beta);
  PLS_CUDA(cudaGraphLaunch(B->graph, B->stream));
}

}  // namespace

}  // namespace pls

using namespace pls;

extern "C" {

perflibs_status_t perflibs_b200_batch_create(perflibs_b200_batch_t *out, int32_t count,
                                             const perflibs_spmat_t *mats, const int32_t *k,
                                             const float *const *Bp, const int64_t *ldb,
                                             float *const *Cp, const int64_t *ldc, void *stream) {
  if (!out || count <= 0 || !mats || !k || !Bp || !ldb || !Cp || !ldc)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  *out = nullptr;
  return status_guard([&]() -> perflibs_status_t {
    std::unique_ptr<Batch> owner(new Batch);  // freed on every early return
    Batch *B = owner.get();
    cudaGetDevice(&B->device);
    if (stream) {
      B->stream = (cudaStream_t)stream;
    } else {
      PLS_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
      B->own_stream = true;
    }
    for (int32_t i = 0; i < count; ++i) {
      Mat *A = mats[i];
      if (!A || A->dt != Dt::F32 || k[i] < 0 || ldb[i] < k[i] || ldc[i] < k[i] ||
          !(A->fmt == Fmt::CSR || A->fmt == Fmt::SELL || A->fmt == Fmt::BSR))
        return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
      InstDesc d{};
      d.B = Bp[i];
      d.C = Cp[i];
      d.ldb = ldb[i];
      d.ldc = ldc[i];
      d.m = A->m;
      d.k = k[i];
      if (A->fmt == Fmt::BSR) {
        d.is_bsr = 1;
        d.bs = A->bsr.bs;
        d.layout = A->bsr.layout;
        d.rp = A->bsr.row_ptr.as<int32_t>();
        d.col = A->bsr.col.as<int32_t>();
        d.val = A->bsr.vals.as<float>();
      } else {
        d.is_bsr = 0;
        d.bs = 1;
        d.rp = A->csr.row_ptr.as<int32_t>();
        d.col = A->csr.col.as<int32_t>();
        d.val = A->csr.vals.as<float>();
      }
      if (d.is_bsr && (int64_t)A->bsr.nnzb * d.bs * d.bs > INT32_MAX)
        return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
      // Lane shape and vector width per instance: 16-byte vectors when k
      // fills at least one and its B and C rows are 16-byte aligned (one
      // vector tile per pass), else scalar columns with up to two per lane.
      const bool v4 = k[i] >= 4 && (uintptr_t)Bp[i] % 16 == 0 && (uintptr_t)Cp[i] % 16 == 0 &&
                      ldb[i] % 4 == 0 && ldc[i] % 4 == 0;
      const RowsShape sh =
          rows_shape(k[i], v4 ? 4 : 1, (double)A->nnz / std::max(A->m, 1), v4 ? 1 : 2);
      d.lg_tk = sh.lg_tk;
      d.lg_tn = sh.lg_tn;
      d.path = v4 ? 0 : (sh.nv == 2 ? 2 : 1);
      if (d.is_bsr && (d.bs == 2 || d.bs == 4 || d.bs == 8) && k[i] > 0) {
        // read as blocks: one column of C per lane, up to 32 lanes per block row
        d.path = 3;
        d.brp = d.rp;
        d.lg_tk = 0;
        while ((1 << d.lg_tk) < k[i] && d.lg_tk < 5)
          ++d.lg_tk;
        d.lg_tn = 0;
      }
      // B has A->n rows of ldb, C has A->m rows of ldc
      if ((int64_t)A->n * ldb[i] >= INT32_MAX || (int64_t)A->m * ldc[i] >= INT32_MAX)
        B->off32 = false;
      B->host.push_back(d);
      B->work_per_row.push_back(((double)A->nnz / std::max(A->m, 1) + 1.0) * std::max(k[i], 1));
    }
    // Every CSR instance, and every BSR instance not read as blocks, is read
    // as scalar CSR rows whose column and value sit side by side (one 8-byte
    // load per entry: each of a row's column lanes loads every entry, so
    // these loads are a large share of the kernel's instructions); such BSR
    // instances are expanded to scalar rows here. BSR instances read as
    // blocks (path 3) get a column-major copy of their blocks instead.
    int64_t packed = 0, srows = 0, cm = 0;
    for (int32_t i = 0; i < count; ++i) {
      const InstDesc &d = B->host[i];
      if (d.path == 3)
        cm += mats[i]->bsr.nnzb * d.bs * d.bs;
      else
        packed += d.is_bsr ? mats[i]->bsr.nnzb * d.bs * d.bs : mats[i]->csr.nnz;
      if (d.is_bsr && d.path != 3)
        srows += (int64_t)d.m + 1;
    }
    B->packed.reserve(sizeof(int2) * std::max<int64_t>(packed, 1));
    B->scalar_rp.reserve(sizeof(int32_t) * std::max<int64_t>(srows, 1));
    B->bsr_cm.reserve(sizeof(float) * std::max<int64_t>(cm, 1));
    packed = srows = cm = 0;
    for (int32_t i = 0; i < count; ++i) {
      InstDesc &d = B->host[i];
      int2 *cv = B->packed.as<int2>() + packed;
      if (d.path == 3) {
        const BsrDev &b = mats[i]->bsr;
        float *out = B->bsr_cm.as<float>() + cm;
        const int64_t e = b.nnzb * b.bs * b.bs;
        if (e > 0)
          k_bsr_colmajor<<<(unsigned)div_up(e, 256), 256, 0, B->stream>>>(
              b.nnzb, b.bs, d.layout == PERFLIBS_ROW_MAJOR, d.val, out);
        d.val = out;
        cm += e;
        d.cv = nullptr;
        continue;
      }
      if (d.is_bsr) {
        const BsrDev &b = mats[i]->bsr;
        int32_t *srp = B->scalar_rp.as<int32_t>() + srows;
        const int64_t rows = (int64_t)b.mb * b.bs;
        k_bsr_scalar_rp<<<(unsigned)div_up(rows + 1, 256), 256, 0, B->stream>>>(b.mb, b.bs, d.rp,
                                                                                srp);
        if (rows > 0)
          k_bsr_pack<<<(unsigned)div_up(rows, 256), 256, 0, B->stream>>>(
              b.mb, b.bs, d.layout == PERFLIBS_ROW_MAJOR, d.rp, d.col, d.val, srp, cv);
        d.rp = srp;
        srows += rows + 1;
        packed += b.nnzb * b.bs * b.bs;
      } else {
        const int64_t nnz = mats[i]->csr.nnz;
        if (nnz > 0)
          k_pack_cv<<<(unsigned)div_up(nnz, 256), 256, 0, B->stream>>>(nnz, d.col, d.val, cv);
        packed += nnz;
      }
      d.cv = cv;
    }
    PLS_LAUNCH_CHECK();
    // Band instances: CSR rows of consecutive columns get a copy of their
    // values alone, which their staged rows read.
    {
      DevBuf flags;
      flags.reserve(sizeof(int) * (size_t)count);
      std::vector<int> hf((size_t)count, 1);
      PLS_CUDA(cudaMemcpyAsync(flags.p, hf.data(), sizeof(int) * count, cudaMemcpyHostToDevice,
                               B->stream));
      for (int32_t i = 0; i < count; ++i) {
        const InstDesc &d = B->host[i];
        if (!d.is_bsr && d.m > 0)
          k_rows_consecutive<<<(unsigned)div_up(d.m, 256), 256, 0, B->stream>>>(
              d.m, d.rp, d.col, flags.as<int>() + i);
      }
      PLS_LAUNCH_CHECK();
      PLS_CUDA(cudaMemcpyAsync(hf.data(), flags.p, sizeof(int) * count, cudaMemcpyDeviceToHost,
                               B->stream));
      PLS_CUDA(cudaStreamSynchronize(B->stream));
      int64_t nb = 0;
      for (int32_t i = 0; i < count; ++i)
        if (!B->host[i].is_bsr && hf[i])
          nb += mats[i]->csr.nnz;
      B->band_vals.reserve(sizeof(float) * std::max<int64_t>(nb, 1));
      nb = 0;
      for (int32_t i = 0; i < count; ++i) {
        InstDesc &d = B->host[i];
        d.band_val = nullptr;
        if (d.is_bsr || !hf[i])
          continue;
        const int64_t nnz = mats[i]->csr.nnz;
        float *out = B->band_vals.as<float>() + nb;
        if (nnz > 0)
          PLS_CUDA(cudaMemcpyAsync(out, d.val, sizeof(float) * nnz, cudaMemcpyDeviceToDevice,
                                   B->stream));
        d.band_val = out;
        nb += nnz;
      }
      PLS_CUDA(cudaStreamSynchronize(B->stream));
    }
    B->inst.reserve(sizeof(InstDesc) * count);
    PLS_CUDA(cudaMemcpyAsync(B->inst.p, B->host.data(), sizeof(InstDesc) * count,
                             cudaMemcpyHostToDevice, B->stream));
    build_staged(B);
    B->counter.reserve(16);
    int sms = 0, per_sm = 0;
    PLS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B->device));
    PLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, B->off32 ? k_batch_spmm<true> : k_batch_spmm<false>, kBatchThreads,
        sizeof(float) * kStageFloats));
    B->grid = sms * std::max(per_sm, 1);
    build_items(B, 64);
    *out = owner.release();
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_batch_set_tile(perflibs_b200_batch_t B, int32_t rows) {
  if (!B || rows < 0)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] {
    if (rows > 0)
      build_items(B, rows);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_batch_tune(perflibs_b200_batch_t B, int32_t *best_tile,
                                           float *best_ms) {
  TraceRange trace("perflibs_b200_batch_tune");
  if (!B)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] {
    const EventPair ev;
    cudaEvent_t e0 = ev.e0, e1 = ev.e1;
    int32_t best = 64;
    bool best_staging = false;
    float bms = 1e30f;
    for (const bool staging : {true, false})
    for (int32_t tile : {8, 32, 128, 512, 2048}) {
      if (staging && B->n_sitems == 0)
        continue;
      B->staging = staging;
      build_items(B, tile);
      run(B, 1.f, 0.f);
      run(B, 1.f, 0.f);
      std::vector<float> t;
      for (int r = 0; r < 7; ++r) {
        PLS_CUDA(cudaEventRecord(e0, B->stream));
        run(B, 1.f, 0.f);
        PLS_CUDA(cudaEventRecord(e1, B->stream));
        PLS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        PLS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t.push_back(ms);
      }
      std::sort(t.begin(), t.end());
      if (t[t.size() / 2] < bms) {
        bms = t[t.size() / 2];
        best = tile;
        best_staging = staging;
      }
    }
    B->staging = best_staging;
    build_items(B, best);
    if (best_tile)
      *best_tile = best;
    if (best_ms)
      *best_ms = bms;
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_batch_set_staging(perflibs_b200_batch_t B, int32_t on) {
  if (!B)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] {
    B->staging = on != 0;
    build_items(B, B->tile);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_batch_stage_info(perflibs_b200_batch_t B, int64_t *staged_items,
                                                 int32_t *on) {
  if (!B)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (staged_items)
    *staged_items = B->n_sitems;
  if (on)
    *on = B->staging ? 1 : 0;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_batch_exec(perflibs_b200_batch_t B, float alpha, float beta) {
  if (!B)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] {
    run(B, alpha, beta);
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_batch_info(perflibs_b200_batch_t B, int64_t *n_items,
                                           int32_t *launches, int32_t *tile) {
  if (!B)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  if (n_items)
    *n_items = B->n_items;
  if (launches)
    *launches = B->n_items > 0 || (B->staging && B->n_sitems > 0) ? 1 : 0;
  if (tile)
    *tile = B->tile;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_batch_destroy(perflibs_b200_batch_t B) {
  delete B;
  return PERFLIBS_STATUS_SUCCESS;
}

}  // extern "C"
