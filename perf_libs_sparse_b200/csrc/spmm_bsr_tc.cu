// BSR x dense SpMM on the fifth-generation tensor cores (tcgen05.mma) for
// block size 8, with the values in BF16 storage, FP32 B and C and FP32
// accumulation.
//
// Formulation. For block row i with blocks (i, j_p), C_i^T = sum_p B_{j_p}^T
// A_{i,j_p}^T, where C_i is the block row's 8 rows of C and B_j the 8 rows
// of B for block column j. One work item is (block row i, a chunk of 128
// columns of C); its accumulator D (128 x 16 FP32, in tensor memory) holds
// C_i^T for the chunk: TMEM lane = column of C, TMEM column = row of the
// block row (columns 8..15 stay zero). Each block is one MMA of kind::tf32,
// M = 128, N = 16, K = 8, both operands K-major without swizzle (8-row x
// 16-byte core matrices, K chunks 128 bytes apart, row groups 256 bytes
// apart):
//   * operand A (M x K): rows 8j .. 8j + 7 of B, columns k0 .. k0 + 127,
//     transposed into the core matrices by the CTA's threads, one column of
//     C per thread (columns past k are zeros);
//   * operand B (K x N): A_{i,j}^T as FP32 (exact for BF16 values), from a
//     K-major copy of the values built at creation; rows N = 8..15 are zero,
//     written once.
// TF32 rounds B to 10 mantissa bits (relative 2^-11); with BF16 values
// (relative 2^-9) the results stay within the BF16 storage mode's 1e-2 of
// the FP64 oracle. FP64 and FP32 storage keep the FMA kernel.
//
// Pipeline (128 threads per CTA, persistent over the items): the threads
// hold the next block's B values in registers (loaded while the previous
// block's MMA runs), write them into a ring of kTcStages shared-memory
// stages, and thread 0 issues the block's MMA; tcgen05.commit frees the
// block's stage (done_bar) and, after an item's last block, marks its D
// buffer complete (d_bar). D is double-buffered in TMEM, so item q's MMAs
// run while the four warps read item q - 1's D (tcgen05.ld, each warp its 32
// lanes) and write C. Every wait has an iteration limit; a wait that runs
// out sets the mapped error flag, the CTA stops, waits (bounded) for its
// MMAs in flight and frees its tensor memory.
#include <algorithm>

#include "common.cuh"
#include "pls_internal.hpp"
#include "tma.cuh"

namespace pls {

namespace {

constexpr int kTcStages = 4;
constexpr int kTcThreads = 128;               // one column of C per thread
constexpr int kTcM = 128;                     // columns of C per item (MMA M)
constexpr int kTcN = 16;                      // MMA N: the block row's 8 rows + 8 zero
constexpr int kTcK = 8;                       // MMA K (kind::tf32): one block
constexpr int kTcAopBytes = kTcM * kTcK * 4;  // 4 KB
constexpr int kTcBopBytes = kTcN * kTcK * 4;  // 512 B, the first 256 B the block's values
constexpr int kTcStageBytes = kTcAopBytes + kTcBopBytes;
constexpr int kTcTmemCols = 32;               // two D buffers of kTcN columns
constexpr int kTcSmem = kTcStages * kTcStageBytes + 128;  // + alignment room

struct TcArgs {
  int32_t mb;       // block rows
  int32_t k, nkc;   // columns of C; chunks of kTcM columns
  int64_t n_items;  // mb * nkc, item = i * nkc + chunk
  int32_t wait_limit;
  // Failure-path tests only: the first wait on a D buffer goes to a barrier
  // that nothing arrives on, so it runs out.
  int32_t stall;
};

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, int cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   tma::smem_addr(dst)),
               "r"(cols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, int cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
// D (TMEM) = A x B (+ D when accumulate), kind::tf32.
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   tma::smem_addr(bar))
               : "memory");
}
// 8 consecutive 32-bit TMEM columns of the warp's 32 lanes (lane = thread).
// The load fills its registers asynchronously: the wait names them as
// read-write operands, so that no use of them is scheduled before it.
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(addr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i)
    v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all in 16-byte units), version 1, layout type (0 no swizzle, 2
// 128-byte swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)layout << 61;
  return d;
}

// Instruction descriptor of the MMA: FP32 accumulator, TF32 operands, both
// K-major, N = kTcN, M = kTcM.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (0u << 15) | (0u << 16) |
                              ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
// Byte offset of element (row r, K index kk) in a K-major operand of 8-row x
// 16-byte core matrices: K chunks of 4 elements 128 bytes apart, groups of 8
// rows 256 bytes apart (the descriptors' leading / stride byte offsets).
__host__ __device__ constexpr int kmajor_off(int r, int kk) {
  return (r / 8) * 256 + (kk / 4) * 128 + (r % 8) * 16 + (kk % 4) * 4;
}

// The CTA's items in order (blockIdx.x, + gridDim.x, ...), skipping block rows
// without blocks, one block at a time.
struct TcCursor {
  int64_t item;
  int32_t p, p1, i, chunk;
  bool valid;
};

__device__ __forceinline__ void tc_seek(TcCursor &c, int64_t item, const TcArgs &a,
                                        const int32_t *__restrict__ rp) {
  for (; item < a.n_items; item += gridDim.x) {
    const int32_t i = (int32_t)(item / a.nkc);
    const int32_t p0 = __ldg(rp + i), p1 = __ldg(rp + i + 1);
    if (p0 < p1) {
      c = TcCursor{item, p0, p1, i, (int32_t)(item % a.nkc), true};
      return;
    }
  }
  c.valid = false;
}

__global__ void __launch_bounds__(kTcThreads)
    k_spmm_bsr_tc(const TcArgs a, const int32_t *__restrict__ rp, const int32_t *__restrict__ col,
                  const float *__restrict__ tcv, const float *__restrict__ B, int64_t ldb,
                  float *__restrict__ C, int64_t ldc, float alpha, float beta, int beta_nz,
                  int *__restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t done_bar[kTcStages], d_bar[2], never_bar;
  __shared__ uint32_t tmem_s;
  unsigned char *smem = smem_raw + ((128u - (tma::smem_addr(smem_raw) & 127u)) & 127u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tmem_alloc(&tmem_s, kTcTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s)
      tma::bar_init(&done_bar[s]);
    tma::bar_init(&d_bar[0]);
    tma::bar_init(&d_bar[1]);
    tma::bar_init(&never_bar);
    tma::bar_init_fence();
  }
  // Rows N = 8 .. 15 of every stage's operand B are zero.
  for (int e = tid; e < kTcStages * 64; e += kTcThreads)
    reinterpret_cast<float *>(smem + (e / 64) * kTcStageBytes + kTcAopBytes + 256)[e % 64] = 0.f;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_s;

  // The thread's column of B for the next block (and, threads 0..15, four of
  // the block's operand-B values), loaded one block ahead.
  TcCursor cur;
  tc_seek(cur, blockIdx.x, a, rp);
  float bn[8], vn[4];
  auto load_next = [&]() {
    const int32_t cm = cur.chunk * kTcM + tid;
    const int64_t r0 = (int64_t)__ldg(col + cur.p) * 8;
#pragma unroll
    for (int r = 0; r < 8; ++r)
      bn[r] = cm < a.k ? __ldg(B + (r0 + r) * ldb + cm) : 0.f;
    if (tid < 16) {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(tcv + (int64_t)cur.p * 64) + tid);
      vn[0] = t.x, vn[1] = t.y, vn[2] = t.z, vn[3] = t.w;
    }
  };
  if (cur.valid)
    load_next();

  uint32_t f = 0;              // blocks staged so far
  uint32_t d_waits[2] = {0, 0};  // waits on d_bar[b] so far (their parities)
  bool ok = true;
  int64_t prev_item = -1;
  bool prev_full = false;
  for (int64_t item = blockIdx.x;; item += gridDim.x) {
    const bool have = item < a.n_items;
    const int qb = (int)(((item - blockIdx.x) / gridDim.x) & 1);  // D buffer of this item
    bool full = false;
    // 1. This item's blocks: stage, then one MMA each into D buffer qb.
    if (have && cur.valid && cur.item == item) {
      full = true;
      const int32_t p0 = cur.p;
      for (bool more = true; more && ok;) {
        const int32_t p = cur.p;
        const bool last = p + 1 == cur.p1;
        const uint32_t s = f % kTcStages;
        if (f >= kTcStages)  // the stage's previous MMA must be done with it
          ok = tma::bar_wait_bounded(&done_bar[s], ((f / kTcStages) - 1) & 1u, a.wait_limit);
        unsigned char *st = smem + s * kTcStageBytes;
        *reinterpret_cast<float4 *>(st + kmajor_off(tid, 0)) = make_float4(bn[0], bn[1], bn[2], bn[3]);
        *reinterpret_cast<float4 *>(st + kmajor_off(tid, 4)) = make_float4(bn[4], bn[5], bn[6], bn[7]);
        if (tid < 16)  // values (kk, nn) at kmajor_off(nn, kk): 16 bytes per thread
          *reinterpret_cast<float4 *>(st + kTcAopBytes + tid * 16) = make_float4(vn[0], vn[1], vn[2], vn[3]);
        if (last)
          tc_seek(cur, item + gridDim.x, a, rp);
        else
          ++cur.p;
        more = !last;
        if (cur.valid)
          load_next();  // in flight during the MMA
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        ok = __syncthreads_and(ok) != 0;
        if (ok && tid == 0) {
          tc_fence_after();
          const uint32_t sa = tma::smem_addr(st);
          mma_tf32(tmem + (uint32_t)(qb * kTcN), smem_desc(sa, 128, 256, 0),
                   smem_desc(sa + kTcAopBytes, 128, 256, 0), kTcIdesc, p > p0 ? 1u : 0u);
          mma_commit(&done_bar[s]);
          if (last)
            mma_commit(&d_bar[qb]);
        }
        ++f;
      }
    }
    // 2. The previous item's epilogue from its D buffer.
    if (ok && prev_item >= 0) {
      const int pb = qb ^ 1;
      const int32_t i = (int32_t)(prev_item / a.nkc);
      const int32_t col0 = (int32_t)(prev_item % a.nkc) * kTcM + 32 * warp + lane;
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (prev_full) {
        const bool stall = a.stall && d_waits[0] + d_waits[1] == 0;
        bool landed = tma::bar_wait_bounded(stall ? &never_bar : &d_bar[pb],
                                            stall ? 0u : d_waits[pb] & 1u, a.wait_limit);
        ++d_waits[pb];
        landed = __all_sync(0xffffffffu, landed);
        if (landed) {
          tc_fence_after();
          tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(pb * kTcN), v);
        }
        ok = landed;
      }
      if (ok && col0 < a.k) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          float *cp = C + ((int64_t)i * 8 + r) * ldc + col0;
          *cp = beta_nz ? alpha * v[r] + beta * *cp : alpha * v[r];
        }
      }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok) != 0;
    if (!ok || !have)
      break;
    prev_item = item;
    prev_full = full;
  }
  if (!ok && tid == 0) {
    *(volatile int *)err = 1;
    __threadfence_system();
  }
  // MMAs still in flight after an expired wait: wait for them (bounded)
  // before the shared and tensor memory go away.
  if (tid == 0)
    for (uint32_t g = (f > kTcStages ? f - kTcStages : 0); g < f; ++g)
      tma::bar_wait_bounded(&done_bar[g % kTcStages], (g / kTcStages) & 1u, a.wait_limit);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    tmem_dealloc(tmem, kTcTmemCols);
}

// K-major FP32 copy of the BSR values for operand B: block p's element
// (row nn, column kk), operand element (K = kk, N = nn), at float
// p * 64 + kmajor_off(nn, kk) / 4.
template <class V>
__global__ void k_bsr_tc_vals(int64_t nnzb, int layout, const V *__restrict__ vals,
                              float *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnzb * 64)
    return;
  const int64_t p = e / 64;
  const int nn = (int)(e % 64) / 8, kk = (int)(e % 8);
  const V v = vals[p * 64 + (layout == PERFLIBS_ROW_MAJOR ? nn * 8 + kk : kk * 8 + nn)];
  out[p * 64 + kmajor_off(nn, kk) / 4] = to_acc<float>(v);
}

}  // namespace

bool spmm_bsr_tc(BsrDev &b, const float *B, int64_t ldb, float *C, int64_t ldc, int k,
                 float alpha, float beta, cudaStream_t s, bool launch) {
  if (b.bs != 8 || b.mb <= 0 || b.nnzb <= 0 || k <= 0 || b.evt() != Vt::BF16)
    return false;
  if (ldb < k)
    return false;
  if (b.tc_err.host && *(volatile int *)b.tc_err.host) {
    *(volatile int *)b.tc_err.host = 0;
    throw Error(PERFLIBS_STATUS_EXECUTION_FAILURE,
                "tensor-core BSR SpMM: a copy or MMA did not complete (reported by an earlier call)");
  }
  if (!launch)
    return true;
  // The operand-B copy of the values, rebuilt when the values change.
  if (b.tc_vals_src != b.ev() || b.tc_vals_version != b.vals_version) {
    b.tc_vals.reserve(sizeof(float) * (size_t)b.nnzb * 64);
    k_bsr_tc_vals<__nv_bfloat16><<<(unsigned)div_up(b.nnzb * 64, 256), 256, 0, s>>>(
        b.nnzb, b.layout, static_cast<const __nv_bfloat16 *>(b.ev()), b.tc_vals.as<float>());
    PLS_LAUNCH_CHECK();
    b.tc_vals_src = b.ev();
    b.tc_vals_version = b.vals_version;
  }
  if (!b.tc_err.host)
    b.tc_err.alloc();
  TcArgs a{};
  a.mb = b.mb;
  a.k = k;
  a.nkc = (int32_t)div_up(k, kTcM);
  a.n_items = (int64_t)a.mb * a.nkc;
  a.wait_limit = g_stage_wait_limit.load();
  a.stall = g_stage_shortfall.load() > 0 ? 1 : 0;
  int dev = 0, sms = 0, per_sm = 0;
  PLS_CUDA(cudaGetDevice(&dev));
  PLS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PLS_CUDA(cudaFuncSetAttribute(k_spmm_bsr_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kTcSmem));
  PLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmm_bsr_tc, kTcThreads,
                                                         kTcSmem));
  // At most 8 CTAs per SM: 8 x 32 of the SM's 512 tensor-memory columns.
  per_sm = std::min(std::max(per_sm, 1), 8);
  const unsigned grid = (unsigned)std::min<int64_t>(a.n_items, (int64_t)sms * per_sm);
  k_spmm_bsr_tc<<<grid, kTcThreads, kTcSmem, s>>>(a, b.row_ptr.as<int32_t>(), b.col.as<int32_t>(),
                                                  b.tc_vals.as<float>(), B, ldb, C, ldc, alpha,
                                                  beta, beta != 0.f, b.tc_err.dev);
  PLS_LAUNCH_CHECK();
  return true;
}

}  // namespace pls
