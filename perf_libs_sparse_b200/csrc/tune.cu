// SpMV kernel selection: the default heuristic, configuration application,
// and the exhaustive GPU autotuner.
//
// The reference's optimize phase ("audition", src/matvec.cpp:189-518) tries
// SELL-C-sigma candidates in a fixed preference order, accepts the first one
// whose padding efficiency beta clears 0.96, and times it against CSR with a
// Welch t-test early exit. Here every candidate is built on the device and
// timed with CUDA events (median of several launches, L2 flushed between
// launches when the matrix would otherwise sit in L2), and the fastest wins.
// The full timing table is kept: it is both the fallback of the learned
// selector and the ground truth its regret is measured against.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

template <class X> __global__ void k_fill(int64_t n, X v, X *p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    p[i] = v;
}

struct DeviceScratch {
  DevBuf flush;  // written between timed launches to evict L2
  size_t l2 = 0;
};

DeviceScratch &scratch(int dev) {
  static std::mutex mu;
  static DeviceScratch per[64];
  std::lock_guard<std::mutex> g(mu);
  DeviceScratch &d = per[dev & 63];
  if (!d.flush.p) {
    int l2 = 0;
    PLS_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    d.l2 = (size_t)l2;
    d.flush.reserve(std::max<size_t>(2 * d.l2, 64u << 20));
  }
  return d;
}

int pow2_floor(double v) {
  int p = 1;
  while (p * 2 <= v && p < 32)
    p *= 2;
  return p;
}

int64_t matrix_bytes(const Mat *A) {
  return A->csr.nnz * (int64_t)(vt_size(A->csr.evt()) + 4) + 4LL * (A->m + 1);
}

}  // namespace

SpmvConfig default_config(const Mat *A) {
  SpmvConfig c;
  c.kind = Kind::CSR_VECTOR;
  const double mean = A->m > 0 ? (double)A->csr.nnz / A->m : 1.0;
  c.tpr = pow2_floor(mean);
  return c;
}

// Make cfg the active SpMV configuration: build the SELL layout or the
// long-row list it needs.
void apply_config(Mat *A, const SpmvConfig &cfg) {
  cudaStream_t s = stream_of(A);
  SpmvConfig c = cfg;
  if (c.kind == Kind::CSR_VECTOR && c.tpr <= 0)
    c.tpr = default_config(A).tpr;
  if (c.kind == Kind::SELL) {
    const bool have = A->sell.nC > 0 && A->sell.C == c.C && A->sell.sigma == c.sigma &&
                      A->sell.vt == A->csr.evt();
    if (!have) {
      A->sell = SellDev{};
      build_sell(A->csr, A->m, c.C, c.sigma, A->sell, s);
    }
    // Spread chunks much wider than the typical one over several lane
    // groups (power-law row lengths).
    const double mean_w = A->sell.nC ? (double)A->sell.size / (A->sell.nC * (double)c.C) : 0;
    const int slice = std::max(64, (int)std::ceil(mean_w * 8));
    if (A->sell.max_width > 4 * slice)
      sell_build_work_list(A->sell, slice, s);
    else
      sell_build_work_list(A->sell, 0, s);
    A->fmt = Fmt::SELL;
  } else {
    if (c.kind == Kind::CSR_SPLIT && A->csr.long_threshold != c.tpr)
      csr_build_long_rows(A->csr, A->m, c.tpr > 0 ? c.tpr : 1024, s);
    if (A->fmt == Fmt::SELL)
      A->fmt = Fmt::CSR;
  }
  A->cfg = c;
}

double time_config(Mat *A, const SpmvConfig &cfg, int reps) {
  apply_config(A, cfg);
  cudaStream_t s = stream_of(A);
  const int64_t xl = A->n, yl = A->m;
  DeviceScratch &sc = scratch(A->device);
  const bool flush = matrix_bytes(A) < (int64_t)(3 * sc.l2);
  const EventPair ev;
  cudaEvent_t e0 = ev.e0, e1 = ev.e1;
  std::vector<float> t;
  auto run = [&]() {
    if (A->dt == Dt::F64) {
      run_spmv<double>(A, PERFLIBS_SPARSE_OPERATION_NOTRANS, A->xbuf.as<double>(),
                       A->ybuf.as<double>(), 1.0, 0.0, s);
    } else {
      run_spmv<float>(A, PERFLIBS_SPARSE_OPERATION_NOTRANS, A->xbuf.as<float>(),
                      A->ybuf.as<float>(), 1.0f, 0.0f, s);
    }
  };
  const size_t xs = A->dt == Dt::F64 ? 8 : 4;
  A->xbuf.reserve(xs * std::max<int64_t>(xl, 1));
  A->ybuf.reserve(xs * std::max<int64_t>(yl, 1));
  if (A->dt == Dt::F64)
    k_fill<double><<<(unsigned)div_up(std::max<int64_t>(xl, 1), 256), 256, 0, s>>>(
        xl, 1.0, A->xbuf.as<double>());
  else
    k_fill<float><<<(unsigned)div_up(std::max<int64_t>(xl, 1), 256), 256, 0, s>>>(
        xl, 1.0f, A->xbuf.as<float>());
  run();
  run();
  for (int r = 0; r < reps; ++r) {
    if (flush)
      PLS_CUDA(cudaMemsetAsync(sc.flush.p, r & 0xff, sc.flush.bytes, s));
    PLS_CUDA(cudaEventRecord(e0, s));
    run();
    PLS_CUDA(cudaEventRecord(e1, s));
    PLS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    PLS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  return t.empty() ? 0.0 : t[t.size() / 2];
}

// The candidate list (also the class list of the learned selector). Sorting
// windows go up to 8192 rows; 0 is the unsorted layout.
std::vector<SpmvConfig> tune_candidates(const Mat *A) {
  std::vector<SpmvConfig> out;
  for (int tpr : {1, 2, 4, 8, 16, 32}) {
    SpmvConfig c;
    c.kind = Kind::CSR_VECTOR;
    c.tpr = tpr;
    out.push_back(c);
  }
  {
    SpmvConfig c;
    c.kind = Kind::CSR_SPLIT;
    c.tpr = 1024;
    out.push_back(c);
  }
  for (int C : {8, 16, 32})
    for (int sigma : {0, 32, 256, 1024, 4096, 8192}) {
      if (sigma != 0 && (sigma < C || sigma % C != 0))
        continue;
      SpmvConfig c;
      c.kind = Kind::SELL;
      c.C = C;
      c.sigma = sigma;
      out.push_back(c);
    }
  return out;
}

void tune_spmv(Mat *A) {
  A->tune_table.clear();
  A->tune_source = TuneSource::NONE;
  if (A->m == 0 || A->csr.nnz == 0) {
    apply_config(A, default_config(A));
    return;
  }
  TuneKey key;
  SpmvConfig cached;
  if (tune_cache_find(A, cached, A->tune_table, key)) {
    apply_config(A, cached);
    A->tune_source = TuneSource::CACHE;
    return;
  }
  const auto cands = tune_candidates(A);
  const int64_t bytes = matrix_bytes(A);
  // About 2 ms of measured work per candidate, 3..25 launches.
  const double est_ms = bytes / 6.0e9;
  const int reps = (int)std::min(25.0, std::max(3.0, 2.0 / std::max(est_ms, 1e-3)));
  for (const auto &c : cands) {
    TuneEntry te;
    te.cfg = c;
    te.ms = time_config(A, c, reps);
    if (c.kind == Kind::SELL && A->sell.size > 0)
      te.beta = (double)A->csr.nnz / (double)A->sell.size;
    A->tune_table.push_back(te);
    if (c.kind == Kind::SELL)
      A->sell = SellDev{};  // one layout on the device at a time
  }
  // Second pass: the finalists (within kRefineBand of the fastest, at most
  // kFinalists) are timed again in interleaved rounds (A B C, A B C, ...), so
  // that a drift of clocks or power state during the first pass cannot decide
  // between near-equal layouts; each keeps the median of its timings. On the
  // C2 matrix C = 16 and C = 32 are within 5%, and a single pass picked the
  // slower one in some runs.
  constexpr double kRefineBand = 0.05;
  constexpr size_t kFinalists = 4;
  constexpr int kRefineRounds = 3;
  std::vector<size_t> order(cands.size());
  for (size_t i = 0; i < order.size(); ++i)
    order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return A->tune_table[a].ms < A->tune_table[b].ms;
  });
  std::vector<size_t> fin;
  for (size_t i : order)
    if (fin.size() < kFinalists &&
        A->tune_table[i].ms <= A->tune_table[order[0]].ms * (1.0 + kRefineBand))
      fin.push_back(i);
  if (fin.size() > 1) {
    std::vector<std::vector<double>> runs(fin.size());
    for (size_t f = 0; f < fin.size(); ++f)
      runs[f].push_back(A->tune_table[fin[f]].ms);
    for (int round = 0; round < kRefineRounds; ++round)
      for (size_t f = 0; f < fin.size(); ++f)
        runs[f].push_back(time_config(A, cands[fin[f]], reps));
    for (size_t f = 0; f < fin.size(); ++f) {
      std::sort(runs[f].begin(), runs[f].end());
      A->tune_table[fin[f]].ms = runs[f][runs[f].size() / 2];
    }
  }
  size_t best = 0;
  for (size_t i = 1; i < A->tune_table.size(); ++i)
    if (A->tune_table[i].ms < A->tune_table[best].ms)
      best = i;
  const SpmvConfig best_cfg = cands[best];
  apply_config(A, best_cfg);
  A->tune_source = TuneSource::TIMED;
  tune_cache_put(key, best_cfg, A->tune_table);
}

}  // namespace pls
