// Autotune cache: checkpoint / resume for the exhaustive tuner.
//
// Every exhaustive tune is recorded under a key made of the GPU model, the
// matrix's dimensions and nonzero count, the API and storage value types,
// and a 64-bit hash of its sparsity structure (row pointers and column
// indices; values do not change a kernel's speed). A later exhaustive
// optimize with the same key takes the recorded configuration and timing
// table without timing anything. The cache lives in the process and can be
// written to and merged from a text file, so a tuning campaign (or the
// selector's training corpus) resumes where it stopped.
//
// The structure hash is a sum over all row pointers and column indices of
// splitmix64(position, value) (Vigna's splitmix64 finaliser as the mixing
// function). A sum is independent of the order the device adds the terms
// in, so the hash is the same on every run.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Positions [0, m] are row pointers, [m + 1, m + 1 + nnz) column indices.
__global__ void k_structure_hash(int32_t m, int64_t nnz, const int32_t *__restrict__ rp,
                                 const int32_t *__restrict__ col,
                                 unsigned long long *__restrict__ out) {
  const int64_t total = (int64_t)m + 1 + nnz;
  uint64_t h = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(i <= m ? __ldg(rp + i) : __ldg(col + (i - m - 1)));
    h += splitmix64(((uint64_t)i << 32) ^ v);
  }
  for (int o = 16; o > 0; o >>= 1)
    h += __shfl_xor_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0)
    atomicAdd(out, (unsigned long long)h);
}

uint64_t structure_hash(const CsrDev &c, int32_t m, cudaStream_t s) {
  DevBuf acc;
  acc.reserve(8);
  PLS_CUDA(cudaMemsetAsync(acc.p, 0, 8, s));
  const int64_t total = (int64_t)m + 1 + c.nnz;
  const unsigned blocks = (unsigned)std::min<int64_t>(div_up(total, 256), 148 * 16);
  k_structure_hash<<<blocks, 256, 0, s>>>(m, c.nnz, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(),
                                          acc.as<unsigned long long>());
  PLS_LAUNCH_CHECK();
  unsigned long long h = 0;
  PLS_CUDA(cudaMemcpyAsync(&h, acc.p, 8, cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  return h;
}

std::string device_signature(int dev) {
  int major = 0, minor = 0, sms = 0;
  PLS_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  PLS_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
  PLS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return "cc" + std::to_string(major) + std::to_string(minor) + "-sm" + std::to_string(sms);
}

struct Entry {
  SpmvConfig best;
  std::vector<TuneEntry> table;
};

std::mutex g_mu;
std::map<TuneKey, Entry> g_cache;

constexpr const char *kMagic = "plsparse_b200_tune_cache";
constexpr int kVersion = 1;

TuneKey key_of(const Mat *A) {
  TuneKey k;
  k.dev = device_signature(A->device);
  k.m = A->m;
  k.n = A->n;
  k.nnz = A->csr.nnz;
  k.hash = structure_hash(A->csr, A->m, stream_of(A));
  k.dt = (int)A->dt;
  k.vt = (int)A->csr.evt();
  return k;
}

bool valid_config(const SpmvConfig &c) {
  switch (c.kind) {
  case Kind::CSR_VECTOR:
    return c.tpr >= 0 && c.tpr <= 32;
  case Kind::CSR_SPLIT:
    return c.tpr > 0;
  case Kind::SELL:
    return (c.C == 8 || c.C == 16 || c.C == 32) && c.sigma >= 0 && c.sigma <= 16384 &&
           (c.sigma == 0 || c.sigma % c.C == 0);
  }
  return false;
}

}  // namespace

bool tune_cache_find(const Mat *A, SpmvConfig &best, std::vector<TuneEntry> &table,
                     TuneKey &key) {
  key = key_of(A);
  std::lock_guard<std::mutex> g(g_mu);
  const auto it = g_cache.find(key);
  if (it == g_cache.end())
    return false;
  best = it->second.best;
  table = it->second.table;
  return true;
}

void tune_cache_put(const TuneKey &key, const SpmvConfig &best,
                    const std::vector<TuneEntry> &table) {
  std::lock_guard<std::mutex> g(g_mu);
  Entry &e = g_cache[key];
  e.best = best;
  e.table = table;
}

}  // namespace pls

using namespace pls;

namespace {

// Closes the file if a write or read throws (host allocation failure).
struct CloseOnThrow {
  FILE *f;
  ~CloseOnThrow() {
    if (f)
      std::fclose(f);
  }
};

perflibs_status_t save_cache(const char *path) {
  std::lock_guard<std::mutex> g(g_mu);
  FILE *f = std::fopen(path, "w");
  if (!f)
    return PERFLIBS_STATUS_EXECUTION_FAILURE;
  CloseOnThrow closer{f};
  bool ok = std::fprintf(f, "%s %d %zu\n", kMagic, kVersion, g_cache.size()) > 0;
  for (const auto &kv : g_cache) {
    const TuneKey &k = kv.first;
    const Entry &e = kv.second;
    ok = ok && std::fprintf(f, "%s %d %d %" PRId64 " %016" PRIx64 " %d %d %d %d %d %d %zu\n",
                            k.dev.c_str(), k.m, k.n, k.nnz, k.hash, k.dt, k.vt,
                            (int)e.best.kind, e.best.C, e.best.sigma, e.best.tpr,
                            e.table.size()) > 0;
    for (const TuneEntry &t : e.table)
      ok = ok && std::fprintf(f, "%d %d %d %d %.9g %.9g\n", (int)t.cfg.kind, t.cfg.C,
                              t.cfg.sigma, t.cfg.tpr, t.ms, t.beta) > 0;
  }
  closer.f = nullptr;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PERFLIBS_STATUS_SUCCESS : PERFLIBS_STATUS_EXECUTION_FAILURE;
}

perflibs_status_t load_cache(const char *path) {
  FILE *f = std::fopen(path, "r");
  if (!f)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  CloseOnThrow closer{f};
  std::map<TuneKey, Entry> read;
  char magic[64] = {0};
  int version = 0;
  size_t count = 0;
  bool ok = std::fscanf(f, "%63s %d %zu", magic, &version, &count) == 3 &&
            std::strcmp(magic, kMagic) == 0 && version == kVersion;
  for (size_t i = 0; ok && i < count; ++i) {
    char dev[64] = {0};
    TuneKey k;
    Entry e;
    int kind = 0;
    size_t rows = 0;
    ok = std::fscanf(f, "%63s %d %d %" SCNd64 " %" SCNx64 " %d %d %d %d %d %d %zu", dev, &k.m,
                     &k.n, &k.nnz, &k.hash, &k.dt, &k.vt, &kind, &e.best.C, &e.best.sigma,
                     &e.best.tpr, &rows) == 12;
    k.dev = dev;
    e.best.kind = (Kind)kind;
    ok = ok && kind >= 0 && kind <= 2 && valid_config(e.best) && k.m >= 0 && k.n >= 0 &&
         k.nnz >= 0 && rows <= 4096;
    for (size_t r = 0; ok && r < rows; ++r) {
      TuneEntry t;
      int tk = 0;
      ok = std::fscanf(f, "%d %d %d %d %lf %lf", &tk, &t.cfg.C, &t.cfg.sigma, &t.cfg.tpr, &t.ms,
                       &t.beta) == 6 &&
           tk >= 0 && tk <= 2;
      t.cfg.kind = (Kind)tk;
      ok = ok && valid_config(t.cfg);
      e.table.push_back(t);
    }
    if (ok)
      read[k] = std::move(e);
  }
  closer.f = nullptr;
  std::fclose(f);
  if (!ok)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  std::lock_guard<std::mutex> g(g_mu);
  for (auto &kv : read)
    g_cache[kv.first] = std::move(kv.second);
  return PERFLIBS_STATUS_SUCCESS;
}

}  // namespace

extern "C" {

perflibs_status_t perflibs_b200_tune_cache_save(const char *path) {
  if (!path)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] { return save_cache(path); });
}

// Merges the file's entries into the cache (an entry replaces one with the
// same key). A file that is not a cache of this version, or is cut short or
// malformed anywhere, changes nothing and is an input error.
perflibs_status_t perflibs_b200_tune_cache_load(const char *path) {
  if (!path)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&] { return load_cache(path); });
}

perflibs_status_t perflibs_b200_tune_cache_clear(void) {
  std::lock_guard<std::mutex> g(g_mu);
  g_cache.clear();
  return PERFLIBS_STATUS_SUCCESS;
}

int64_t perflibs_b200_tune_cache_size(void) {
  std::lock_guard<std::mutex> g(g_mu);
  return (int64_t)g_cache.size();
}

}  // extern "C"
