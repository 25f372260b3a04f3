// Structure statistics of a CSR matrix, computed on the device: the input
// of the learned selector (the reference's only tuning statistic is mgmd,
// src/matrix_statistics.cpp:23-93, plus the SELL padding efficiency beta,
// src/sell_c_sigma.cpp:369-379; the rest are added here).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

namespace {

constexpr int kHistExact = 4096;  // exact bins for row lengths 0..4095
constexpr int kHistLog = 32;      // then one bin per power of two

struct RowStats {
  double s1, s2, s3, s4;  // sums of L, L^2, L^3, L^4
  double dist_sum;        // sum |i - j|
  double mgmd_sum;        // sum over rows of exp(mean log gap)
  unsigned long long near;  // nonzeros with |i - j| <= 32
  unsigned long long empty;
  int min_len, max_len;
  long long max_dist;
};

__device__ __forceinline__ void atomic_add_d(double *p, double v) { atomicAdd(p, v); }

__global__ void k_row_stats(int32_t m, const int32_t *__restrict__ rp,
                            const int32_t *__restrict__ col, RowStats *st,
                            unsigned int *hist) {
  double s1 = 0, s2 = 0, s3 = 0, s4 = 0, dsum = 0, mg = 0;
  unsigned long long near = 0, empty = 0;
  int mn = INT32_MAX, mx = 0;
  long long md = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = rp[i], e = rp[i + 1];
    const int32_t L = e - b;
    const double l = L;
    s1 += l;
    s2 += l * l;
    s3 += l * l * l;
    s4 += l * l * l * l;
    mn = min(mn, L);
    mx = max(mx, L);
    if (L == 0)
      empty++;
    const int bin = L < kHistExact ? L : kHistExact + min(kHistLog - 1, 31 - __clz(L) - 12);
    atomicAdd(hist + bin, 1u);
    double lg = 0;
    int32_t prev = 0;
    for (int32_t j = b; j < e; ++j) {
      const int32_t cj = col[j];
      const long long d = llabs((long long)cj - i);
      dsum += (double)d;
      md = max(md, d);
      if (d <= 32)
        near++;
      if (j > b)
        lg += log(fabs((double)cj - (double)prev));
      prev = cj;
    }
    // The reference divides the summed logs of the L-1 gaps by L
    // (src/matrix_statistics.cpp:70-79).
    if (L)
      mg += exp(lg / l);
  }
  atomic_add_d(&st->s1, s1);
  atomic_add_d(&st->s2, s2);
  atomic_add_d(&st->s3, s3);
  atomic_add_d(&st->s4, s4);
  atomic_add_d(&st->dist_sum, dsum);
  atomic_add_d(&st->mgmd_sum, mg);
  atomicAdd(&st->near, near);
  atomicAdd(&st->empty, empty);
  atomicMin(&st->min_len, mn);
  atomicMax(&st->max_len, mx);
  atomicMax(&st->max_dist, md);
}

double percentile(const std::vector<unsigned int> &h, int64_t m, double q) {
  const double target = q * (double)m;
  double acc = 0;
  for (int b = 0; b < (int)h.size(); ++b) {
    acc += h[b];
    if (acc >= target && h[b] > 0) {
      if (b < kHistExact)
        return b;
      return std::ldexp(1.0, b - kHistExact + 12);
    }
  }
  return 0;
}

}  // namespace

int64_t count_blocks(const CsrDev &c, int32_t m, int32_t n, int bs, cudaStream_t s);
int64_t sell_padded_size(const CsrDev &c, int32_t m, int C, int sigma, cudaStream_t s);

void compute_features(const Mat *A, float *out) {
  const CsrDev &c = A->csr;
  cudaStream_t s = stream_of(A);
  const int32_t m = A->m, n = A->n;
  const int64_t nnz = c.nnz;
  DevBuf stb, hb;
  stb.reserve(sizeof(RowStats));
  hb.reserve(sizeof(unsigned int) * (kHistExact + kHistLog));
  RowStats init{};
  init.min_len = INT32_MAX;
  PLS_CUDA(cudaMemcpyAsync(stb.p, &init, sizeof(RowStats), cudaMemcpyHostToDevice, s));
  PLS_CUDA(cudaMemsetAsync(hb.p, 0, sizeof(unsigned int) * (kHistExact + kHistLog), s));
  if (m > 0) {
    const unsigned blocks = (unsigned)std::min<int64_t>(div_up(m, 256), 148 * 16);
    k_row_stats<<<blocks, 256, 0, s>>>(m, c.row_ptr.as<int32_t>(), c.col.as<int32_t>(),
                                       stb.as<RowStats>(), hb.as<unsigned int>());
    PLS_LAUNCH_CHECK();
  }
  RowStats st;
  std::vector<unsigned int> hist(kHistExact + kHistLog);
  PLS_CUDA(cudaMemcpyAsync(&st, stb.p, sizeof(RowStats), cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaMemcpyAsync(hist.data(), hb.p, sizeof(unsigned int) * hist.size(),
                           cudaMemcpyDeviceToHost, s));
  PLS_CUDA(cudaStreamSynchronize(s));
  const double M = std::max(m, 1), N = std::max(n, 1);
  const double mean = st.s1 / M;
  const double var = std::max(0.0, st.s2 / M - mean * mean);
  const double sd = std::sqrt(var);
  // Central moments from raw moments.
  const double m3 = st.s3 / M - 3 * mean * st.s2 / M + 2 * mean * mean * mean;
  const double m4 = st.s4 / M - 4 * mean * st.s3 / M + 6 * mean * mean * st.s2 / M -
                    3 * mean * mean * mean * mean;
  const double skew = var > 0 ? m3 / (var * sd) : 0.0;
  const double kurt = var > 0 ? m4 / (var * var) - 3.0 : 0.0;
  const int mn = m > 0 ? st.min_len : 0;
  double f[PERFLIBS_B200_NFEATURES];
  f[0] = std::log2(m + 1.0);
  f[1] = std::log2(n + 1.0);
  f[2] = std::log2(nnz + 1.0);
  f[3] = mean;
  f[4] = sd;
  f[5] = skew;
  f[6] = kurt;
  f[7] = std::log2(1.0 + mn);
  f[8] = std::log2(1.0 + st.max_len);
  f[9] = st.empty / M;
  f[10] = std::log2(1.0 + percentile(hist, m, 0.50));
  f[11] = std::log2(1.0 + percentile(hist, m, 0.90));
  f[12] = std::log2(1.0 + percentile(hist, m, 0.99));
  f[13] = mean > 0 ? std::log2(std::max(1.0, st.max_len / mean)) : 0.0;
  f[14] = nnz > 0 ? st.dist_sum / nnz / N : 0.0;
  f[15] = st.max_dist / N;
  f[16] = nnz > 0 ? (double)st.near / nnz : 0.0;
  int k = 17;
  for (int bs : {2, 4, 8}) {
    const int64_t nb = nnz > 0 ? count_blocks(c, m, n, bs, s) : 0;
    f[k++] = nb > 0 ? (double)nnz / ((double)bs * bs * nb) : 0.0;
  }
  const int sells[3][2] = {{8, 0}, {32, 0}, {32, 1024}};
  for (auto &cs : sells) {
    const int64_t sz = nnz > 0 ? sell_padded_size(c, m, cs[0], cs[1], s) : 0;
    f[k++] = sz > 0 ? (double)nnz / sz : 1.0;
  }
  f[23] = std::log2(1.0 + st.mgmd_sum / M);
  for (int i = 0; i < PERFLIBS_B200_NFEATURES; ++i)
    out[i] = (float)f[i];
}

}  // namespace pls
