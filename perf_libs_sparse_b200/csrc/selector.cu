// Learned format / parameter selector: an MLP NF -> 64 -> 64 -> K (ReLU,
// softmax), FP32, trained with soft-target cross-entropy and Adam, entirely
// by the kernels in this file. One training step (gather a shuffled
// mini-batch, normalise, forward, loss, backward, Adam) is captured once as
// a CUDA graph and replayed; the step counter and batch offset live in
// device memory so replays need no host work.
//
// The network is tiny (about 7k parameters), so the kernels are plain
// thread-per-output dot products: the work is launch-bound, which is what
// the graph replay addresses.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "pls_internal.hpp"

namespace pls {

constexpr int NF = PERFLIBS_B200_NFEATURES;
constexpr int H = 64;

namespace {

__global__ void k_gather_batch(int B, int K, const int32_t *__restrict__ perm,
                               const int32_t *__restrict__ off, const float *__restrict__ X,
                               const float *__restrict__ T, float *__restrict__ xb,
                               float *__restrict__ tb) {
  const int i = blockIdx.x;
  const int src = perm[*off + i];
  for (int f = threadIdx.x; f < NF; f += blockDim.x)
    xb[i * NF + f] = X[(int64_t)src * NF + f];
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    tb[i * K + k] = T[(int64_t)src * K + k];
}

__global__ void k_normalize(int B, const float *__restrict__ x, const float *__restrict__ mean,
                            const float *__restrict__ inv_std, float *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < B * NF) {
    const int f = t % NF;
    out[t] = (x[t] - mean[f]) * inv_std[f];
  }
}

// Y[b, o] = act(sum_i X[b, i] W[o, i] + bias[o])
__global__ void k_linear_fwd(int B, int in, int out, const float *__restrict__ X,
                             const float *__restrict__ W, const float *__restrict__ bias,
                             float *__restrict__ Y, int relu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * out)
    return;
  const int b = t / out, o = t % out;
  float s = bias[o];
  for (int i = 0; i < in; ++i)
    s = fmaf(X[b * in + i], W[o * in + i], s);
  Y[t] = relu ? fmaxf(s, 0.f) : s;
}

// Row-wise softmax of Z, loss += -sum T log P / B, dZ = (P - T) / B.
__global__ void k_softmax_xent(int B, int K, const float *__restrict__ Z,
                               const float *__restrict__ T, float *__restrict__ P,
                               float *__restrict__ dZ, float *__restrict__ loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B)
    return;
  const float *z = Z + b * K;
  float mx = -INFINITY;
  for (int k = 0; k < K; ++k)
    mx = fmaxf(mx, z[k]);
  float sum = 0;
  for (int k = 0; k < K; ++k)
    sum += __expf(z[k] - mx);
  const float lse = mx + __logf(sum);
  float l = 0;
  for (int k = 0; k < K; ++k) {
    const float p = __expf(z[k] - lse);
    if (P)
      P[b * K + k] = p;
    const float t = T ? T[b * K + k] : 0.f;
    if (T)
      l -= t * (z[k] - lse);
    if (dZ)
      dZ[b * K + k] = (p - t) / B;
  }
  if (loss && T)
    atomicAdd(loss, l / B);
}

// dW[o, i] = sum_b dY[b, o] X[b, i]; db[o] = sum_b dY[b, o].
__global__ void k_linear_bwd_w(int B, int in, int out, const float *__restrict__ dY,
                               const float *__restrict__ X, float *__restrict__ dW,
                               float *__restrict__ db) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= out * (in + 1))
    return;
  const int o = t / (in + 1), i = t % (in + 1);
  float s = 0;
  if (i < in) {
    for (int b = 0; b < B; ++b)
      s = fmaf(dY[b * out + o], X[b * in + i], s);
    dW[o * in + i] = s;
  } else {
    for (int b = 0; b < B; ++b)
      s += dY[b * out + o];
    db[o] = s;
  }
}

// dX[b, i] = (sum_o dY[b, o] W[o, i]) * (Hprev[b, i] > 0)
__global__ void k_linear_bwd_x(int B, int in, int out, const float *__restrict__ dY,
                               const float *__restrict__ W, const float *__restrict__ Hprev,
                               float *__restrict__ dX) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * in)
    return;
  const int b = t / in, i = t % in;
  float s = 0;
  for (int o = 0; o < out; ++o)
    s = fmaf(dY[b * out + o], W[o * in + i], s);
  dX[t] = Hprev[t] > 0.f ? s : 0.f;
}

struct AdamState {
  int t;
  float bc1, bc2;
};

__global__ void k_adam_prep(AdamState *st, float b1, float b2) {
  st->t += 1;
  st->bc1 = 1.f - powf(b1, (float)st->t);
  st->bc2 = 1.f - powf(b2, (float)st->t);
}

__global__ void k_adam(int64_t P, float *__restrict__ w, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, const AdamState *st,
                       float lr, float b1, float b2, float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P)
    return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / st->bc1, vh = vi / st->bc2;
  w[i] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_advance(int32_t *off, int B) { *off += B; }

__global__ void k_zero(float *p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    p[i] = 0.f;
}

unsigned nb(int64_t n, int t = 256) { return (unsigned)div_up(std::max<int64_t>(n, 1), t); }

}  // namespace

}  // namespace pls

struct perflibs_b200_selector_s {
  int K = 0;
  int device = 0;
  int64_t P = 0;       // trainable parameters
  int64_t Ptot = 0;    // + normalisation
  pls::DevBuf params, grads, adam_m, adam_v, state;
  cudaStream_t stream = nullptr;

  // Offsets into the parameter vector.
  int64_t oW1() const { return 0; }
  int64_t ob1() const { return (int64_t)pls::H * pls::NF; }
  int64_t oW2() const { return ob1() + pls::H; }
  int64_t ob2() const { return oW2() + (int64_t)pls::H * pls::H; }
  int64_t oW3() const { return ob2() + pls::H; }
  int64_t ob3() const { return oW3() + (int64_t)K * pls::H; }
  int64_t omean() const { return ob3() + K; }
  int64_t oistd() const { return omean() + pls::NF; }
  float *p(int64_t o) const { return params.as<float>() + o; }
  float *g(int64_t o) const { return grads.as<float>() + o; }
};

namespace pls {

using Sel = perflibs_b200_selector_s;

namespace {

struct Activations {
  DevBuf xn, h1, h2, z, p, dz, dh2, dh1, loss;
  void reserve(int B, int K) {
    xn.reserve(4 * (size_t)B * NF);
    h1.reserve(4 * (size_t)B * H);
    h2.reserve(4 * (size_t)B * H);
    z.reserve(4 * (size_t)B * K);
    p.reserve(4 * (size_t)B * K);
    dz.reserve(4 * (size_t)B * K);
    dh2.reserve(4 * (size_t)B * H);
    dh1.reserve(4 * (size_t)B * H);
    loss.reserve(4);
  }
};

// Forward (and, with T, loss + backward into S->grads) on B samples whose
// raw features are at x (device).
void forward_backward(Sel *S, int B, const float *x, const float *T, Activations &a,
                      bool backward, cudaStream_t s) {
  const int K = S->K;
  k_normalize<<<nb((int64_t)B * NF), 256, 0, s>>>(B, x, S->p(S->omean()), S->p(S->oistd()),
                                                  a.xn.as<float>());
  k_linear_fwd<<<nb((int64_t)B * H), 256, 0, s>>>(B, NF, H, a.xn.as<float>(), S->p(S->oW1()),
                                                  S->p(S->ob1()), a.h1.as<float>(), 1);
  k_linear_fwd<<<nb((int64_t)B * H), 256, 0, s>>>(B, H, H, a.h1.as<float>(), S->p(S->oW2()),
                                                  S->p(S->ob2()), a.h2.as<float>(), 1);
  k_linear_fwd<<<nb((int64_t)B * K), 256, 0, s>>>(B, H, K, a.h2.as<float>(), S->p(S->oW3()),
                                                  S->p(S->ob3()), a.z.as<float>(), 0);
  k_zero<<<1, 32, 0, s>>>(a.loss.as<float>(), 1);
  k_softmax_xent<<<nb(B, 128), 128, 0, s>>>(B, K, a.z.as<float>(), T, a.p.as<float>(),
                                            backward ? a.dz.as<float>() : nullptr,
                                            a.loss.as<float>());
  if (!backward)
    return;
  k_linear_bwd_w<<<nb((int64_t)K * (H + 1)), 256, 0, s>>>(B, H, K, a.dz.as<float>(),
                                                          a.h2.as<float>(), S->g(S->oW3()),
                                                          S->g(S->ob3()));
  k_linear_bwd_x<<<nb((int64_t)B * H), 256, 0, s>>>(B, H, K, a.dz.as<float>(), S->p(S->oW3()),
                                                    a.h2.as<float>(), a.dh2.as<float>());
  k_linear_bwd_w<<<nb((int64_t)H * (H + 1)), 256, 0, s>>>(B, H, H, a.dh2.as<float>(),
                                                          a.h1.as<float>(), S->g(S->oW2()),
                                                          S->g(S->ob2()));
  k_linear_bwd_x<<<nb((int64_t)B * H), 256, 0, s>>>(B, H, H, a.dh2.as<float>(), S->p(S->oW2()),
                                                    a.h1.as<float>(), a.dh1.as<float>());
  k_linear_bwd_w<<<nb((int64_t)H * (NF + 1)), 256, 0, s>>>(B, NF, H, a.dh1.as<float>(),
                                                           a.xn.as<float>(), S->g(S->oW1()),
                                                           S->g(S->ob1()));
}

}  // namespace

}  // namespace pls

using namespace pls;

namespace pls {
int selector_classes(perflibs_b200_selector_t S) { return S ? S->K : 0; }
}  // namespace pls

extern "C" {

perflibs_status_t perflibs_b200_selector_create(perflibs_b200_selector_t *out, int32_t K,
                                                uint64_t seed) {
  if (!out || K <= 0 || K > 4096)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  *out = nullptr;
  Sel *S = nullptr;
  const perflibs_status_t st = status_guard([&] {
    S = new Sel;
    S->K = K;
    cudaGetDevice(&S->device);
    S->P = S->ob3() + K;
    S->Ptot = S->P + 2 * NF;
    S->params.reserve(4 * S->Ptot);
    S->grads.reserve(4 * S->P);
    S->adam_m.reserve(4 * S->P);
    S->adam_v.reserve(4 * S->P);
    S->state.reserve(64);
    PLS_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    // He-uniform initialisation, zero biases, identity normalisation.
    std::vector<float> h(S->Ptot, 0.f);
    std::mt19937_64 rng(seed);
    auto init = [&](int64_t off, int fan_in, int64_t count) {
      const float lim = std::sqrt(6.f / fan_in);
      std::uniform_real_distribution<float> u(-lim, lim);
      for (int64_t i = 0; i < count; ++i)
        h[off + i] = u(rng);
    };
    init(S->oW1(), NF, (int64_t)H * NF);
    init(S->oW2(), H, (int64_t)H * H);
    init(S->oW3(), H, (int64_t)K * H);
    for (int f = 0; f < NF; ++f)
      h[S->oistd() + f] = 1.f;
    PLS_CUDA(cudaMemcpy(S->params.p, h.data(), 4 * S->Ptot, cudaMemcpyHostToDevice));
    PLS_CUDA(cudaDeviceSynchronize());  // legacy-stream copy, may still be in flight
    return PERFLIBS_STATUS_SUCCESS;
  });
  if (st != PERFLIBS_STATUS_SUCCESS) {
    perflibs_b200_selector_destroy(S);  // null, or what was made before the failure
    return st;
  }
  *out = S;
  return PERFLIBS_STATUS_SUCCESS;
}

perflibs_status_t perflibs_b200_selector_destroy(perflibs_b200_selector_t S) {
  if (S) {
    if (S->stream)
      cudaStreamDestroy(S->stream);
    delete S;
  }
  return PERFLIBS_STATUS_SUCCESS;
}

int64_t perflibs_b200_selector_param_count(perflibs_b200_selector_t S) {
  return S ? S->Ptot : -1;
}

perflibs_status_t perflibs_b200_selector_get_params(perflibs_b200_selector_t S, float *params) {
  if (!S || !params)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return cudaMemcpy(params, S->params.p, 4 * S->Ptot, cudaMemcpyDeviceToHost) == cudaSuccess
             ? PERFLIBS_STATUS_SUCCESS
             : PERFLIBS_STATUS_EXECUTION_FAILURE;
}

perflibs_status_t perflibs_b200_selector_set_params(perflibs_b200_selector_t S,
                                                    const float *params) {
  if (!S || !params)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  // Legacy-stream copy from pageable memory: synchronise before the
  // selector's own stream reads the parameters.
  return cudaMemcpy(S->params.p, params, 4 * S->Ptot, cudaMemcpyHostToDevice) == cudaSuccess &&
                 cudaDeviceSynchronize() == cudaSuccess
             ? PERFLIBS_STATUS_SUCCESS
             : PERFLIBS_STATUS_EXECUTION_FAILURE;
}

perflibs_status_t perflibs_b200_selector_loss_grad(perflibs_b200_selector_t S, const float *X,
                                                   const float *T, int32_t n, float *loss,
                                                   float *grad) {
  if (!S || !X || !T || n <= 0)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&]() -> perflibs_status_t {
    cudaStream_t s = S->stream;
    DevBuf xd, td;
    xd.reserve(4 * (size_t)n * NF);
    td.reserve(4 * (size_t)n * S->K);
    PLS_CUDA(cudaMemcpyAsync(xd.p, X, 4 * (size_t)n * NF, cudaMemcpyHostToDevice, s));
    PLS_CUDA(cudaMemcpyAsync(td.p, T, 4 * (size_t)n * S->K, cudaMemcpyHostToDevice, s));
    Activations a;
    a.reserve(n, S->K);
    forward_backward(S, n, xd.as<float>(), td.as<float>(), a, true, s);
    PLS_LAUNCH_CHECK();
    if (loss)
      PLS_CUDA(cudaMemcpyAsync(loss, a.loss.p, 4, cudaMemcpyDeviceToHost, s));
    if (grad)
      PLS_CUDA(cudaMemcpyAsync(grad, S->grads.p, 4 * S->P, cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_selector_train(perflibs_b200_selector_t S, const float *X,
                                               const float *T, int32_t n, int32_t epochs,
                                               int32_t batch, float lr, uint64_t seed,
                                               float *final_loss) {
  if (!S || !X || !T || n <= 0 || epochs <= 0 || batch <= 0)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&]() -> perflibs_status_t {
    cudaStream_t s = S->stream;
    const int K = S->K;
    const int B = std::min(batch, n);
    const int steps = n / B;
    // Feature normalisation fitted on the training set (host, once).
    {
      std::vector<float> mean(NF, 0.f), istd(NF, 1.f);
      for (int f = 0; f < NF; ++f) {
        double m = 0, v = 0;
        for (int i = 0; i < n; ++i)
          m += X[(int64_t)i * NF + f];
        m /= n;
        for (int i = 0; i < n; ++i) {
          const double d = X[(int64_t)i * NF + f] - m;
          v += d * d;
        }
        v /= n;
        mean[f] = (float)m;
        istd[f] = v > 1e-12 ? (float)(1.0 / std::sqrt(v)) : 1.f;
      }
      PLS_CUDA(cudaMemcpyAsync(S->p(S->omean()), mean.data(), 4 * NF, cudaMemcpyHostToDevice, s));
      PLS_CUDA(cudaMemcpyAsync(S->p(S->oistd()), istd.data(), 4 * NF, cudaMemcpyHostToDevice, s));
    }
    DevBuf xd, td, perm, xb, tb;
    xd.reserve(4 * (size_t)n * NF);
    td.reserve(4 * (size_t)n * K);
    perm.reserve(4 * (size_t)n);
    xb.reserve(4 * (size_t)B * NF);
    tb.reserve(4 * (size_t)B * K);
    PLS_CUDA(cudaMemcpyAsync(xd.p, X, 4 * (size_t)n * NF, cudaMemcpyHostToDevice, s));
    PLS_CUDA(cudaMemcpyAsync(td.p, T, 4 * (size_t)n * K, cudaMemcpyHostToDevice, s));
    PLS_CUDA(cudaMemsetAsync(S->adam_m.p, 0, 4 * S->P, s));
    PLS_CUDA(cudaMemsetAsync(S->adam_v.p, 0, 4 * S->P, s));
    PLS_CUDA(cudaMemsetAsync(S->state.p, 0, 64, s));
    auto *st = S->state.as<AdamState>();
    auto *off = reinterpret_cast<int32_t *>(S->state.as<char>() + 32);
    Activations a;
    a.reserve(B, K);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;

    // One training step, captured once.
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    PLS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    k_gather_batch<<<B, 32, 0, s>>>(B, K, perm.as<int32_t>(), off, xd.as<float>(), td.as<float>(),
                                    xb.as<float>(), tb.as<float>());
    forward_backward(S, B, xb.as<float>(), tb.as<float>(), a, true, s);
    k_adam_prep<<<1, 1, 0, s>>>(st, b1, b2);
    k_adam<<<nb(S->P), 256, 0, s>>>(S->P, S->params.as<float>(), S->grads.as<float>(),
                                     S->adam_m.as<float>(), S->adam_v.as<float>(), st, lr, b1, b2,
                                     eps);
    k_advance<<<1, 1, 0, s>>>(off, B);
    PLS_CUDA(cudaStreamEndCapture(s, &graph));
    PLS_CUDA(cudaGraphInstantiate(&exec, graph, 0));

    std::mt19937_64 rng(seed);
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(idx.begin(), idx.end(), rng);
      PLS_CUDA(cudaMemcpyAsync(perm.p, idx.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, s));
      PLS_CUDA(cudaMemsetAsync(off, 0, 4, s));
      for (int k = 0; k < steps; ++k)
        PLS_CUDA(cudaGraphLaunch(exec, s));
      // The host buffer `idx` is rewritten next epoch: wait for the copy.
      PLS_CUDA(cudaStreamSynchronize(s));
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (final_loss) {
      // Loss over the whole training set with the final parameters.
      Activations full;
      full.reserve(n, K);
      forward_backward(S, n, xd.as<float>(), td.as<float>(), full, false, s);
      PLS_CUDA(cudaMemcpyAsync(final_loss, full.loss.p, 4, cudaMemcpyDeviceToHost, s));
    }
    PLS_CUDA(cudaStreamSynchronize(s));
    return PERFLIBS_STATUS_SUCCESS;
  });
}

perflibs_status_t perflibs_b200_selector_predict(perflibs_b200_selector_t S, const float *X,
                                                 int32_t n, float *probs, int32_t *cls) {
  if (!S || !X || n <= 0)
    return PERFLIBS_STATUS_INPUT_PARAMETER_ERROR;
  return status_guard([&]() -> perflibs_status_t {
    cudaStream_t s = S->stream;
    const int K = S->K;
    DevBuf xd;
    xd.reserve(4 * (size_t)n * NF);
    PLS_CUDA(cudaMemcpyAsync(xd.p, X, 4 * (size_t)n * NF, cudaMemcpyHostToDevice, s));
    Activations a;
    a.reserve(n, K);
    forward_backward(S, n, xd.as<float>(), nullptr, a, false, s);
    PLS_LAUNCH_CHECK();
    std::vector<float> p((size_t)n * K);
    PLS_CUDA(cudaMemcpyAsync(p.data(), a.p.p, 4 * p.size(), cudaMemcpyDeviceToHost, s));
    PLS_CUDA(cudaStreamSynchronize(s));
    if (probs)
      std::memcpy(probs, p.data(), 4 * p.size());
    if (cls)
      for (int i = 0; i < n; ++i)
        cls[i] = (int32_t)(std::max_element(p.begin() + (size_t)i * K, p.begin() + (size_t)(i + 1) * K) -
                           (p.begin() + (size_t)i * K));
    return PERFLIBS_STATUS_SUCCESS;
  });
}

}  // extern "C"
