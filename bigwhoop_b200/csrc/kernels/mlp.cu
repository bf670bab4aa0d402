// The rate-control warm start's network: a 34 -> 64 -> 64 -> 1 multilayer perceptron (ReLU
// hidden layers, linear output, FP32), with hand-written CUDA kernels for inference, the
// gradient of the mean squared error and Adam training.
//
// Parameters, one float array of kMlpParams values in this order:
//   W1[64][34], b1[64], W2[64][64], b2[64], W3[64], b3
// Inputs: the 34 rate-control features (tier2.cpp, rate_features); output: the predicted
// final slope threshold / 65536.
//
// Gradients are deterministic: every sample's gradient is written to its own row and the rows
// are summed in sample order, so training gives the same weights on every run.
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "device_common.cuh"

namespace bwcb {

extern const float kBuiltinRateModel[];
extern const int kBuiltinRateModelSize;

namespace {

constexpr int kIn = kMlpInputs, kHid = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid,
              kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid;
static_assert(kOffB3 + 1 == kMlpParams, "parameter layout");

// one CTA (64 threads) per sample: hidden activations and the output
__global__ void __launch_bounds__(kHid) mlp_forward_kernel(const float *__restrict__ P,
                                                           const float *__restrict__ X, int n,
                                                           float *__restrict__ H1,
                                                           float *__restrict__ H2,
                                                           float *__restrict__ Y) {
  __shared__ float x[kIn], h1[kHid], h2[kHid];
  const int s = blockIdx.x, j = threadIdx.x;
  if (s >= n) return;
  if (j < kIn) x[j] = X[(size_t)s * kIn + j];
  __syncthreads();
  float a = P[kOffB1 + j];
  for (int i = 0; i < kIn; ++i) a += P[kOffW1 + j * kIn + i] * x[i];
  h1[j] = a > 0.f ? a : 0.f;
  __syncthreads();
  float b = P[kOffB2 + j];
  for (int k = 0; k < kHid; ++k) b += P[kOffW2 + j * kHid + k] * h1[k];
  h2[j] = b > 0.f ? b : 0.f;
  if (H1) H1[(size_t)s * kHid + j] = h1[j];
  if (H2) H2[(size_t)s * kHid + j] = h2[j];
  __syncthreads();
  if (j == 0) {
    float y = P[kOffB3];
    for (int k = 0; k < kHid; ++k) y += P[kOffW3 + k] * h2[k];
    Y[s] = y;
  }
}

// one CTA per sample: that sample's gradient of (y - t)^2 / n, written to row s of G
__global__ void __launch_bounds__(kHid) mlp_backward_kernel(const float *__restrict__ P,
                                                            const float *__restrict__ X,
                                                            const float *__restrict__ T, int n,
                                                            const float *__restrict__ H1,
                                                            const float *__restrict__ H2,
                                                            const float *__restrict__ Y,
                                                            float *__restrict__ G) {
  __shared__ float x[kIn], h1[kHid], d2[kHid];
  const int s = blockIdx.x, j = threadIdx.x;
  if (s >= n) return;
  float *g = G + (size_t)s * kMlpParams;
  if (j < kIn) x[j] = X[(size_t)s * kIn + j];
  h1[j] = H1[(size_t)s * kHid + j];
  const float h2 = H2[(size_t)s * kHid + j];
  const float dy = 2.f * (Y[s] - T[s]) / (float)n;
  // output layer
  g[kOffW3 + j] = dy * h2;
  if (j == 0) g[kOffB3] = dy;
  d2[j] = (h2 > 0.f) ? dy * P[kOffW3 + j] : 0.f;
  __syncthreads();
  // second layer: row j of W2
  for (int k = 0; k < kHid; ++k) g[kOffW2 + j * kHid + k] = d2[j] * h1[k];
  g[kOffB2 + j] = d2[j];
  // first layer: unit j
  float d1 = 0.f;
  for (int m = 0; m < kHid; ++m) d1 += d2[m] * P[kOffW2 + m * kHid + j];
  d1 = (h1[j] > 0.f) ? d1 : 0.f;
  for (int i = 0; i < kIn; ++i) g[kOffW1 + j * kIn + i] = d1 * x[i];
  g[kOffB1 + j] = d1;
}

// sum of the per-sample rows, in sample order; loss = sum (y - t)^2 / n
__global__ void mlp_reduce_kernel(const float *__restrict__ G, int n, float *__restrict__ grad,
                                  const float *__restrict__ Y, const float *__restrict__ T,
                                  float *loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    float a = 0.f;
    for (int s = 0; s < n; ++s) a += G[(size_t)s * kMlpParams + p];
    grad[p] = a;
  }
  if (p == 0 && loss) {
    float l = 0.f;
    for (int s = 0; s < n; ++s) l += (Y[s] - T[s]) * (Y[s] - T[s]);
    *loss = l / (float)n;
  }
}

// Adam step t (1-based)
__global__ void adam_kernel(float *__restrict__ P, const float *__restrict__ grad,
                            float *__restrict__ M, float *__restrict__ V, float lr, int t) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float g = grad[p];
  const float m = b1 * M[p] + (1.f - b1) * g;
  const float v = b2 * V[p] + (1.f - b2) * g * g;
  M[p] = m;
  V[p] = v;
  const float mh = m / (1.f - powf(b1, (float)t));
  const float vh = v / (1.f - powf(b2, (float)t));
  P[p] -= lr * mh / (sqrtf(vh) + eps);
}

template <typename T>
T *dalloc(size_t count) {
  void *p = nullptr;
  if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
  return static_cast<T *>(p);
}

struct Scratch {
  float *P = nullptr, *X = nullptr, *T = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr,
        *G = nullptr, *grad = nullptr, *loss = nullptr, *M = nullptr, *V = nullptr;
  bool ok = false;
  Scratch(int n) {
    P = dalloc<float>(kMlpParams);
    X = dalloc<float>((size_t)n * kIn);
    T = dalloc<float>(n);
    H1 = dalloc<float>((size_t)n * kHid);
    H2 = dalloc<float>((size_t)n * kHid);
    Y = dalloc<float>(n);
    G = dalloc<float>((size_t)n * kMlpParams);
    grad = dalloc<float>(kMlpParams);
    loss = dalloc<float>(1);
    M = dalloc<float>(kMlpParams);
    V = dalloc<float>(kMlpParams);
    ok = P && X && T && H1 && H2 && Y && G && grad && loss && M && V;
  }
  ~Scratch() {
    float *all[] = {P, X, T, H1, H2, Y, G, grad, loss, M, V};
    for (float *p : all)
      if (p) cudaFree(p);
  }
};

void gradient_on_device(Scratch &w, int n, cudaStream_t s) {
  mlp_forward_kernel<<<n, kHid, 0, s>>>(w.P, w.X, n, w.H1, w.H2, w.Y);
  mlp_backward_kernel<<<n, kHid, 0, s>>>(w.P, w.X, w.T, n, w.H1, w.H2, w.Y, w.G);
  mlp_reduce_kernel<<<(kMlpParams + 255) / 256, 256, 0, s>>>(w.G, n, w.grad, w.Y, w.T, w.loss);
}

// model for rate-control warm starts: the built-in one (compiled from data/pcrd_mlp.npy) until
// bwc_b200_set_rate_model replaces or disables it
std::mutex g_model_mutex;
bool g_model_init = false;
bool g_model_set = false;
std::vector<float> g_model;

void init_model_locked() {
  if (g_model_init) return;
  g_model_init = true;
  if (kBuiltinRateModelSize == kMlpParams) {
    g_model.assign(kBuiltinRateModel, kBuiltinRateModel + kMlpParams);
    g_model_set = true;
  }
}
float *g_model_dev[64] = {};
float *g_io_dev[64] = {};
cudaStream_t g_model_stream[64] = {};

}  // namespace

bool mlp_predict(const float *features, int n, float *out) {
  std::lock_guard<std::mutex> lock(g_model_mutex);
  init_model_locked();
  if (!g_model_set || n <= 0 || n > 64) return false;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  if (!g_model_dev[dev]) {
    g_model_dev[dev] = dalloc<float>(kMlpParams);
    g_io_dev[dev] = dalloc<float>(64 * (kIn + 1));
    if (!g_model_dev[dev] || !g_io_dev[dev] ||
        cudaStreamCreateWithFlags(&g_model_stream[dev], cudaStreamNonBlocking) != cudaSuccess)
      return false;
    cudaMemcpy(g_model_dev[dev], g_model.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice);
  }
  cudaStream_t s = g_model_stream[dev];
  float *X = g_io_dev[dev], *Y = X + 64 * kIn;
  cudaMemcpyAsync(X, features, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice, s);
  mlp_forward_kernel<<<n, kHid, 0, s>>>(g_model_dev[dev], X, n, nullptr, nullptr, Y);
  cudaMemcpyAsync(out, Y, n * sizeof(float), cudaMemcpyDeviceToHost, s);
  return cudaStreamSynchronize(s) == cudaSuccess;
}

}  // namespace bwcb

using namespace bwcb;

extern "C" int bwc_b200_mlp_forward(const float *params, const float *X, uint32 n, float *y) {
  if (!params || !X || !y || !n) return 1;
  Scratch w((int)n);
  if (!w.ok) return 1;
  cudaMemcpy(w.P, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(w.X, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
  mlp_forward_kernel<<<n, kHid>>>(w.P, w.X, (int)n, nullptr, nullptr, w.Y);
  cudaMemcpy(y, w.Y, n * sizeof(float), cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

extern "C" int bwc_b200_mlp_gradient(const float *params, const float *X, const float *t,
                                     uint32 n, float *grad, float *loss) {
  if (!params || !X || !t || !grad || !n) return 1;
  Scratch w((int)n);
  if (!w.ok) return 1;
  cudaMemcpy(w.P, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(w.X, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(w.T, t, n * sizeof(float), cudaMemcpyHostToDevice);
  gradient_on_device(w, (int)n, 0);
  cudaMemcpy(grad, w.grad, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost);
  if (loss) cudaMemcpy(loss, w.loss, sizeof(float), cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

extern "C" int bwc_b200_mlp_train(float *params, const float *X, const float *t, uint32 n,
                                  uint32 epochs, uint32 batch, float lr, uint64 seed,
                                  float *loss_per_epoch) {
  if (!params || !X || !t || !n || !batch) return 1;
  const uint32_t B = batch < n ? batch : n;
  Scratch w((int)B);
  float *M = w.M, *V = w.V;
  if (!w.ok) return 1;
  cudaMemcpy(w.P, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(M, 0, kMlpParams * sizeof(float));
  cudaMemset(V, 0, kMlpParams * sizeof(float));
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  std::vector<float> xb((size_t)B * kIn), tb(B);
  uint64_t rng = seed * 6364136223846793005ull + 1442695040888963407ull;
  int step = 0;
  for (uint32_t e = 0; e < epochs; ++e) {
    for (uint32_t i = n - 1; i > 0; --i) {   // Fisher-Yates with a 64-bit LCG
      rng = rng * 6364136223846793005ull + 1442695040888963407ull;
      const uint32_t j = (uint32_t)((rng >> 33) % (i + 1));
      std::swap(order[i], order[j]);
    }
    double epoch_loss = 0;
    int nb = 0;
    for (uint32_t b0 = 0; b0 + B <= n; b0 += B) {
      for (uint32_t k = 0; k < B; ++k) {
        const uint32_t r = order[b0 + k];
        for (int q = 0; q < kIn; ++q) xb[(size_t)k * kIn + q] = X[(size_t)r * kIn + q];
        tb[k] = t[r];
      }
      cudaMemcpy(w.X, xb.data(), xb.size() * sizeof(float), cudaMemcpyHostToDevice);
      cudaMemcpy(w.T, tb.data(), tb.size() * sizeof(float), cudaMemcpyHostToDevice);
      gradient_on_device(w, (int)B, 0);
      adam_kernel<<<(kMlpParams + 255) / 256, 256>>>(w.P, w.grad, M, V, lr, ++step);
      float l = 0;
      cudaMemcpy(&l, w.loss, sizeof(float), cudaMemcpyDeviceToHost);
      epoch_loss += l;
      ++nb;
    }
    if (loss_per_epoch) loss_per_epoch[e] = nb ? (float)(epoch_loss / nb) : 0.f;
  }
  cudaMemcpy(params, w.P, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

extern "C" int bwc_b200_set_rate_model(const float *params) {
  std::lock_guard<std::mutex> lock(g_model_mutex);
  g_model_init = true;
  if (!params) {
    g_model_set = false;
    return 0;
  }
  g_model.assign(params, params + kMlpParams);
  g_model_set = true;
  for (int d = 0; d < 64; ++d)
    if (g_model_dev[d]) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(d);
      cudaMemcpy(g_model_dev[d], g_model.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice);
      cudaSetDevice(cur);
    }
  return 0;
}
