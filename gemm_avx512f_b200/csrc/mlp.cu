// mlp.cu -- the learned configuration selector's network: training and
// batched inference kernels, written out by hand (no library GEMM).
//
// Network: x (7 features) -> 64 ReLU -> 64 ReLU -> 48 linear outputs, the
// predicted log2(ms) of each DGEMM configuration (tuner.cu).  Parameters are
// one flat float array: W1[7][64], b1[64], W2[64][64], b2[64], W3[64][48],
// b3[48].  Loss: mean squared error over the finite targets (configurations
// that were not timed carry non-finite targets and are masked out).
// Training: minibatch Adam (Kingma & Ba 2015) on the GPU.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "b2_methods.cuh"
#include "b2_profile.cuh"

namespace b2 {
namespace {

constexpr int IN = 7, H = 64, OUT = 48;
constexpr int P_W1 = 0, P_B1 = P_W1 + IN * H, P_W2 = P_B1 + H, P_B2 = P_W2 + H * H;
constexpr int P_W3 = P_B2 + H, P_B3 = P_W3 + H * OUT, NPARAM = P_B3 + OUT;

// Y[b][o] = act(bias[o] + sum_i X[b][i] W[i][o])
__global__ void dense_fwd(const float *__restrict__ X, const float *__restrict__ W,
                          const float *__restrict__ bias, float *__restrict__ Y, int B, int in,
                          int out, int relu) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * out) return;
  const int b = idx / out, o = idx % out;
  float a = bias[o];
  for (int i = 0; i < in; ++i) a = fmaf(X[b * in + i], W[i * out + o], a);
  Y[idx] = relu ? fmaxf(a, 0.f) : a;
}

// dY = 2 mask (Y - T) / count; loss += mask (Y - T)^2 / count
__global__ void loss_grad(const float *__restrict__ Y, const float *__restrict__ T,
                          float *__restrict__ dY, float *loss, int n, float inv_count) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const float t = T[idx];
  float d = 0.f;
  if (isfinite(t)) {
    d = Y[idx] - t;
    atomicAdd(loss, d * d * inv_count);
  }
  dY[idx] = 2.f * d * inv_count;
}

// dW[i][o] = sum_b A[b][i] G[b][o];  db[o] = sum_b G[b][o]
__global__ void dense_wgrad(const float *__restrict__ A, const float *__restrict__ G,
                            float *__restrict__ dW, float *__restrict__ db, int B, int in,
                            int out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < in * out) {
    const int i = idx / out, o = idx % out;
    float a = 0.f;
    for (int b = 0; b < B; ++b) a = fmaf(A[b * in + i], G[b * out + o], a);
    dW[idx] = a;
  } else if (idx < in * out + out) {
    const int o = idx - in * out;
    float a = 0.f;
    for (int b = 0; b < B; ++b) a += G[b * out + o];
    db[o] = a;
  }
}

// dA[b][i] = [Hin[b][i] > 0] sum_o G[b][o] W[i][o]   (Hin = the ReLU output feeding W)
__global__ void dense_xgrad_relu(const float *__restrict__ G, const float *__restrict__ W,
                                 const float *__restrict__ Hin, float *__restrict__ dA, int B,
                                 int in, int out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * in) return;
  const int b = idx / in, i = idx % in;
  if (Hin[idx] <= 0.f) { dA[idx] = 0.f; return; }
  float a = 0.f;
  for (int o = 0; o < out; ++o) a = fmaf(G[b * out + o], W[i * out + o], a);
  dA[idx] = a;
}

__global__ void adam_step(float *__restrict__ w, const float *__restrict__ g,
                          float *__restrict__ m, float *__restrict__ v, int n, float lr, float b1,
                          float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void gather_rows(const float *__restrict__ src, const int *__restrict__ idx,
                            float *__restrict__ dst, int B, int width) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * width) return;
  const int b = t / width, c = t % width;
  dst[t] = src[(long long)idx[b] * width + c];
}

inline int blocks(long long n) { return (int)((n + 255) / 256); }

struct Net {
  float *w = nullptr, *g = nullptr;  // parameters and gradients (NPARAM each)
  float *h1 = nullptr, *h2 = nullptr, *y = nullptr, *dy = nullptr, *dh2 = nullptr, *dh1 = nullptr;
  float *loss = nullptr;
  int cap = 0;
  int alloc(int B) {
    cap = B;
    const size_t f = sizeof(float);
    if (cudaMalloc(&w, NPARAM * f) || cudaMalloc(&g, NPARAM * f) || cudaMalloc(&h1, (size_t)B * H * f) ||
        cudaMalloc(&h2, (size_t)B * H * f) || cudaMalloc(&y, (size_t)B * OUT * f) ||
        cudaMalloc(&dy, (size_t)B * OUT * f) || cudaMalloc(&dh2, (size_t)B * H * f) ||
        cudaMalloc(&dh1, (size_t)B * H * f) || cudaMalloc(&loss, f)) {
      (void)cudaGetLastError();
      return B2_ERR_NOMEM;
    }
    return B2_OK;
  }
  ~Net() {
    for (float *p : {w, g, h1, h2, y, dy, dh2, dh1, loss}) cudaFree(p);
  }
  void forward(const float *x, int B, cudaStream_t s) {
    B2_PROF("mlp_forward", s);
    dense_fwd<<<blocks((long long)B * H), 256, 0, s>>>(x, w + P_W1, w + P_B1, h1, B, IN, H, 1);
    dense_fwd<<<blocks((long long)B * H), 256, 0, s>>>(h1, w + P_W2, w + P_B2, h2, B, H, H, 1);
    dense_fwd<<<blocks((long long)B * OUT), 256, 0, s>>>(h2, w + P_W3, w + P_B3, y, B, H, OUT, 0);
  }
  // loss and gradients (into g) for targets t; count = finite targets
  void backward(const float *x, const float *t, int B, float inv_count, cudaStream_t s) {
    B2_PROF("mlp_backward", s);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    loss_grad<<<blocks((long long)B * OUT), 256, 0, s>>>(y, t, dy, loss, B * OUT, inv_count);
    dense_wgrad<<<blocks(H * OUT + OUT), 256, 0, s>>>(h2, dy, g + P_W3, g + P_B3, B, H, OUT);
    dense_xgrad_relu<<<blocks((long long)B * H), 256, 0, s>>>(dy, w + P_W3, h2, dh2, B, H, OUT);
    dense_wgrad<<<blocks(H * H + H), 256, 0, s>>>(h1, dh2, g + P_W2, g + P_B2, B, H, H);
    dense_xgrad_relu<<<blocks((long long)B * H), 256, 0, s>>>(dh2, w + P_W2, h1, dh1, B, H, H);
    dense_wgrad<<<blocks(IN * H + H), 256, 0, s>>>(x, dh1, g + P_W1, g + P_B1, B, IN, H);
  }
};

float finite_count(const float *T, long long n) {
  long long c = 0;
  for (long long i = 0; i < n; ++i) c += std::isfinite(T[i]) ? 1 : 0;
  return (float)(c > 0 ? c : 1);
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" {

int b2_mlp_forward(const float *weights, int n, const float *X, float *Y) {
  if (!weights || n < 0 || (n > 0 && (!X || !Y))) return B2_ERR_ARG;
  if (n == 0) return B2_OK;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  cudaStream_t s = c->stream;
  Net net;
  int rc = net.alloc(n);
  float *dx = nullptr;
  if (rc == B2_OK && cudaMalloc(&dx, (size_t)n * IN * sizeof(float)) != cudaSuccess) rc = B2_ERR_NOMEM;
  if (rc == B2_OK) {
    cudaMemcpyAsync(net.w, weights, NPARAM * sizeof(float), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dx, X, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, s);
    net.forward(dx, n, s);
    cudaMemcpyAsync(Y, net.y, (size_t)n * OUT * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "mlp forward");
  }
  cudaFree(dx);
  return rc;
}

int b2_mlp_gradient(const float *weights, int n, const float *X, const float *T, float *loss,
                    float *grad) {
  if (!weights || n < 1 || !X || !T || !loss || !grad) return B2_ERR_ARG;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  cudaStream_t s = c->stream;
  Net net;
  int rc = net.alloc(n);
  float *dx = nullptr, *dt = nullptr;
  if (rc == B2_OK && (cudaMalloc(&dx, (size_t)n * IN * 4) != cudaSuccess ||
                      cudaMalloc(&dt, (size_t)n * OUT * 4) != cudaSuccess))
    rc = B2_ERR_NOMEM;
  if (rc == B2_OK) {
    cudaMemcpyAsync(net.w, weights, NPARAM * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dx, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dt, T, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, s);
    net.forward(dx, n, s);
    net.backward(dx, dt, n, 1.f / finite_count(T, (long long)n * OUT), s);
    cudaMemcpyAsync(grad, net.g, NPARAM * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(loss, net.loss, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "mlp gradient");
  }
  cudaFree(dx);
  cudaFree(dt);
  return rc;
}

// Train on n samples (features X[n][7], targets T[n][48], non-finite = masked)
// with minibatch Adam; weights_in (may be NULL: seeded Glorot-uniform init)
// -> weights_out; final_loss = mean squared error over the whole set.
int b2_mlp_train(int n, const float *X, const float *T, int epochs, int batch, float lr, int seed,
                 const float *weights_in, float *weights_out, float *final_loss) {
  if (n < 1 || !X || !T || !weights_out || epochs < 0 || batch < 1) return B2_ERR_ARG;
  Ctx *c = ctx();
  if (!c) return B2_ERR_NO_DEVICE;
  cudaStream_t s = c->stream;
  if (batch > n) batch = n;
  std::vector<float> w0(NPARAM);
  if (weights_in) {
    memcpy(w0.data(), weights_in, NPARAM * 4);
  } else {
    std::mt19937 gen((unsigned)seed);
    auto init = [&](int off, int fan_in, int fan_out) {
      const float lim = sqrtf(6.f / (float)(fan_in + fan_out));
      std::uniform_real_distribution<float> u(-lim, lim);
      for (int i = 0; i < fan_in * fan_out; ++i) w0[off + i] = u(gen);
    };
    std::fill(w0.begin(), w0.end(), 0.f);
    init(P_W1, IN, H);
    init(P_W2, H, H);
    init(P_W3, H, OUT);
  }
  Net net, full;
  int rc = net.alloc(batch);
  if (rc == B2_OK) rc = full.alloc(n);
  float *dX = nullptr, *dT = nullptr, *bx = nullptr, *bt = nullptr, *m = nullptr, *v = nullptr;
  int *didx = nullptr;
  if (rc == B2_OK &&
      (cudaMalloc(&dX, (size_t)n * IN * 4) || cudaMalloc(&dT, (size_t)n * OUT * 4) ||
       cudaMalloc(&bx, (size_t)batch * IN * 4) || cudaMalloc(&bt, (size_t)batch * OUT * 4) ||
       cudaMalloc(&m, NPARAM * 4) || cudaMalloc(&v, NPARAM * 4) ||
       cudaMalloc(&didx, (size_t)n * 4))) {
    (void)cudaGetLastError();
    rc = B2_ERR_NOMEM;
  }
  if (rc == B2_OK) {
    cudaMemcpyAsync(dX, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dT, T, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(net.w, w0.data(), NPARAM * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(m, 0, NPARAM * 4, s);
    cudaMemsetAsync(v, 0, NPARAM * 4, s);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::mt19937 gen((unsigned)seed + 1u);
    // per-batch normalisation by the batch's finite targets (precomputed per
    // epoch on the host from the permutation)
    int step = 0;
    for (int ep = 0; ep < epochs && rc == B2_OK; ++ep) {
      std::shuffle(perm.begin(), perm.end(), gen);
      cudaMemcpyAsync(didx, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s);
      const float lr_ep = lr * (0.5f * (1.f + cosf(3.14159265f * ep / (float)(epochs > 0 ? epochs : 1))) * 0.95f + 0.05f);
      for (int b0 = 0; b0 + batch <= n; b0 += batch) {
        long long cnt = 0;
        for (int i = 0; i < batch; ++i)
          for (int o = 0; o < OUT; ++o) cnt += std::isfinite(T[(long long)perm[b0 + i] * OUT + o]);
        gather_rows<<<blocks((long long)batch * IN), 256, 0, s>>>(dX, didx + b0, bx, batch, IN);
        gather_rows<<<blocks((long long)batch * OUT), 256, 0, s>>>(dT, didx + b0, bt, batch, OUT);
        net.forward(bx, batch, s);
        net.backward(bx, bt, batch, 1.f / (float)(cnt > 0 ? cnt : 1), s);
        ++step;
        const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
        adam_step<<<blocks(NPARAM), 256, 0, s>>>(net.w, net.g, m, v, NPARAM, lr_ep, 0.9f, 0.999f,
                                                  1e-8f, c1, c2);
      }
      if (cudaGetLastError() != cudaSuccess) rc = B2_ERR_CUDA;
    }
    // final loss over the whole set
    cudaMemcpyAsync(full.w, net.w, NPARAM * 4, cudaMemcpyDeviceToDevice, s);
    full.forward(dX, n, s);
    full.backward(dX, dT, n, 1.f / finite_count(T, (long long)n * OUT), s);
    float L = 0.f;
    cudaMemcpyAsync(&L, full.loss, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(weights_out, net.w, NPARAM * 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "mlp train");
    if (final_loss) *final_loss = L;
  }
  for (void *p : {(void *)dX, (void *)dT, (void *)bx, (void *)bt, (void *)m, (void *)v, (void *)didx})
    cudaFree(p);
  return rc;
}

}  // extern "C"
