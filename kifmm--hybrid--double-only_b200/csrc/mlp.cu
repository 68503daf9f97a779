// Cost-model network: a 3-layer perceptron (FP32) trained and evaluated on the
// GPU by the kernels below (no counterpart in the reference, which takes its
// leaf size from the command line).
//
//   H1 = relu(X W1 + b1)   X: B x F,  W1: F x H
//   H2 = relu(H1 W2 + b2)  W2: H x H
//   Y  = H2 W3 + b3        W3: H x O
//   loss = mean over B x O of (Y - T)^2
//
// Parameters are one packed float array [W1 | b1 | W2 | b2 | W3 | b3], each
// weight matrix row-major (input index major).  Gradients use the same
// layout.  Training is full-batch Adam (beta1 0.9, beta2 0.999, eps 1e-8).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "host.h"

namespace kfmm {
namespace {

constexpr int kMlpThreads = 256;

struct Layout {
  int F, H, O;
  size_t w1, b1, w2, b2, w3, b3, total;
  Layout(int f, int h, int o) : F(f), H(h), O(o) {
    w1 = 0;
    b1 = w1 + (size_t)F * H;
    w2 = b1 + H;
    b2 = w2 + (size_t)H * H;
    w3 = b2 + H;
    b3 = w3 + (size_t)H * O;
    total = b3 + O;
  }
};

// Y[b, o] = bias[o] + sum_i X[b, i] W[i, o]; relu optional; one thread per output
__global__ void dense_forward(int B, int I, int O, const float* X, const float* W,
                              const float* bias, float* Y, int relu) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < B * O; q += gridDim.x * blockDim.x) {
    const int b = q / O, o = q % O;
    float s = bias[o];
    for (int i = 0; i < I; ++i) s = fmaf(X[(size_t)b * I + i], W[(size_t)i * O + o], s);
    Y[q] = relu ? fmaxf(s, 0.f) : s;
  }
}

// dY of the output layer: 2 (Y - T) / (B O)
__global__ void loss_grad(int n, const float* Y, const float* T, float* dY, float* sq) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float d = Y[q] - T[q];
    dY[q] = 2.f * d / (float)n;
    sq[q] = d * d;
  }
}

// dW[i, o] = sum_b X[b, i] dY[b, o]  and  dbias[o] = sum_b dY[b, o]
__global__ void dense_weight_grad(int B, int I, int O, const float* X, const float* dY, float* dW,
                                  float* dbias) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < (I + 1) * O;
       q += gridDim.x * blockDim.x) {
    const int i = q / O, o = q % O;
    float s = 0.f;
    if (i < I)
      for (int b = 0; b < B; ++b) s = fmaf(X[(size_t)b * I + i], dY[(size_t)b * O + o], s);
    else
      for (int b = 0; b < B; ++b) s += dY[(size_t)b * O + o];
    if (i < I) dW[q] = s;
    else dbias[o] = s;
  }
}

// dX[b, i] = (sum_o dY[b, o] W[i, o]) * (H[b, i] > 0), H the layer's relu output
__global__ void dense_input_grad(int B, int I, int O, const float* dY, const float* W,
                                 const float* H, float* dX) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < B * I; q += gridDim.x * blockDim.x) {
    const int b = q / I, i = q % I;
    float s = 0.f;
    for (int o = 0; o < O; ++o) s = fmaf(dY[(size_t)b * O + o], W[(size_t)i * O + o], s);
    dX[q] = H[q] > 0.f ? s : 0.f;
  }
}

__global__ void adam_step(int n, float* p, const float* g, float* m, float* v, float lr,
                          float c1, float c2) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    m[q] = 0.9f * m[q] + 0.1f * g[q];
    v[q] = 0.999f * v[q] + 0.001f * g[q] * g[q];
    p[q] -= lr * (m[q] / c1) / (sqrtf(v[q] / c2) + 1e-8f);
  }
}

__global__ void sum_kernel(int n, const float* x, float* out) {
  __shared__ float red[kMlpThreads];
  float s = 0.f;
  for (int q = threadIdx.x; q < n; q += blockDim.x) s += x[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

inline int blocks_for(size_t n) {
  return (int)std::min<size_t>((n + kMlpThreads - 1) / kMlpThreads, 1024);
}

struct Net {
  Layout L;
  int B;
  float *p, *g, *X, *T, *H1, *H2, *Y, *dY, *dH2, *dH1, *sq, *loss, *m, *v;
  std::vector<void*> allocs;
  Net(int f, int h, int o, int b) : L(f, h, o), B(b) {}
  ~Net() {
    for (void* a : allocs) cudaFree(a);
  }
  cudaError_t alloc(float** q, size_t n) {
    void* a = nullptr;
    cudaError_t e = cudaMalloc(&a, std::max<size_t>(n, 1) * sizeof(float));
    if (e == cudaSuccess) allocs.push_back(a);
    *q = (float*)a;
    return e;
  }
  cudaError_t init(bool train) {
    cudaError_t e;
    const size_t n = L.total;
    if ((e = alloc(&p, n)) || (e = alloc(&X, (size_t)B * L.F)) || (e = alloc(&H1, (size_t)B * L.H)) ||
        (e = alloc(&H2, (size_t)B * L.H)) || (e = alloc(&Y, (size_t)B * L.O)))
      return e;
    if (!train) return cudaSuccess;
    if ((e = alloc(&g, n)) || (e = alloc(&T, (size_t)B * L.O)) || (e = alloc(&dY, (size_t)B * L.O)) ||
        (e = alloc(&dH2, (size_t)B * L.H)) || (e = alloc(&dH1, (size_t)B * L.H)) ||
        (e = alloc(&sq, (size_t)B * L.O)) || (e = alloc(&loss, 1)) || (e = alloc(&m, n)) ||
        (e = alloc(&v, n)))
      return e;
    cudaMemset(m, 0, n * sizeof(float));
    return cudaMemset(v, 0, n * sizeof(float));
  }
  void forward() {
    dense_forward<<<blocks_for((size_t)B * L.H), kMlpThreads>>>(B, L.F, L.H, X, p + L.w1,
                                                                 p + L.b1, H1, 1);
    dense_forward<<<blocks_for((size_t)B * L.H), kMlpThreads>>>(B, L.H, L.H, H1, p + L.w2,
                                                                 p + L.b2, H2, 1);
    dense_forward<<<blocks_for((size_t)B * L.O), kMlpThreads>>>(B, L.H, L.O, H2, p + L.w3,
                                                                 p + L.b3, Y, 0);
  }
  void backward() {
    const int n = B * L.O;
    loss_grad<<<blocks_for(n), kMlpThreads>>>(n, Y, T, dY, sq);
    sum_kernel<<<1, kMlpThreads>>>(n, sq, loss);
    dense_weight_grad<<<blocks_for((size_t)(L.H + 1) * L.O), kMlpThreads>>>(B, L.H, L.O, H2, dY,
                                                                             g + L.w3, g + L.b3);
    dense_input_grad<<<blocks_for((size_t)B * L.H), kMlpThreads>>>(B, L.H, L.O, dY, p + L.w3,
                                                                    H2, dH2);
    dense_weight_grad<<<blocks_for((size_t)(L.H + 1) * L.H), kMlpThreads>>>(B, L.H, L.H, H1, dH2,
                                                                             g + L.w2, g + L.b2);
    dense_input_grad<<<blocks_for((size_t)B * L.H), kMlpThreads>>>(B, L.H, L.H, dH2, p + L.w2,
                                                                    H1, dH1);
    dense_weight_grad<<<blocks_for((size_t)(L.F + 1) * L.H), kMlpThreads>>>(B, L.F, L.H, X, dH1,
                                                                             g + L.w1, g + L.b1);
  }
};

#define MLP_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_error(std::string("mlp: ") + #call + ": " + cudaGetErrorString(e_));            \
      return KFMM_ERR_CUDA;                                                               \
    }                                                                                     \
  } while (0)

bool bad_shape(int F, int H, int O, int B) {
  return F < 1 || H < 1 || O < 1 || B < 1 || F > 4096 || H > 4096 || O > 4096;
}

}  // namespace
}  // namespace kfmm

using namespace kfmm;

extern "C" kfmm_status kfmm_mlp_param_count(int F, int H, int O, long long* count) {
  if (!count || bad_shape(F, H, O, 1)) {
    set_error("kfmm_mlp_param_count: bad shape");
    return KFMM_ERR_INVALID;
  }
  *count = (long long)Layout(F, H, O).total;
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_mlp_forward(int F, int H, int O, const float* params, int B,
                                        const float* X, float* Y) {
  if (!params || !X || !Y || bad_shape(F, H, O, B)) {
    set_error("kfmm_mlp_forward: bad argument");
    return KFMM_ERR_INVALID;
  }
  Net net(F, H, O, B);
  MLP_CUDA(net.init(false));
  MLP_CUDA(cudaMemcpy(net.p, params, sizeof(float) * net.L.total, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(net.X, X, sizeof(float) * (size_t)B * F, cudaMemcpyHostToDevice));
  net.forward();
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaMemcpy(Y, net.Y, sizeof(float) * (size_t)B * O, cudaMemcpyDeviceToHost));
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_mlp_gradients(int F, int H, int O, const float* params, int B,
                                          const float* X, const float* T, float* grads,
                                          float* loss) {
  if (!params || !X || !T || !grads || !loss || bad_shape(F, H, O, B)) {
    set_error("kfmm_mlp_gradients: bad argument");
    return KFMM_ERR_INVALID;
  }
  Net net(F, H, O, B);
  MLP_CUDA(net.init(true));
  MLP_CUDA(cudaMemcpy(net.p, params, sizeof(float) * net.L.total, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(net.X, X, sizeof(float) * (size_t)B * F, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(net.T, T, sizeof(float) * (size_t)B * O, cudaMemcpyHostToDevice));
  net.forward();
  net.backward();
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaMemcpy(grads, net.g, sizeof(float) * net.L.total, cudaMemcpyDeviceToHost));
  float s = 0.f;
  MLP_CUDA(cudaMemcpy(&s, net.loss, sizeof(float), cudaMemcpyDeviceToHost));
  *loss = s / (float)(B * O);
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_mlp_train(int F, int H, int O, float* params, int B, const float* X,
                                      const float* T, int steps, float lr, float* losses) {
  if (!params || !X || !T || steps < 1 || !(lr > 0.f) || bad_shape(F, H, O, B)) {
    set_error("kfmm_mlp_train: bad argument");
    return KFMM_ERR_INVALID;
  }
  Net net(F, H, O, B);
  MLP_CUDA(net.init(true));
  MLP_CUDA(cudaMemcpy(net.p, params, sizeof(float) * net.L.total, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(net.X, X, sizeof(float) * (size_t)B * F, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(net.T, T, sizeof(float) * (size_t)B * O, cudaMemcpyHostToDevice));
  const int n = (int)net.L.total;
  for (int s = 1; s <= steps; ++s) {
    net.forward();
    net.backward();
    const float c1 = 1.f - std::pow(0.9f, (float)s), c2 = 1.f - std::pow(0.999f, (float)s);
    adam_step<<<blocks_for(n), kMlpThreads>>>(n, net.p, net.g, net.m, net.v, lr, c1, c2);
    if (losses) {
      float l = 0.f;
      MLP_CUDA(cudaMemcpy(&l, net.loss, sizeof(float), cudaMemcpyDeviceToHost));
      losses[s - 1] = l / (float)(B * O);
    }
  }
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaMemcpy(params, net.p, sizeof(float) * net.L.total, cudaMemcpyDeviceToHost));
  return KFMM_OK;
}
