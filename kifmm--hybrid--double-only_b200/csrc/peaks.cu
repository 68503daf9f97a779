// Throughput micro-benchmarks that give the roofline denominators the
// driver's peak file does not carry: FP64 and FP32 FMA, FP32 rsqrt (MUFU),
// FP64 rsqrt, and FP64 DMMA (mma.sync m8n8k4).  Each kernel runs long
// independent chains on every SM; the result is written only under a
// never-true condition so nothing is optimised away.
#include <cuda_runtime.h>

#include <string>

#include "kifmm_b200.h"

namespace kfmm {
void set_error(const std::string& msg);
}

namespace {

constexpr int kIters = 4096;

__global__ void fma64_kernel(double seed, double* sink) {
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x + i;
  const double b = 0.999999, c = 1e-9;
  for (int it = 0; it < kIters; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fma(a[i], b, c);
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == -1.2345) sink[0] = s;
}

__global__ void fma32_kernel(float seed, float* sink) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x + i;
  const float b = 0.9999f, c = 1e-6f;
  for (int it = 0; it < kIters; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], b, c);
  float s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == -1.2345f) sink[0] = s;
}

__global__ void rsqrt32_kernel(float seed, float* sink) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x + i;
  for (int it = 0; it < kIters / 4; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = rsqrtf(a[i]);
  float s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == -1.2345f) sink[0] = s;
}

__global__ void rsqrt64_kernel(double seed, double* sink) {
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x + i;
  for (int it = 0; it < kIters / 16; ++it)
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = rsqrt(a[i]);
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  if (s == -1.2345) sink[0] = s;
}

__global__ void dmma_kernel(double seed, double* sink) {
  double d[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = seed;
  const double a = 0.5 + threadIdx.x * 1e-3, b = 0.25;
  for (int it = 0; it < kIters / 8; ++it)
#pragma unroll
    for (int i = 0; i < 4; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(d[i][0]), "+d"(d[i][1])
                   : "d"(a), "d"(b));
  double s = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) s += d[i][0] + d[i][1];
  if (s == -1.2345) sink[0] = s;
}

}  // namespace

extern "C" kfmm_status kfmm_measure_peak(int what, double* value) {
  if (!value || what < 0 || what > 4) {
    kfmm::set_error("kfmm_measure_peak: bad argument");
    return KFMM_ERR_INVALID;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 8;
  double* sink = nullptr;
  if (cudaMalloc(&sink, 64) != cudaSuccess) {
    kfmm::set_error("kfmm_measure_peak: cudaMalloc failed");
    return KFMM_ERR_ALLOC;
  }
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  auto launch = [&]() {
    switch (what) {
      case 0: fma64_kernel<<<blocks, threads>>>(1.0, sink); break;
      case 1: fma32_kernel<<<blocks, threads>>>(1.0f, (float*)sink); break;
      case 2: rsqrt32_kernel<<<blocks, threads>>>(1.0f, (float*)sink); break;
      case 3: rsqrt64_kernel<<<blocks, threads>>>(1.0, sink); break;
      case 4: dmma_kernel<<<blocks, threads>>>(1.0, sink); break;
    }
  };
  launch();
  cudaEventRecord(a);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) launch();
  cudaEventRecord(b);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) {
    kfmm::set_error(std::string("kfmm_measure_peak: ") + cudaGetErrorString(e));
    return KFMM_ERR_CUDA;
  }
  const double n = (double)blocks * threads * reps;
  const double s = ms * 1e-3;
  switch (what) {
    case 0:
    case 1: *value = n * kIters * 8 * 2 / s / 1e12; break;         // TFLOP/s
    case 2: *value = n * (kIters / 4) * 8 / s / 1e12; break;      // T rsqrt/s
    case 3: *value = n * (kIters / 16) * 8 / s / 1e12; break;     // T rsqrt/s
    case 4: *value = n / 32 * (kIters / 8) * 4 * 512 / s / 1e12; break;  // TFLOP/s
  }
  return KFMM_OK;
}
