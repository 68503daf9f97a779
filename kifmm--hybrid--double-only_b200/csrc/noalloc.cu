// Allocation-free upward pass for leaves (kfmm_s2m_noalloc).
//
// Who needs this: callers that may not allocate device memory when they call
// into the solver.  A host framework that owns all device memory through its
// own pool (and forbids stray cudaMalloc/cudaFree, which also synchronise the
// device), or a solver step that runs while such a framework holds the
// memory budget, can still turn source points into upward equivalent
// densities here: the caller passes every input and output buffer, and the
// only scratch (the check potentials) lives in a fixed array that is part of
// the loaded library image.
//
// The scratch array below exists once per GPU that loads this library and
// stays resident until the process exits.  All calls on a device share it and
// it keeps the last call's contents; every call overwrites the part it uses
// before reading it.  Calls whose work overlaps on the GPU (e.g. issued on two
// streams at once) race on it and must be serialised by the caller.
//
// The per-device set-up (symbol addresses, the surface table) is done once
// and remembered for the life of the process; a cudaDeviceReset between calls
// would discard the table behind that record, so callers must not reset a
// device they keep using through this entry point.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "host.h"
#include "kifmm_b200.h"

namespace kfmm {
namespace {

// Check potentials of one call: nleaves * Q doubles at most (8 MiB).
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 20;
static __device__ __align__(256) double g_s2m_scratch[kNoAllocScratchDoubles];

// UC check-surface points (unit box) for NP = 3..8, 3 doubles per point.
constexpr int kMaxQ = 488;  // NP = 8
static __device__ __align__(16) double g_uc_surface[6][3 * kMaxQ];

constexpr int kMaxDevices = 64;
struct DeviceSetup {
  bool done = false;
  double* scratch = nullptr;  // device address of g_s2m_scratch
  double* uc = nullptr;       // device address of g_uc_surface
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

constexpr double kOOFP_NA = 1.0 / (4.0 * 3.14159265358979323846);
constexpr int kNaThreads = 128;

// Check potential at the UC surface of each leaf from the leaf's own sources
// (the S2M check step of fmm/omp.cc:70-88); block = (leaf, 128 surface points).
__global__ void __launch_bounds__(kNaThreads)
s2m_check_noalloc_kernel(int Q, const double* __restrict__ uc, const double* __restrict__ src4,
                         const int* __restrict__ leaf_beg, const int* __restrict__ leaf_num,
                         const double* __restrict__ leaf_ctr, double* __restrict__ chk) {
  __shared__ double4 stage[kNaThreads];
  const int leaf = blockIdx.x;
  const int q = blockIdx.y * kNaThreads + threadIdx.x;
  const double cx = leaf_ctr[4 * leaf], cy = leaf_ctr[4 * leaf + 1], cz = leaf_ctr[4 * leaf + 2],
               r = leaf_ctr[4 * leaf + 3];
  double tx = 0, ty = 0, tz = 0;
  if (q < Q) {
    tx = __dadd_rn(cx, __dmul_rn(r, uc[3 * q]));
    ty = __dadd_rn(cy, __dmul_rn(r, uc[3 * q + 1]));
    tz = __dadd_rn(cz, __dmul_rn(r, uc[3 * q + 2]));
  }
  const int beg = leaf_beg[leaf], num = leaf_num[leaf];
  const double4* s4 = reinterpret_cast<const double4*>(src4);
  double acc = 0.0;
  for (int c0 = 0; c0 < num; c0 += kNaThreads) {
    const int cnt = min(kNaThreads, num - c0);
    __syncthreads();
    if (threadIdx.x < cnt) stage[threadIdx.x] = s4[beg + c0 + threadIdx.x];
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const double4 s = stage[j];
      const double dx = tx - s.x, dy = ty - s.y, dz = tz - s.z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      acc = fma(s.w, r2 > 0.0 ? rsqrt(r2) : 0.0, acc);
    }
  }
  if (q < Q) chk[(size_t)leaf * Q + q] = kOOFP_NA * acc;
}

// uden[leaf] = r_leaf * UC2UE * chk[leaf]  (r_leaf = 2^-depth, fmm/omp.cc:88-99)
__global__ void __launch_bounds__(kNaThreads)
s2m_solve_noalloc_kernel(int P, int Q, const double* __restrict__ uc2ue,
                         const double* __restrict__ chk, const double* __restrict__ leaf_ctr,
                         double* __restrict__ uden) {
  extern __shared__ double c_s[];
  const int leaf = blockIdx.x;
  for (int q = threadIdx.x; q < Q; q += kNaThreads) c_s[q] = chk[(size_t)leaf * Q + q];
  __syncthreads();
  const double scale = leaf_ctr[4 * leaf + 3];
  for (int m = threadIdx.x; m < P; m += kNaThreads) {
    double acc = 0.0;
    for (int q = 0; q < Q; ++q) acc = fma(uc2ue[(size_t)q * P + m], c_s[q], acc);
    uden[(size_t)leaf * P + m] = scale * acc;
  }
}

kfmm_status setup_device(int dev, DeviceSetup** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("kfmm_s2m_noalloc: device ordinal out of range");
    return KFMM_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSetup& s = g_setup[dev];
  if (!s.done) {
    cudaError_t e = cudaGetSymbolAddress((void**)&s.scratch, g_s2m_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.uc, g_uc_surface);
    if (e != cudaSuccess) {
      set_error(std::string("kfmm_s2m_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return KFMM_ERR_CUDA;
    }
    std::vector<double> tab((size_t)6 * 3 * kMaxQ, 0.0);
    for (int np = 3; np <= 8; ++np) {
      Surfaces S;
      make_surfaces(np, &S);
      std::copy(S.uc.begin(), S.uc.end(), tab.begin() + (size_t)(np - 3) * 3 * kMaxQ);
    }
    e = cudaMemcpyToSymbol(g_uc_surface, tab.data(), sizeof(double) * tab.size());
    // A copy from pageable memory may return before the data has landed;
    // the kernels run on the caller's stream, which need not wait on the
    // legacy stream, so the table is made complete here.
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_error(std::string("kfmm_s2m_noalloc: surface table upload: ") + cudaGetErrorString(e));
      return KFMM_ERR_CUDA;
    }
    s.done = true;
  }
  *out = &s;
  return KFMM_OK;
}

}  // namespace
}  // namespace kfmm

using namespace kfmm;

extern "C" kfmm_status kfmm_s2m_noalloc(int np, int nleaves, const double* src4,
                                        const int* leaf_beg, const int* leaf_num,
                                        const double* leaf_ctr, const double* uc2ue,
                                        double* uden, void* stream) {
  int P = 0, Q = 0;
  if (kfmm_sizes(np, &P, &Q, nullptr) != KFMM_OK) return KFMM_ERR_UNSUPPORTED;
  if (nleaves < 0 || (nleaves > 0 && (!src4 || !leaf_beg || !leaf_num || !leaf_ctr || !uc2ue ||
                                      !uden))) {
    set_error("kfmm_s2m_noalloc: bad argument");
    return KFMM_ERR_INVALID;
  }
  if ((size_t)nleaves * Q > kNoAllocScratchDoubles) {
    set_error("kfmm_s2m_noalloc: nleaves * Q = " + std::to_string((size_t)nleaves * Q) +
              " exceeds the fixed scratch of " + std::to_string(kNoAllocScratchDoubles) +
              " doubles; split the leaves into smaller calls");
    return KFMM_ERR_INVALID;
  }
  if (nleaves == 0) return KFMM_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("kfmm_s2m_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return KFMM_ERR_CUDA;
  }
  DeviceSetup* s = nullptr;
  kfmm_status st = setup_device(dev, &s);
  if (st != KFMM_OK) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  dim3 g1(nleaves, (Q + kNaThreads - 1) / kNaThreads);
  s2m_check_noalloc_kernel<<<g1, kNaThreads, 0, cs>>>(Q, s->uc + (size_t)(np - 3) * 3 * kMaxQ,
                                                      src4, leaf_beg, leaf_num, leaf_ctr,
                                                      s->scratch);
  s2m_solve_noalloc_kernel<<<nleaves, kNaThreads, sizeof(double) * Q, cs>>>(P, Q, uc2ue,
                                                                            s->scratch,
                                                                            leaf_ctr, uden);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("kfmm_s2m_noalloc: launch: ") + cudaGetErrorString(e));
    return KFMM_ERR_CUDA;
  }
  return KFMM_OK;
}
