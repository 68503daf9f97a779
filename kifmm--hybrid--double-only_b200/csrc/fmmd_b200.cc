// fmmd--b200: drop-in for the reference's `fmmd--cuda` driver.
//
//   fmmd--b200 <#pts> {uniform,ellipseUniformAngles,ellipsoidSurface} <#pts-per-box>
//   env NP (expansion order, default 6), NV (validation targets, default
//   1000), C (1: targets are the sources), KFMM_MIXED=1 for the mixed form,
//   KFMM_CPU_SHARE_PPM=<n> for the hybrid CPU+GPU evaluation (the host's
//   cores sum that share of the U list, in parts per million; 1000000 is the
//   schedule of the reference's fmmd--hybrid2, fmm/run--hybrid2.cu:25-47),
//   KFMM_DUMP_POT=<file> to write the potentials (original order, raw doubles).
//
// Same sequence and output lines as fmm/driver.cc:211-371: seed 26, points,
// densities, octree + lists, preproc, run (phase timings on stderr), then the
// driver's check: an exact FP64 direct sum at NV sampled targets and the
// relative L2 error.  Everything runs through include/kifmm_b200.h; the direct
// sum runs on the GPU (kfmm_direct_evaluation).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "kifmm_b200.h"

static int env_int(const char* name, int def) {
  const char* s = std::getenv(name);
  if (!s) return def;
  long t = std::atol(s);
  return t > 0 ? (int)t : def;
}

#define CHECK(x)                                                           \
  do {                                                                     \
    kfmm_status s_ = (x);                                                  \
    if (s_ != KFMM_OK) {                                                   \
      std::fprintf(stderr, "%s failed (%d): %s\n", #x, (int)s_, kfmm_last_error()); \
      return 1;                                                            \
    }                                                                      \
  } while (0)

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s <N> <distribution> <pts/box> \n", argv[0]);
    return 255;
  }
  const int n = std::atoi(argv[1]);
  const char* dist = argv[2];
  const int ppb = std::atoi(argv[3]);
  const int np = env_int("NP", 6), nv = env_int("NV", 1000);
  const int coincide = env_int("C", 0) == 1 ? 1 : 0;
  const bool mixed = env_int("KFMM_MIXED", 0) == 1;
  const int cpu_share = std::min(env_int("KFMM_CPU_SHARE_PPM", 0), 1000000);

  std::vector<double> sx(n), sy(n), sz(n), den(n), tx(n), ty(n), tz(n), pot(n);
  std::vector<int> ids(nv);
  CHECK(kfmm_generate_points(n, dist, coincide, 26, sx.data(), sy.data(), sz.data(), den.data(),
                             tx.data(), ty.data(), tz.data(), nv, ids.data()));
  kfmm_tree* tree = nullptr;
  CHECK(kfmm_tree_build(n, sx.data(), sy.data(), sz.data(), n, tx.data(), ty.data(), tz.data(),
                        ppb, &tree));
  kfmm_tree_desc desc;
  CHECK(kfmm_tree_describe(tree, &desc));
  std::fprintf(stderr, "Preprocessing...\n");
  kfmm_plan* plan = nullptr;
  kfmm_tuning tuning = {};
  tuning.cpu_share_ppm = cpu_share;
  CHECK(kfmm_plan_create_tuned(&desc, np, mixed ? KFMM_MIXED : KFMM_PLAIN_FP64, nullptr,
                               cpu_share ? &tuning : nullptr, &plan));
  std::fprintf(stderr, "Finished setup.\n");
  std::fprintf(stderr, "Evaluation...\n");
  CHECK(kfmm_enable_timing(plan, 1));
  CHECK(kfmm_evaluate(plan, sx.data(), sy.data(), sz.data(), den.data(), tx.data(), ty.data(),
                      tz.data(), pot.data(), nullptr));
  if (const char* path = std::getenv("KFMM_DUMP_POT")) {
    FILE* f = std::fopen(path, "wb");
    if (!f || std::fwrite(pot.data(), sizeof(double), n, f) != (size_t)n) {
      std::fprintf(stderr, "KFMM_DUMP_POT: cannot write %s\n", path);
      return 1;
    }
    std::fclose(f);
  }
  float ms[6];
  CHECK(kfmm_phase_times(plan, ms));
  const double t_up = ms[0] * 1e-3, t_v = ms[1] * 1e-3, t_x = ms[2] * 1e-3,
               t_down = ms[3] * 1e-3, t_near = ms[4] * 1e-3, t_copy = ms[5] * 1e-3;
  const double total = t_up + t_v + t_x + t_down + t_near + t_copy;
  std::fprintf(stderr, "=== Statistics ===\n");
  std::fprintf(stdout, "Code: b200-%s%s\n", mixed ? "mixed" : "fp64", cpu_share ? "-hybrid" : "");
  std::fprintf(stdout, "Floating-point word size: %lu bytes\n", (unsigned long)sizeof(double));
  std::fprintf(stderr, "== Timing for FMM3d ==\n");
  // U, W and the direct X list run in one fused kernel, reported as "U list"
  std::fprintf(stderr, "  Up    : %g secs (%.1f%%)\n", t_up, t_up / total * 100);
  std::fprintf(stderr, "  U list: %g secs (%.1f%%)\n", t_near, t_near / total * 100);
  std::fprintf(stderr, "  V list: %g secs (%.1f%%)\n", t_v, t_v / total * 100);
  std::fprintf(stderr, "  W list: %g secs (%.1f%%)\n", 0.0, 0.0);
  std::fprintf(stderr, "  X list: %g secs (%.1f%%)\n", t_x, t_x / total * 100);
  std::fprintf(stderr, "  Down  : %g secs (%.1f%%)\n", t_down + t_copy,
               (t_down + t_copy) / total * 100);
  std::fprintf(stderr, "  ==> Total Execution Time: %g secs\n", total);

  // fmm/driver.cc:142-206, on the device
  std::vector<double> cx(nv), cy(nv), cz(nv), direct(nv, 0.0);
  for (int k = 0; k < nv; ++k) {
    cx[k] = tx[ids[k]];
    cy[k] = ty[ids[k]];
    cz[k] = tz[ids[k]];
  }
  double *d[8] = {};
  const size_t bs = sizeof(double) * n, bt = sizeof(double) * nv;
  cudaMalloc(&d[0], bs); cudaMalloc(&d[1], bs); cudaMalloc(&d[2], bs); cudaMalloc(&d[3], bs);
  cudaMalloc(&d[4], bt); cudaMalloc(&d[5], bt); cudaMalloc(&d[6], bt); cudaMalloc(&d[7], bt);
  cudaMemcpy(d[0], sx.data(), bs, cudaMemcpyHostToDevice);
  cudaMemcpy(d[1], sy.data(), bs, cudaMemcpyHostToDevice);
  cudaMemcpy(d[2], sz.data(), bs, cudaMemcpyHostToDevice);
  cudaMemcpy(d[3], den.data(), bs, cudaMemcpyHostToDevice);
  cudaMemcpy(d[4], cx.data(), bt, cudaMemcpyHostToDevice);
  cudaMemcpy(d[5], cy.data(), bt, cudaMemcpyHostToDevice);
  cudaMemcpy(d[6], cz.data(), bt, cudaMemcpyHostToDevice);
  cudaMemset(d[7], 0, bt);
  CHECK(kfmm_direct_evaluation(nv, d[4], d[5], d[6], d[7], n, d[0], d[1], d[2], d[3], nullptr));
  if (cudaMemcpy(direct.data(), d[7], bt, cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "direct sum failed: %s\n", cudaGetErrorString(cudaGetLastError()));
    return 1;
  }
  for (double* p : d) cudaFree(p);
  double vn = 0, en = 0;
  for (int k = 0; k < nv; ++k) {
    const double fmm = pot[ids[k]], e = direct[k] - fmm;
    vn += fmm * fmm;
    en += e * e;
  }
  kfmm_stats st;
  CHECK(kfmm_plan_stats(plan, &st));
  std::fprintf(stdout, "Inputs: %d | %s | %d \n", n, dist, ppb);
  std::fprintf(stdout, "Estimated no. of flops (Ulist): %g\n", 11.0 * st.u_pairs);
  std::fprintf(stdout, "Estimated no. of flops (Vlist): %g\n", 8.0 * st.hadamard_cmacs);
  std::fprintf(stderr, "Relative error: %e\n", std::sqrt(en) / std::sqrt(vn));
  kfmm_plan_destroy(plan);
  kfmm_tree_destroy(tree);
  return 0;
}
