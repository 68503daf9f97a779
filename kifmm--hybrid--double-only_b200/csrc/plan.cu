// Plan (preproc) and run of the KIFMM evaluator: the C ABI of
// include/kifmm_b200.h over the kernels of kernels.cuh.
//
// Phase order of kfmm_run:
//   up    : S2M check potentials (P2P) -> UC2UE level GEMM; M2M per level,
//           deepest first (fmm/cuda.cu:571-600, fmm/omp.cc:61-227)
//   vlist : forward FFT of every source box, sibling-group Hadamard, inverse
//           FFT into the downward check potential (fmm/cuda.cu:718-1196)
//   xlist : S2L onto check surfaces (fmm/cuda.cu:2380-2493)
//   down  : L2L per level, shallowest first (fmm/cuda.cu:1981-2045)
//   ulist : one fused kernel per target chunk: U list, W list, direct X list,
//           and L2T (fmm/cuda.cu:604-663, 2070-2197, 1804-1872)
//   copy  : potentials back to original order (fmm/cuda.cu:2543-2565)
// The reference adds U/W/X/L2T contributions into one array in four passes;
// here each target's potential is summed once in registers and written once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "host.h"
#include "kernels.cuh"

namespace kfmm {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }

#define KF_CUDA(call)                                                               \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
      return KFMM_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

#define KF_CHECK_LAUNCH(what)                                                       \
  do {                                                                              \
    cudaError_t e_ = cudaGetLastError();                                            \
    if (e_ != cudaSuccess) {                                                        \
      set_error(std::string(what) + ": " + cudaGetErrorString(e_));                 \
      return KFMM_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

struct GemmBatch {
  const double* A;
  int M, K;
  int chunks, mrows, nsplit, ksplit;  // launch shape, fixed at plan time
  const double* B;
  int* boff;  // device
  double* C;
  int* coff;  // device
  double* alpha;  // device or null
  double alpha_const;
  int ncol;
  int accumulate;
};

}  // namespace kfmm

using namespace kfmm;

struct kfmm_plan {
  int np = 0, P = 0, Q = 0, F = 0, Fpad = 0, nn = 0, ns = 0, nt = 0, maxdepth = 0;
  kfmm_precision prec = KFMM_PLAIN_FP64;
  std::vector<void*> allocs;
  // tree on device
  double4* ctr = nullptr;
  int *d_depth = nullptr, *d_src_beg = nullptr, *d_src_num = nullptr;
  int *d_src_perm = nullptr, *d_trg_perm = nullptr;
  int *d_src_inv = nullptr, *d_trg_inv = nullptr;  // original index -> leaf-order position
  // points
  double *o_sx = nullptr, *o_sy = nullptr, *o_sz = nullptr, *o_w = nullptr;
  double *o_tx = nullptr, *o_ty = nullptr, *o_tz = nullptr;
  double4 *src4 = nullptr, *trg4 = nullptr;
  // mixed form: FP32 leaf-local sources and the leaf of each source; FP32
  // node centres (exact: dyadic, depth <= 20)
  float4* src4f = nullptr;
  int* d_src_leaf = nullptr;
  float4* ctrf = nullptr;
  double *pot_leaf = nullptr, *pot_orig = nullptr;
  bool have_src = false, have_trg = false;
  // expansions
  double *uden = nullptr, *dchk = nullptr, *dden = nullptr, *chk_up = nullptr, *chk_m = nullptr;
  void *spec = nullptr, *effv = nullptr;  // double2 (FP64) or float2 (mixed)
  size_t cplx = sizeof(double2);
  // operators
  double *d_uc2ue = nullptr, *d_ue2uc = nullptr, *d_dc2de = nullptr, *d_de2dc_stack = nullptr;
  double* d_m2m = nullptr;  // mixed form: UC2UE x UE2UC, P x 8P (one product per M2M level)
  void* d_trans = nullptr;
  double *d_sp_ue = nullptr, *d_sp_uc = nullptr, *d_sp_de = nullptr, *d_sp_dc = nullptr;
  float *d_spf_ue = nullptr, *d_spf_de = nullptr;
  double *d_cs = nullptr, *d_sn = nullptr;
  int *d_surf_idx = nullptr, *d_surf_ijk = nullptr;
  // work lists
  P2PJob *s2m_jobs = nullptr, *nf_jobs = nullptr, *s2l_jobs = nullptr;
  int *s2m_ent = nullptr, *nf_ent = nullptr, *s2l_ent = nullptr;
  int n_s2m = 0, n_nf = 0, n_s2l = 0;
  std::vector<float> nf_class;  // cost class of each near-field job (-log1.25 cost)
  // the near field's jobs before chunking (one per target leaf, all its
  // targets) and their source counts, kept to re-chunk on a new job size
  std::vector<P2PJob> nf_leaf;
  std::vector<double> nf_leaf_ns;
  bool nf_w_heavy = false;     // W-list surfaces carry > 1% of the near-field pairs
  int* job_counter = nullptr;  // persistent P2P work counters: S2M, S2L, near field
  // [0] set by kernels whose bounded waits ran out, zeroed per solve; [1]
  // collects [0] over the kfmm_evaluate_async calls since the last wait
  int* d_error = nullptr;
  long long wait_limit = kMbarSpinLimit;  // tries of the V-list tile-copy wait
  int had32_groups_per_block = 0;
  int p2p_grid = 0;            // resident P2P blocks on the device
  bool nf_minb5 = false;       // mixed near field with 5 resident blocks per SM
  kfmm_tuning tune{};          // launch choices asked for at creation (0 = automatic)
  int p2p_grid5 = 0;
  std::vector<GemmBatch> up_gemms, down_gemms;
  int *fft_nodes = nullptr, *ifft_nodes = nullptr;
  int n_fft = 0, n_ifft = 0;
  int *win = nullptr, *members = nullptr;
  int n_groups = 0;
  // mixed form: x-neighbour pairs of groups and the groups left single
  unsigned long long* pair_rows = nullptr;  // per pair window: rows holding an entry
  unsigned long long* single_rows = nullptr;
  int *pair_win = nullptr, *pair_members = nullptr, *single_win = nullptr,
      *single_members = nullptr;
  int n_pairs = 0, n_singles = 0;
  int pair_per_block = 0;
  // tensor-core Hadamard (mixed form) on the complete levels it takes: levels,
  // box -> node maps and the MMAs' B operands; the spectra, the error flag and
  // the unit counter are filled in at launch
  HadTcParams tc{};
  int n_tc_levels = 0;
  int* tc_counter = nullptr;
  // hybrid evaluation (kfmm_tuning.cpu_share_ppm): the host evaluates the
  // U lists of these target leaves; their GPU near-field jobs skip the U
  // entries.  Per leaf: its targets host_trg[tbeg, tbeg + tcnt) (original
  // indices) and its U entries host_u[ubeg, uend), each a range of host_src
  // (the original indices of one source leaf's points).
  struct HostLeaf {
    int tbeg, tcnt, ubeg, uend;
  };
  std::vector<HostLeaf> host_leaves;
  std::vector<int> host_trg, host_src;
  std::vector<int2> host_u;
  double host_pairs = 0.0;
  kfmm_stats stats{};
  int num_sms = 148;
  double* splitk = nullptr;   // split-K partial sums, shared by the level GEMMs
  size_t splitk_doubles = 0;
  bool timing = false;
  // timing marks (kfmm_enable_timing): 0 start, 1 S2M pairs done, 2 up done,
  // 3 forward FFT, 4 Hadamard, 5 inverse FFT (V done), 6 S2L (X done),
  // 7 down done, 8 near field done, 9 copy done
  static constexpr int kMarks = 10;
  cudaEvent_t ev[kMarks] = {};
  // kfmm_evaluate(_async): host->device copies and the target gather run on
  // `side`, the potentials' device->host copy on `d2h`, the solve on the
  // caller's stream; the events order successive solves (see
  // kfmm_evaluate_async)
  cudaStream_t side = nullptr, d2h = nullptr;
  cudaEvent_t ev_h2d_src = nullptr, ev_gsrc = nullptr, ev_gtrg = nullptr, ev_nf = nullptr,
              ev_d2h = nullptr;
};

namespace {

int fft_src_resident(int np, bool mixed);  // resident blocks per SM of the forward FFT

template <class T>
kfmm_status dalloc(kfmm_plan* p, T** ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) count = 1;
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, count * sizeof(T));
  if (e != cudaSuccess) {
    set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return KFMM_ERR_ALLOC;
  }
  p->allocs.push_back(v);
  *ptr = (T*)v;
  return KFMM_OK;
}

template <class T>
void dfree(kfmm_plan* p, T*& ptr) {
  if (!ptr) return;
  auto it = std::find(p->allocs.begin(), p->allocs.end(), (void*)ptr);
  if (it != p->allocs.end()) p->allocs.erase(it);
  cudaFree(ptr);
  ptr = nullptr;
}

template <class T>
kfmm_status upload(kfmm_plan* p, T** ptr, const std::vector<T>& h) {
  kfmm_status s = dalloc(p, ptr, h.size());
  if (s != KFMM_OK) return s;
  if (!h.empty()) KF_CUDA(cudaMemcpy(*ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return KFMM_OK;
}

#define KF_TRY(x)                  \
  do {                             \
    kfmm_status s_ = (x);          \
    if (s_ != KFMM_OK) return s_;  \
  } while (0)

// Split K when the launch would give fewer than two blocks per SM.  The split
// count minimises (waves of blocks) x (16-deep K slices per block) plus the
// split-K partial sums' traffic, 16 B per entry per split, counted at ~12.5 MB
// per slice-wave (the kernel's measured rate): one wave of half-K blocks
// beats two waves of third-K blocks.  Up to max(8, K / 64) ways unless the
// plan's tuning says otherwise (measured on 4M points: allowing 8 ways to the
// short-K products, K = P or Q, took 0.25 ms off the ellipsoid-surface solve
// at NP=4 and 0.05 ms off the uniform one at NP=6, against K / 64 ways).
constexpr int kSplitKAuto = 8;
void choose_split(const kfmm_plan* p, GemmBatch& g) {
  const int M = g.M, K = g.K;
  const int blocks = g.chunks * ((g.ncol + kGemmBN - 1) / kGemmBN);
  const int want = 2 * p->num_sms;
  g.nsplit = 1;
  g.ksplit = (K + kGemmBK - 1) / kGemmBK * kGemmBK;
  if (blocks >= want) return;
  double best = 1e300;
  const int smax = p->tune.splitk_max > 0 ? p->tune.splitk_max : std::max(kSplitKAuto, K / 64);
  for (int s = 1; s <= smax; ++s) {
    const int ks = ((K + s - 1) / s + kGemmBK - 1) / kGemmBK * kGemmBK;
    const int ns = (K + ks - 1) / ks;
    const double waves = std::ceil((double)blocks * ns / want);
    const double traffic = ns > 1 ? ns * 16.0 * M * (double)g.ncol / 12.5e6 : 0.0;
    const double cost = waves * (ks / kGemmBK) + traffic;
    if (cost < best) {
      best = cost;
      g.nsplit = ns;
      g.ksplit = ks;
    }
  }
}

// Split-K scratch the plan's level products need (doubles).
size_t splitk_need(const kfmm_plan* p) {
  size_t n = 0;
  for (const auto* v : {&p->up_gemms, &p->down_gemms})
    for (const GemmBatch& g : *v)
      if (g.nsplit > 1) n = std::max(n, (size_t)g.nsplit * g.ncol * g.M);
  return n;
}

// Split-K partial-sum buffer at least as large as the level products need.
kfmm_status ensure_splitk(kfmm_plan* p) {
  const size_t need = splitk_need(p);
  if (need > p->splitk_doubles) {
    dfree(p, p->splitk);
    KF_TRY(dalloc(p, &p->splitk, need));
    p->splitk_doubles = need;
  }
  return KFMM_OK;
}

// Kernel launches of one kfmm_run (kfmm_plan_stats.launches).
void count_launches(kfmm_plan* p) {
  int reduces = 0;
  for (const auto* v : {&p->up_gemms, &p->down_gemms})
    for (const GemmBatch& g : *v) reduces += g.nsplit > 1;
  p->stats.tensor_levels = p->n_tc_levels;
  p->stats.host_pairs = p->host_pairs;
  p->stats.launches = reduces + (p->n_s2m > 0) + (int)p->up_gemms.size() + (p->n_fft > 0) +
                      (p->prec == KFMM_MIXED ? (p->n_pairs > 0) + (p->n_singles > 0)
                                             : (p->n_groups > 0)) +
                      (p->n_tc_levels > 0) + (p->n_ifft > 0) + (p->n_s2l > 0) +
                      (int)p->down_gemms.size() + (p->n_nf > 0) +
                      (p->prec == KFMM_MIXED ? 0 : 1);  // the plain form's scatter pass
}

kfmm_status add_gemm(kfmm_plan* p, std::vector<GemmBatch>& out, const double* A, int M, int K,
                     const double* B, const std::vector<int>& boff, double* C,
                     const std::vector<int>& coff, const std::vector<double>* alpha,
                     double alpha_const, int accumulate) {
  if (boff.empty()) return KFMM_OK;
  // the GEMM kernel copies aligned pairs of doubles
  bool even = M % 2 == 0 && K % 2 == 0;
  for (int o : boff) even = even && o % 2 == 0;
  if (!even) {
    set_error("add_gemm: operator sizes and column offsets must be even");
    return KFMM_ERR_UNSUPPORTED;
  }
  GemmBatch g{};
  g.A = A;
  g.M = M;
  g.K = K;
  g.B = B;
  g.C = C;
  g.ncol = (int)boff.size();
  g.accumulate = accumulate;
  g.alpha_const = alpha_const;
  KF_TRY(upload(p, &g.boff, boff));
  KF_TRY(upload(p, &g.coff, coff));
  if (alpha) KF_TRY(upload(p, &g.alpha, *alpha));
  g.chunks = (M + kGemmRows - 1) / kGemmRows;
  g.mrows = ((M + g.chunks - 1) / g.chunks + 7) / 8 * 8;
  choose_split(p, g);
  p->stats.gemm_flops += 2.0 * M * (double)K * g.ncol;
  out.push_back(g);
  return KFMM_OK;
}

kfmm_status launch_gemms(const kfmm_plan* p, const std::vector<GemmBatch>& gs, cudaStream_t st) {
  for (const GemmBatch& b : gs) {
    GemmArgs a{b.A, b.M, b.K, b.ksplit, b.nsplit > 1 ? p->splitk : nullptr, b.B, b.boff, b.C,
               b.coff, b.alpha, b.alpha_const, b.ncol, b.accumulate};
    dim3 grid(b.chunks, (b.ncol + kGemmBN - 1) / kGemmBN, b.nsplit);
    if (b.accumulate)
      gemm_fp64_dmma_kernel<true><<<grid, kGemmThreads, kGemmSmemBytes, st>>>(a, b.mrows);
    else
      gemm_fp64_dmma_kernel<false><<<grid, kGemmThreads, kGemmSmemBytes, st>>>(a, b.mrows);
    KF_CHECK_LAUNCH("gemm_fp64_dmma_kernel");
    if (b.nsplit > 1) {
      const size_t total = (size_t)b.ncol * b.M;
      const int blocks = (int)std::min<size_t>((total + 255) / 256, 4 * (size_t)p->num_sms);
      gemm_splitk_reduce_kernel<<<blocks, 256, 0, st>>>(a, b.nsplit);
      KF_CHECK_LAUNCH("gemm_splitk_reduce_kernel");
    }
  }
  return KFMM_OK;
}

P2PParams p2p_params(const kfmm_plan* p, const P2PJob* jobs, const int* ent, double* out) {
  P2PParams q;
  q.jobs = jobs;
  q.entries = ent;
  q.src4 = p->src4;
  q.trg4 = p->trg4;
  q.ctr = p->ctr;
  q.src_beg = p->d_src_beg;
  q.src_num = p->d_src_num;
  q.uden = p->uden;
  q.dden = p->dden;
  q.sp_ue = p->d_sp_ue;
  q.sp_uc = p->d_sp_uc;
  q.sp_de = p->d_sp_de;
  q.sp_dc = p->d_sp_dc;
  q.out = out;
  q.P = p->P;
  q.Q = p->Q;
  return q;
}

P2PMixedParams p2p_mixed_params(const kfmm_plan* p, const P2PParams& q,
                                const int* out_perm = nullptr) {
  P2PMixedParams m;
  m.p = q;
  m.src4f = p->src4f;
  m.ctrf = p->ctrf;
  m.spf_ue = p->d_spf_ue;
  m.spf_de = p->d_spf_de;
  m.out_perm = out_perm;
  return m;
}

// The near field's output: the mixed form writes the potentials in original
// order directly (its kernel takes the target permutation), the plain form
// in leaf order for the scatter pass.
double* near_field_out(const kfmm_plan* p) {
  return p->prec == KFMM_MIXED ? p->pot_orig : p->pot_leaf;
}

FFTParams fft_params(const kfmm_plan* p) {
  FFTParams f{};
  f.np = p->np;
  f.P = p->P;
  f.F = p->F;
  f.nn = p->nn;
  f.depth = p->d_depth;
  f.surf_idx = p->d_surf_idx;
  f.surf_ijk = p->d_surf_ijk;
  f.cs = p->d_cs;
  f.sn = p->d_sn;
  return f;
}

kfmm_status validate_desc(const kfmm_tree_desc* d) {
  if (!d || d->num_nodes <= 0 || d->num_src <= 0 || d->num_trg <= 0 || !d->parent || !d->child ||
      !d->depth || !d->tag || !d->path || !d->src_beg || !d->src_num || !d->trg_beg ||
      !d->trg_num || !d->src_perm || !d->trg_perm || !d->u_ptr || !d->v_ptr || !d->w_ptr ||
      !d->x_ptr || (d->u_ptr[d->num_nodes] > 0 && !d->u_idx) ||
      (d->v_ptr[d->num_nodes] > 0 && !d->v_idx) || (d->w_ptr[d->num_nodes] > 0 && !d->w_idx) ||
      (d->x_ptr[d->num_nodes] > 0 && !d->x_idx)) {
    set_error("kfmm_plan_create: incomplete tree description");
    return KFMM_ERR_INVALID;
  }
  const int nn = d->num_nodes;
  for (int i = 0; i < nn; ++i) {
    if (d->child[i] != -1 && (d->child[i] <= i || d->child[i] + 8 > nn)) {
      set_error("kfmm_plan_create: child index out of range");
      return KFMM_ERR_INVALID;
    }
    if (d->depth[i] < 0 || d->depth[i] > 20) {
      set_error("kfmm_plan_create: depth out of range");
      return KFMM_ERR_INVALID;
    }
    if (d->child[i] == -1) {
      if (d->src_num[i] < 0 || d->src_beg[i] < 0 || d->src_beg[i] + d->src_num[i] > d->num_src ||
          d->trg_num[i] < 0 || d->trg_beg[i] < 0 || d->trg_beg[i] + d->trg_num[i] > d->num_trg) {
        set_error("kfmm_plan_create: leaf point range out of bounds");
        return KFMM_ERR_INVALID;
      }
    }
  }
  const int* ptrs[4] = {d->u_ptr, d->v_ptr, d->w_ptr, d->x_ptr};
  const int* idxs[4] = {d->u_idx, d->v_idx, d->w_idx, d->x_idx};
  for (int k = 0; k < 4; ++k) {
    if (ptrs[k][0] != 0) {
      set_error("kfmm_plan_create: list pointer must start at 0");
      return KFMM_ERR_INVALID;
    }
    for (int i = 0; i < nn; ++i)
      if (ptrs[k][i + 1] < ptrs[k][i]) {
        set_error("kfmm_plan_create: list pointers not monotone");
        return KFMM_ERR_INVALID;
      }
    for (int j = 0; j < ptrs[k][nn]; ++j)
      if (idxs[k][j] < 0 || idxs[k][j] >= nn) {
        set_error("kfmm_plan_create: list entry out of range");
        return KFMM_ERR_INVALID;
      }
  }
  // permutations: every original index exactly once (the point reorders
  // scatter through their inverses)
  for (int pass = 0; pass < 2; ++pass) {
    const int n = pass ? d->num_trg : d->num_src;
    const int* perm = pass ? d->trg_perm : d->src_perm;
    std::vector<char> seen(n, 0);
    for (int i = 0; i < n; ++i) {
      if (perm[i] < 0 || perm[i] >= n || seen[perm[i]]) {
        set_error(pass ? "kfmm_plan_create: target permutation is not a permutation"
                       : "kfmm_plan_create: source permutation is not a permutation");
        return KFMM_ERR_INVALID;
      }
      seen[perm[i]] = 1;
    }
  }
  return KFMM_OK;
}

// Key of a position within one level (coordinates < 2^21: plans accept depth <= 21).
inline long long key_of(int x, int y, int z) {
  return (long long)x | ((long long)y << 21) | ((long long)z << 42);
}

constexpr double kCostClassWidth = 1.05;  // cost ratio spanned by one job-order class

// The near field's jobs: each target leaf's targets in chunks of 32 * rows
// (rows: the tuning's job_rows, else 4 for mixed plans whose W-list surfaces
// carry more than 1% of the pairs, else 6), ordered largest first by cost
// class (target slots x sources, in classes 5% wide); within a class the
// jobs keep their tree order, so warps working at the same time read
// neighbouring leaves' sources and the L2 cache serves the repeats (4M
// points, NP=6 uniform / NP=4 ellipsoid surface, mixed near field: classes
// 25% wide 4.44 / 2.32 ms, 12% 4.39 / 2.28, 5% 4.39 / 2.27, 100% 4.48 /
// 2.50).  The
// mixed near field runs with 5 resident blocks per SM on the same clouds
// (or when the tuning says so).  Measured on 4M points on the ellipsoid
// surface, NP=4, 256 per box: 2.32 ms against 2.50 ms with 6 blocks and 6
// rows; uniform clouds keep 6 and 6 (4.42 ms, against 4.70 ms with 4 rows).
kfmm_status build_nf_jobs(kfmm_plan* p) {
  int rows = p->prec == KFMM_MIXED && p->nf_w_heavy ? 4 : kMaxSlots;
  if (p->tune.job_rows > 0) rows = std::min(p->tune.job_rows, kMaxSlots);
  const int chunk = 32 * rows;
  std::vector<P2PJob> jobs;
  std::vector<double> ns;
  for (size_t l = 0; l < p->nf_leaf.size(); ++l) {
    const P2PJob& L = p->nf_leaf[l];
    for (int c = 0; c < L.tcnt; c += chunk) {
      P2PJob j = L;
      j.tbeg = L.tbeg + c;
      j.tcnt = std::min(chunk, L.tcnt - c);
      j.out = L.out + c;
      jobs.push_back(j);
      ns.push_back(p->nf_leaf_ns[l]);
    }
  }
  std::vector<std::pair<double, int>> key(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) {
    const double cost = std::max(1.0, ns[j] * ((jobs[j].tcnt + 31) / 32));
    key[j] = {-std::floor(std::log(cost) / std::log(kCostClassWidth)), (int)j};
  }
  std::stable_sort(key.begin(), key.end(),
                   [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
                     return a.first < b.first;
                   });
  std::vector<P2PJob> out(jobs.size());
  p->nf_class.resize(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) {
    out[j] = jobs[key[j].second];
    p->nf_class[j] = (float)key[j].first;
  }
  dfree(p, p->nf_jobs);
  KF_TRY(upload(p, &p->nf_jobs, out));
  p->n_nf = (int)out.size();
  p->nf_minb5 = p->prec == KFMM_MIXED &&
                (p->tune.nf_blocks == 5 || (p->tune.nf_blocks == 0 && p->nf_w_heavy));
  return KFMM_OK;
}

// Mixed Hadamard launch shape: one CTA per SM over (chunks x frequency
// blocks).  A chunk holds k windows per warp (every warp the same count, so
// none idles at the end of its CTA); k minimises the span ceil(CTAs / SMs) x
// (k + 0.1), the 0.1 standing for a CTA's translation-tile load, unless the
// tuning fixes k.
void set_had_blocks(kfmm_plan* p) {
  const int nfb = p->Fpad / kFB;
  auto per_block = [&](int items, int warps) {
    if (p->tune.had_windows > 0) return warps * std::min(p->tune.had_windows, 8);
    int pick = warps;
    double best = 1e300;
    for (int k = 1; k <= 8; ++k) {
      const long long ctas = (long long)((items + warps * k - 1) / (warps * k)) * nfb;
      const double span = std::ceil((double)ctas / p->num_sms) * (k + 0.1);
      if (span < best) {
        best = span;
        pick = warps * k;
      }
    }
    return pick;
  };
  p->had32_groups_per_block = per_block(p->n_singles, kHad32Warps);
  p->pair_per_block = per_block(p->n_pairs, kHadPairWarps);
}

kfmm_status check_tuning(const kfmm_tuning* t) {
  if (t && (t->nf_blocks < 0 || t->nf_blocks > 6 || (t->nf_blocks > 0 && t->nf_blocks < 5) ||
            t->job_rows < 0 || t->job_rows > kMaxSlots || t->had_windows < 0 ||
            t->had_windows > 8 || t->splitk_max < 0 || t->had_tensor < 0 ||
            t->had_tensor > 2 || t->cpu_share_ppm < 0 || t->cpu_share_ppm > 1000000)) {
    set_error("kfmm_tuning: tuning value out of range");
    return KFMM_ERR_INVALID;
  }
  return KFMM_OK;
}

kfmm_status build_plan(kfmm_plan* p, const kfmm_tree_desc* d, const kfmm_operator_set* user) {
  const int nn = d->num_nodes, np = p->np;
  {
    int dev = 0;
    KF_CUDA(cudaGetDevice(&dev));
    KF_CUDA(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev));
  }
  Operators op = operators_for(np);
  if (user) {
    const size_t P0 = op.P, Q0 = op.Q;
    if (!user->uc2ue || !user->ue2uc || !user->dc2de || !user->de2dc) {
      set_error("kfmm_plan_create_with_operators: uc2ue, ue2uc, dc2de and de2dc are required");
      return KFMM_ERR_INVALID;
    }
    op.uc2ue.assign(user->uc2ue, user->uc2ue + P0 * Q0);
    op.ue2uc.assign(user->ue2uc, user->ue2uc + 8 * P0 * Q0);
    op.dc2de.assign(user->dc2de, user->dc2de + P0 * P0);
    op.de2dc.assign(user->de2dc, user->de2dc + 8 * P0 * P0);
    if (user->ue2dc) op.ue2dc.assign(user->ue2dc, user->ue2dc + (size_t)343 * 2 * op.F);
  }
  Surfaces S;
  make_surfaces(np, &S);
  const int P = S.P, Q = S.Q, F = S.F;
  p->P = P;
  p->Q = Q;
  p->F = F;
  p->nn = nn;
  p->ns = d->num_src;
  p->nt = d->num_trg;
  auto is_leaf = [&](int i) { return d->child[i] == -1; };
  auto has_src = [&](int i) { return (d->tag[i] & kSrcTag) != 0; };
  auto has_trg = [&](int i) { return (d->tag[i] & kTrgTag) != 0; };
  int maxd = 0;
  for (int i = 0; i < nn; ++i) maxd = std::max(maxd, d->depth[i]);
  p->maxdepth = maxd;
  if (maxd > 21) {  // key_of packs 21 bits per coordinate
    set_error("kfmm_plan_create: trees deeper than 21 levels are not supported");
    return KFMM_ERR_UNSUPPORTED;
  }

  // --- tree arrays
  std::vector<double4> ctr(nn);
  for (int i = 0; i < nn; ++i) {
    double c[3];
    for (int k = 0; k < 3; ++k) c[k] = -1.0 + (2.0 * 1.0) * (d->path[3 * i + k] + 0.5) / double(1 << d->depth[i]);
    ctr[i] = make_double4(c[0], c[1], c[2], 1.0 / double(1 << d->depth[i]));
  }
  KF_TRY(upload(p, &p->ctr, ctr));
  {
    std::vector<float4> cf(nn);
    for (int i = 0; i < nn; ++i)
      cf[i] = make_float4((float)ctr[i].x, (float)ctr[i].y, (float)ctr[i].z, (float)ctr[i].w);
    KF_TRY(upload(p, &p->ctrf, cf));
  }
  KF_TRY(upload(p, &p->d_depth, std::vector<int>(d->depth, d->depth + nn)));
  KF_TRY(upload(p, &p->d_src_beg, std::vector<int>(d->src_beg, d->src_beg + nn)));
  KF_TRY(upload(p, &p->d_src_num, std::vector<int>(d->src_num, d->src_num + nn)));
  KF_TRY(upload(p, &p->d_src_perm, std::vector<int>(d->src_perm, d->src_perm + d->num_src)));
  KF_TRY(upload(p, &p->d_trg_perm, std::vector<int>(d->trg_perm, d->trg_perm + d->num_trg)));
  {
    std::vector<int> si(d->num_src), ti(d->num_trg);
    for (int i = 0; i < d->num_src; ++i) si[d->src_perm[i]] = i;
    for (int i = 0; i < d->num_trg; ++i) ti[d->trg_perm[i]] = i;
    KF_TRY(upload(p, &p->d_src_inv, si));
    KF_TRY(upload(p, &p->d_trg_inv, ti));
    if (p->prec == KFMM_MIXED) {
      // each source's leaf, by original index (the source gather reads it
      // beside the coordinates, coalesced)
      std::vector<int> leaf_of(d->num_src, 0);
      for (int i = 0; i < nn; ++i)
        if (d->child[i] == -1)
          for (int k = 0; k < d->src_num[i]; ++k) leaf_of[d->src_perm[d->src_beg[i] + k]] = i;
      KF_TRY(upload(p, &p->d_src_leaf, leaf_of));
      KF_TRY(dalloc(p, &p->src4f, d->num_src));
    }
  }

  // --- operators and surfaces
  KF_TRY(upload(p, &p->d_uc2ue, op.uc2ue));
  KF_TRY(upload(p, &p->d_ue2uc, op.ue2uc));  // Q x 8P, the 8 blocks side by side
  if (p->prec == KFMM_MIXED) {
    // M2M as one operator: uden_parent = 2^-d UC2UE (sum_c UE2UC_c 2^(d+1) uden_c)
    // = 2 (UC2UE UE2UC) [uden_c] (fmm/omp_sse_block.cc:103-155), the product
    // formed once here in FP64 (column-major, P x 8P)
    std::vector<double> m((size_t)P * 8 * P, 0.0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < 8 * P; ++k)
      for (int q = 0; q < Q; ++q) {
        const double u = op.ue2uc[(size_t)k * Q + q];
        for (int i = 0; i < P; ++i) m[(size_t)k * P + i] += op.uc2ue[(size_t)q * P + i] * u;
      }
    KF_TRY(upload(p, &p->d_m2m, m));
  }
  KF_TRY(upload(p, &p->d_dc2de, op.dc2de));
  {
    std::vector<double> st((size_t)8 * P * P);  // 8P x P: the 8 blocks stacked
    for (int c = 0; c < 8; ++c)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i)
          st[(size_t)j * 8 * P + c * P + i] = op.de2dc[(size_t)c * P * P + (size_t)j * P + i];
    KF_TRY(upload(p, &p->d_de2dc_stack, st));
  }
  p->Fpad = (F + kFB - 1) / kFB * kFB;
  p->cplx = p->prec == KFMM_MIXED ? sizeof(float2) : sizeof(double2);
  // Offsets with |delta|_inf <= 1 are adjacent boxes, never V-list pairs: the
  // table keeps zeros there whatever the supplied operators hold, and the
  // Hadamard kernels skip them.
  auto adjacent = [](int id) {
    return std::abs(id % 7 - 3) <= 1 && std::abs(id / 7 % 7 - 3) <= 1 && std::abs(id / 49 - 3) <= 1;
  };
  if (p->prec == KFMM_MIXED) {
    // [fb][343][32]: one contiguous 87,808-byte tile per block of 32
    // frequencies (hadamard_fp32_kernel)
    const int nfb = p->Fpad / kFB;
    std::vector<float2> tr((size_t)nfb * 343 * kFB, make_float2(0.f, 0.f));
    for (int id = 0; id < 343; ++id)
      for (int f = 0; f < F && !adjacent(id); ++f)
        tr[((size_t)(f / kFB) * 343 + id) * kFB + f % kFB] =
            make_float2((float)op.ue2dc[2 * ((size_t)id * F + f)],
                        (float)op.ue2dc[2 * ((size_t)id * F + f) + 1]);
    float2* d = nullptr;
    KF_TRY(upload(p, &d, tr));
    p->d_trans = d;
  } else {
    std::vector<double2> tr((size_t)343 * p->Fpad, make_double2(0.0, 0.0));
    for (int id = 0; id < 343; ++id)
      for (int f = 0; f < F && !adjacent(id); ++f)
        tr[(size_t)id * p->Fpad + f] = make_double2(op.ue2dc[2 * ((size_t)id * F + f)],
                                                    op.ue2dc[2 * ((size_t)id * F + f) + 1]);
    double2* d = nullptr;
    KF_TRY(upload(p, &d, tr));
    p->d_trans = d;
  }
  KF_TRY(upload(p, &p->d_sp_ue, S.ue));
  KF_TRY(upload(p, &p->d_sp_uc, S.uc));
  KF_TRY(upload(p, &p->d_sp_de, S.de));
  KF_TRY(upload(p, &p->d_sp_dc, S.dc));
  KF_TRY(upload(p, &p->d_spf_ue, std::vector<float>(S.ue.begin(), S.ue.end())));
  KF_TRY(upload(p, &p->d_spf_de, std::vector<float>(S.de.begin(), S.de.end())));
  {
    const int n = 2 * np;
    std::vector<double> cs(n), sn(n);
    for (int m = 0; m < n; ++m) {
      cs[m] = std::cos(2.0 * M_PI * m / n);
      sn[m] = std::sin(2.0 * M_PI * m / n);
    }
    KF_TRY(upload(p, &p->d_cs, cs));
    KF_TRY(upload(p, &p->d_sn, sn));
    std::vector<int> sidx(np * np * np, -1), sijk;
    int cnt = 0;
    for (int i = 0; i < np; i++)
      for (int j = 0; j < np; j++)
        for (int k = 0; k < np; k++)
          if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
            sidx[(i * np + j) * np + k] = cnt++;
            sijk.push_back(i);
            sijk.push_back(j);
            sijk.push_back(k);
          }
    KF_TRY(upload(p, &p->d_surf_idx, sidx));
    KF_TRY(upload(p, &p->d_surf_ijk, sijk));
  }

  // --- work arrays
  KF_TRY(dalloc(p, &p->o_sx, p->ns));
  KF_TRY(dalloc(p, &p->o_sy, p->ns));
  KF_TRY(dalloc(p, &p->o_sz, p->ns));
  KF_TRY(dalloc(p, &p->o_w, p->ns));
  KF_TRY(dalloc(p, &p->o_tx, p->nt));
  KF_TRY(dalloc(p, &p->o_ty, p->nt));
  KF_TRY(dalloc(p, &p->o_tz, p->nt));
  if (p->prec != KFMM_MIXED) KF_TRY(dalloc(p, &p->src4, p->ns));  // mixed kernels read src4f
  KF_TRY(dalloc(p, &p->trg4, p->nt));
  KF_TRY(dalloc(p, &p->pot_leaf, p->nt));
  KF_TRY(dalloc(p, &p->pot_orig, p->nt));
  KF_TRY(dalloc(p, &p->uden, (size_t)nn * P));
  KF_TRY(dalloc(p, &p->dchk, (size_t)nn * P));
  KF_TRY(dalloc(p, &p->dden, (size_t)nn * P));
  {
    unsigned char *a = nullptr, *b = nullptr;
    KF_TRY(dalloc(p, &a, (size_t)nn * p->Fpad * p->cplx));
    KF_TRY(dalloc(p, &b, (size_t)nn * p->Fpad * p->cplx));
    p->spec = a;
    p->effv = b;
  }
  KF_CUDA(cudaMemset(p->uden, 0, sizeof(double) * (size_t)nn * P));
  KF_CUDA(cudaMemset(p->dden, 0, sizeof(double) * (size_t)nn * P));
  KF_CUDA(cudaMemset(p->dchk, 0, sizeof(double) * (size_t)nn * P));
  KF_CUDA(cudaMemset(p->spec, 0, p->cplx * (size_t)nn * p->Fpad));
  KF_CUDA(cudaMemset(p->effv, 0, p->cplx * (size_t)nn * p->Fpad));

  const int chunk = 32 * kMaxSlots;  // targets per S2M / S2L job (near field: build_nf_jobs)
  auto add_chunks = [&](std::vector<P2PJob>& jobs, int tnode, int tkind, int tbeg0, int tcount,
                        int ebeg, int eend, int out0, int mode) {
    for (int c = 0; c < tcount; c += chunk) {
      P2PJob j;
      j.tnode = tnode;
      j.tkind = tkind;
      j.tbeg = tbeg0 + c;
      j.tcnt = std::min(chunk, tcount - c);
      j.ebeg = ebeg;
      j.eend = eend;
      j.out = out0 + c;
      j.mode = mode;
      jobs.push_back(j);
    }
  };
  auto src_count = [&](int ent) -> int {
    int kind = ent >> 28, node = ent & 0x0fffffff;
    return kind == 0 ? d->src_num[node] : P;
  };
  // For the persistent P2P kernel: largest first, by cost class (target slots
  // x sources, in classes 5% wide); within a class the jobs keep their tree
  // order, so warps working at the same time read neighbouring leaves' sources
  // and the L2 cache serves the repeats.
  auto order_jobs = [&](std::vector<P2PJob>& jobs, const std::vector<int>& ent,
                        std::vector<float>* class_out = nullptr) {
    std::vector<std::pair<double, int>> key(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
      double ns = 0;
      for (int k = jobs[j].ebeg; k < jobs[j].eend; ++k) ns += src_count(ent[k]);
      const double cost = std::max(1.0, ns * ((jobs[j].tcnt + 31) / 32));
      key[j] = {-std::floor(std::log(cost) / std::log(kCostClassWidth)), (int)j};
    }
    std::stable_sort(key.begin(), key.end(),
                     [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
                       return a.first < b.first;
                     });
    std::vector<P2PJob> out(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) out[j] = jobs[key[j].second];
    jobs.swap(out);
    if (class_out) {
      class_out->resize(jobs.size());
      for (size_t j = 0; j < jobs.size(); ++j) (*class_out)[j] = (float)key[j].first;
    }
  };

  // --- up: S2M jobs + UC2UE GEMM, then M2M per level
  {
    std::vector<P2PJob> jobs;
    std::vector<int> ent, boff, coff;
    std::vector<double> alpha;
    int slot = 0;
    for (int i = 0; i < nn; ++i) {
      if (!is_leaf(i) || !has_src(i)) continue;
      int e = (int)ent.size();
      ent.push_back(i);
      add_chunks(jobs, i, 1, 0, Q, e, e + 1, slot * Q, 0);
      p->stats.s2m_pairs += (double)Q * d->src_num[i];
      boff.push_back(slot * Q);
      coff.push_back(i * P);
      alpha.push_back(std::ldexp(1.0, -d->depth[i]));
      ++slot;
    }
    order_jobs(jobs, ent);
    p->n_s2m = (int)jobs.size();
    KF_TRY(upload(p, &p->s2m_jobs, jobs));
    KF_TRY(upload(p, &p->s2m_ent, ent));
    KF_TRY(dalloc(p, &p->chk_up, (size_t)std::max(slot, 1) * Q));
    KF_TRY(add_gemm(p, p->up_gemms, p->d_uc2ue, P, Q, p->chk_up, boff, p->uden, coff, &alpha, 0, 0));
    int maxpar = 1;
    std::vector<std::vector<int>> par(maxd + 1);
    for (int i = 0; i < nn; ++i)
      if (!is_leaf(i) && has_src(i)) par[d->depth[i]].push_back(i);
    for (int dd = 0; dd <= maxd; ++dd) maxpar = std::max(maxpar, (int)par[dd].size());
    if (p->prec != KFMM_MIXED) KF_TRY(dalloc(p, &p->chk_m, (size_t)maxpar * Q));
    // Equivalent densities of depth 0 and 1 nodes are never read: V lists
    // start at depth 2 and W-list nodes lie below a depth >= 1 leaf's
    // colleagues, so at depth >= 2.  M2M stops at parents of depth 2.
    for (int dd = maxd - 1; dd >= 2; --dd) {
      if (par[dd].empty()) continue;
      std::vector<int> b1, c1, b2, c2;
      for (size_t k = 0; k < par[dd].size(); ++k) {
        b1.push_back(d->child[par[dd][k]] * P);
        c1.push_back((int)k * Q);
        b2.push_back((int)k * Q);
        c2.push_back(par[dd][k] * P);
      }
      if (p->prec == KFMM_MIXED) {
        // one product of the fused operator: half the flops of the two
        // (P x 8P against Q x 8P + P x Q), no intermediate check potentials
        KF_TRY(add_gemm(p, p->up_gemms, p->d_m2m, P, 8 * P, p->uden, b1, p->uden, c2, nullptr,
                        2.0, 0));
      } else {
        KF_TRY(add_gemm(p, p->up_gemms, p->d_ue2uc, Q, 8 * P, p->uden, b1, p->chk_m, c1, nullptr,
                        std::ldexp(1.0, dd + 1), 0));
        KF_TRY(add_gemm(p, p->up_gemms, p->d_uc2ue, P, Q, p->chk_m, b2, p->uden, c2, nullptr,
                        std::ldexp(1.0, -dd), 0));
      }
    }
  }

  // --- V list
  {
    std::vector<int> fn, ifn;
    for (int i = 0; i < nn; ++i)
      if (has_src(i) && d->depth[i] >= 2) fn.push_back(i);
    for (int i = 0; i < nn; ++i)
      if (has_trg(i) && d->v_ptr[i + 1] > d->v_ptr[i]) ifn.push_back(i);
    p->n_fft = (int)fn.size();
    p->n_ifft = (int)ifn.size();
    KF_TRY(upload(p, &p->fft_nodes, fn));
    KF_TRY(upload(p, &p->ifft_nodes, ifn));
    std::vector<std::unordered_map<long long, int>> at(maxd + 1);
    for (int i = 0; i < nn; ++i)
      at[d->depth[i]][key_of(d->path[3 * i], d->path[3 * i + 1], d->path[3 * i + 2])] = i;
    std::vector<int> win, mem, gparent;
    for (int pn = 0; pn < nn; ++pn) {
      if (is_leaf(pn)) continue;
      int m[8], any = 0;
      for (int c = 0; c < 8; ++c) {
        int ch = d->child[pn] + c;
        m[c] = (has_trg(ch) && d->v_ptr[ch + 1] > d->v_ptr[ch]) ? ch : -1;
        any |= m[c] >= 0;
      }
      if (!any) continue;
      const int cd = d->depth[pn] + 1, lim = 1 << cd;
      int w[216];
      for (int wz = 0; wz < 6; ++wz)
        for (int wy = 0; wy < 6; ++wy)
          for (int wx = 0; wx < 6; ++wx) {
            int x = 2 * d->path[3 * pn] - 2 + wx, y = 2 * d->path[3 * pn + 1] - 2 + wy,
                z = 2 * d->path[3 * pn + 2] - 2 + wz;
            int id = -1;
            if (x >= 0 && y >= 0 && z >= 0 && x < lim && y < lim && z < lim) {
              auto it = at[cd].find(key_of(x, y, z));
              if (it != at[cd].end() && has_src(it->second)) id = it->second;
            }
            w[wx + 6 * wy + 36 * wz] = id;
          }
      // The window must reproduce every member's V list exactly.
      for (int c = 0; c < 8; ++c) {
        if (m[c] < 0) continue;
        std::vector<int> fromwin;
        for (int q = 0; q < 216; ++q) {
          int dx = q % 6 - 2 - (c >> 2), dy = (q / 6) % 6 - 2 - ((c >> 1) & 1), dz = q / 36 - 2 - (c & 1);
          if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) >= 2 && w[q] >= 0)
            fromwin.push_back(w[q]);
        }
        std::sort(fromwin.begin(), fromwin.end());
        std::vector<int> vl(d->v_idx + d->v_ptr[m[c]], d->v_idx + d->v_ptr[m[c] + 1]);
        std::sort(vl.begin(), vl.end());
        if (fromwin != vl) {
          set_error("kfmm_plan_create: V list of node " + std::to_string(m[c]) +
                    " is not the same-depth far part of its parent's neighbourhood");
          return KFMM_ERR_INVALID;
        }
        p->stats.v_pairs += (double)vl.size();
        p->stats.hadamard_cmacs += (double)vl.size() * F;
      }
      win.insert(win.end(), w, w + 216);
      mem.insert(mem.end(), m, m + 8);
      gparent.push_back(pn);
    }
    p->n_groups = (int)mem.size() / 8;
    // Mixed form: levels whose boxes are all present go to the tensor-core
    // kernel (hadamard_tc_kernel); it reads box -> node maps of the level
    std::vector<char> tc_level(maxd + 1, 0);
    // (only when the tuning asks for it: on B200 the CUDA-core kernels below
    // measured faster, 1.53 against 3.21 ms at 4M points, NP=6: with 16
    // output columns per frequency each MMA streams its whole A tile for 16
    // columns, a sixteenth of the tensor cores' rate)
    if (p->prec == KFMM_MIXED && p->n_groups && p->tune.had_tensor == 2) {
      std::vector<int> groups_at(maxd + 1, 0);
      for (int g = 0; g < p->n_groups; ++g) ++groups_at[d->depth[gparent[g]] + 1];
      for (int cd = 2; cd <= std::min(maxd, 7); ++cd) {
        const long long nb = 1ll << (3 * cd);
        if (groups_at[cd] == 0 || (long long)at[cd].size() != nb) continue;
        if (p->n_tc_levels == kTcMaxLevels) break;
        tc_level[cd] = 1;
        const int n = 1 << cd;
        std::vector<int> sm(nb, -1), tm(nb, -1);
        for (const auto& kv : at[cd]) {
          const int node = kv.second;
          const int x = d->path[3 * node], y = d->path[3 * node + 1], z = d->path[3 * node + 2];
          const size_t q = ((size_t)z * n + y) * n + x;
          if (has_src(node)) sm[q] = node;
          if (has_trg(node) && d->v_ptr[node + 1] > d->v_ptr[node]) tm[q] = node;
        }
        TcLevel& L = p->tc.lv[p->n_tc_levels++];
        L.n = n;
        L.ntx = (n / 2 + kTcGX - 1) / kTcGX;
        L.nty = (n / 2 + kTcGY - 1) / kTcGY;
        L.col0 = p->tc.cols;
        p->tc.cols += L.ntx * L.nty;
        int* dm = nullptr;
        KF_TRY(upload(p, &dm, sm));
        L.srcmap = dm;
        KF_TRY(upload(p, &dm, tm));
        L.trgmap = dm;
      }
      if (p->n_tc_levels) {
        // B operands per frequency, in the order the kernel issues its MMAs
        // (plane wz, row pair q, MMA i of the pair): for MMA i its two K
        // chunks (window row, box pair); per chunk the K elements re S(wx),
        // im S(wx), re S(wx+1), im S(wx+1); columns n = 2 c + (re | im of E_c).
        // B is stored K-major as core matrices [n block][K chunk][8 rows][16 B]
        // (LBO 128 B, SBO 256 B), TF32 hi = rn(t), lo = rn(t - hi).
        auto tf32 = [](float x) {
          unsigned u;
          std::memcpy(&u, &x, 4);
          u = (u + 0x1000u) & 0xffffe000u;  // nearest, ties away from zero
          float r;
          std::memcpy(&r, &u, 4);
          return r;
        };
        std::vector<float> bt((size_t)F * 2 * kTcMma * 128, 0.f);
        for (int f = 0; f < F; ++f)
          for (int j = 0; j < kTcMma; ++j) {
            const int wz = j / 9, q = (j % 9) / 3, i = j % 3;
            for (int kc = 0; kc < 2; ++kc) {
              // (row, box pair) of this chunk: i 0 -> (2q, 0), (2q, 1); i 1 -> (2q, 2),
              // (2q + 1, 0); i 2 -> (2q + 1, 1), (2q + 1, 2)
              const int slot = 2 * i + kc;
              const int wy = 2 * q + slot / 3, pr = slot % 3;
              for (int nrow = 0; nrow < 16; ++nrow) {
                const int c = nrow >> 1, o = nrow & 1;
                for (int e = 0; e < 4; ++e) {
                  const int wx = 2 * pr + (e >> 1), part = e & 1;
                  const int dx = wx - 2 - (c >> 2), dy = wy - 2 - ((c >> 1) & 1),
                            dz = wz - 2 - (c & 1);
                  const int id = (dx + 3) + 7 * (dy + 3) + 49 * (dz + 3);
                  float tr = 0.f, ti = 0.f;
                  if (!adjacent(id)) {
                    tr = (float)op.ue2dc[2 * ((size_t)id * F + f)];
                    ti = (float)op.ue2dc[2 * ((size_t)id * F + f) + 1];
                  }
                  const float v = part == 0 ? (o == 0 ? tr : ti) : (o == 0 ? -ti : tr);
                  const float hi = tf32(v), lo = tf32(v - hi);
                  const size_t at0 = (((size_t)f * 2) * kTcMma + j) * 128 +
                                     ((nrow >> 3) * 2 + kc) * 32 + (nrow & 7) * 4 + e;
                  bt[at0] = hi;
                  bt[at0 + (size_t)kTcMma * 128] = lo;
                }
              }
            }
          }
        float* db = nullptr;
        KF_TRY(upload(p, &db, bt));
        p->tc.btab = (const unsigned char*)db;
        p->tc.nn = nn;
        p->tc.F = F;
        p->tc.nlevels = p->n_tc_levels;
        KF_TRY(dalloc(p, &p->tc_counter, 1));
      }
    }
    if (p->prec == KFMM_MIXED && p->n_groups) {
      // pair groups whose parents are x-neighbours (x even, x + 1): their
      // windows share 4 of 6 x-positions and form one 8 x 6 x 6 window
      // per parent depth: parent position -> group
      std::vector<std::unordered_map<long long, int>> gat(maxd + 1);
      for (int g = 0; g < p->n_groups; ++g) {
        const int pn = gparent[g];
        gat[d->depth[pn]][key_of(d->path[3 * pn], d->path[3 * pn + 1], d->path[3 * pn + 2])] = g;
      }
      std::vector<char> used(p->n_groups, 0);
      for (int g = 0; g < p->n_groups; ++g) used[g] = tc_level[d->depth[gparent[g]] + 1];
      std::vector<int> pwin, pmem, swin, smem;
      for (int g = 0; g < p->n_groups; ++g) {
        if (used[g]) continue;
        const int pn = gparent[g];
        int partner = -1;
        if ((d->path[3 * pn] & 1) == 0) {
          auto& level = gat[d->depth[pn]];
          auto it = level.find(key_of(d->path[3 * pn] + 1, d->path[3 * pn + 1], d->path[3 * pn + 2]));
          if (it != level.end() && !used[it->second]) partner = it->second;
        }
        used[g] = 1;
        if (partner < 0) {
          swin.insert(swin.end(), &win[(size_t)g * 216], &win[(size_t)g * 216] + 216);
          smem.insert(smem.end(), &mem[(size_t)g * 8], &mem[(size_t)g * 8] + 8);
          continue;
        }
        used[partner] = 1;
        int w8[288];
        for (int q = 0; q < 36; ++q)
          for (int x = 0; x < 8; ++x) {
            const int a = x < 6 ? win[(size_t)g * 216 + q * 6 + x] : -2;
            const int b = x >= 2 ? win[(size_t)partner * 216 + q * 6 + x - 2] : -2;
            if (a != -2 && b != -2 && a != b) {
              set_error("kfmm_plan_create: neighbouring V-list windows disagree");
              return KFMM_ERR_INVALID;
            }
            w8[q * 8 + x] = a != -2 ? a : b;
          }
        pwin.insert(pwin.end(), w8, w8 + 288);
        pmem.insert(pmem.end(), &mem[(size_t)g * 8], &mem[(size_t)g * 8] + 8);
        pmem.insert(pmem.end(), &mem[(size_t)partner * 8], &mem[(size_t)partner * 8] + 8);
      }
      p->n_pairs = (int)pmem.size() / 16;
      p->n_singles = (int)smem.size() / 8;
      KF_TRY(upload(p, &p->pair_win, pwin));
      {
        std::vector<unsigned long long> prow(pmem.size() / 16, 0ull);
        for (size_t g = 0; g < prow.size(); ++g)
          for (int r = 0; r < 36; ++r)
            for (int x = 0; x < 8; ++x)
              if (pwin[g * 288 + r * 8 + x] >= 0) prow[g] |= 1ull << r;
        KF_TRY(upload(p, &p->pair_rows, prow));
        std::vector<unsigned long long> srow(smem.size() / 8, 0ull);
        for (size_t g = 0; g < srow.size(); ++g)
          for (int r = 0; r < 36; ++r)
            for (int x = 0; x < 6; ++x)
              if (swin[g * 216 + r * 6 + x] >= 0) srow[g] |= 1ull << r;
        KF_TRY(upload(p, &p->single_rows, srow));
      }
      KF_TRY(upload(p, &p->pair_members, pmem));
      KF_TRY(upload(p, &p->single_win, swin));
      KF_TRY(upload(p, &p->single_members, smem));
    }
    KF_TRY(upload(p, &p->win, win));
    KF_TRY(upload(p, &p->members, mem));
    p->stats.spectra_bytes = 16.0 * F * ((double)fn.size() + (double)ifn.size());
  }

  // --- X list S2L jobs
  {
    std::vector<P2PJob> jobs;
    std::vector<int> ent;
    for (int t = 0; t < nn; ++t) {
      if (!has_trg(t)) continue;
      int xb = d->x_ptr[t], xe = d->x_ptr[t + 1];
      if (xe == xb) continue;
      if (is_leaf(t) && d->trg_num[t] < P) continue;  // handled directly in the near field
      int e0 = (int)ent.size();
      int ns = 0;
      for (int k = xb; k < xe; ++k) {
        ent.push_back(d->x_idx[k]);
        ns += d->src_num[d->x_idx[k]];
      }
      add_chunks(jobs, t, 2, 0, P, e0, (int)ent.size(), t * P, 1);
      p->stats.s2l_pairs += (double)P * ns;
    }
    order_jobs(jobs, ent);
    p->n_s2l = (int)jobs.size();
    KF_TRY(upload(p, &p->s2l_jobs, jobs));
    KF_TRY(upload(p, &p->s2l_ent, ent));
  }

  // --- down: L2L per level
  for (int dd = 2; dd <= maxd; ++dd) {
    if (dd >= 3) {
      std::vector<int> b1, c1;
      for (int i = 0; i < nn; ++i)
        if (d->depth[i] == dd - 1 && !is_leaf(i) && has_trg(i)) {
          b1.push_back(i * P);
          c1.push_back(d->child[i] * P);
        }
      KF_TRY(add_gemm(p, p->down_gemms, p->d_de2dc_stack, 8 * P, P, p->dden, b1, p->dchk, c1,
                      nullptr, std::ldexp(1.0, dd - 1), 1));
    }
    std::vector<int> b2;
    for (int i = 0; i < nn; ++i)
      if (d->depth[i] == dd && has_trg(i)) b2.push_back(i * P);
    KF_TRY(add_gemm(p, p->down_gemms, p->d_dc2de, P, P, p->dchk, b2, p->dden, b2, nullptr,
                    std::ldexp(1.0, -dd), 0));
  }

  // --- near field: U + W + direct X + L2T
  {
    std::vector<P2PJob> jobs;
    std::vector<int> ent;
    // Pairs with W-list UE surfaces: where they carry more than 1% of the
    // pairs (clouds on surfaces), the mixed near field runs with 5 resident
    // blocks per SM and jobs of at most 4 rows (128 targets): measured on 4M
    // points on the ellipsoid surface, NP=4, 256 per box: 2.32 ms against
    // 2.50 ms with 6 blocks and 6 rows; uniform clouds keep 6 and 6 (4.42 ms,
    // against 4.70 ms with 4 rows).
    double w_pairs = 0.0;
    for (int t = 0; t < nn; ++t) {
      if (!is_leaf(t) || !has_trg(t) || d->trg_num[t] == 0) continue;
      for (int k = d->w_ptr[t]; k < d->w_ptr[t + 1]; ++k) {
        const int s = d->w_idx[k];
        if (!(is_leaf(s) && d->src_num[s] < P)) w_pairs += (double)d->trg_num[t] * P;
      }
    }
    double all_pairs = 0.0;
    for (int t = 0; t < nn; ++t) {
      if (!is_leaf(t) || !has_trg(t)) continue;
      double ns = 0;
      for (int k = d->u_ptr[t]; k < d->u_ptr[t + 1]; ++k) ns += d->src_num[d->u_idx[k]];
      all_pairs += ns * d->trg_num[t];
    }
    p->nf_w_heavy = w_pairs > 0.01 * (all_pairs + w_pairs);
    // Hybrid: the host takes the U lists of the cheapest target leaves (by
    // U-list pairs, ties in node order) up to cpu_share_ppm of all U pairs.
    std::vector<char> on_host(nn, 0);
    if (p->tune.cpu_share_ppm > 0) {
      std::vector<std::pair<double, int>> cost;
      for (int t = 0; t < nn; ++t) {
        if (!is_leaf(t) || !has_trg(t) || d->trg_num[t] == 0) continue;
        double ns = 0;
        for (int k = d->u_ptr[t]; k < d->u_ptr[t + 1]; ++k) ns += d->src_num[d->u_idx[k]];
        cost.push_back({ns * d->trg_num[t], t});
      }
      std::stable_sort(cost.begin(), cost.end(),
                       [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
                         return a.first < b.first;
                       });
      const double want = all_pairs * (p->tune.cpu_share_ppm * 1e-6);
      std::vector<int> src_at(nn, -1);  // source leaf -> its range in host_src
      for (const auto& c : cost) {
        if (p->host_pairs + c.first > want && p->tune.cpu_share_ppm < 1000000) break;
        const int t = c.second;
        on_host[t] = 1;
        p->host_pairs += c.first;
        kfmm_plan::HostLeaf L;
        L.tbeg = (int)p->host_trg.size();
        L.tcnt = d->trg_num[t];
        for (int i = 0; i < L.tcnt; ++i) p->host_trg.push_back(d->trg_perm[d->trg_beg[t] + i]);
        L.ubeg = (int)p->host_u.size();
        for (int k = d->u_ptr[t]; k < d->u_ptr[t + 1]; ++k) {
          const int s = d->u_idx[k];
          if (src_at[s] < 0) {
            src_at[s] = (int)p->host_src.size();
            for (int i = 0; i < d->src_num[s]; ++i)
              p->host_src.push_back(d->src_perm[d->src_beg[s] + i]);
          }
          p->host_u.push_back(make_int2(src_at[s], src_at[s] + d->src_num[s]));
        }
        L.uend = (int)p->host_u.size();
        p->host_leaves.push_back(L);
      }
    }
    for (int t = 0; t < nn; ++t) {
      if (!is_leaf(t) || !has_trg(t) || d->trg_num[t] == 0) continue;
      int e0 = (int)ent.size();
      for (int k = d->u_ptr[t]; k < d->u_ptr[t + 1]; ++k) ent.push_back(d->u_idx[k]);
      const int e_after_u = (int)ent.size();
      for (int k = d->w_ptr[t]; k < d->w_ptr[t + 1]; ++k) {
        int s = d->w_idx[k];
        bool direct = is_leaf(s) && d->src_num[s] < P;  // fmm/omp.cc:675
        ent.push_back(direct ? s : ((1 << 28) | s));
      }
      if (d->trg_num[t] < P)  // fmm/omp.cc:724
        for (int k = d->x_ptr[t]; k < d->x_ptr[t + 1]; ++k) ent.push_back(d->x_idx[k]);
      if (d->depth[t] >= 2) ent.push_back((2 << 28) | t);
      if (on_host[t]) e0 = e_after_u;  // the host sums this leaf's U list
      int ns = 0;
      for (int k = e0; k < (int)ent.size(); ++k) ns += src_count(ent[k]);
      P2PJob j;
      j.tnode = t;
      j.tkind = 0;
      j.tbeg = d->trg_beg[t];
      j.tcnt = d->trg_num[t];
      j.ebeg = e0;
      j.eend = (int)ent.size();
      j.out = d->trg_beg[t];
      j.mode = 0;
      p->nf_leaf.push_back(j);
      p->nf_leaf_ns.push_back(ns);
      p->stats.u_pairs += (double)d->trg_num[t] * ns;
    }
    KF_TRY(upload(p, &p->nf_ent, ent));
    KF_TRY(build_nf_jobs(p));
  }

  fft_src_resident(p->np, p->prec == KFMM_MIXED);  // the occupancy query, before any capture
  KF_CUDA(cudaFuncSetAttribute(gemm_fp64_dmma_kernel<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmemBytes));
  KF_CUDA(cudaFuncSetAttribute(gemm_fp64_dmma_kernel<true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmemBytes));
  KF_CUDA(cudaFuncSetAttribute(hadamard_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kTcSmemBytes));
  KF_CUDA(cudaFuncSetAttribute(hadamard_fp32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kHad32TileBytes));
  KF_CUDA(cudaFuncSetAttribute(hadamard_fp32_pair_kernel,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kHadPairSmemBytes));
  set_had_blocks(p);

  KF_TRY(ensure_splitk(p));
  KF_TRY(dalloc(p, &p->job_counter, 3));
  KF_TRY(dalloc(p, &p->d_error, 2));
  KF_CUDA(cudaMemset(p->d_error, 0, 2 * sizeof(int)));
  {
    int occ = 0;
    if (p->prec == KFMM_MIXED)
      KF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p2p_warp_kernel<true>,
                                                            32 * kWarpJobsPerBlock, 0));
    else
      KF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p2p_warp_kernel<false>,
                                                            32 * kWarpJobsPerBlock, 0));
    p->p2p_grid = std::max(1, occ) * p->num_sms;
    int occ5 = 0;
    KF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ5, p2p_warp_kernel<true, 5>,
                                                          32 * kWarpJobsPerBlock, 0));
    p->p2p_grid5 = std::max(1, occ5) * p->num_sms;
  }
  p->stats.num_nodes = nn;
  p->stats.P = P;
  p->stats.Q = Q;
  p->stats.F = F;
  count_launches(p);
  for (int i = 0; i < kfmm_plan::kMarks; ++i) KF_CUDA(cudaEventCreate(&p->ev[i]));
  KF_CUDA(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
  KF_CUDA(cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&p->ev_h2d_src, &p->ev_gsrc, &p->ev_gtrg, &p->ev_nf, &p->ev_d2h})
    KF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return KFMM_OK;
}

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

// Resident blocks per SM of a kernel (queried once per instance).
template <class Kern>
int resident_blocks(Kern kern, int threads) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, 0) != cudaSuccess ||
      occ < 1)
    occ = 1;
  return occ;
}

// Resident blocks per SM of the forward FFT kernel of NP; the first call (at
// plan creation, outside any stream capture) makes the query.
template <int NP>
int fft_src_resident(bool mixed) {
  static const int occ32 = resident_blocks(fft_src_np_kernel<NP, float2>, kFFTThreads);
  static const int occ64 = resident_blocks(fft_src_np_kernel<NP, double2>, kFFTThreads);
  return mixed ? occ32 : occ64;
}

int fft_src_resident(int np, bool mixed) {
  switch (np) {
    case 3: return fft_src_resident<3>(mixed);
    case 4: return fft_src_resident<4>(mixed);
    case 5: return fft_src_resident<5>(mixed);
    case 6: return fft_src_resident<6>(mixed);
    case 7: return fft_src_resident<7>(mixed);
    default: return fft_src_resident<8>(mixed);
  }
}

template <int NP>
void fft_launch_np(bool mixed, bool forward, int nboxes, int num_sms, FFTParams f,
                   cudaStream_t st) {
  constexpr int B = fft_boxes_per_block<NP>();
  const int nblocks = (nboxes + B - 1) / B;
  f.nboxes = nboxes;
  if (forward) {
    // persistent: one wave of blocks, each taking groups of boxes in turn
    const int grid = std::max(1, std::min(nblocks, num_sms * fft_src_resident<NP>(mixed)));
    if (mixed) fft_src_np_kernel<NP, float2><<<grid, kFFTThreads, 0, st>>>(f);
    else fft_src_np_kernel<NP, double2><<<grid, kFFTThreads, 0, st>>>(f);
  } else {
    if (mixed) ifft_trg_np_kernel<NP, float2><<<nblocks, kFFTThreads, 0, st>>>(f);
    else ifft_trg_np_kernel<NP, double2><<<nblocks, kFFTThreads, 0, st>>>(f);
  }
}

kfmm_status launch_fft(int np, bool mixed, bool forward, int nboxes, int num_sms,
                       const FFTParams& f, void* stream) {
  switch (np) {
    case 3: fft_launch_np<3>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    case 4: fft_launch_np<4>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    case 5: fft_launch_np<5>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    case 6: fft_launch_np<6>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    case 7: fft_launch_np<7>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    case 8: fft_launch_np<8>(mixed, forward, nboxes, num_sms, f, S(stream)); break;
    default: set_error("launch_fft: NP out of range"); return KFMM_ERR_UNSUPPORTED;
  }
  KF_CHECK_LAUNCH(forward ? "fft_src_np_kernel" : "ifft_trg_np_kernel");
  return KFMM_OK;
}

kfmm_status launch_p2p(const kfmm_plan* p, int which, int njobs, const P2PParams& q,
                       void* stream, const char* what) {
  const int blocks = std::min(p->p2p_grid, (njobs + kWarpJobsPerBlock - 1) / kWarpJobsPerBlock);
  int* counter = p->job_counter + which;
  KF_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), S(stream)));
  if (p->prec == KFMM_MIXED && which == 2 && p->nf_minb5)
    p2p_warp_kernel<true, 5><<<std::min(p->p2p_grid5, (njobs + kWarpJobsPerBlock - 1) /
                                                          kWarpJobsPerBlock),
                               32 * kWarpJobsPerBlock, 0, S(stream)>>>(
        p2p_mixed_params(p, q, p->d_trg_perm), njobs, counter);
  else if (p->prec == KFMM_MIXED)
    p2p_warp_kernel<true><<<blocks, 32 * kWarpJobsPerBlock, 0, S(stream)>>>(
        p2p_mixed_params(p, q, which == 2 ? p->d_trg_perm : nullptr), njobs, counter);
  else
    p2p_warp_kernel<false><<<blocks, 32 * kWarpJobsPerBlock, 0, S(stream)>>>(q, njobs, counter);
  KF_CHECK_LAUNCH(std::string("p2p kernel (") + what + ")");
  return KFMM_OK;
}

void mark(kfmm_plan* p, int i, cudaStream_t st) {
  if (p->timing) cudaEventRecord(p->ev[i], st);
}

// Waits for `stream` and reports whether a kernel of the plan's last solve
// gave up a bounded wait (the flag is zeroed at the start of every V list).
kfmm_status sync_and_check(kfmm_plan* p, cudaStream_t st) {
  int err = 0;
  KF_CUDA(cudaMemcpyAsync(&err, p->d_error, sizeof(int), cudaMemcpyDeviceToHost, st));
  KF_CUDA(cudaStreamSynchronize(st));
  if (err) {
    set_error("a kernel's bounded wait ran out (V-list translation tile copy)");
    return KFMM_ERR_CUDA;
  }
  return KFMM_OK;
}

}  // namespace

extern "C" {

const char* kfmm_last_error(void) { return g_error.c_str(); }
const char* kfmm_version(void) { return "kifmm_b200 0.1 (sm_100a)"; }

kfmm_status kfmm_plan_create(const kfmm_tree_desc* tree, int np, kfmm_precision precision,
                             kfmm_plan** out) {
  return kfmm_plan_create_with_operators(tree, np, precision, nullptr, out);
}

kfmm_status kfmm_plan_create_with_operators(const kfmm_tree_desc* tree, int np,
                                            kfmm_precision precision,
                                            const kfmm_operator_set* ops, kfmm_plan** out) {
  return kfmm_plan_create_tuned(tree, np, precision, ops, nullptr, out);
}

kfmm_status kfmm_plan_create_tuned(const kfmm_tree_desc* tree, int np, kfmm_precision precision,
                                   const kfmm_operator_set* ops, const kfmm_tuning* tuning,
                                   kfmm_plan** out) {
  if (!out) {
    set_error("kfmm_plan_create: out is NULL");
    return KFMM_ERR_INVALID;
  }
  *out = nullptr;
  if (np < 3 || np > 8) {
    set_error("kfmm_plan_create: NP must be in 3..8");
    return KFMM_ERR_UNSUPPORTED;
  }
  if (precision != KFMM_PLAIN_FP64 && precision != KFMM_MIXED) {
    set_error("kfmm_plan_create: unknown precision");
    return KFMM_ERR_INVALID;
  }
  KF_TRY(validate_desc(tree));
  KF_TRY(check_tuning(tuning));
  kfmm_plan* p = new kfmm_plan();
  p->np = np;
  p->prec = precision;
  if (tuning) p->tune = *tuning;
  kfmm_status s = build_plan(p, tree, ops);
  if (s != KFMM_OK) {
    std::string keep = g_error;
    kfmm_plan_destroy(p);
    g_error = keep;
    return s;
  }
  *out = p;
  return KFMM_OK;
}

kfmm_status kfmm_plan_destroy(kfmm_plan* p) {
  if (!p) return KFMM_OK;
  for (void* v : p->allocs) cudaFree(v);
  for (int i = 0; i < kfmm_plan::kMarks; ++i)
    if (p->ev[i]) cudaEventDestroy(p->ev[i]);
  for (cudaEvent_t e : {p->ev_h2d_src, p->ev_gsrc, p->ev_gtrg, p->ev_nf, p->ev_d2h})
    if (e) cudaEventDestroy(e);
  if (p->side) cudaStreamDestroy(p->side);
  if (p->d2h) cudaStreamDestroy(p->d2h);
  delete p;
  return KFMM_OK;
}

kfmm_status kfmm_plan_set_tuning(kfmm_plan* p, const kfmm_tuning* tuning) {
  if (!p) {
    set_error("kfmm_plan_set_tuning: null plan");
    return KFMM_ERR_INVALID;
  }
  KF_TRY(check_tuning(tuning));
  const kfmm_tuning old = p->tune;
  p->tune = tuning ? *tuning : kfmm_tuning{};
  p->tune.had_tensor = old.had_tensor;  // the levels' kernels are chosen at creation
  p->tune.cpu_share_ppm = old.cpu_share_ppm;  // and so is the host's share
  KF_CUDA(cudaDeviceSynchronize());  // no launch of the plan may still read what changes
  if (p->tune.job_rows != old.job_rows || p->tune.nf_blocks != old.nf_blocks)
    KF_TRY(build_nf_jobs(p));
  set_had_blocks(p);
  if (p->tune.splitk_max != old.splitk_max) {
    for (auto* v : {&p->up_gemms, &p->down_gemms})
      for (GemmBatch& g : *v) choose_split(p, g);
    KF_TRY(ensure_splitk(p));
    count_launches(p);
  }
  return KFMM_OK;
}

kfmm_status kfmm_set_sources_device(kfmm_plan* p, const double* sx, const double* sy,
                                    const double* sz, const double* den, void* stream) {
  if (!p || !sx || !sy || !sz || !den) {
    set_error("kfmm_set_sources_device: null argument");
    return KFMM_ERR_INVALID;
  }
  if (p->prec == KFMM_MIXED) {
    scatter_sources_mixed_kernel<<<4 * p->num_sms, 256, 0, S(stream)>>>(
        p->ns, p->d_src_inv, p->d_src_leaf, sx, sy, sz, den, p->ctr, p->src4f);
  } else {
    scatter_points_kernel<<<4 * p->num_sms, 256, 0, S(stream)>>>(p->ns, p->d_src_inv, sx, sy, sz,
                                                                 den, p->src4);
  }
  KF_CHECK_LAUNCH("source gather");
  p->have_src = true;
  return KFMM_OK;
}

kfmm_status kfmm_set_targets_device(kfmm_plan* p, const double* tx, const double* ty,
                                    const double* tz, void* stream) {
  if (!p || !tx || !ty || !tz) {
    set_error("kfmm_set_targets_device: null argument");
    return KFMM_ERR_INVALID;
  }
  scatter_points_kernel<<<4 * p->num_sms, 256, 0, S(stream)>>>(p->nt, p->d_trg_inv, tx, ty, tz,
                                                               nullptr, p->trg4);
  KF_CHECK_LAUNCH("scatter_points_kernel");
  p->have_trg = true;
  return KFMM_OK;
}

kfmm_status kfmm_set_sources(kfmm_plan* p, const double* sx, const double* sy, const double* sz,
                             const double* den, void* stream) {
  if (!p || !sx || !sy || !sz || !den) {
    set_error("kfmm_set_sources: null argument");
    return KFMM_ERR_INVALID;
  }
  const size_t b = sizeof(double) * p->ns;
  KF_CUDA(cudaMemcpyAsync(p->o_sx, sx, b, cudaMemcpyHostToDevice, S(stream)));
  KF_CUDA(cudaMemcpyAsync(p->o_sy, sy, b, cudaMemcpyHostToDevice, S(stream)));
  KF_CUDA(cudaMemcpyAsync(p->o_sz, sz, b, cudaMemcpyHostToDevice, S(stream)));
  KF_CUDA(cudaMemcpyAsync(p->o_w, den, b, cudaMemcpyHostToDevice, S(stream)));
  return kfmm_set_sources_device(p, p->o_sx, p->o_sy, p->o_sz, p->o_w, stream);
}

kfmm_status kfmm_set_targets(kfmm_plan* p, const double* tx, const double* ty, const double* tz,
                             void* stream) {
  if (!p || !tx || !ty || !tz) {
    set_error("kfmm_set_targets: null argument");
    return KFMM_ERR_INVALID;
  }
  const size_t b = sizeof(double) * p->nt;
  KF_CUDA(cudaMemcpyAsync(p->o_tx, tx, b, cudaMemcpyHostToDevice, S(stream)));
  KF_CUDA(cudaMemcpyAsync(p->o_ty, ty, b, cudaMemcpyHostToDevice, S(stream)));
  KF_CUDA(cudaMemcpyAsync(p->o_tz, tz, b, cudaMemcpyHostToDevice, S(stream)));
  return kfmm_set_targets_device(p, p->o_tx, p->o_ty, p->o_tz, stream);
}

kfmm_status kfmm_up_calc(kfmm_plan* p, void* stream) {
  if (!p || !p->have_src) {
    set_error("kfmm_up_calc: plan has no sources");
    return KFMM_ERR_STATE;
  }
  if (p->n_s2m) {
    KF_TRY(launch_p2p(p, 0, p->n_s2m, p2p_params(p, p->s2m_jobs, p->s2m_ent, p->chk_up), stream,
                      "s2m"));
  }
  mark(p, 1, S(stream));
  return launch_gemms(p, p->up_gemms, S(stream));
}

kfmm_status kfmm_vlist_calc(kfmm_plan* p, void* stream) {
  if (!p) return KFMM_ERR_INVALID;
  // the error flag reports this solve's waits only
  KF_CUDA(cudaMemsetAsync(p->d_error, 0, sizeof(int), S(stream)));
  KF_CUDA(cudaMemsetAsync(p->dchk, 0, sizeof(double) * (size_t)p->nn * p->P, S(stream)));
  mark(p, 2, S(stream));
  FFTParams f = fft_params(p);
  const bool mixed = p->prec == KFMM_MIXED;
  if (p->n_fft) {
    f.nodes = p->fft_nodes;
    f.pln = p->uden;
    f.specout = p->spec;
    KF_TRY(launch_fft(p->np, mixed, true, p->n_fft, p->num_sms, f, stream));
  }
  mark(p, 3, S(stream));
  if (p->n_groups) {
    if (mixed) {
      if (p->n_pairs) {
        const int ppb = p->pair_per_block;
        HadPairParams h{p->nn, p->n_pairs, ppb, p->pair_win, p->pair_members, p->pair_rows,
                        (const float2*)p->d_trans, (const float2*)p->spec, (float2*)p->effv,
                        p->d_error, p->wait_limit};
        dim3 grid((p->n_pairs + ppb - 1) / ppb, p->Fpad / kFB);
        hadamard_fp32_pair_kernel<<<grid, kHadPairThreads, kHadPairSmemBytes, S(stream)>>>(h);
        KF_CHECK_LAUNCH("hadamard_fp32_pair_kernel");
      }
      if (p->n_singles) {
        const int gpb = p->had32_groups_per_block;
        Had32Params h{p->nn, p->n_singles, gpb, p->single_win, p->single_members, p->single_rows,
                      (const float2*)p->d_trans, (const float2*)p->spec, (float2*)p->effv,
                      p->d_error, p->wait_limit};
        dim3 grid((p->n_singles + gpb - 1) / gpb, p->Fpad / kFB);
        hadamard_fp32_kernel<<<grid, kHad32Threads, kHad32TileBytes, S(stream)>>>(h);
        KF_CHECK_LAUNCH("hadamard_fp32_kernel");
      }
      if (p->n_tc_levels) {
        KF_CUDA(cudaMemsetAsync(p->tc_counter, 0, sizeof(int), S(stream)));
        HadTcParams h = p->tc;
        h.spec = (const float2*)p->spec;
        h.effv = (float2*)p->effv;
        h.next_unit = p->tc_counter;
        h.error = p->d_error;
        h.wait_limit = p->wait_limit;
        hadamard_tc_kernel<<<p->num_sms, kTcThreads, kTcSmemBytes, S(stream)>>>(h);
        KF_CHECK_LAUNCH("hadamard_tc_kernel");
      }
    } else {
      HadamardParams h{p->nn, p->n_groups, kHadGroupsPerBlock, p->win, p->members,
                       (const double2*)p->d_trans, p->Fpad, (const double2*)p->spec,
                       (double2*)p->effv};
      dim3 grid((p->n_groups + kHadGroupsPerBlock - 1) / kHadGroupsPerBlock, p->Fpad / kFB);
      hadamard_kernel<<<grid, kHadThreads, 0, S(stream)>>>(h);
      KF_CHECK_LAUNCH("hadamard_kernel");
    }
  }
  mark(p, 4, S(stream));
  if (p->n_ifft) {
    f.nodes = p->ifft_nodes;
    f.specin = p->effv;
    f.plnout = p->dchk;
    KF_TRY(launch_fft(p->np, mixed, false, p->n_ifft, p->num_sms, f, stream));
  }
  return KFMM_OK;
}

kfmm_status kfmm_xlist_calc(kfmm_plan* p, void* stream) {
  if (!p) return KFMM_ERR_INVALID;
  if (p->n_s2l) {
    KF_TRY(launch_p2p(p, 1, p->n_s2l, p2p_params(p, p->s2l_jobs, p->s2l_ent, p->dchk), stream,
                      "s2l"));
  }
  return KFMM_OK;
}

kfmm_status kfmm_down_calc(kfmm_plan* p, void* stream) {
  if (!p) return KFMM_ERR_INVALID;
  return launch_gemms(p, p->down_gemms, S(stream));
}

namespace {
kfmm_status near_field(kfmm_plan* p, void* stream) {
  if (!p || !p->have_trg || !p->have_src) {
    set_error("kfmm_ulist_calc: plan has no points");
    return KFMM_ERR_STATE;
  }
  if (p->n_nf) {
    KF_TRY(launch_p2p(p, 2, p->n_nf, p2p_params(p, p->nf_jobs, p->nf_ent, near_field_out(p)),
                      stream, "near field"));
  }
  return KFMM_OK;
}

// A hybrid plan's GPU near field leaves out the host's U lists: only
// kfmm_evaluate, which adds them, may run it.
kfmm_status refuse_hybrid(const kfmm_plan* p, const char* who) {
  if (p && !p->host_leaves.empty()) {
    set_error(std::string(who) +
              ": the plan evaluates part of its U list on the host "
              "(kfmm_tuning.cpu_share_ppm): use kfmm_evaluate");
    return KFMM_ERR_UNSUPPORTED;
  }
  return KFMM_OK;
}
}  // namespace

kfmm_status kfmm_ulist_calc(kfmm_plan* p, void* stream) {
  KF_TRY(refuse_hybrid(p, "kfmm_ulist_calc"));
  return near_field(p, stream);
}

kfmm_status kfmm_copy_trg_val(kfmm_plan* p, double* pot_host, void* stream) {
  if (!p) return KFMM_ERR_INVALID;
  if (p->prec != KFMM_MIXED) {  // the mixed near field wrote pot_orig itself
    scatter_pot_kernel<<<592, 256, 0, S(stream)>>>(p->nt, p->d_trg_perm, p->pot_leaf,
                                                   p->pot_orig);
    KF_CHECK_LAUNCH("scatter_pot_kernel");
  }
  if (pot_host) {
    KF_CUDA(cudaMemcpyAsync(pot_host, p->pot_orig, sizeof(double) * p->nt, cudaMemcpyDeviceToHost,
                            S(stream)));
    return sync_and_check(p, S(stream));
  }
  return KFMM_OK;
}

kfmm_status kfmm_get_potentials_device(kfmm_plan* p, double* pot_dev, void* stream) {
  if (!p || !pot_dev) return KFMM_ERR_INVALID;
  KF_CUDA(cudaMemcpyAsync(pot_dev, p->pot_orig, sizeof(double) * p->nt, cudaMemcpyDeviceToDevice,
                          S(stream)));
  return sync_and_check(p, S(stream));
}

kfmm_status kfmm_set_wait_limit(kfmm_plan* p, long long tries) {
  if (!p) return KFMM_ERR_INVALID;
  p->wait_limit = tries < 0 ? kMbarSpinLimit : tries;
  return KFMM_OK;
}

}  // extern "C"

namespace {
// up, V, X (S2L) and down: everything before the near field
kfmm_status run_far_field(kfmm_plan* p, void* stream) {
  cudaStream_t st = S(stream);
  mark(p, 0, st);
  KF_TRY(kfmm_up_calc(p, stream));
  KF_TRY(kfmm_vlist_calc(p, stream));
  mark(p, 5, st);
  KF_TRY(kfmm_xlist_calc(p, stream));
  mark(p, 6, st);
  KF_TRY(kfmm_down_calc(p, stream));
  mark(p, 7, st);
  return KFMM_OK;
}
}  // namespace

extern "C" {

kfmm_status kfmm_run(kfmm_plan* p, void* stream) {
  if (!p) {
    set_error("kfmm_run: null plan");
    return KFMM_ERR_INVALID;
  }
  if (!p->have_src || !p->have_trg) {
    set_error("kfmm_run: set sources and targets first");
    return KFMM_ERR_STATE;
  }
  KF_TRY(refuse_hybrid(p, "kfmm_run"));
  KF_TRY(run_far_field(p, stream));
  KF_TRY(near_field(p, stream));
  mark(p, 8, S(stream));
  KF_TRY(kfmm_copy_trg_val(p, nullptr, stream));
  mark(p, 9, S(stream));
  return KFMM_OK;
}

namespace {
kfmm_status evaluate_async(kfmm_plan* p, const double* sx, const double* sy, const double* sz,
                           const double* den, const double* tx, const double* ty,
                           const double* tz, double* pot, void* stream) {
  if (!p || !pot || !sx || !sy || !sz || !den || !tx || !ty || !tz) {
    set_error("kfmm_evaluate_async: null argument");
    return KFMM_ERR_INVALID;
  }
  // Streams: copies and the target gather on `side`, the solve on `stream`,
  // the potentials' copy back on `d2h`.  The events keep each buffer's
  // readers and writers of successive calls in order, and nothing else, so a
  // call's copies overlap the previous call's solve:
  //   staging o_s*  : H2D(i) after gather_src(i-1)          (ev_gsrc)
  //   staging o_t*  : H2D(i) after gather_trg(i-1)          (side order)
  //   trg4          : gather_trg(i) after near field(i-1)   (ev_nf)
  //   src4 / src4f  : gather_src(i) after near field(i-1)   (stream order)
  //   pot_orig      : near field(i) after D2H(i-1)          (ev_d2h)
  cudaStream_t st = S(stream), sd = p->side;
  const size_t bs = sizeof(double) * p->ns, bt = sizeof(double) * p->nt;
  KF_CUDA(cudaStreamWaitEvent(sd, p->ev_gsrc, 0));
  KF_CUDA(cudaMemcpyAsync(p->o_sx, sx, bs, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_sy, sy, bs, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_sz, sz, bs, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_w, den, bs, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaEventRecord(p->ev_h2d_src, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_tx, tx, bt, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_ty, ty, bt, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaMemcpyAsync(p->o_tz, tz, bt, cudaMemcpyHostToDevice, sd));
  KF_CUDA(cudaStreamWaitEvent(sd, p->ev_nf, 0));
  KF_TRY(kfmm_set_targets_device(p, p->o_tx, p->o_ty, p->o_tz, sd));
  KF_CUDA(cudaEventRecord(p->ev_gtrg, sd));

  KF_CUDA(cudaStreamWaitEvent(st, p->ev_h2d_src, 0));
  KF_TRY(kfmm_set_sources_device(p, p->o_sx, p->o_sy, p->o_sz, p->o_w, stream));
  KF_CUDA(cudaEventRecord(p->ev_gsrc, st));
  KF_TRY(run_far_field(p, stream));
  KF_CUDA(cudaStreamWaitEvent(st, p->ev_gtrg, 0));
  KF_CUDA(cudaStreamWaitEvent(st, p->ev_d2h, 0));
  KF_TRY(near_field(p, stream));
  mark(p, 8, st);
  KF_TRY(kfmm_copy_trg_val(p, nullptr, stream));
  mark(p, 9, st);
  error_fold_kernel<<<1, 1, 0, st>>>(p->d_error);
  KF_CHECK_LAUNCH("error_fold_kernel");
  KF_CUDA(cudaEventRecord(p->ev_nf, st));

  KF_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_nf, 0));
  KF_CUDA(cudaMemcpyAsync(pot, p->pot_orig, bt, cudaMemcpyDeviceToHost, p->d2h));
  KF_CUDA(cudaEventRecord(p->ev_d2h, p->d2h));
  return KFMM_OK;
}

// The host's share of a hybrid plan's U list (exact FP64 as fmm/omp.cc:259-283:
// pairs at r = 0 skipped), from the original-order host arrays; add[j] for
// target host_trg[j].
void host_ulist(const kfmm_plan* p, const double* sx, const double* sy, const double* sz,
                const double* den, const double* tx, const double* ty, const double* tz,
                double* add) {
  const int nl = (int)p->host_leaves.size();
#pragma omp parallel for schedule(dynamic, 1)
  for (int h = 0; h < nl; ++h) {
    const kfmm_plan::HostLeaf& L = p->host_leaves[h];
    for (int i = 0; i < L.tcnt; ++i) {
      const int t = p->host_trg[L.tbeg + i];
      const double x = tx[t], y = ty[t], z = tz[t];
      double sum = 0.0;
      for (int e = L.ubeg; e < L.uend; ++e) {
        const int2 r = p->host_u[e];
        for (int k = r.x; k < r.y; ++k) {
          const int s = p->host_src[k];
          const double dx = x - sx[s], dy = y - sy[s], dz = z - sz[s];
          const double r2 = dx * dx + dy * dy + dz * dz;
          if (r2 > 0.0) sum += den[s] / std::sqrt(r2);
        }
      }
      add[L.tbeg + i] = kOOFP * sum;
    }
  }
}
}  // namespace

kfmm_status kfmm_evaluate_async(kfmm_plan* p, const double* sx, const double* sy,
                                const double* sz, const double* den, const double* tx,
                                const double* ty, const double* tz, double* pot, void* stream) {
  KF_TRY(refuse_hybrid(p, "kfmm_evaluate_async"));
  return evaluate_async(p, sx, sy, sz, den, tx, ty, tz, pot, stream);
}

kfmm_status kfmm_evaluate_join(kfmm_plan* p, void* stream) {
  if (!p) {
    set_error("kfmm_evaluate_join: null plan");
    return KFMM_ERR_INVALID;
  }
  KF_CUDA(cudaStreamWaitEvent(S(stream), p->ev_d2h, 0));
  return KFMM_OK;
}

kfmm_status kfmm_evaluate_wait(kfmm_plan* p, void* stream) {
  KF_TRY(kfmm_evaluate_join(p, stream));
  int err[2] = {0, 0};
  KF_CUDA(cudaMemcpyAsync(err, p->d_error, 2 * sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
  KF_CUDA(cudaStreamSynchronize(S(stream)));
  if (err[1]) {
    KF_CUDA(cudaMemsetAsync(p->d_error + 1, 0, sizeof(int), S(stream)));
    KF_CUDA(cudaStreamSynchronize(S(stream)));
    set_error("a kernel's bounded wait ran out (V-list translation tile copy)");
    return KFMM_ERR_CUDA;
  }
  return KFMM_OK;
}

kfmm_status kfmm_evaluate(kfmm_plan* p, const double* sx, const double* sy, const double* sz,
                          const double* den, const double* tx, const double* ty,
                          const double* tz, double* pot, void* stream) {
  if (!p || !pot || !tx || !ty || !tz) {
    set_error("kfmm_evaluate: null argument");
    return KFMM_ERR_INVALID;
  }
  if (p->host_leaves.empty()) {
    KF_TRY(evaluate_async(p, sx, sy, sz, den, tx, ty, tz, pot, stream));
    return kfmm_evaluate_wait(p, stream);
  }
  // hybrid: a host thread (and its OpenMP team) sums the host's U lists
  // while this thread queues the GPU's work and waits for it (with pageable
  // host arrays the copies themselves hold this thread); the sums are then
  // added to the downloaded potentials
  std::vector<double> add(p->host_trg.size());
  std::thread host([&] { host_ulist(p, sx, sy, sz, den, tx, ty, tz, add.data()); });
  kfmm_status st = evaluate_async(p, sx, sy, sz, den, tx, ty, tz, pot, stream);
  if (st == KFMM_OK) st = kfmm_evaluate_wait(p, stream);
  host.join();
  if (st != KFMM_OK) return st;
  for (size_t j = 0; j < add.size(); ++j) pot[p->host_trg[j]] += add[j];
  return KFMM_OK;
}

kfmm_status kfmm_direct_evaluation(int nt, const double* tx, const double* ty, const double* tz,
                                   double* pot, int ns, const double* sx, const double* sy,
                                   const double* sz, const double* den, void* stream) {
  if (nt < 0 || ns < 0 || (nt > 0 && (!tx || !ty || !tz || !pot)) ||
      (ns > 0 && (!sx || !sy || !sz || !den))) {
    set_error("kfmm_direct_evaluation: bad argument");
    return KFMM_ERR_INVALID;
  }
  if (nt == 0 || ns == 0) return KFMM_OK;
  direct_fp64_kernel<<<(nt + 127) / 128, 128, 0, S(stream)>>>(nt, tx, ty, tz, pot, ns, sx, sy, sz,
                                                              den);
  KF_CHECK_LAUNCH("direct_fp64_kernel");
  return KFMM_OK;
}

kfmm_status kfmm_read_array(kfmm_plan* p, int which, double* out, size_t count) {
  if (!p || !out) return KFMM_ERR_INVALID;
  const void* src = nullptr;
  size_t avail = 0;
  switch (which) {
    case 0: src = p->uden; avail = (size_t)p->nn * p->P; break;
    case 1: src = p->dchk; avail = (size_t)p->nn * p->P; break;
    case 2: src = p->dden; avail = (size_t)p->nn * p->P; break;
    case 3: src = p->pot_leaf; avail = (size_t)p->nt; break;
    case 4:
      if (p->prec == KFMM_MIXED) {
        set_error("kfmm_read_array: spectra of a mixed plan are FP32");
        return KFMM_ERR_INVALID;
      }
      src = p->spec;
      avail = (size_t)p->nn * p->Fpad * 2;
      break;
    default:
      set_error("kfmm_read_array: unknown array");
      return KFMM_ERR_INVALID;
  }
  if (count > avail) {
    set_error("kfmm_read_array: count exceeds array size");
    return KFMM_ERR_INVALID;
  }
  KF_CUDA(cudaDeviceSynchronize());
  if (which == 3 && p->prec == KFMM_MIXED) {  // leaf-order view of pot_orig
    gather_pot_kernel<<<592, 256>>>(p->nt, p->d_trg_perm, p->pot_orig, p->pot_leaf);
    KF_CHECK_LAUNCH("gather_pot_kernel");
    KF_CUDA(cudaDeviceSynchronize());
  }
  KF_CUDA(cudaMemcpy(out, src, count * sizeof(double), cudaMemcpyDeviceToHost));
  return KFMM_OK;
}

kfmm_status kfmm_plan_stats(const kfmm_plan* p, kfmm_stats* s) {
  if (!p || !s) return KFMM_ERR_INVALID;
  *s = p->stats;
  return KFMM_OK;
}

struct kfmm_batch {
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // fused near field of all plans: per-plan kernel arguments, (plan, job)
  // pairs in cost-class order, the job counter
  void* d_params = nullptr;  // P2PMixedParams (mixed plans) or P2PParams
  int2* d_jobs = nullptr;
  int* d_counter = nullptr;
  std::vector<kfmm_plan*> plans;  // for the error flags kfmm_batch_wait reads
};

static void batch_release(kfmm_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_params) cudaFree(b->d_params);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_counter) cudaFree(b->d_counter);
  for (cudaEvent_t e : b->events) cudaEventDestroy(e);
  for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
  delete b;
}

kfmm_status kfmm_batch_create(kfmm_plan* const* plans, int nplans, int nstreams,
                              kfmm_batch** out) {
  if (!plans || !out || nplans < 1 || nstreams < 1 || nstreams > 32) {
    set_error("kfmm_batch_create: need plans, nplans >= 1 and 1 <= nstreams <= 32");
    return KFMM_ERR_INVALID;
  }
  *out = nullptr;
  for (int i = 0; i < nplans; ++i) {
    if (!plans[i] || !plans[i]->have_src || !plans[i]->have_trg) {
      set_error("kfmm_batch_create: plan " + std::to_string(i) + " is null or has no points");
      return KFMM_ERR_STATE;
    }
    KF_TRY(refuse_hybrid(plans[i], "kfmm_batch_create"));
  }
  nstreams = std::min(nstreams, nplans);
  kfmm_batch* b = new kfmm_batch();
  b->plans.assign(plans, plans + nplans);
  auto fail = [&](cudaError_t e, const char* what) {
    set_error(std::string("kfmm_batch_create: ") + what + ": " + cudaGetErrorString(e));
    batch_release(b);
    return KFMM_ERR_CUDA;
  };
  cudaError_t e;
  b->streams.resize(nstreams + 1);
  for (auto& st : b->streams) {
    st = nullptr;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess)
      return fail(e, "cudaStreamCreate");
  }
  b->events.resize(nstreams + 1);
  for (auto& ev : b->events) {
    ev = nullptr;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
      return fail(e, "cudaEventCreate");
  }
  // Plans of one precision share one near-field launch: their far fields run
  // on the branch streams, then a single persistent launch takes the jobs of
  // all plans, largest cost class first, so small solves do not leave SMs
  // idle.
  bool fused = true;
  size_t njobs = 0;
  for (int i = 0; i < nplans; ++i) {
    fused = fused && plans[i]->prec == plans[0]->prec;
    njobs += plans[i]->n_nf;
  }
  fused = fused && njobs > 0 && njobs < (size_t)INT32_MAX;
  // A single solve is captured as its own launches (its near field keeps the
  // by-value argument block of the regular kernel).
  const bool single = nplans == 1;
  if (single) fused = false;
  if (fused) {
    const bool mixed = plans[0]->prec == KFMM_MIXED;
    std::vector<P2PParams> params(nplans);
    std::vector<P2PMixedParams> mparams(mixed ? nplans : 0);
    std::vector<std::pair<float, int2>> order;
    order.reserve(njobs);
    for (int i = 0; i < nplans; ++i) {
      kfmm_plan* p = plans[i];
      params[i] = p2p_params(p, p->nf_jobs, p->nf_ent, near_field_out(p));
      if (mixed) mparams[i] = p2p_mixed_params(p, params[i], p->d_trg_perm);
      for (int j = 0; j < p->n_nf; ++j) order.push_back({p->nf_class[j], make_int2(i, j)});
    }
    std::stable_sort(order.begin(), order.end(),
                     [](const std::pair<float, int2>& a, const std::pair<float, int2>& c) {
                       return a.first < c.first;
                     });
    std::vector<int2> jobs(njobs);
    for (size_t j = 0; j < njobs; ++j) jobs[j] = order[j].second;
    const size_t pbytes = mixed ? sizeof(P2PMixedParams) * nplans : sizeof(P2PParams) * nplans;
    const void* psrc = mixed ? (const void*)mparams.data() : (const void*)params.data();
    if ((e = cudaMalloc(&b->d_params, pbytes)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_jobs, sizeof(int2) * njobs)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_counter, sizeof(int))) != cudaSuccess)
      return fail(e, "cudaMalloc");
    if ((e = cudaMemcpy(b->d_params, psrc, pbytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(b->d_jobs, jobs.data(), sizeof(int2) * njobs, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
      return fail(e, "cudaMemcpy");
  }
  cudaStream_t origin = b->streams[nstreams];
  if ((e = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return fail(e, "cudaStreamBeginCapture");
  // fork: every branch stream waits on the origin, then runs its plans
  auto fork = [&]() {
    cudaEventRecord(b->events[nstreams], origin);
    for (int k = 0; k < nstreams; ++k) cudaStreamWaitEvent(b->streams[k], b->events[nstreams], 0);
  };
  auto join = [&]() {
    for (int k = 0; k < nstreams; ++k) {
      cudaEventRecord(b->events[k], b->streams[k]);
      cudaStreamWaitEvent(origin, b->events[k], 0);
    }
  };
  if (!single) fork();
  kfmm_status st = KFMM_OK;
  for (int i = 0; i < nplans && st == KFMM_OK; ++i) {
    const bool timing = plans[i]->timing;
    plans[i]->timing = false;
    cudaStream_t on = single ? origin : b->streams[i % nstreams];
    st = fused ? run_far_field(plans[i], on) : kfmm_run(plans[i], on);
    plans[i]->timing = timing;
  }
  if (!single) join();
  if (fused && st == KFMM_OK) {
    cudaMemsetAsync(b->d_counter, 0, sizeof(int), origin);
    const int blocks = std::min(plans[0]->p2p_grid,
                                (int)((njobs + kWarpJobsPerBlock - 1) / kWarpJobsPerBlock));
    if (plans[0]->prec == KFMM_MIXED)
      p2p_fused_kernel<true><<<blocks, 32 * kWarpJobsPerBlock, 0, origin>>>(
          (const P2PMixedParams*)b->d_params, b->d_jobs, (int)njobs, b->d_counter);
    else
      p2p_fused_kernel<false><<<blocks, 32 * kWarpJobsPerBlock, 0, origin>>>(
          (const P2PParams*)b->d_params, b->d_jobs, (int)njobs, b->d_counter);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("kfmm_batch_create: fused near-field launch failed");
      st = KFMM_ERR_CUDA;
    }
    fork();
    for (int i = 0; i < nplans && st == KFMM_OK; ++i)
      st = kfmm_copy_trg_val(plans[i], nullptr, b->streams[i % nstreams]);
    join();
  }
  e = cudaStreamEndCapture(origin, &b->graph);
  if (st != KFMM_OK) {
    batch_release(b);
    return st;
  }
  if (e != cudaSuccess) return fail(e, "cudaStreamEndCapture");
  if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
    return fail(e, "cudaGraphInstantiate");
  *out = b;
  return KFMM_OK;
}

kfmm_status kfmm_batch_launch(kfmm_batch* b, void* stream) {
  if (!b || !b->exec) {
    set_error("kfmm_batch_launch: null batch");
    return KFMM_ERR_INVALID;
  }
  KF_CUDA(cudaGraphLaunch(b->exec, S(stream)));
  return KFMM_OK;
}

kfmm_status kfmm_batch_wait(kfmm_batch* b, void* stream) {
  if (!b) {
    set_error("kfmm_batch_wait: null batch");
    return KFMM_ERR_INVALID;
  }
  std::vector<int> err(b->plans.size(), 0);
  for (size_t i = 0; i < b->plans.size(); ++i)
    KF_CUDA(cudaMemcpyAsync(&err[i], b->plans[i]->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                            S(stream)));
  KF_CUDA(cudaStreamSynchronize(S(stream)));
  for (size_t i = 0; i < err.size(); ++i)
    if (err[i]) {
      set_error("kfmm_batch_wait: a bounded wait ran out in solve " + std::to_string(i) +
                " (V-list translation tile copy)");
      return KFMM_ERR_CUDA;
    }
  return KFMM_OK;
}

kfmm_status kfmm_batch_destroy(kfmm_batch* b) {
  batch_release(b);
  return KFMM_OK;
}

kfmm_status kfmm_enable_timing(kfmm_plan* p, int enable) {
  if (!p) return KFMM_ERR_INVALID;
  p->timing = enable != 0;
  return KFMM_OK;
}

kfmm_status kfmm_phase_times(const kfmm_plan* p, float* ms) {
  if (!p || !ms) return KFMM_ERR_INVALID;
  if (!p->timing) {
    set_error("kfmm_phase_times: timing not enabled");
    return KFMM_ERR_STATE;
  }
  KF_CUDA(cudaEventSynchronize(p->ev[9]));
  const int edge[7] = {0, 2, 5, 6, 7, 8, 9};  // up, vlist, xlist, down, ulist, copy
  for (int i = 0; i < 6; ++i)
    KF_CUDA(cudaEventElapsedTime(&ms[i], p->ev[edge[i]], p->ev[edge[i + 1]]));
  return KFMM_OK;
}

kfmm_status kfmm_kernel_times(const kfmm_plan* p, float* ms) {
  if (!p || !ms) return KFMM_ERR_INVALID;
  if (!p->timing) {
    set_error("kfmm_kernel_times: timing not enabled");
    return KFMM_ERR_STATE;
  }
  KF_CUDA(cudaEventSynchronize(p->ev[9]));
  for (int i = 0; i < 9; ++i) KF_CUDA(cudaEventElapsedTime(&ms[i], p->ev[i], p->ev[i + 1]));
  return KFMM_OK;
}

}  // extern "C"
