/*
 * kifmm_b200 — C ABI of a B200 (sm_100a) evaluator for the kernel-independent
 * fast multipole method, 3-D Laplace kernel phi(t) = sum_s w_s / (4 pi |t-s|).
 *
 * It replaces the GPU evaluator plug-in of the reference benchmark (the
 * functions fmm/evaluate.h:18-57 declares and fmm/evaluate--cuda.cu,
 * fmm/run--cuda.cu and fmm/cuda.cu implement for `fmmd--cuda`).  Those are C++
 * symbols over std::vector trees; this ABI carries the same information as
 * plain pointers and sizes.  Every call returns a status; nothing exits the
 * process.  Host arrays belong to the caller, device memory belongs to the
 * plan.  Calls on one plan are not re-entrant.  `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).
 */
#ifndef KIFMM_B200_H
#define KIFMM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  KFMM_OK = 0,
  KFMM_ERR_INVALID = 1,     /* bad argument or inconsistent tree */
  KFMM_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  KFMM_ERR_ALLOC = 3,       /* host or device allocation failed */
  KFMM_ERR_UNSUPPORTED = 4, /* e.g. NP outside 3..8 */
  KFMM_ERR_STATE = 5        /* call out of order (e.g. run before points) */
} kfmm_status;

typedef enum {
  KFMM_PLAIN_FP64 = 0, /* FP64 throughout */
  KFMM_MIXED = 1       /* FP32 + compensated sums for P2P and M2L products */
} kfmm_precision;

/* Point sets.  Generators restate fmm/input.cc:30-84 (create) and the density
 * draw of fmm/driver.cc:244,266: srand48(seed) then the reference's drand48
 * sequence.  distribution: "uniform" ([-1,1)^3), "ellipseUniformAngles",
 * or "ellipsoidSurface" (semi-axes 0.5,0.5,0.05 centred at 0.5, densities in
 * [-1,1); not in the reference).  coincide != 0 makes targets the sources
 * (env C of fmm/util.c:177).  If check_ids is not NULL, num_check validation
 * indices are drawn next from the same stream (fmm/driver.cc:149-152). */
kfmm_status kfmm_generate_points(int n, const char* distribution, int coincide, long seed,
                                 double* sx, double* sy, double* sz, double* den,
                                 double* tx, double* ty, double* tz,
                                 int num_check, int* check_ids);

/* Octree + U/V/W/X lists: restates src_tree / trg_tree / compute_lists
 * (fmm/input.cc:204-298, 304-381, 387-460).  Node order, point order, tags
 * and lists are identical to the reference's vector<NodeTree>. */
typedef struct kfmm_tree kfmm_tree;

typedef struct {
  int num_nodes;
  int num_levels;      /* node_level has num_levels+1 entries */
  int num_src, num_trg;
  const int* parent;   /* -1 for the root */
  const int* child;    /* first of 8 contiguous children, -1 for a leaf */
  const int* depth;
  const int* tag;      /* bit 1: has sources, bit 2: has targets */
  const int* path;     /* 3 per node: path2Node */
  const int* src_beg;  /* leaf-order source range (leaves only) */
  const int* src_num;
  const int* trg_beg;
  const int* trg_num;
  const int* src_perm; /* leaf-order position -> original source index */
  const int* trg_perm; /* leaf-order position -> original target index */
  const int* node_level;
  const int *u_ptr, *u_idx; /* CSR lists, num_nodes+1 pointers each */
  const int *v_ptr, *v_idx;
  const int *w_ptr, *w_idx;
  const int *x_ptr, *x_idx;
} kfmm_tree_desc;

kfmm_status kfmm_tree_build(int num_src, const double* sx, const double* sy,
                            const double* sz, int num_trg, const double* tx,
                            const double* ty, const double* tz, int pts_max,
                            kfmm_tree** out);
/* The same tree as kfmm_tree_build (identical description), with the point
 * work done on the current CUDA device on `stream`: exact Morton keys of
 * the reference's octant comparisons, radix sorts, a breadth-first split
 * over the sorted keys; lists on the host (fmm/input.cc:204-460, replaced
 * by this GPU path).  Trees of more than 21 levels give
 * KFMM_ERR_UNSUPPORTED.  Host input arrays. */
kfmm_status kfmm_tree_build_device(int num_src, const double* sx, const double* sy,
                                   const double* sz, int num_trg, const double* tx,
                                   const double* ty, const double* tz, int pts_max,
                                   void* stream, kfmm_tree** out);
kfmm_status kfmm_tree_describe(const kfmm_tree* tree, kfmm_tree_desc* desc);
void kfmm_tree_destroy(kfmm_tree* tree);

/* Surface sizes for NP (fmm/trans.cc:26,67): P=|UE|=|DE|=|DC|, Q=|UC|,
 * F = complex spectrum length (np+1)(2np)^2. */
kfmm_status kfmm_sizes(int np, int* P, int* Q, int* F);

/* FP64 host precompute of the translation operators (fmm/trans.cc:144-268,
 * fmm/vecmatop.cc:34-78, fmm/omp_sse_block.cc:432-478).  Column-major like the
 * reference: uc2ue P x Q, ue2uc 8 x (Q x P), dc2de P x P, de2dc 8 x (P x P),
 * ue2dc 343 x F complex (interleaved re,im; zero where |delta|_inf <= 1).
 * Any output pointer may be NULL. */
kfmm_status kfmm_operators(int np, double* uc2ue, double* ue2uc, double* dc2de,
                           double* de2dc, double* ue2dc);

/* Plan = preproc (fmm/evaluate--cuda.cu:1441-2239): uploads tree, lists and
 * operators to the current CUDA device and allocates every work array. */
typedef struct kfmm_plan kfmm_plan;

kfmm_status kfmm_plan_create(const kfmm_tree_desc* tree, int np, kfmm_precision precision,
                             kfmm_plan** out);

/* Operator matrices supplied by the caller, layouts as kfmm_operators()
 * writes them.  The drop-in preproc passes the matrices its own trans.cc
 * computed (fmm/evaluate--cuda.cu:1628-1643 uploads the same set), so results
 * do not depend on which LAPACK produced the pseudo-inverses: with kappa ~
 * 0.1^-(np+1) a different SVD moves the potentials by ~1e-10 (NP=6). */
typedef struct {
  const double* uc2ue; /* P x Q */
  const double* ue2uc; /* 8 x (Q x P) */
  const double* dc2de; /* P x P */
  const double* de2dc; /* 8 x (P x P) */
  const double* ue2dc; /* 343 x F complex; NULL: computed here */
} kfmm_operator_set;

kfmm_status kfmm_plan_create_with_operators(const kfmm_tree_desc* tree, int np,
                                            kfmm_precision precision,
                                            const kfmm_operator_set* ops, kfmm_plan** out);

/* Kernel launch choices (no reference counterpart; the reference fixes its
 * thread-block sizes at compile time, fmm/cuda.cu:35-105).  0 in a field
 * keeps the plan's own choice.  The autotuner sweeps them.
 *   nf_blocks   mixed near field compiled for 5 or 6 resident blocks per SM
 *               (automatic: 5 when W-list surfaces carry > 1% of the pairs)
 *   job_rows    near-field jobs of at most 32 * job_rows targets, 1..6
 *               (automatic: 4 for mixed plans whose W lists carry > 1% of the
 *               pairs, else 6)
 *   had_windows mixed Hadamard: sibling windows per warp of a CTA, 1..8
 *               (automatic: the shortest span in waves of one CTA per SM)
 *   splitk_max  level products: largest split-K factor (automatic:
 *               max(8, K / 64))
 *   had_tensor  mixed Hadamard on the tcgen05 tensor cores (TF32, three
 *               passes) for levels whose boxes are all present: 2 every
 *               complete level; 0 automatic and 1 none (the CUDA-core kernels,
 *               measured faster on B200); fixed when the plan is created
 *               (kfmm_plan_set_tuning keeps the creation's choice)
 *   cpu_share_ppm hybrid evaluation (fmm/run--hybrid2.cu:25-47, where the
 *               host's cores run the U list while the GPU runs up, V and
 *               down): the host CPU takes the U-list point pairs of the
 *               cheapest target leaves up to this share of all of them, in
 *               parts per million (1,000,000: the whole U list, the
 *               reference's schedule), in FP64, while the GPU runs the rest;
 *               fixed at creation.  Such plans evaluate through
 *               kfmm_evaluate only (kfmm_run, kfmm_evaluate_async,
 *               kfmm_ulist_calc and batches refuse them), and their
 *               device-side potentials (kfmm_get_potentials_device,
 *               kfmm_read_array) lack the host's share. */
typedef struct {
  int nf_blocks;
  int job_rows;
  int had_windows;
  int splitk_max;
  int had_tensor;
  int cpu_share_ppm;
} kfmm_tuning;

/* kfmm_plan_create_with_operators with launch choices; ops and tuning may be
 * NULL. */
kfmm_status kfmm_plan_create_tuned(const kfmm_tree_desc* tree, int np, kfmm_precision precision,
                                   const kfmm_operator_set* ops, const kfmm_tuning* tuning,
                                   kfmm_plan** out);
/* New launch choices for an existing plan (NULL: all automatic): the
 * near-field jobs are re-chunked, the other choices are launch shapes; it
 * waits for the device first.  A batch that holds the plan must be created
 * again afterwards.  Only the split-K factor changes the order of any sum. */
kfmm_status kfmm_plan_set_tuning(kfmm_plan* plan, const kfmm_tuning* tuning);
kfmm_status kfmm_plan_destroy(kfmm_plan* plan);

/* Points in ORIGINAL order.  Host variants copy host->device inside the call
 * (on `stream`); device variants take device pointers.  Targets are needed
 * once per tree; densities may change between runs. */
kfmm_status kfmm_set_sources(kfmm_plan* plan, const double* sx, const double* sy,
                             const double* sz, const double* den, void* stream);
kfmm_status kfmm_set_targets(kfmm_plan* plan, const double* tx, const double* ty,
                             const double* tz, void* stream);
kfmm_status kfmm_set_sources_device(kfmm_plan* plan, const double* sx, const double* sy,
                                    const double* sz, const double* den, void* stream);
kfmm_status kfmm_set_targets_device(kfmm_plan* plan, const double* tx, const double* ty,
                                    const double* tz, void* stream);

/* run (fmm/run--cuda.cu:27-345): every phase below, in order, asynchronously
 * on `stream`; potentials stay on the device in original order. */
kfmm_status kfmm_run(kfmm_plan* plan, void* stream);

/* The phases, one by one (fmm/evaluate.h:35-52).  Call in this order. */
kfmm_status kfmm_up_calc(kfmm_plan* plan, void* stream);    /* S2M + M2M */
kfmm_status kfmm_vlist_calc(kfmm_plan* plan, void* stream); /* FFT, Hadamard, IFFT */
kfmm_status kfmm_xlist_calc(kfmm_plan* plan, void* stream); /* S2L part of X */
kfmm_status kfmm_down_calc(kfmm_plan* plan, void* stream);  /* L2L */
/* U list + W list + direct part of X + L2T, fused: each target's potential is
 * accumulated once, in registers, and written once (KFMM_MIXED plans: already
 * at the target's original index). */
kfmm_status kfmm_ulist_calc(kfmm_plan* plan, void* stream);
/* copy_trg_val (fmm/cuda.cu:2543-2565): potentials to original order on the
 * device (plain plans: a scatter; mixed plans: already there); pot_host (may
 * be NULL) additionally receives them (synchronous).
 * kfmm_get_potentials_device copies them to device memory and waits for
 * `stream`.  Both report KFMM_ERR_CUDA when a kernel of the last solve gave up
 * a bounded wait (the mixed V list's translation-tile copy); the flag is
 * cleared at the start of every solve, so a later solve that completes is
 * reported as KFMM_OK again.  (The reference exits on any CUDA error,
 * fmm/cuda.cu:19-30.) */
kfmm_status kfmm_copy_trg_val(kfmm_plan* plan, double* pot_host, void* stream);
kfmm_status kfmm_get_potentials_device(kfmm_plan* plan, double* pot_dev, void* stream);

/* Tries of the bounded waits in the plan's kernels (no reference
 * counterpart).  tries >= 0 sets the limit, tries < 0 restores the default
 * (2^24).  A limit of 0 makes the V-list tile-copy wait give up at once: the
 * solve then reports KFMM_ERR_CUDA, which tests use to drive the error path
 * without a fault (the copy still lands before the kernel exits). */
kfmm_status kfmm_set_wait_limit(kfmm_plan* plan, long long tries);

/* End-to-end: host inputs (original order) -> host potentials
 * (synchronous; kfmm_evaluate_async followed by kfmm_evaluate_wait).  For a
 * hybrid plan (kfmm_tuning.cpu_share_ppm > 0) the calling thread's OpenMP
 * team sums the host's share of the U list in FP64 from the host arrays
 * while the GPU works, and adds it to the downloaded potentials
 * (fmm/run--hybrid2.cu:25-47). */
kfmm_status kfmm_evaluate(kfmm_plan* plan, const double* sx, const double* sy,
                          const double* sz, const double* den, const double* tx,
                          const double* ty, const double* tz, double* pot, void* stream);

/* The same, queued without waiting (no reference counterpart: the reference
 * runs one synchronous solve per process).  The solve runs on `stream`, after
 * the work already queued there; the host->device copies run on a copy stream
 * of the plan and the potentials' device->host copy on another, so with
 * pinned host arrays the copies of one call overlap the solve of the previous
 * one: back-to-back calls are bounded by the larger of the device time and
 * the transfer time, not their sum.  The host arrays must stay unchanged, and
 * `pot` unread, until the call has completed: kfmm_evaluate_join makes
 * `stream` wait for every call queued on the plan (without blocking the
 * host), kfmm_evaluate_wait blocks until then and reports KFMM_ERR_CUDA if any
 * of those solves gave up a bounded wait.  Calls on one plan are not
 * re-entrant; queue them from one host thread on one stream. */
kfmm_status kfmm_evaluate_async(kfmm_plan* plan, const double* sx, const double* sy,
                                const double* sz, const double* den, const double* tx,
                                const double* ty, const double* tz, double* pot, void* stream);
kfmm_status kfmm_evaluate_join(kfmm_plan* plan, void* stream);
kfmm_status kfmm_evaluate_wait(kfmm_plan* plan, void* stream);

/* ulist__direct_evaluation (fmm/evaluate.h:27): pot[i] += sum_j den[j] /
 * (4 pi |t_i - s_j|), skipping r == 0.  Device pointers, FP64. */
kfmm_status kfmm_direct_evaluation(int nt, const double* tx, const double* ty,
                                   const double* tz, double* pot, int ns,
                                   const double* sx, const double* sy, const double* sz,
                                   const double* den, void* stream);

/* Introspection for parity tests: copy a per-node array (node-major, P or Q
 * doubles per node) to host.  which: 0 src_upw_equ_den, 1 trg_dwn_chk_val,
 * 2 trg_dwn_equ_den, 3 potentials in leaf order, 4 source spectra (2F per
 * node).  Synchronous. */
kfmm_status kfmm_read_array(kfmm_plan* plan, int which, double* host_out, size_t count);

typedef struct {
  double u_pairs;      /* target-source pairs of the near-field kernel */
  double s2m_pairs;    /* pairs of the S2M check-potential kernel */
  double s2l_pairs;    /* pairs of the X-list S2L kernel */
  double v_pairs;      /* V-list (target, source) box pairs */
  double hadamard_cmacs; /* complex multiply-adds the Hadamard kernel issues */
  double gemm_flops;   /* 2*m*n*k over all level GEMMs */
  double spectra_bytes; /* source + target spectra bytes, one pass each */
  int num_nodes, P, Q, F;
  int launches;        /* kernels one kfmm_run launches */
  int tensor_levels;   /* levels whose Hadamard runs on the tcgen05 tensor cores */
  double host_pairs;   /* U-list pairs the host sums (hybrid plans) */
} kfmm_stats;
kfmm_status kfmm_plan_stats(const kfmm_plan* plan, kfmm_stats* stats);

/* Per-phase device times of the last kfmm_run with timing enabled (ms):
 * [up, vlist, xlist, down, ulist, copy].  enable != 0 records CUDA events. */
kfmm_status kfmm_enable_timing(kfmm_plan* plan, int enable);
kfmm_status kfmm_phase_times(const kfmm_plan* plan, float* ms6);
/* Finer split of the same run (ms): [S2M pair sums, upward level products
 * (UC2UE, M2M; includes zeroing the downward check potentials), forward FFT,
 * Hadamard, inverse FFT, S2L, downward level products (L2L), near field,
 * copy]. */
kfmm_status kfmm_kernel_times(const kfmm_plan* plan, float* ms9);

/* Allocation-free S2M for a batch of leaves; it has no counterpart in the
 * reference.  For callers that may not allocate device memory at call time
 * (a host framework that owns all device memory through its own pool, or a
 * solver step run while such a framework holds the memory budget):
 * everything is passed in, and the only scratch, the leaves' check
 * potentials, lives in a fixed 8 MiB array inside the library image (one per
 * GPU that loads the library, resident until the process exits).
 *   src4     device, leaf-ordered sources as (x, y, z, w) quadruples
 *   leaf_beg, leaf_num  device, each leaf's source range in src4
 *   leaf_ctr device, 4 doubles per leaf: centre x, y, z and radius 2^-depth
 *   uc2ue    device, the P x Q UC2UE operator (column-major, kfmm_operators)
 *   uden     device output, nleaves x P upward equivalent densities
 * Limit: nleaves * Q <= 1,048,576 (3542 leaves at NP=6); larger batches are
 * rejected with KFMM_ERR_INVALID.  The first call on a device sets that
 * device up (symbol addresses, a small surface table, then a device
 * synchronisation) and should come before any stream capture; the set-up is
 * remembered for the life of the process, so the device must not be reset
 * (cudaDeviceReset) between calls.  All calls on a device share the scratch,
 * which keeps the last call's contents: calls that overlap on the GPU race
 * and must be serialised by the caller.  No cudaMalloc/cudaFree or
 * allocating library call is made. */
kfmm_status kfmm_s2m_noalloc(int np, int nleaves, const double* src4, const int* leaf_beg,
                             const int* leaf_num, const double* leaf_ctr, const double* uc2ue,
                             double* uden, void* stream);

/* Batched solves (no counterpart in the reference, which runs one solve per
 * process).  kfmm_batch_create captures kfmm_run of every plan into one CUDA
 * graph whose branches are spread over `nstreams` concurrent streams (1 to
 * 32); kfmm_batch_launch replays all solves with one graph launch on
 * `stream`.  The plans keep their own device buffers: set their points
 * (kfmm_set_sources/targets, or *_device) before a launch and read results
 * with kfmm_copy_trg_val / kfmm_get_potentials_device after it.  Phase timing
 * is switched off on the plans while they are captured.  A plan may belong to
 * one batch at a time and must outlive it; calls on a batch are not
 * re-entrant. */
typedef struct kfmm_batch kfmm_batch;
kfmm_status kfmm_batch_create(kfmm_plan* const* plans, int nplans, int nstreams,
                              kfmm_batch** out);
kfmm_status kfmm_batch_launch(kfmm_batch* batch, void* stream);
/* Waits for `stream` and reports KFMM_ERR_CUDA if any solve of the last
 * launch gave up a bounded wait (see kfmm_set_wait_limit). */
kfmm_status kfmm_batch_wait(kfmm_batch* batch, void* stream);
kfmm_status kfmm_batch_destroy(kfmm_batch* batch);

/* Cost-model network (no counterpart in the reference, which takes the leaf
 * size from its command line): a 3-layer perceptron in FP32,
 *   Y = relu(relu(X W1 + b1) W2 + b2) W3 + b3,  X: B x F, hidden H, Y: B x O,
 * trained on the GPU by hand-written forward, backward and Adam kernels on
 * the loss mean((Y - T)^2).  params: packed [W1 | b1 | W2 | b2 | W3 | b3],
 * weights row-major (input index major), kfmm_mlp_param_count floats; grads
 * in the same layout.  Host arrays; the calls synchronise.  kfmm_mlp_train
 * runs `steps` full-batch Adam steps (lr, beta 0.9 / 0.999), updates params
 * in place and writes each step's loss to losses (may be NULL). */
kfmm_status kfmm_mlp_param_count(int F, int H, int O, long long* count);
kfmm_status kfmm_mlp_forward(int F, int H, int O, const float* params, int B, const float* X,
                             float* Y);
kfmm_status kfmm_mlp_gradients(int F, int H, int O, const float* params, int B,
                               const float* X, const float* T, float* grads, float* loss);
kfmm_status kfmm_mlp_train(int F, int H, int O, float* params, int B, const float* X,
                           const float* T, int steps, float lr, float* losses);

/* Throughput of the current device's execution pipes, measured by
 * micro-benchmarks (no reference counterpart; roofline denominators):
 * what 0: FP64 FMA TFLOP/s, 1: FP32 FMA TFLOP/s, 2: FP32 rsqrt 1e12/s (MUFU),
 * 3: FP64 rsqrt 1e12/s, 4: FP64 DMMA (mma.sync m8n8k4) TFLOP/s. */
kfmm_status kfmm_measure_peak(int what, double* value);

const char* kfmm_last_error(void);
const char* kfmm_version(void);

#ifdef __cplusplus
}
#endif

#endif
