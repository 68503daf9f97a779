// The reference plug-in interface (fmm/evaluate.h:18-57) implemented over the
// kifmm_b200 C ABI.  Linking this file instead of fmm/evaluate--cuda.cu,
// fmm/run--cuda.cu and fmm/cuda.cu with the reference's common objects
// (driver, input, trans, evaluate, svdrep, vecmatop, util, reals) gives a
// drop-in `fmmd--cuda`: same driver, same tree and lists, same operator
// matrices (built by the reference's own trans.cc and passed to the plan),
// evaluation on the B200.  It compiles against the reference's headers; the
// recipe is the fmmd--b200-dropin rule of oracle/Makefile.
//
// env: KFMM_MIXED=1 selects the mixed-precision form; KFMM_CPU_SHARE_PPM=<n>
// the hybrid CPU+GPU evaluation (1000000: the whole U list on the host's
// cores while the GPU runs the rest, the schedule of fmm/run--hybrid2.cu, so
// this file then stands in for fmmd--hybrid2's run); KFMM_DUMP_POT=<file>
// writes the potentials (original target order, raw doubles) after run(), so
// tests can compare them per target with the reference's.
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "evaluate.h"
#include "kifmm_b200.h"
#include "node.h"
#include "trans.h"
#include "util.h"

struct FMMWrapper {
  AllNodes* AN;
  kfmm_plan* plan;
  int num_trg;
};

static void fail(const char* what) {
  fprintf(stderr, "%s: %s\n", what, kfmm_last_error());
  exit(-1);  // the reference's own error behaviour (fmm/cuda.cu:19-30)
}

const char* get_implementation_name(void) {
  const char* m = getenv("KFMM_MIXED");
  return (m && atoi(m) == 1) ? "b200-mixed" : "b200-fp64";
}

int get_num_threads(void) { return 1; }

// 1/(4 pi r) kernel matrix for the operator precompute (fmm/omp.cc:289-318)
int kernel(int sn, int tn, real_t* x1, real_t* x2, real_t* x3, real_t* y1, real_t* y2, real_t* y3,
           real_t* mat) {
  for (int i = 0; i < sn; i++)
    for (int j = 0; j < tn; j++) {
      real_t x = x1[i] - y1[j], y = x2[i] - y2[j], z = x3[i] - y3[j];
      real_t r = sqrt(x * x + y * y + z * z);
      if (r != 0) mat[j + i * tn] = OOFP_R / r;
    }
  return 0;
}

// exact FP64 direct sum, used by the driver's validate (fmm/driver.cc:185)
int ulist__direct_evaluation(Node trg, Node src) {
  for (int i = 0; i < trg.num_pts; i++) {
    real_t td = 0.0;
    for (int j = 0; j < src.num_pts; j++) {
      real_t x = trg.x[i] - src.x[j], y = trg.y[i] - src.y[j], z = trg.z[i] - src.z[j];
      real_t r = sqrt(x * x + y * y + z * z);
      if (r != 0) td += src.den_pot[j] / r;
    }
    trg.den_pot[i] += OOFP_R * td;
  }
  return 0;
}

int pointwise_mult(int n, FFT_COMPLEX* x, int ix, FFT_COMPLEX* y, int iy, FFT_COMPLEX* z, int iz) {
  for (int i = 0; i < n; i++) {
    (*z)[0] += ((*x)[0] * (*y)[0] - (*x)[1] * (*y)[1]);
    (*z)[1] += ((*x)[0] * (*y)[1] + (*x)[1] * (*y)[0]);
    x += ix;
    y += iy;
    z += iz;
  }
  return 0;
}

FMMWrapper_t* preproc(AllNodes* A) {
  std::vector<NodeTree>& nv = *A->N;
  const int nn = (int)nv.size();
  static std::vector<int> parent, child, depth, tag, path, sb, sn, tb, tn, sperm, tperm, level;
  static std::vector<int> lp[4], li[4];
  parent.resize(nn); child.resize(nn); depth.resize(nn); tag.resize(nn); path.resize(3 * nn);
  sb.resize(nn); sn.resize(nn); tb.resize(nn); tn.resize(nn);
  sperm.clear(); tperm.clear();
  for (int k = 0; k < 4; ++k) { lp[k].assign(1, 0); li[k].clear(); }
  for (int i = 0; i < nn; ++i) {
    NodeTree& t = nv[i];
    parent[i] = t.parent; child[i] = t.child; depth[i] = t.depth; tag[i] = t.tag;
    for (int d = 0; d < 3; ++d) path[3 * i + d] = t.path2Node(d);
    sb[i] = t.srcBeg; sn[i] = t.srcNum; tb[i] = t.trgBeg; tn[i] = t.trgNum;
    sperm.insert(sperm.end(), t.srcOwnVecIdxs.begin(), t.srcOwnVecIdxs.end());
    tperm.insert(tperm.end(), t.trgOwnVecIdxs.begin(), t.trgOwnVecIdxs.end());
    std::vector<int>* L[4] = {&t.Unodes, &t.Vnodes, &t.Wnodes, &t.Xnodes};
    for (int k = 0; k < 4; ++k) {
      li[k].insert(li[k].end(), L[k]->begin(), L[k]->end());
      lp[k].push_back((int)li[k].size());
    }
  }
  level.assign(A->nodeLevel->begin(), A->nodeLevel->end());
  kfmm_tree_desc d;
  d.num_nodes = nn;
  d.num_levels = (int)level.size() - 1;
  d.num_src = (int)sperm.size();
  d.num_trg = (int)tperm.size();
  d.parent = parent.data(); d.child = child.data(); d.depth = depth.data(); d.tag = tag.data();
  d.path = path.data(); d.src_beg = sb.data(); d.src_num = sn.data(); d.trg_beg = tb.data();
  d.trg_num = tn.data(); d.src_perm = sperm.data(); d.trg_perm = tperm.data();
  d.node_level = level.data();
  d.u_ptr = lp[0].data(); d.u_idx = li[0].data(); d.v_ptr = lp[1].data(); d.v_idx = li[1].data();
  d.w_ptr = lp[2].data(); d.w_idx = li[2].data(); d.x_ptr = lp[3].data(); d.x_idx = li[3].data();

  // operators from the reference's own trans.cc (as fmm/evaluate--cuda.cu's
  // preproc does before uploading them)
  Trans_matrix* TM = A->TM;
  Pos* SP = A->SP;
  compute_UC2UE_mat(TM, SP);
  TM->UE2UC = (real_t**)malloc(sizeof(real_t*) * 8);
  TM->DE2DC = (real_t**)malloc(sizeof(real_t*) * 8);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) {
        Index3 idx(a, b, c);
        compute_UE2UC_mat(idx, TM, SP);
      }
  compute_DC2DE_mat(TM, SP);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) {
        Index3 idx(a, b, c);
        compute_DE2DC_mat(idx, TM, SP);
      }
  const int P = pln_size(UE, SP), Q = pln_size(UC, SP);
  static std::vector<double> ue2uc, de2dc;
  ue2uc.resize((size_t)8 * P * Q);
  de2dc.resize((size_t)8 * P * P);
  for (int c = 0; c < 8; ++c) {
    memcpy(&ue2uc[(size_t)c * P * Q], TM->UE2UC[c], sizeof(double) * P * Q);
    memcpy(&de2dc[(size_t)c * P * P], TM->DE2DC[c], sizeof(double) * P * P);
  }
  kfmm_operator_set ops = {TM->UC2UE, ue2uc.data(), TM->DC2DE, de2dc.data(), NULL};
  const char* m = getenv("KFMM_MIXED");
  kfmm_precision prec = (m && atoi(m) == 1) ? KFMM_MIXED : KFMM_PLAIN_FP64;
  FMMWrapper_t* F = (FMMWrapper_t*)calloc(1, sizeof(FMMWrapper_t));
  F->AN = A;
  F->num_trg = d.num_trg;
  kfmm_tuning tuning;
  memset(&tuning, 0, sizeof(tuning));
  if (const char* h = getenv("KFMM_CPU_SHARE_PPM")) {
    const long v = atol(h);
    tuning.cpu_share_ppm = v < 0 ? 0 : (v > 1000000 ? 1000000 : (int)v);
  }
  if (kfmm_plan_create_tuned(&d, getenv__accuracy(), prec, &ops,
                             tuning.cpu_share_ppm ? &tuning : NULL, &F->plan) != KFMM_OK)
    fail("kfmm_plan_create_tuned");
  return F;
}

int run(FMMWrapper_t* F) {
  AllNodes* A = F->AN;
  if (kfmm_enable_timing(F->plan, 1) != KFMM_OK) fail("kfmm_enable_timing");
  if (kfmm_evaluate(F->plan, A->sx_orig, A->sy_orig, A->sz_orig, A->den_orig, A->tx_orig,
                    A->ty_orig, A->tz_orig, A->pot_orig, NULL) != KFMM_OK)
    fail("kfmm_evaluate");
  if (const char* path = getenv("KFMM_DUMP_POT")) {
    FILE* f = fopen(path, "wb");
    if (!f || fwrite(A->pot_orig, sizeof(double), F->num_trg, f) != (size_t)F->num_trg) {
      fprintf(stderr, "KFMM_DUMP_POT: cannot write %s\n", path);
      exit(-1);
    }
    fclose(f);
  }
  float ms[6];
  if (kfmm_phase_times(F->plan, ms) != KFMM_OK) fail("kfmm_phase_times");
  long double t_up = ms[0] * 1e-3L, t_v = ms[1] * 1e-3L, t_x = ms[2] * 1e-3L;
  long double t_down = (ms[3] + ms[5]) * 1e-3L, t_u = ms[4] * 1e-3L;
  long double t_total = t_up + t_v + t_x + t_down + t_u;
  fprintf(stderr, "=== Statistics ===\n");
  fprintf(stdout, "Code: %s\n", get_implementation_name());
  fprintf(stdout, "Floating-point word size: %lu bytes\n", sizeof(real_t));
  fprintf(stderr, "== Timing for FMM3d ==\n");
  fprintf(stderr, "  Up    : %Lg secs (%.1Lf%%)\n", t_up, t_up / t_total * 100);
  fprintf(stderr, "  U list: %Lg secs (%.1Lf%%)\n", t_u, t_u / t_total * 100);
  fprintf(stderr, "  V list: %Lg secs (%.1Lf%%)\n", t_v, t_v / t_total * 100);
  fprintf(stderr, "  W list: %Lg secs (%.1Lf%%)\n", (long double)0, (long double)0);
  fprintf(stderr, "  X list: %Lg secs (%.1Lf%%)\n", t_x, t_x / t_total * 100);
  fprintf(stderr, "  Down  : %Lg secs (%.1Lf%%)\n", t_down, t_down / t_total * 100);
  fprintf(stderr, "  ==> Total Execution Time: %Lg secs\n", t_total);
  return 0;
}
