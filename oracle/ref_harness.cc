/*
 * Test infrastructure: a driver for the reference KIFMM CPU evaluator that
 * dumps its tree, operators, per-phase arrays and potentials to a binary file.
 *
 * It is linked against the reference's own objects (fmm/input.cc, trans.cc,
 * evaluate.cc, evaluate--basic.cc, svdrep.cc, vecmatop.cc, util.c, reals*.c and
 * either omp.cc or omp_sse_block.cc), compiled in place from the reference tree
 * by oracle/Makefile, and replaces only fmm/driver.cc's main() (driver.cc:211-371),
 * whose call sequence it follows:
 *   srand48(26) -> create -> densities drand48 -> src_tree -> trg_tree ->
 *   get_input -> trans_setup -> allocate expansions -> work_division_U/V ->
 *   preproc -> run -> validate.
 * Differences from driver.cc, all deliberate:
 *   - every expansion array is zeroed after allocation (driver.cc:318-322 relies
 *     on fresh mmap'd pages being zero);
 *   - the validation accumulator is zeroed (driver.cc:157 never zeroes chkPot);
 *   - allocations of 4 KiB and more are served from fresh (zeroed) pages
 *     (mallopt M_MMAP_THRESHOLD): compute_fft_src never zeroes its per-thread
 *     regular-grid buffer (fmm/omp.cc:396-397, fmm/omp_sse_block.cc same
 *     lines), so its spectra are only right when that buffer starts at zero;
 *   - distribution "ellipsoidSurface" (not in the reference) is generated here:
 *     semi-axes (0.5, 0.5, 0.05) centred at (0.5, 0.5, 0.5), azimuth then polar
 *     angle drawn per point exactly as input.cc:66-70 draws them, densities
 *     2*drand48()-1.
 *
 * usage: ref_harness <N> <distribution> <pts/box> <out.bin> [notime|tree]
 *   env NP, C, NV as for the reference driver (fmm/util.c).
 *   "tree": build tree and lists only, skip evaluation.
 */
#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <malloc.h>
#include <time.h>

#include <vector>

#include "evaluate.h"
#include "input.h"
#include "node.h"
#include "reals.h"
#include "reals_aligned.h"
#include "trans.h"
#include "util.h"

static FILE* g_out = NULL;

static void put(const char* name, int dtype, long long count, const void* data) {
  char nm[32];
  memset(nm, 0, sizeof(nm));
  strncpy(nm, name, 31);
  fwrite(nm, 1, 32, g_out);
  int dt = dtype;
  fwrite(&dt, sizeof(int), 1, g_out);
  fwrite(&count, sizeof(long long), 1, g_out);
  size_t esz = dtype == 0 ? sizeof(double) : sizeof(int);
  if (count > 0) fwrite(data, esz, (size_t)count, g_out);
}
static void putd(const char* n, long long c, const double* d) { put(n, 0, c, d); }
static void puti(const char* n, long long c, const int* d) { put(n, 1, c, d); }

static double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void gen_ellipsoid_surface(int N, AllNodes* A, int coincide) {
  const double ax[3] = {0.5, 0.5, 0.05};
  const double c[3] = {0.5, 0.5, 0.5};
  for (int i = 0; i < N; i++) {
    double phi = 2 * M_PI * drand48();
    double theta = M_PI * drand48();
    A->sx_orig[i] = c[0] + ax[0] * sin(theta) * cos(phi);
    A->sy_orig[i] = c[1] + ax[1] * sin(theta) * sin(phi);
    A->sz_orig[i] = c[2] + ax[2] * cos(theta);
  }
  if (coincide) {
    A->tx_orig = A->sx_orig;
    A->ty_orig = A->sy_orig;
    A->tz_orig = A->sz_orig;
    return;
  }
  for (int i = 0; i < N; i++) {
    double phi = 2 * M_PI * drand48();
    double theta = M_PI * drand48();
    A->tx_orig[i] = c[0] + ax[0] * sin(theta) * cos(phi);
    A->ty_orig[i] = c[1] + ax[1] * sin(theta) * sin(phi);
    A->tz_orig[i] = c[2] + ax[2] * cos(theta);
  }
}

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s <N> <distribution> <pts/box> <out.bin> [tree]\n", argv[0]);
    return 2;
  }
  int N = atoi(argv[1]);
  const char* dist = argv[2];
  int pts_max = atoi(argv[3]);
  bool tree_only = argc > 5 && strcmp(argv[5], "tree") == 0;
  mallopt(M_MMAP_THRESHOLD, 4096);
  g_out = fopen(argv[4], "wb");
  if (!g_out) return 3;

  srand48(26);
  std::vector<NodeTree> nodeVec;
  std::vector<int> nodeLevel;
  AllNodes* A = (AllNodes*)calloc(1, sizeof(AllNodes));
  A->tx_orig = reals_alloc__aligned(N);
  A->ty_orig = reals_alloc__aligned(N);
  A->tz_orig = reals_alloc__aligned(N);
  A->pot_orig = reals_alloc__aligned(N);
  A->sx_orig = reals_alloc__aligned(N);
  A->sy_orig = reals_alloc__aligned(N);
  A->sz_orig = reals_alloc__aligned(N);
  A->den_orig = reals_alloc__aligned(N);
  A->N = &nodeVec;
  A->nodeLevel = &nodeLevel;

  int coincide = getenv__coincide();
  bool signed_den = false;
  if (strcmp(dist, "ellipsoidSurface") == 0) {
    gen_ellipsoid_surface(N, A, coincide);
    signed_den = true;
  } else {
    create(N, (char*)dist, A);
  }
  for (int i = 0; i < N; i++) A->den_orig[i] = signed_den ? 2.0 * drand48() - 1.0 : drand48();

  double t0 = now_s();
  src_tree(N, pts_max, A);
  trg_tree(N, A);
  double t_tree = now_s() - t0;

  int nn = (int)nodeVec.size();
  int np = getenv__accuracy();
  int meta[8] = {N, np, pts_max, nn, coincide, 0, 0, 0};
  puti("meta", 8, meta);
  putd("sx", N, A->sx_orig);
  putd("sy", N, A->sy_orig);
  putd("sz", N, A->sz_orig);
  putd("den", N, A->den_orig);
  putd("tx", N, A->tx_orig);
  putd("ty", N, A->ty_orig);
  putd("tz", N, A->tz_orig);
  {
    std::vector<int> parent(nn), child(nn), depth(nn), tag(nn), path(3 * nn), sb(nn), sn(nn),
        tb(nn), tn(nn);
    std::vector<int> sperm, tperm;
    std::vector<int> lp[4], li[4];
    for (int k = 0; k < 4; ++k) lp[k].push_back(0);
    for (int i = 0; i < nn; ++i) {
      NodeTree& t = nodeVec[i];
      parent[i] = t.parent;
      child[i] = t.child;
      depth[i] = t.depth;
      tag[i] = t.tag;
      for (int d = 0; d < 3; ++d) path[3 * i + d] = t.path2Node(d);
      sb[i] = t.srcBeg;
      sn[i] = t.srcNum;
      tb[i] = t.trgBeg;
      tn[i] = t.trgNum;
      for (size_t k = 0; k < t.srcOwnVecIdxs.size(); ++k) sperm.push_back(t.srcOwnVecIdxs[k]);
      for (size_t k = 0; k < t.trgOwnVecIdxs.size(); ++k) tperm.push_back(t.trgOwnVecIdxs[k]);
      std::vector<int>* L[4] = {&t.Unodes, &t.Vnodes, &t.Wnodes, &t.Xnodes};
      for (int k = 0; k < 4; ++k) {
        for (size_t j = 0; j < L[k]->size(); ++j) li[k].push_back((*L[k])[j]);
        lp[k].push_back((int)li[k].size());
      }
    }
    puti("parent", nn, parent.data());
    puti("child", nn, child.data());
    puti("depth", nn, depth.data());
    puti("tag", nn, tag.data());
    puti("path", 3LL * nn, path.data());
    puti("src_beg", nn, sb.data());
    puti("src_num", nn, sn.data());
    puti("trg_beg", nn, tb.data());
    puti("trg_num", nn, tn.data());
    puti("src_perm", (long long)sperm.size(), sperm.data());
    puti("trg_perm", (long long)tperm.size(), tperm.data());
    puti("node_level", (long long)nodeLevel.size(), nodeLevel.data());
    const char* nm[4][2] = {{"u_ptr", "u_idx"}, {"v_ptr", "v_idx"}, {"w_ptr", "w_idx"}, {"x_ptr", "x_idx"}};
    for (int k = 0; k < 4; ++k) {
      puti(nm[k][0], (long long)lp[k].size(), lp[k].data());
      puti(nm[k][1], (long long)li[k].size(), li[k].data());
    }
  }
  double tm[4] = {t_tree, 0, 0, 0};
  if (tree_only) {
    putd("timing", 4, tm);
    fclose(g_out);
    return 0;
  }

  A->tx = reals_alloc__aligned(N);
  A->ty = reals_alloc__aligned(N);
  A->tz = reals_alloc__aligned(N);
  A->pot = reals_alloc__aligned(N);
  A->sx = reals_alloc__aligned(N);
  A->sy = reals_alloc__aligned(N);
  A->sz = reals_alloc__aligned(N);
  A->den = reals_alloc__aligned(N);
  A->Ns = (Node*)_mm_malloc(nn * sizeof(Node), IDEAL_ALIGNMENT);
  A->Nt = (Node*)_mm_malloc(nn * sizeof(Node), IDEAL_ALIGNMENT);
  get_input(A);

  Pos* SP = (Pos*)malloc(sizeof(Pos) * 4);
  Pos* RP = (Pos*)malloc(sizeof(Pos));
  trans_setup(SP, RP);
  A->SP = SP;
  A->RP = RP;
  A->TM = (Trans_matrix*)calloc(1, sizeof(Trans_matrix));
  int P = pln_size(UE, SP), Q = pln_size(UC, SP), E = eff_data_size(UE);
  A->src_upw_equ_den = reals_alloc__aligned((size_t)nn * P);
  A->eff_den = reals_alloc__aligned((size_t)nn * E);
  A->trg_dwn_equ_den = reals_alloc__aligned((size_t)nn * pln_size(DE, SP));
  A->trg_dwn_chk_val = reals_alloc__aligned((size_t)nn * pln_size(DC, SP));
  A->eff_val = reals_alloc__aligned((size_t)nn * eff_data_size(DC));
  memset(A->src_upw_equ_den, 0, sizeof(double) * (size_t)nn * P);
  memset(A->eff_den, 0, sizeof(double) * (size_t)nn * E);
  memset(A->trg_dwn_equ_den, 0, sizeof(double) * (size_t)nn * pln_size(DE, SP));
  memset(A->trg_dwn_chk_val, 0, sizeof(double) * (size_t)nn * pln_size(DC, SP));
  memset(A->eff_val, 0, sizeof(double) * (size_t)nn * eff_data_size(DC));
  memset(A->pot_orig, 0, sizeof(double) * (size_t)N);

  work_division_U(A);
  work_division_V(A);
  FMMWrapper_t* F = preproc(A);
  double t1 = now_s();
  run(F);
  double t_run = now_s() - t1;

  int meta2[4] = {P, Q, E, pln_size(DE, SP)};
  puti("sizes", 4, meta2);
  putd("uc2ue", (long long)P * Q, A->TM->UC2UE);
  for (int c = 0; c < 8; ++c) {
    char nm[32];
    snprintf(nm, sizeof nm, "ue2uc_%d", c);
    putd(nm, (long long)P * Q, A->TM->UE2UC[c]);
    snprintf(nm, sizeof nm, "de2dc_%d", c);
    putd(nm, (long long)P * P, A->TM->DE2DC[c]);
  }
  putd("dc2de", (long long)P * P, A->TM->DC2DE);
  {
    std::vector<double> T((size_t)343 * E, 0.0);
    for (int i = 0; i < 343; ++i) {
      int a = i % 7 - 3, b = (i / 7) % 7 - 3, c = i / 49 - 3;
      if (abs(a) > 1 || abs(b) > 1 || abs(c) > 1)
        memcpy(&T[(size_t)i * E], A->TM->UE2DC[i], sizeof(double) * E);
    }
    putd("ue2dc", (long long)343 * E, T.data());
  }
  putd("src_upw_equ_den", (long long)nn * P, A->src_upw_equ_den);
  putd("trg_dwn_chk_val", (long long)nn * P, A->trg_dwn_chk_val);
  putd("trg_dwn_equ_den", (long long)nn * P, A->trg_dwn_equ_den);
  if ((long long)nn * E <= (1LL << 24)) putd("eff_den", (long long)nn * E, A->eff_den);
  putd("pot_leaf", N, A->pot);
  putd("pot", N, A->pot_orig);

  /* validation: driver.cc:142-206 with the accumulator zeroed */
  int nv = getenv__validate();
  std::vector<int> ids(nv);
  std::vector<double> direct(nv, 0.0);
  for (int k = 0; k < nv; ++k) ids[k] = (int)floor(drand48() * N);
  Node src;
  src.x = A->sx_orig;
  src.y = A->sy_orig;
  src.z = A->sz_orig;
  src.den_pot = A->den_orig;
  src.num_pts = N;
  for (int k = 0; k < nv; ++k) {
    Node t;
    double x = A->tx_orig[ids[k]], y = A->ty_orig[ids[k]], z = A->tz_orig[ids[k]];
    t.x = &x;
    t.y = &y;
    t.z = &z;
    t.den_pot = &direct[k];
    t.num_pts = 1;
    ulist__direct_evaluation(t, src);
  }
  double vn = 0, en = 0;
  for (int k = 0; k < nv; ++k) {
    double d = direct[k] - A->pot_orig[ids[k]];
    vn += A->pot_orig[ids[k]] * A->pot_orig[ids[k]];
    en += d * d;
  }
  double rerr = sqrt(en) / sqrt(vn);
  puti("check_ids", nv, ids.data());
  putd("check_direct", nv, direct.data());
  tm[1] = t_run;
  tm[2] = rerr;
  putd("timing", 4, tm);
  fprintf(stderr, "Relative error: %e\n", rerr);
  fclose(g_out);
  return 0;
}
