// Host-side structures shared by the tree builder, the operator precompute
// and the plan.  Internal to libkifmm_b200; the public surface is
// include/kifmm_b200.h.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "kifmm_b200.h"

namespace kfmm {

constexpr int kSrcTag = 1;  // LET_SRCNODE (fmm/input.h:12)
constexpr int kTrgTag = 2;  // LET_TRGNODE (fmm/input.h:13)

// 1/(4 pi) exactly as the reference's OOFP_R macro evaluates it
// (fmm/evaluate.h:10).
constexpr double kOneOver4Pi = 1.0 / (4.0 * 3.14159265358979323846);

void set_error(const std::string& msg);

struct Tree {
  int num_src = 0, num_trg = 0;
  std::vector<int> parent, child, depth, tag, path;  // path: 3 per node
  std::vector<int> src_beg, src_num, trg_beg, trg_num;
  std::vector<int> src_perm, trg_perm;
  std::vector<int> node_level;
  std::vector<int> list_ptr[4], list_idx[4];  // U, V, W, X
  int num_nodes() const { return (int)parent.size(); }
};
// Fills T.list_ptr / list_idx from the tree structure and tags.
void build_lists(Tree& T);

// Surface sample grids and regular grid (fmm/trans.cc:14-88).
struct Surfaces {
  int np = 0, P = 0, Q = 0, G = 0, F = 0;
  std::vector<double> ue, uc, de, dc;  // 3 per point, xyz interleaved
};
void make_surfaces(int np, Surfaces* s);

struct Operators {
  int np = 0, P = 0, Q = 0, F = 0;
  std::vector<double> uc2ue;  // P x Q col-major
  std::vector<double> ue2uc;  // 8 x (Q x P)
  std::vector<double> dc2de;  // P x P
  std::vector<double> de2dc;  // 8 x (P x P)
  std::vector<double> ue2dc;  // 343 x F complex interleaved
};
// Computes (or returns a cached copy of) the operators for np.
const Operators& operators_for(int np);

}  // namespace kfmm

struct kfmm_tree {
  kfmm::Tree t;
};
