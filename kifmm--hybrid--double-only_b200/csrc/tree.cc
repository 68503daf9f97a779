// Point generators and the adaptive octree with its U/V/W/X interaction lists.
//
// The node numbering, point order, tags and list contents reproduce the
// reference's vector<NodeTree> (fmm/input.h:18-49) exactly; the algorithms are
// restated here over flat arrays:
//   - points split breadth-first, a node splitting when it holds more than
//     pts_max sources (fmm/input.cc:204-298); children are appended as a block
//     of 8, child (a,b,c) at offset 4a+2b+c (input.cc:142-147);
//   - a point goes to octant (x>=cx, y>=cy, z>=cz) and keeps its parent order
//     (input.cc:250-256), so each leaf lists its points by increasing index;
//   - leaf-order offsets are running sums over non-empty leaves in node order
//     (input.cc:282-296 sources, 436-449 targets);
//   - lists scan the 6x6x6 block of the parent's neighbourhood, descend to the
//     deepest existing node, and classify by depth and adjacency, with a
//     breadth-first descent into adjacent same-depth non-leaves for the W and
//     U lists of leaves (input.cc:304-381).  Lists keep only source-bearing
//     nodes, sorted by node index (input.cc:369-380 iterate std::set).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <new>

#include "host.h"

namespace kfmm {

namespace {

// Centre coordinate d of a node: -1 + 2 (p + 0.5) / 2^depth, evaluated in the
// same order as fmm/input.cc:122-135 (every intermediate is exact).
inline double center_coord(int p, int depth) {
  return -1.0 + (2.0 * 1.0) * (p + 0.5) / double(1 << depth);
}

struct Builder {
  Tree& T;
  explicit Builder(Tree& t) : T(t) {}

  int find_node(int wdepth, const int* wpath) const {
    int cur = 0;
    while (T.depth[cur] < wdepth && T.child[cur] != -1) {
      int sh = wdepth - T.depth[cur] - 1;
      int c = ((wpath[0] >> sh) & 1) * 4 + ((wpath[1] >> sh) & 1) * 2 + ((wpath[2] >> sh) & 1);
      cur = T.child[cur] + c;
    }
    return cur;
  }

  bool adjacent(int a, int b) const {
    int md = std::max(T.depth[a], T.depth[b]);
    int ra = 1 << (md - T.depth[a]);
    int rb = 1 << (md - T.depth[b]);
    int rad = ra + rb, linf = 0;
    bool within = true;
    for (int d = 0; d < 3; ++d) {
      int ca = (2 * T.path[3 * a + d] + 1) * ra;
      int cb = (2 * T.path[3 * b + d] + 1) * rb;
      int dif = std::abs(ca - cb);
      within = within && dif <= rad;
      linf = std::max(linf, dif);
    }
    return within && linf == rad;
  }

  void lists_of(int n, std::vector<int>* out) const {
    std::vector<int> U, V, W, X;
    const bool leaf = T.child[n] == -1;
    const int dep = T.depth[n];
    if (T.parent[n] != -1) {
      const int* pp = &T.path[3 * T.parent[n]];
      const int lim = 1 << dep;
      std::deque<int> q;
      for (int i = -2; i < 4; ++i)
        for (int j = -2; j < 4; ++j)
          for (int k = -2; k < 4; ++k) {
            int tp[3] = {2 * pp[0] + i, 2 * pp[1] + j, 2 * pp[2] + k};
            if (tp[0] < 0 || tp[1] < 0 || tp[2] < 0 || tp[0] >= lim || tp[1] >= lim ||
                tp[2] >= lim)
              continue;
            if (tp[0] == T.path[3 * n] && tp[1] == T.path[3 * n + 1] && tp[2] == T.path[3 * n + 2])
              continue;
            int r = find_node(dep, tp);
            bool adj = adjacent(r, n);
            if (T.depth[r] < dep) {
              if (adj) {
                if (leaf) U.push_back(r);
              } else {
                X.push_back(r);
              }
            }
            if (T.depth[r] == dep) {
              if (!adj) {
                V.push_back(r);
              } else if (leaf) {
                q.clear();
                q.push_back(r);
                while (!q.empty()) {
                  int f = q.front();
                  q.pop_front();
                  if (!adjacent(f, n)) {
                    W.push_back(f);
                  } else if (T.child[f] == -1) {
                    U.push_back(f);
                  } else {
                    for (int c = 0; c < 8; ++c) q.push_back(T.child[f] + c);
                  }
                }
              }
            }
          }
    }
    if (leaf) U.push_back(n);
    std::vector<int>* L[4] = {&U, &V, &W, &X};
    for (int k = 0; k < 4; ++k) {
      std::vector<int>& v = *L[k];
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      out[k].clear();
      for (int id : v)
        if (T.tag[id] & kSrcTag) out[k].push_back(id);
    }
  }
};

// Stable 8-way split of perm[b, e) by octant about centre c.
void split_octants(const double* x, const double* y, const double* z, int* perm, int b,
                   int e, const double c[3], std::vector<int>& tmp, int cnt[8]) {
  std::memset(cnt, 0, sizeof(int) * 8);
  tmp.resize((size_t)(e - b));
  for (int i = b; i < e; ++i) {
    int p = perm[i];
    int o = (x[p] >= c[0]) * 4 + (y[p] >= c[1]) * 2 + (z[p] >= c[2]);
    cnt[o]++;
  }
  int off[8];
  off[0] = 0;
  for (int o = 1; o < 8; ++o) off[o] = off[o - 1] + cnt[o - 1];
  for (int i = b; i < e; ++i) {
    int p = perm[i];
    int o = (x[p] >= c[0]) * 4 + (y[p] >= c[1]) * 2 + (z[p] >= c[2]);
    tmp[off[o]++] = p;
  }
  std::memcpy(perm + b, tmp.data(), sizeof(int) * (size_t)(e - b));
}

}  // namespace

constexpr int kMaxHostDepth = 30;
struct TooDeep {};

static void build_tree(Tree& T, int ns, const double* sx, const double* sy, const double* sz,
                       int nt, const double* tx, const double* ty, const double* tz,
                       int pts_max) {
  T.num_src = ns;
  T.num_trg = nt;
  // Each node owns a contiguous range of sperm; children split the range.
  std::vector<int> sperm(ns), rb, re;
  for (int i = 0; i < ns; ++i) sperm[i] = i;
  T.parent.assign(1, -1);
  T.child.assign(1, -1);
  T.depth.assign(1, 0);
  T.path.assign(3, 0);
  rb.assign(1, 0);
  re.assign(1, ns);
  T.node_level.assign(1, 0);
  std::vector<int> tmp;
  int beg = 0, end = 1;
  while (beg < end) {
    for (int k = beg; k < end; ++k) {
      if (re[k] - rb[k] <= pts_max) continue;
      // more than pts_max coincident points never separate: the reference
      // splits forever; here the depth is capped where the integer box
      // coordinates would overflow
      if (T.depth[k] >= kMaxHostDepth) throw TooDeep();
      int first = (int)T.parent.size();
      T.child[k] = first;
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int c = 0; c < 2; ++c) {
            T.parent.push_back(k);
            T.child.push_back(-1);
            T.depth.push_back(T.depth[k] + 1);
            T.path.push_back(2 * T.path[3 * k] + a);
            T.path.push_back(2 * T.path[3 * k + 1] + b);
            T.path.push_back(2 * T.path[3 * k + 2] + c);
          }
      double cc[3];
      for (int d = 0; d < 3; ++d) cc[d] = center_coord(T.path[3 * k + d], T.depth[k]);
      int cnt[8];
      split_octants(sx, sy, sz, sperm.data(), rb[k], re[k], cc, tmp, cnt);
      int o = rb[k];
      for (int c = 0; c < 8; ++c) {
        rb.push_back(o);
        re.push_back(o + cnt[c]);
        o += cnt[c];
      }
    }
    beg = end;
    end = (int)T.parent.size();
    T.node_level.push_back(beg);
  }
  const int nn = T.num_nodes();
  T.tag.assign(nn, 0);
  T.src_beg.assign(nn, 0);
  T.src_num.assign(nn, 0);
  T.trg_beg.assign(nn, 0);
  T.trg_num.assign(nn, 0);
  T.src_perm.clear();
  T.src_perm.reserve(ns);
  int sum = 0;
  for (int i = 0; i < nn; ++i) {
    int cnt = re[i] - rb[i];
    if (cnt <= 0) continue;
    T.tag[i] |= kSrcTag;
    if (T.child[i] == -1) {
      T.src_beg[i] = sum;
      T.src_num[i] = cnt;
      sum += cnt;
      T.src_perm.insert(T.src_perm.end(), sperm.begin() + rb[i], sperm.begin() + re[i]);
    }
  }
  // Targets descend the source tree (fmm/input.cc:387-434).
  std::vector<int> tperm(nt), tb(nn, 0), te(nn, 0);
  for (int i = 0; i < nt; ++i) tperm[i] = i;
  te[0] = nt;
  for (int k = 0; k < nn; ++k) {
    if (T.child[k] == -1) continue;
    double cc[3];
    for (int d = 0; d < 3; ++d) cc[d] = center_coord(T.path[3 * k + d], T.depth[k]);
    int cnt[8];
    split_octants(tx, ty, tz, tperm.data(), tb[k], te[k], cc, tmp, cnt);
    int o = tb[k];
    for (int c = 0; c < 8; ++c) {
      tb[T.child[k] + c] = o;
      te[T.child[k] + c] = o + cnt[c];
      o += cnt[c];
    }
  }
  T.trg_perm.clear();
  T.trg_perm.reserve(nt);
  sum = 0;
  for (int i = 0; i < nn; ++i) {
    int cnt = te[i] - tb[i];
    if (cnt <= 0) continue;
    T.tag[i] |= kTrgTag;
    if (T.child[i] == -1) {
      T.trg_beg[i] = sum;
      T.trg_num[i] = cnt;
      sum += cnt;
      T.trg_perm.insert(T.trg_perm.end(), tperm.begin() + tb[i], tperm.begin() + te[i]);
    }
  }
  build_lists(T);
}

// U/V/W/X lists of every target-bearing node (nodes are independent: built in
// parallel, concatenated in node order).
void build_lists(Tree& T) {
  const int nn = T.num_nodes();
  Builder B(T);
  std::vector<std::vector<int>> per(4 * (size_t)nn);
#pragma omp parallel
  {
    std::vector<int> L[4];
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < nn; ++i) {
      if (!(T.tag[i] & kTrgTag)) continue;
      B.lists_of(i, L);
      for (int k = 0; k < 4; ++k) per[4 * (size_t)i + k] = L[k];
    }
  }
  for (int k = 0; k < 4; ++k) {
    T.list_ptr[k].assign(1, 0);
    T.list_idx[k].clear();
    for (int i = 0; i < nn; ++i) {
      const std::vector<int>& v = per[4 * (size_t)i + k];
      T.list_idx[k].insert(T.list_idx[k].end(), v.begin(), v.end());
      T.list_ptr[k].push_back((int)T.list_idx[k].size());
    }
  }
}

}  // namespace kfmm

using namespace kfmm;

extern "C" kfmm_status kfmm_generate_points(int n, const char* distribution, int coincide,
                                            long seed, double* sx, double* sy, double* sz,
                                            double* den, double* tx, double* ty, double* tz,
                                            int num_check, int* check_ids) {
  if (n <= 0 || !distribution || !sx || !sy || !sz || !den || !tx || !ty || !tz) {
    set_error("kfmm_generate_points: bad argument");
    return KFMM_ERR_INVALID;
  }
  srand48(seed);
  bool signed_den = false;
  if (std::strcmp(distribution, "uniform") == 0) {
    // fmm/input.cc:36-57
    for (int i = 0; i < n; i++) {
      sx[i] = (2.0 * drand48() - 1.0);
      sy[i] = (2.0 * drand48() - 1.0);
      sz[i] = (2.0 * drand48() - 1.0);
    }
    if (!coincide) {
      for (int i = 0; i < n; i++) {
        tx[i] = (2.0 * drand48() - 1.0);
        ty[i] = (2.0 * drand48() - 1.0);
        tz[i] = (2.0 * drand48() - 1.0);
      }
    } else {
      std::memcpy(tx, sx, sizeof(double) * n);
      std::memcpy(ty, sy, sizeof(double) * n);
      std::memcpy(tz, sz, sizeof(double) * n);
    }
  } else if (std::strcmp(distribution, "ellipseUniformAngles") == 0) {
    // fmm/input.cc:59-79: sources then targets, whatever `coincide` says
    const double r = 0.49;
    const double c[3] = {0.5, 0.5, 0.5};
    double* X[2] = {sx, tx};
    double* Y[2] = {sy, ty};
    double* Z[2] = {sz, tz};
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < n; i++) {
        double phi = 2 * M_PI * drand48();
        double theta = M_PI * drand48();
        X[s][i] = c[0] + 0.25 * r * sin(theta) * cos(phi);
        Y[s][i] = c[1] + 0.25 * r * sin(theta) * sin(phi);
        Z[s][i] = c[2] + r * cos(theta);
      }
  } else if (std::strcmp(distribution, "ellipsoidSurface") == 0) {
    // Thin ellipsoid shell inside the root box; same angle law as above.
    const double ax[3] = {0.5, 0.5, 0.05};
    const double c[3] = {0.5, 0.5, 0.5};
    double* X[2] = {sx, tx};
    double* Y[2] = {sy, ty};
    double* Z[2] = {sz, tz};
    for (int s = 0; s < (coincide ? 1 : 2); ++s)
      for (int i = 0; i < n; i++) {
        double phi = 2 * M_PI * drand48();
        double theta = M_PI * drand48();
        X[s][i] = c[0] + ax[0] * sin(theta) * cos(phi);
        Y[s][i] = c[1] + ax[1] * sin(theta) * sin(phi);
        Z[s][i] = c[2] + ax[2] * cos(theta);
      }
    if (coincide) {
      std::memcpy(tx, sx, sizeof(double) * n);
      std::memcpy(ty, sy, sizeof(double) * n);
      std::memcpy(tz, sz, sizeof(double) * n);
    }
    signed_den = true;
  } else {
    set_error(std::string("kfmm_generate_points: unknown distribution ") + distribution);
    return KFMM_ERR_INVALID;
  }
  // fmm/driver.cc:266-267
  for (int i = 0; i < n; i++) den[i] = signed_den ? 2.0 * drand48() - 1.0 : drand48();
  // fmm/driver.cc:149-152
  if (check_ids)
    for (int k = 0; k < num_check; k++) check_ids[k] = int(floor(drand48() * n));
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_tree_build(int num_src, const double* sx, const double* sy,
                                       const double* sz, int num_trg, const double* tx,
                                       const double* ty, const double* tz, int pts_max,
                                       kfmm_tree** out) {
  if (!out || num_src <= 0 || num_trg <= 0 || pts_max <= 0 || !sx || !sy || !sz || !tx ||
      !ty || !tz) {
    set_error("kfmm_tree_build: bad argument");
    return KFMM_ERR_INVALID;
  }
  for (int i = 0; i < num_src; ++i)
    if (!(sx[i] >= -1.0 && sx[i] <= 1.0 && sy[i] >= -1.0 && sy[i] <= 1.0 && sz[i] >= -1.0 &&
          sz[i] <= 1.0)) {
      set_error("kfmm_tree_build: sources must lie in the root box [-1,1]^3");
      return KFMM_ERR_INVALID;
    }
  for (int i = 0; i < num_trg; ++i)
    if (!(tx[i] >= -1.0 && tx[i] <= 1.0 && ty[i] >= -1.0 && ty[i] <= 1.0 && tz[i] >= -1.0 &&
          tz[i] <= 1.0)) {
      set_error("kfmm_tree_build: targets must lie in the root box [-1,1]^3");
      return KFMM_ERR_INVALID;
    }
  kfmm_tree* t = new (std::nothrow) kfmm_tree();
  if (!t) {
    set_error("kfmm_tree_build: out of host memory");
    return KFMM_ERR_ALLOC;
  }
  try {
    build_tree(t->t, num_src, sx, sy, sz, num_trg, tx, ty, tz, pts_max);
  } catch (const std::bad_alloc&) {
    delete t;
    set_error("kfmm_tree_build: out of host memory");
    return KFMM_ERR_ALLOC;
  } catch (const TooDeep&) {
    delete t;
    set_error("kfmm_tree_build: more than pts_max coincident sources: the tree would need more "
              "than 30 levels");
    return KFMM_ERR_UNSUPPORTED;
  }
  *out = t;
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_tree_describe(const kfmm_tree* tree, kfmm_tree_desc* d) {
  if (!tree || !d) {
    set_error("kfmm_tree_describe: null argument");
    return KFMM_ERR_INVALID;
  }
  const Tree& T = tree->t;
  d->num_nodes = T.num_nodes();
  d->num_levels = (int)T.node_level.size() - 1;
  d->num_src = T.num_src;
  d->num_trg = T.num_trg;
  d->parent = T.parent.data();
  d->child = T.child.data();
  d->depth = T.depth.data();
  d->tag = T.tag.data();
  d->path = T.path.data();
  d->src_beg = T.src_beg.data();
  d->src_num = T.src_num.data();
  d->trg_beg = T.trg_beg.data();
  d->trg_num = T.trg_num.data();
  d->src_perm = T.src_perm.data();
  d->trg_perm = T.trg_perm.data();
  d->node_level = T.node_level.data();
  d->u_ptr = T.list_ptr[0].data();
  d->u_idx = T.list_idx[0].data();
  d->v_ptr = T.list_ptr[1].data();
  d->v_idx = T.list_idx[1].data();
  d->w_ptr = T.list_ptr[2].data();
  d->w_idx = T.list_idx[2].data();
  d->x_ptr = T.list_ptr[3].data();
  d->x_idx = T.list_idx[3].data();
  return KFMM_OK;
}

extern "C" void kfmm_tree_destroy(kfmm_tree* tree) { delete tree; }
