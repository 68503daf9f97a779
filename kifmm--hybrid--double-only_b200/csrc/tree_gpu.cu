// Octree construction with the point work on the GPU (kfmm_tree_build_device).
//
// Produces exactly the tree of kfmm_tree_build (node numbering, tags, point
// permutations, lists; fmm/input.cc:204-460) in a different way:
//
//   1. Every point gets the integer cell (px, py, pz) at depth 21 that the
//      reference's comparisons "x >= centre" (fmm/input.cc:250-256) select
//      level by level.  The centres -1 + (2p + 1) / 2^d are exact dyadic
//      numbers, so the comparisons select p = floor((x + 1) 2^20) in exact
//      arithmetic; the kernel takes the floating-point estimate and corrects
//      it against the exact cell boundaries -1 + p / 2^20 (exact in FP64).
//      Interleaving the bits, x highest at every level, gives a 63-bit
//      Morton key whose order is the order of the child indices 4a + 2b + c
//      (fmm/input.cc:142-147) level by level.
//   2. The source keys are sorted (CUB radix sort).  A node is then a
//      contiguous range of the sorted keys; the host grows the tree breadth
//      first, splitting a node when its range holds more than pts_max
//      sources, and finds the children's ranges by binary search.
//   3. Each source is keyed (leaf node index, original index) and sorted:
//      the result is the reference's leaf-order permutation (leaves in node
//      order, points of a leaf by increasing index, input.cc:282-296).
//   4. Each target descends the tree on the GPU to its deepest node and is
//      keyed and sorted the same way (input.cc:387-449).
//   5. Lists are built on the host from the finished structure (build_lists).
//
// Trees deeper than 21 levels are refused (KFMM_ERR_UNSUPPORTED): use
// kfmm_tree_build for them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <cub/cub.cuh>
#include <new>
#include <string>
#include <vector>

#include "host.h"

namespace kfmm {
namespace {

constexpr int kMaxDepth = 21;
constexpr double kCell = 2.0 / (double)(1 << kMaxDepth);  // cell width at depth 21

__host__ __device__ __forceinline__ unsigned cell_of(double x) {
  const int top = (1 << kMaxDepth) - 1;
  int p = (int)floor((x + 1.0) / kCell);
  p = p < 0 ? 0 : (p > top ? top : p);
  // exact boundaries -1 + p 2^-20
  while (p > 0 && x < -1.0 + (double)p * kCell) --p;
  while (p < top && x >= -1.0 + (double)(p + 1) * kCell) ++p;
  return (unsigned)p;
}

__host__ __device__ __forceinline__ unsigned long long spread3(unsigned v) {
  unsigned long long x = v & 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

__global__ void morton_kernel(int n, const double* x, const double* y, const double* z,
                              unsigned long long* key, int* idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    key[i] = spread3(cell_of(x[i])) << 2 | spread3(cell_of(y[i])) << 1 | spread3(cell_of(z[i]));
    if (idx) idx[i] = i;
  }
}

// sorted position j -> (leaf node << 32 | original index), leaves given by
// their first sorted position (ascending) and node index
__global__ void leaf_key_kernel(int n, const int* sorted_idx, int nleaves, const int* leaf_lo,
                                const int* leaf_node, unsigned long long* out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    int a = 0, b = nleaves - 1;  // last leaf with lo <= j
    while (a < b) {
      const int m = (a + b + 1) >> 1;
      if (leaf_lo[m] <= j) a = m;
      else b = m - 1;
    }
    out[j] = (unsigned long long)leaf_node[a] << 32 | (unsigned)sorted_idx[j];
  }
}

// target i descends from the root to its deepest node
__global__ void descend_kernel(int n, const unsigned long long* key, const int* child,
                               unsigned long long* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long k = key[i];
    int node = 0;
    for (int d = 0; d < kMaxDepth && child[node] != -1; ++d)
      node = child[node] + (int)((k >> (3 * (kMaxDepth - 1 - d))) & 7);
    out[i] = (unsigned long long)node << 32 | (unsigned)i;
  }
}

struct DeviceBuffers {
  std::vector<void*> ptrs;
  ~DeviceBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t n) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) ptrs.push_back(v);
    *p = (T*)v;
    return e;
  }
};

#define KF_TREE_TRY(x)            \
  do {                            \
    kfmm_status s_ = (x);         \
    if (s_ != KFMM_OK) return s_; \
  } while (0)

#define TB_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      set_error(std::string("kfmm_tree_build_device: ") + #call + ": " +             \
                cudaGetErrorString(e_));                                             \
      return KFMM_ERR_CUDA;                                                          \
    }                                                                                \
  } while (0)

kfmm_status sort_u64(DeviceBuffers& B, unsigned long long* keys, int* vals, int n,
                     cudaStream_t st) {
  unsigned long long* k2;
  int* v2 = nullptr;
  TB_CUDA(B.alloc(&k2, n));
  if (vals) TB_CUDA(B.alloc(&v2, n));
  size_t bytes = 0;
  if (vals)
    TB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, k2, vals, v2, n, 0, 64, st));
  else
    TB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys, k2, n, 0, 64, st));
  void* tmp;
  TB_CUDA(B.alloc((unsigned char**)&tmp, bytes));
  if (vals)
    TB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, keys, k2, vals, v2, n, 0, 64, st));
  else
    TB_CUDA(cub::DeviceRadixSort::SortKeys(tmp, bytes, keys, k2, n, 0, 64, st));
  TB_CUDA(cudaMemcpyAsync(keys, k2, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice,
                          st));
  if (vals) TB_CUDA(cudaMemcpyAsync(vals, v2, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  return KFMM_OK;
}

kfmm_status build_on_device(Tree& T, int ns, const double* sx, const double* sy,
                            const double* sz, int nt, const double* tx, const double* ty,
                            const double* tz, int pts_max, cudaStream_t st) {
  DeviceBuffers B;
  double *dx, *dy, *dz;
  unsigned long long* skey;
  int* sidx;
  const int grid = 1024, threads = 256;
  T.num_src = ns;
  T.num_trg = nt;

  // 1-2. source keys, sorted
  TB_CUDA(B.alloc(&dx, ns));
  TB_CUDA(B.alloc(&dy, ns));
  TB_CUDA(B.alloc(&dz, ns));
  TB_CUDA(B.alloc(&skey, ns));
  TB_CUDA(B.alloc(&sidx, ns));
  TB_CUDA(cudaMemcpyAsync(dx, sx, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(dy, sy, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(dz, sz, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
  morton_kernel<<<grid, threads, 0, st>>>(ns, dx, dy, dz, skey, sidx);
  TB_CUDA(cudaGetLastError());
  KF_TREE_TRY(sort_u64(B, skey, sidx, ns, st));
  std::vector<unsigned long long> keys(ns);
  TB_CUDA(cudaMemcpyAsync(keys.data(), skey, sizeof(unsigned long long) * ns,
                          cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));

  // grow the tree breadth first over the sorted keys
  T.parent.assign(1, -1);
  T.child.assign(1, -1);
  T.depth.assign(1, 0);
  T.path.assign(3, 0);
  T.node_level.assign(1, 0);
  std::vector<int> lo(1, 0), hi(1, ns);
  std::vector<unsigned long long> prefix(1, 0);
  int beg = 0, end = 1;
  while (beg < end) {
    for (int k = beg; k < end; ++k) {
      if (hi[k] - lo[k] <= pts_max) continue;
      const int d = T.depth[k];
      if (d >= kMaxDepth) {
        set_error("kfmm_tree_build_device: the tree needs more than 21 levels; use "
                  "kfmm_tree_build");
        return KFMM_ERR_UNSUPPORTED;
      }
      const int first = (int)T.parent.size();
      T.child[k] = first;
      const int shift = 3 * (kMaxDepth - d - 1);
      int o = lo[k];
      for (int c = 0; c < 8; ++c) {
        const unsigned long long pc = prefix[k] << 3 | (unsigned long long)c;
        const unsigned long long limit = (pc + 1) << shift;  // first key past child c
        const int e = c == 7 ? hi[k]
                             : (int)(std::lower_bound(keys.begin() + o, keys.begin() + hi[k],
                                                      limit) -
                                     keys.begin());
        T.parent.push_back(k);
        T.child.push_back(-1);
        T.depth.push_back(d + 1);
        T.path.push_back(2 * T.path[3 * k] + (c >> 2));
        T.path.push_back(2 * T.path[3 * k + 1] + ((c >> 1) & 1));
        T.path.push_back(2 * T.path[3 * k + 2] + (c & 1));
        lo.push_back(o);
        hi.push_back(e);
        prefix.push_back(pc);
        o = e;
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
  std::vector<int> leaf_lo, leaf_node;  // non-empty source leaves by first position
  int sum = 0;
  for (int i = 0; i < nn; ++i) {
    const int cnt = hi[i] - lo[i];
    if (cnt <= 0) continue;
    T.tag[i] |= kSrcTag;
    if (T.child[i] == -1) {
      T.src_beg[i] = sum;
      T.src_num[i] = cnt;
      sum += cnt;
      leaf_lo.push_back(lo[i]);
      leaf_node.push_back(i);
    }
  }
  {
    std::vector<int> order(leaf_lo.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return leaf_lo[a] < leaf_lo[b]; });
    std::vector<int> l2(order.size()), n2(order.size());
    for (size_t i = 0; i < order.size(); ++i) {
      l2[i] = leaf_lo[order[i]];
      n2[i] = leaf_node[order[i]];
    }
    leaf_lo.swap(l2);
    leaf_node.swap(n2);
  }

  // 3. sources by (leaf, index)
  int *dlo, *dnode, *dchild;
  unsigned long long* lkey;
  TB_CUDA(B.alloc(&dlo, leaf_lo.size()));
  TB_CUDA(B.alloc(&dnode, leaf_node.size()));
  TB_CUDA(B.alloc(&lkey, ns));
  TB_CUDA(cudaMemcpyAsync(dlo, leaf_lo.data(), sizeof(int) * leaf_lo.size(),
                          cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(dnode, leaf_node.data(), sizeof(int) * leaf_node.size(),
                          cudaMemcpyHostToDevice, st));
  leaf_key_kernel<<<grid, threads, 0, st>>>(ns, sidx, (int)leaf_lo.size(), dlo, dnode, lkey);
  TB_CUDA(cudaGetLastError());
  KF_TREE_TRY(sort_u64(B, lkey, nullptr, ns, st));
  std::vector<unsigned long long> sk(ns);
  TB_CUDA(cudaMemcpyAsync(sk.data(), lkey, sizeof(unsigned long long) * ns,
                          cudaMemcpyDeviceToHost, st));

  // 4. targets: keys, descent, sort by (node, index)
  double *ex, *ey, *ez;
  unsigned long long *tkey, *tleaf;
  TB_CUDA(B.alloc(&ex, nt));
  TB_CUDA(B.alloc(&ey, nt));
  TB_CUDA(B.alloc(&ez, nt));
  TB_CUDA(B.alloc(&tkey, nt));
  TB_CUDA(B.alloc(&tleaf, nt));
  TB_CUDA(B.alloc(&dchild, nn));
  TB_CUDA(cudaMemcpyAsync(ex, tx, sizeof(double) * nt, cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(ey, ty, sizeof(double) * nt, cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(ez, tz, sizeof(double) * nt, cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemcpyAsync(dchild, T.child.data(), sizeof(int) * nn, cudaMemcpyHostToDevice, st));
  morton_kernel<<<grid, threads, 0, st>>>(nt, ex, ey, ez, tkey, nullptr);
  TB_CUDA(cudaGetLastError());
  descend_kernel<<<grid, threads, 0, st>>>(nt, tkey, dchild, tleaf);
  TB_CUDA(cudaGetLastError());
  KF_TREE_TRY(sort_u64(B, tleaf, nullptr, nt, st));
  std::vector<unsigned long long> tk(nt);
  TB_CUDA(cudaMemcpyAsync(tk.data(), tleaf, sizeof(unsigned long long) * nt,
                          cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));

  T.src_perm.resize(ns);
  for (int j = 0; j < ns; ++j) T.src_perm[j] = (int)(unsigned)sk[j];
  std::vector<int> tcount(nn, 0);
  T.trg_perm.resize(nt);
  for (int j = 0; j < nt; ++j) {
    T.trg_perm[j] = (int)(unsigned)tk[j];
    ++tcount[(int)(tk[j] >> 32)];
  }
  // a node holds targets when a node below it (or itself) does: children
  // always have larger indices than their parent
  std::vector<int> tsub(tcount);
  for (int i = nn - 1; i > 0; --i) tsub[T.parent[i]] += tsub[i];
  sum = 0;
  for (int i = 0; i < nn; ++i) {
    if (tsub[i] <= 0) continue;
    T.tag[i] |= kTrgTag;
    if (T.child[i] == -1) {
      T.trg_beg[i] = sum;
      T.trg_num[i] = tsub[i];
      sum += tsub[i];
    }
  }
  return KFMM_OK;
}

}  // namespace
}  // namespace kfmm

using namespace kfmm;

extern "C" kfmm_status kfmm_tree_build_device(int num_src, const double* sx, const double* sy,
                                              const double* sz, int num_trg, const double* tx,
                                              const double* ty, const double* tz, int pts_max,
                                              void* stream, kfmm_tree** out) {
  if (!out || num_src <= 0 || num_trg <= 0 || pts_max <= 0 || !sx || !sy || !sz || !tx ||
      !ty || !tz) {
    set_error("kfmm_tree_build_device: bad argument");
    return KFMM_ERR_INVALID;
  }
  *out = nullptr;
  for (int i = 0; i < num_src; ++i)
    if (!(sx[i] >= -1.0 && sx[i] <= 1.0 && sy[i] >= -1.0 && sy[i] <= 1.0 && sz[i] >= -1.0 &&
          sz[i] <= 1.0)) {
      set_error("kfmm_tree_build_device: sources must lie in the root box [-1,1]^3");
      return KFMM_ERR_INVALID;
    }
  for (int i = 0; i < num_trg; ++i)
    if (!(tx[i] >= -1.0 && tx[i] <= 1.0 && ty[i] >= -1.0 && ty[i] <= 1.0 && tz[i] >= -1.0 &&
          tz[i] <= 1.0)) {
      set_error("kfmm_tree_build_device: targets must lie in the root box [-1,1]^3");
      return KFMM_ERR_INVALID;
    }
  kfmm_tree* t = new (std::nothrow) kfmm_tree();
  if (!t) {
    set_error("kfmm_tree_build_device: out of host memory");
    return KFMM_ERR_ALLOC;
  }
  try {
    kfmm_status s = build_on_device(t->t, num_src, sx, sy, sz, num_trg, tx, ty, tz, pts_max,
                                    (cudaStream_t)stream);
    if (s != KFMM_OK) {
      delete t;
      return s;
    }
    build_lists(t->t);
  } catch (const std::bad_alloc&) {
    delete t;
    set_error("kfmm_tree_build_device: out of host memory");
    return KFMM_ERR_ALLOC;
  }
  *out = t;
  return KFMM_OK;
}
