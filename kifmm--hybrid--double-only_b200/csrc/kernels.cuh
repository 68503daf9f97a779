// Device kernels of the KIFMM evaluator (sm_100a).  Included by plan.cu only.
//
// Data layout in HBM (all node-major, node = index into the BFS node array):
//   src4[i]      leaf-ordered sources (x, y, z, w), plain form double4
//   src4f[i]     mixed form: (x, y, z) - leaf centre, w      float4
//   trg4[i]      leaf-ordered targets (x, y, z, 0)            double4
//   ctr[n]       node centre and radius (cx, cy, cz, r)       double4
//   uden/dchk/dden[n*P + k]   upward equivalent density, downward check
//                potential, downward equivalent density      double
//   spec/effv[fb][n][32]      source / target spectra, frequency-blocked
//                (see spec_index)             double2 or float2 (mixed)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace kfmm {

constexpr double kOOFP = 1.0 / (4.0 * 3.14159265358979323846);

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// ---------------------------------------------------------------------------
// P2P engine.  A job evaluates one set of targets against a list of source
// sets ("entries").  Targets: real points of a leaf (kind 0) or the UC (1) /
// DC (2) check surface of a node.  Entries: (kind << 28) | node, kind 0 =
// the node's source points, 1 = the node's UE surface carrying uden, 2 = the
// node's DE surface carrying dden.  Output: out[job.out + i] = (or +=)
// 1/(4 pi) sum_j w_j / |t_i - s_j|, pairs with r == 0 skipped
// (fmm/omp.cc:259-283).
// ---------------------------------------------------------------------------
struct P2PJob {
  int tnode, tkind, tbeg, tcnt;
  int ebeg, eend, out, mode;  // mode 0 write, 1 add
};

struct P2PParams {
  const P2PJob* jobs;
  const int* entries;
  const double4* src4;
  const double4* trg4;
  const double4* ctr;
  const int* src_beg;
  const int* src_num;
  const double* uden;
  const double* dden;
  const double* sp_ue;  // 3 per point
  const double* sp_uc;
  const double* sp_de;
  const double* sp_dc;
  double* out;
  int P, Q;
};

// The mixed form's kernels take these besides (a separate struct: the plain
// form's kernel keeps its argument block, and ptxas its register allocation).
struct P2PMixedParams {
  P2PParams p;
  // leaf-order sources as FP32 offsets from their leaf's centre with the
  // density in FP32 (made once per upload); node centres in FP32
  const float4* src4f;
  const float4* ctrf;
  const float* spf_ue;  // the unit UE / DE surfaces in FP32, 3 per point
  const float* spf_de;
  // near field: target i of a job goes to out[out_perm[J.out + i]], the
  // original order (no scatter pass afterwards); null: out[J.out + i]
  const int* out_perm;
};
template <bool kMixed>
using P2PArgs = typename std::conditional<kMixed, P2PMixedParams, P2PParams>::type;
__device__ __forceinline__ const P2PParams& base_of(const P2PParams& a) { return a; }
__device__ __forceinline__ const P2PParams& base_of(const P2PMixedParams& a) { return a.p; }

__device__ __forceinline__ double3 surface_point(const double4 c, const double* sp, int k) {
  // centre + radius * unit-surface point, unfused as fmm/trans.cc:92-100
  double3 r;
  r.x = __dadd_rn(c.x, __dmul_rn(c.w, sp[3 * k]));
  r.y = __dadd_rn(c.y, __dmul_rn(c.w, sp[3 * k + 1]));
  r.z = __dadd_rn(c.z, __dmul_rn(c.w, sp[3 * k + 2]));
  return r;
}

// Mixed precision P2P (kMixed below): coordinates are taken relative to the
// target set's own node centre and rounded to FP32, so the FP32 differences
// keep ~1e-7 of the box size; 1/r comes from the FP32 reciprocal square root;
// terms are summed in FP32 over blocks of 32 sources and the block sums in
// FP64; the result is scaled by 1/(4 pi) in FP64.  Leaf sources are stored as
// FP32 offsets from their own leaf's centre (src4f); the offset between the
// leaf's and the target node's centres is exact in FP32 (centres are
// -1 + (2i + 1) 2^-d: the difference of two is a multiple of 2^-20 below 2 in
// magnitude for the depths <= 20 that plans accept), so a source costs one
// FP32 rounding more than a direct conversion, and half the bytes.

// ---------------------------------------------------------------------------
// Warp-autonomous P2P.  One warp owns one job of up to 32*kMaxSlots targets
// (slot k of lane l is target l + 32k) and walks the job's source sets on its
// own, without block barriers.  Sources are fetched 32 at a time, one per lane
// (coalesced), prepared in the lane, and written to the warp's own shared
// buffer; after __syncwarp every lane reads each source back as a broadcast.
// The next 32 sources are fetched into registers while the current ones are
// used.  Each source then meets the lane's `slots` targets: independent
// dependency chains per source.  r = 0 can only occur between a leaf's own
// sources and targets (equal coordinates always fall in the same leaf), so
// only the self entry carries the r > 0 test (fmm/omp.cc:280).
//
// The kernel is persistent: a grid of (SMs x resident blocks) warps takes jobs
// from an atomic counter; the host orders the jobs by decreasing cost, so the
// largest start first and the tail is short.
// ---------------------------------------------------------------------------
constexpr int kWarpJobsPerBlock = 4;
constexpr int kMaxSlots = 6;  // targets per lane: jobs hold up to 192 targets
#ifndef KFMM_P2P_MIXED_MINB
#define KFMM_P2P_MIXED_MINB 6  // resident blocks per SM asked of the mixed P2P kernel
#endif

__device__ __forceinline__ void load_entry_source(const P2PParams& p, int kind, int node,
                                                  int base, int idx, double3& s, double& w) {
  if (kind == 0) {
    const double4 v = p.src4[base + idx];
    s = make_double3(v.x, v.y, v.z);
    w = v.w;
  } else {
    s = surface_point(p.ctr[node], kind == 1 ? p.sp_ue : p.sp_de, idx);
    w = (kind == 1 ? p.uden : p.dden)[(size_t)node * p.P + idx];
  }
}

template <int NS, bool kGuard>
__device__ __forceinline__ void pairs_fp64(const double (&tx)[NS], const double (&ty)[NS],
                                           const double (&tz)[NS], double (&acc)[NS],
                                           const double4* buf, int cnt) {
#pragma unroll 2
  for (int k = 0; k < cnt; ++k) {
    const double4 s = buf[k];
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      const double dx = tx[t] - s.x, dy = ty[t] - s.y, dz = tz[t] - s.z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      double inv = rsqrt(r2);
      if (kGuard) inv = r2 > 0.0 ? inv : 0.0;
      acc[t] = fma(s.w, inv, acc[t]);
    }
  }
}

// Packed FP32 pairs (sm_100 f32x2 instructions): one instruction updates two
// targets.  t* hold two targets' coordinates; the source components arrive
// duplicated in both halves.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  return ((unsigned long long)__float_as_uint(hi) << 32) | __float_as_uint(lo);
}
__device__ __forceinline__ float lo_of(unsigned long long v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float hi_of(unsigned long long v) {
  return __uint_as_float((unsigned)(v >> 32));
}

template <bool kGuard>
__device__ __forceinline__ unsigned long long pair_term2(unsigned long long tx,
                                                         unsigned long long ty,
                                                         unsigned long long tz, ulonglong2 sxy,
                                                         ulonglong2 szw, unsigned long long blk) {
  unsigned long long out;
  if (kGuard) {
    asm("{\n"
        " .reg .b64 dx, dy, dz, r2, inv;\n"
        " .reg .f32 a, b, ia, ib;\n"
        " .reg .pred pa, pb;\n"
        " sub.f32x2 dx, %1, %4;\n"
        " sub.f32x2 dy, %2, %5;\n"
        " sub.f32x2 dz, %3, %6;\n"
        " mul.f32x2 r2, dx, dx;\n"
        " fma.rn.f32x2 r2, dy, dy, r2;\n"
        " fma.rn.f32x2 r2, dz, dz, r2;\n"
        " mov.b64 {a, b}, r2;\n"
        " rsqrt.approx.ftz.f32 ia, a;\n"
        " rsqrt.approx.ftz.f32 ib, b;\n"
        " setp.gt.f32 pa, a, 0f00000000;\n"
        " setp.gt.f32 pb, b, 0f00000000;\n"
        " selp.f32 ia, ia, 0f00000000, pa;\n"
        " selp.f32 ib, ib, 0f00000000, pb;\n"
        " mov.b64 inv, {ia, ib};\n"
        " fma.rn.f32x2 %0, %7, inv, %8;\n"
        "}\n"
        : "=l"(out)
        : "l"(tx), "l"(ty), "l"(tz), "l"(sxy.x), "l"(sxy.y), "l"(szw.x), "l"(szw.y), "l"(blk));
  } else {
    asm("{\n"
        " .reg .b64 dx, dy, dz, r2, inv;\n"
        " .reg .f32 a, b, ia, ib;\n"
        " sub.f32x2 dx, %1, %4;\n"
        " sub.f32x2 dy, %2, %5;\n"
        " sub.f32x2 dz, %3, %6;\n"
        " mul.f32x2 r2, dx, dx;\n"
        " fma.rn.f32x2 r2, dy, dy, r2;\n"
        " fma.rn.f32x2 r2, dz, dz, r2;\n"
        " mov.b64 {a, b}, r2;\n"
        " rsqrt.approx.ftz.f32 ia, a;\n"
        " rsqrt.approx.ftz.f32 ib, b;\n"
        " mov.b64 inv, {ia, ib};\n"
        " fma.rn.f32x2 %0, %7, inv, %8;\n"
        "}\n"
        : "=l"(out)
        : "l"(tx), "l"(ty), "l"(tz), "l"(sxy.x), "l"(sxy.y), "l"(szw.x), "l"(szw.y), "l"(blk));
  }
  return out;
}

// Scalar FP32 pair, for the odd target of a lane with an odd slot count.
template <bool kGuard>
__device__ __forceinline__ float pair_term1(float tx, float ty, float tz, float sx, float sy,
                                            float sz, float w, float blk) {
  float out;
  if (kGuard) {
    asm("{\n"
        " .reg .f32 dx, dy, dz, r2, inv;\n"
        " .reg .pred pa;\n"
        " sub.f32 dx, %1, %4;\n"
        " sub.f32 dy, %2, %5;\n"
        " sub.f32 dz, %3, %6;\n"
        " mul.f32 r2, dx, dx;\n"
        " fma.rn.f32 r2, dy, dy, r2;\n"
        " fma.rn.f32 r2, dz, dz, r2;\n"
        " rsqrt.approx.ftz.f32 inv, r2;\n"
        " setp.gt.f32 pa, r2, 0f00000000;\n"
        " selp.f32 inv, inv, 0f00000000, pa;\n"
        " fma.rn.f32 %0, %7, inv, %8;\n"
        "}\n"
        : "=f"(out)
        : "f"(tx), "f"(ty), "f"(tz), "f"(sx), "f"(sy), "f"(sz), "f"(w), "f"(blk));
  } else {
    asm("{\n"
        " .reg .f32 dx, dy, dz, r2, inv;\n"
        " sub.f32 dx, %1, %4;\n"
        " sub.f32 dy, %2, %5;\n"
        " sub.f32 dz, %3, %6;\n"
        " mul.f32 r2, dx, dx;\n"
        " fma.rn.f32 r2, dy, dy, r2;\n"
        " fma.rn.f32 r2, dz, dz, r2;\n"
        " rsqrt.approx.ftz.f32 inv, r2;\n"
        " fma.rn.f32 %0, %7, inv, %8;\n"
        "}\n"
        : "=f"(out)
        : "f"(tx), "f"(ty), "f"(tz), "f"(sx), "f"(sy), "f"(sz), "f"(w), "f"(blk));
  }
  return out;
}

// NS targets per lane: NS / 2 packed pairs, plus one scalar target when NS is
// odd (the high half of the last packed register is then unused).  Terms are
// summed in FP32 over blocks of 32 sources (one chunk); the block sums are
// accumulated in FP64 (acc), which keeps the long sum close to a compensated
// FP32 sum and leaves the FP32 pipe to the pair terms.  (The FP32 -> FP64
// conversions take XU slots beside the reciprocal square roots: blocks of 16
// measured 0.11 ms slower at 4M points, with a 2% smaller rel-L2 error.)
// buf: per source {x,x},{y,y} then {z,z},{w,w} (two ulonglong2 per source).
template <int NS, bool kGuard>
__device__ __forceinline__ void pairs_mixed(const unsigned long long (&tx)[(NS + 1) / 2],
                                            const unsigned long long (&ty)[(NS + 1) / 2],
                                            const unsigned long long (&tz)[(NS + 1) / 2],
                                            double (&acc)[NS], const ulonglong2* buf, int cnt) {
  constexpr int NP2 = NS / 2, ODD = NS & 1, kBlock = 32;
  for (int k = 0; k < cnt; k += kBlock) {
    const int m = min(kBlock, cnt - k);
    unsigned long long blk[NP2 > 0 ? NP2 : 1];
    float blk1 = 0.f;
#pragma unroll
    for (int t = 0; t < NP2; ++t) blk[t] = 0ull;
    auto step = [&](int u) {
      const ulonglong2 a = buf[2 * (k + u)], b = buf[2 * (k + u) + 1];
#pragma unroll
      for (int t = 0; t < NP2; ++t) blk[t] = pair_term2<kGuard>(tx[t], ty[t], tz[t], a, b, blk[t]);
      if (ODD)
        blk1 = pair_term1<kGuard>(lo_of(tx[NP2]), lo_of(ty[NP2]), lo_of(tz[NP2]), lo_of(a.x),
                                  lo_of(a.y), lo_of(b.x), lo_of(b.y), blk1);
    };
    if (m == kBlock) {
      constexpr int kUnroll = NS > 4 ? 2 : 4;  // bounds the live pair temporaries
#pragma unroll kUnroll
      for (int u = 0; u < kBlock; ++u) step(u);
    } else {
      for (int u = 0; u < m; ++u) step(u);
    }
#pragma unroll
    for (int t = 0; t < NP2; ++t) {
      acc[2 * t] += (double)lo_of(blk[t]);
      acc[2 * t + 1] += (double)hi_of(blk[t]);
    }
    if (ODD) acc[NS - 1] += (double)blk1;
  }
}

// Target i of job J (i < J.tcnt), absolute FP64 coordinates.
__device__ __forceinline__ double3 job_target(const P2PParams& p, const P2PJob& J,
                                              const double4 org, int i) {
  if (J.tkind == 0) {
    const double4 w = p.trg4[J.tbeg + i];
    return make_double3(w.x, w.y, w.z);
  }
  return surface_point(org, J.tkind == 1 ? p.sp_uc : p.sp_dc, J.tbeg + i);
}

// Cursor over a job's entries, 32 sources at a time: entry e, sources
// [c0, c0 + 32).  It keeps the entry node's centre relative to the target
// node's centre in FP32 (dlt, exact) and the entry node's radius (a power of
// two).
struct EntryCursor {
  int e, eend, c0, kind, node, count, base;
  float3 dlt;
  float rad;
  __device__ __forceinline__ void open(const P2PMixedParams& a, const float4 orgf) {
    const P2PParams& p = a.p;
    for (; e < eend; ++e) {
      const int ent = p.entries[e];
      kind = ent >> 28;
      node = ent & 0x0fffffff;
      count = kind == 0 ? p.src_num[node] : p.P;
      base = kind == 0 ? p.src_beg[node] : 0;
      if (count > 0) break;
    }
    if (e < eend) {
      const float4 k = a.ctrf[node];
      dlt = make_float3(k.x - orgf.x, k.y - orgf.y, k.z - orgf.z);
      rad = k.w;
    }
  }
  __device__ __forceinline__ void advance(const P2PMixedParams& a, const float4 orgf) {
    c0 += 32;
    if (c0 >= count) {
      ++e;
      c0 = 0;
      open(a, orgf);
    }
  }
  // Source c0 + lane of the current entry relative to the entry node's
  // centre: the leaf point's stored offset, or rad * (FP32 unit-surface
  // point), which is exact.  dlt is added when the chunk is written to the
  // warp's buffer, so this load stays in flight across the pair loop.
  __device__ __forceinline__ float4 source(const P2PMixedParams& a, int lane) const {
    const int idx = c0 + lane;
    if (kind == 0) return a.src4f[base + idx];
    const float* sp = (kind == 1 ? a.spf_ue : a.spf_de) + 3 * idx;
    const double w = (kind == 1 ? a.p.uden : a.p.dden)[(size_t)node * a.p.P + idx];
    return make_float4(rad * sp[0], rad * sp[1], rad * sp[2], (float)w);
  }
};

// Mixed form of a row job (see warp-autonomous P2P above): slot k of lane l
// is target l + 32k; each chunk of 32 sources goes through the warp's shared
// buffer in the target node's FP32 frame and is read back as broadcasts.
template <int NS>
__device__ __forceinline__ void warp_job_mixed(const P2PMixedParams& a, const P2PJob& J, int lane,
                                               void* wbuf) {
  const P2PParams& p = a.p;
  const double4 org = p.ctr[J.tnode];
  const float4 orgf = a.ctrf[J.tnode];
  constexpr int NP2C = (NS + 1) / 2;
  unsigned long long tx[NP2C], ty[NP2C], tz[NP2C];
  {
    float q[NS][3];
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      const int i = lane + 32 * t;
      double3 v = make_double3(org.x, org.y, org.z);
      if (i < J.tcnt) v = job_target(p, J, org, i);
      q[t][0] = (float)(v.x - org.x);
      q[t][1] = (float)(v.y - org.y);
      q[t][2] = (float)(v.z - org.z);
    }
#pragma unroll
    for (int t = 0; t < NP2C; ++t) {
      const int u = 2 * t + 1 < NS ? 2 * t + 1 : 2 * t;
      tx[t] = pack2(q[2 * t][0], q[u][0]);
      ty[t] = pack2(q[2 * t][1], q[u][1]);
      tz[t] = pack2(q[2 * t][2], q[u][2]);
    }
  }
  EntryCursor c{J.ebeg, J.eend, 0, 0, 0, 0, 0, make_float3(0.f, 0.f, 0.f), 0.f};
  c.open(a, orgf);
  float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
  if (c.e < c.eend && lane < min(32, c.count)) s = c.source(a, lane);
  double acc[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) acc[t] = 0.0;
  ulonglong2* buf = (ulonglong2*)wbuf;
  while (c.e < c.eend) {
    const int cnt = min(32, c.count - c.c0);
    const bool guard = c.kind == 0 && J.tkind == 0 && c.node == J.tnode;
    if (lane < cnt) {
      const float x = s.x + c.dlt.x, y = s.y + c.dlt.y, z = s.z + c.dlt.z;
      buf[2 * lane] = make_ulonglong2(pack2(x, x), pack2(y, y));
      buf[2 * lane + 1] = make_ulonglong2(pack2(z, z), pack2(s.w, s.w));
    }
    __syncwarp();
    c.advance(a, orgf);
    if (c.e < c.eend && lane < min(32, c.count - c.c0)) s = c.source(a, lane);
    if (guard) pairs_mixed<NS, true>(tx, ty, tz, acc, buf, cnt);
    else pairs_mixed<NS, false>(tx, ty, tz, acc, buf, cnt);
    __syncwarp();
  }
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    const int i = lane + 32 * t;
    if (i < J.tcnt) {
      const double r = kOOFP * acc[t];
      double* o = p.out + (a.out_perm ? a.out_perm[J.out + i] : J.out + i);
      if (J.mode) *o += r;
      else *o = r;
    }
  }
}

// Plain FP64 form of a row job: the same walk, sources staged as double4.
template <int NS>
__device__ __forceinline__ void warp_job_fp64(const P2PParams& p, const P2PJob& J, int lane,
                                              void* wbuf) {
  const double4 org = p.ctr[J.tnode];
  double q[NS][3];
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    const int i = lane + 32 * t;
    double3 v = make_double3(org.x, org.y, org.z);
    if (i < J.tcnt) {
      if (J.tkind == 0) {
        const double4 w = p.trg4[J.tbeg + i];
        v = make_double3(w.x, w.y, w.z);
      } else {
        v = surface_point(org, J.tkind == 1 ? p.sp_uc : p.sp_dc, J.tbeg + i);
      }
    }
    q[t][0] = v.x;
    q[t][1] = v.y;
    q[t][2] = v.z;
  }
  // chunk cursor over the job's entries: entry e, sources [c0, c0 + 32)
  int e = J.ebeg, c0 = 0, kind = 0, node = 0, count = 0, base = 0;
  auto open_entry = [&]() {  // first entry at or after e with sources
    for (; e < J.eend; ++e) {
      const int ent = p.entries[e];
      kind = ent >> 28;
      node = ent & 0x0fffffff;
      count = kind == 0 ? p.src_num[node] : p.P;
      base = kind == 0 ? p.src_beg[node] : 0;
      if (count > 0) return;
    }
  };
  open_entry();
  double3 s = make_double3(0.0, 0.0, 0.0);
  double w = 0.0;
  if (e < J.eend && lane < min(32, count - c0)) load_entry_source(p, kind, node, base, c0 + lane, s, w);

  double sum[NS];
  {
    double tx[NS], ty[NS], tz[NS], acc[NS];
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      tx[t] = q[t][0];
      ty[t] = q[t][1];
      tz[t] = q[t][2];
      acc[t] = 0.0;
    }
    double4* buf = (double4*)wbuf;
    while (e < J.eend) {
      const int cnt = min(32, count - c0);
      const bool guard = kind == 0 && J.tkind == 0 && node == J.tnode;
      if (lane < cnt) buf[lane] = make_double4(s.x, s.y, s.z, w);
      __syncwarp();
      c0 += 32;
      if (c0 >= count) {
        ++e;
        c0 = 0;
        open_entry();
      }
      if (e < J.eend && lane < min(32, count - c0))
        load_entry_source(p, kind, node, base, c0 + lane, s, w);
      if (guard) pairs_fp64<NS, true>(tx, ty, tz, acc, buf, cnt);
      else pairs_fp64<NS, false>(tx, ty, tz, acc, buf, cnt);
      __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < NS; ++t) sum[t] = acc[t];
  }
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    const int i = lane + 32 * t;
    if (i < J.tcnt) {
      const double r = kOOFP * sum[t];
      double* o = p.out + J.out + i;
      if (J.mode) *o += r;
      else *o = r;
    }
  }
}

template <bool kMixed, int NS>
__device__ __forceinline__ void warp_job(const P2PArgs<kMixed>& a, const P2PJob& J, int lane,
                                         void* wbuf) {
  if constexpr (kMixed) warp_job_mixed<NS>(a, J, lane, wbuf);
  else warp_job_fp64<NS>(a, J, lane, wbuf);
}

template <bool kMixed>
__device__ __forceinline__ void run_job(const P2PArgs<kMixed>& a, const P2PJob& J, int lane,
                                        void* wb) {
  switch ((J.tcnt + 31) >> 5) {
    case 1: warp_job<kMixed, 1>(a, J, lane, wb); break;
    case 2: warp_job<kMixed, 2>(a, J, lane, wb); break;
    case 3: warp_job<kMixed, 3>(a, J, lane, wb); break;
    case 4: warp_job<kMixed, 4>(a, J, lane, wb); break;
    case 5: warp_job<kMixed, 5>(a, J, lane, wb); break;
    default: warp_job<kMixed, kMaxSlots>(a, J, lane, wb); break;
  }
}

__device__ __forceinline__ int next_job_of_warp(int* next_job, int lane) {
  int j = 0;
  if (lane == 0) j = atomicAdd(next_job, 1);
  return __shfl_sync(0xffffffffu, j, 0);
}

// Persistent: each warp takes jobs from *next_job until none are left.  The
// counter is zeroed on the stream before every launch.  kMinBlocks: resident
// blocks per SM asked of ptxas; the plan runs the mixed near field with 5
// (96 registers, no spills) when W-list surfaces carry more than 1% of its
// pairs: measured 8-11% faster on ellipsoid-surface clouds, 1-2% slower than
// 6 on uniform ones, whatever the NP.
template <bool kMixed, int kMinBlocks = kMixed ? KFMM_P2P_MIXED_MINB : 4>
__global__ void __launch_bounds__(32 * kWarpJobsPerBlock, kMinBlocks)
p2p_warp_kernel(P2PArgs<kMixed> a, int njobs, int* next_job) {
  __shared__ __align__(16) unsigned char smem[kWarpJobsPerBlock][32 * 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  void* wb = smem[wid];
  for (;;) {
    int j = 0;
    if (lane == 0) j = atomicAdd(next_job, 1);
    j = __shfl_sync(0xffffffffu, j, 0);
    if (j >= njobs) return;
    const P2PJob J = base_of(a).jobs[j];  // a register copy: the output stores may alias
    run_job<kMixed>(a, J, lane, wb);
  }
}

// The near fields of many plans in one persistent launch (batched solves):
// job j is job jobs[j].y of plan jobs[j].x, whose arrays params[jobs[j].x]
// describes.
template <bool kMixed>
__global__ void __launch_bounds__(32 * kWarpJobsPerBlock, kMixed ? KFMM_P2P_MIXED_MINB : 4)
p2p_fused_kernel(const P2PArgs<kMixed>* params, const int2* jobs, int njobs, int* next_job) {
  __shared__ __align__(16) unsigned char smem[kWarpJobsPerBlock][32 * 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  void* wb = smem[wid];
  for (;;) {
    const int j = next_job_of_warp(next_job, lane);
    if (j >= njobs) return;
    const int2 pj = jobs[j];
    const P2PArgs<kMixed>& a = params[pj.x];
    const P2PJob J = base_of(a).jobs[pj.y];
    run_job<kMixed>(a, J, lane, wb);
  }
}

// ---------------------------------------------------------------------------
// Level GEMM on FP64 tensor cores (mma.sync m8n8k4 DMMA):
//   C[:, j] = alpha_j * A * B[:, j]   (+ C[:, j] when accumulate)
// A: M x K column-major (lda = M).  Column j of B starts at B + boff[j]
// (K contiguous values), column j of C at C + coff[j] (M values).
// ---------------------------------------------------------------------------
struct GemmArgs {
  const double* A;
  int M, K;
  int ksplit;        // K range per blockIdx.z (multiple of kGemmBK)
  double* partial;   // split-K: partial sums [z][ncol][M] (no alpha), else NULL
  const double* B;
  const int* boff;
  double* C;
  const int* coff;
  const double* alpha;  // per column, or NULL -> alpha_const
  double alpha_const;
  int ncol;
  int accumulate;
};

__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// A block computes rows [m0, m0 + mrows) of C (mrows <= 160, a multiple of 8)
// for kGemmBN columns.  8 warps = 4 (rows) x 2 (columns); each warp owns 5 x 4
// m8n8 tiles, i.e. 20 DMMA per 4-deep k step for 9 shared loads.  16-deep
// slices of A and B stream into a 3-stage shared-memory ring by asynchronous
// 16-byte copies (cp.async, zero-filled outside the matrices), so no
// registers hold data in flight and two blocks fit on an SM.  Requires M, K
// and every column offset even (16-byte aligned pairs of doubles); the host
// checks this when it builds a batch.
constexpr int kGemmRows = 160, kGemmBN = 64, kGemmBK = 16, kGemmThreads = 256;
constexpr int kGemmStages = 3;
constexpr int kGemmAStride = kGemmRows + 8;  // doubles; 8 and 4 (mod 16): every bank pair
constexpr int kGemmBStride = kGemmBK + 4;    // hit exactly twice by a warp's fragment reads
constexpr int kGemmStageDoubles = kGemmBK * kGemmAStride + kGemmBN * kGemmBStride;
constexpr size_t kGemmSmemBytes = sizeof(double) * kGemmStages * kGemmStageDoubles;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(smem)),
               "l"(gmem), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// kAcc: the launch accumulates onto C (its epilogue reads C; see there).
template <bool kAcc>
__global__ void __launch_bounds__(kGemmThreads, 2) gemm_fp64_dmma_kernel(GemmArgs g, int mrows) {
  extern __shared__ __align__(16) double gsm[];
  __shared__ int boff_s[kGemmBN];
  __shared__ int coff_s[kAcc ? kGemmBN : 1];
  __shared__ double alpha_s[kAcc ? kGemmBN : 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int m0 = blockIdx.x * mrows, n0 = blockIdx.y * kGemmBN;
  const int mend = min(g.M, m0 + mrows);
  const int kb = blockIdx.z * g.ksplit, ke = min(g.K, kb + g.ksplit);
  const int nslices = ke > kb ? (ke - kb + kGemmBK - 1) / kGemmBK : 0;
  if (tid < kGemmBN) {
    const bool in = n0 + tid < g.ncol;
    boff_s[tid] = in ? g.boff[n0 + tid] : -1;
    if constexpr (kAcc) {
      coff_s[tid] = in ? g.coff[n0 + tid] : 0;
      alpha_s[tid] = in ? (g.alpha ? g.alpha[n0 + tid] : g.alpha_const) : 0.0;
    }
  }
  double acc[5][4][2];
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  __syncthreads();
  auto issue = [&](int s) {
    double* As = gsm + (s % kGemmStages) * kGemmStageDoubles;
    double* Bs = As + kGemmBK * kGemmAStride;
    const int k0 = kb + s * kGemmBK;
#pragma unroll
    for (int r = 0; r < kGemmRows * kGemmBK / 2 / kGemmThreads; ++r) {
      const int q = tid + r * kGemmThreads;
      const int k = q / (kGemmRows / 2), m = 2 * (q % (kGemmRows / 2));
      const int gm = m0 + m, gk = k0 + k;
      const bool ok = gm < mend && gk < ke;
      cp_async16(As + k * kGemmAStride + m, ok ? g.A + (size_t)gk * g.M + gm : g.A, ok);
    }
#pragma unroll
    for (int r = 0; r < kGemmBN * kGemmBK / 2 / kGemmThreads; ++r) {
      const int q = tid + r * kGemmThreads;
      const int n = q / (kGemmBK / 2), k = 2 * (q % (kGemmBK / 2));
      const int gk = k0 + k, bo = boff_s[n];
      const bool ok = bo >= 0 && gk < ke;
      cp_async16(Bs + n * kGemmBStride + k, ok ? g.B + (size_t)bo + gk : g.B, ok);
    }
  };
#pragma unroll
  for (int s = 0; s < kGemmStages - 1; ++s) {
    if (s < nslices) issue(s);
    cp_async_commit();
  }
  for (int s = 0; s < nslices; ++s) {
    cp_async_wait<kGemmStages - 2>();
    __syncthreads();
    if (s + kGemmStages - 1 < nslices) issue(s + kGemmStages - 1);
    cp_async_commit();
    const double* As = gsm + (s % kGemmStages) * kGemmStageDoubles;
    const double* Bs = As + kGemmBK * kGemmAStride;
#pragma unroll
    for (int kk = 0; kk < kGemmBK; kk += 4) {
      double af[5], bf[4];
#pragma unroll
      for (int mi = 0; mi < 5; ++mi)
        af[mi] = As[(kk + (lane & 3)) * kGemmAStride + wm * 40 + mi * 8 + (lane >> 2)];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
        bf[ni] = Bs[(wn * 32 + ni * 8 + (lane >> 2)) * kGemmBStride + kk + (lane & 3)];
#pragma unroll
      for (int mi = 0; mi < 5; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) dmma_884(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
    }
  }
  cp_async_wait<0>();
  if constexpr (!kAcc) {
#pragma unroll
    for (int mi = 0; mi < 5; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int m = m0 + wm * 40 + mi * 8 + (lane >> 2);
          const int n = n0 + wn * 32 + ni * 8 + (lane & 3) * 2 + h;
          if (m < mend && n < g.ncol) {
            if (g.partial) {
              g.partial[((size_t)blockIdx.z * g.ncol + n) * g.M + m] = acc[mi][ni][h];
            } else {
              const double a = g.alpha ? g.alpha[n] : g.alpha_const;
              g.C[(size_t)g.coff[n] + m] = a * acc[mi][ni][h];
            }
          }
        }
  } else {
    // Accumulating epilogue, one row of tiles (8 outputs a thread) at a time:
    // the outputs to accumulate onto are all read before any is written
    // (distinct columns never share memory), so the eight loads overlap instead
    // of each waiting behind the previous store (the accumulating down-pass
    // products at 4M points, NP=6: 0.28 -> 0.25 ms).
#pragma unroll
    for (int mi = 0; mi < 5; ++mi) {
      const int m = m0 + wm * 40 + mi * 8 + (lane >> 2);
      double old[4][2];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int nl = wn * 32 + ni * 8 + (lane & 3) * 2 + h;
          old[ni][h] = !g.partial && m < mend && n0 + nl < g.ncol ? g.C[(size_t)coff_s[nl] + m]
                                                                  : 0.0;
        }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int nl = wn * 32 + ni * 8 + (lane & 3) * 2 + h, n = n0 + nl;
          if (m < mend && n < g.ncol) {
            if (g.partial) {
              g.partial[((size_t)blockIdx.z * g.ncol + n) * g.M + m] = acc[mi][ni][h];
            } else {
              const double v = alpha_s[nl] * acc[mi][ni][h];
              g.C[(size_t)coff_s[nl] + m] = old[ni][h] + v;
            }
          }
        }
    }
  }
}

// Split-K: sum the partial products in split order (deterministic), then
// scale and store as the single-pass kernel would.  A grid-wide pass: the
// sums of every output tile proceed in parallel (a reduction by each tile's
// last-arriving block instead serialises 8 x 160 x 64 loads per tile at the
// end of the launch, measured 0.3 ms slower per solve at 4M points, NP=6).
__global__ void gemm_splitk_reduce_kernel(GemmArgs g, int nsplit) {
  const size_t total = (size_t)g.ncol * g.M;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(q / g.M), m = (int)(q % g.M);
    double sum = 0.0;
    for (int z = 0; z < nsplit; ++z) sum += g.partial[((size_t)z * g.ncol + n) * g.M + m];
    const double a = g.alpha ? g.alpha[n] : g.alpha_const;
    double* c = g.C + (size_t)g.coff[n] + m;
    const double v = a * sum;
    if (g.accumulate) *c += v;
    else *c = v;
  }
}

// ---------------------------------------------------------------------------
// V list.  Grids: the (2np)^3 regular grid, x fastest; surface sample (i,j,k)
// sits at (x,y,z) = (i,j,k) + np/2 (fmm/trans.cc:336-358, 395-418).
// Spectrum index (kz * n + ky) * (np + 1) + kx (r2c halves x).
// Both transforms are pruned to the np^3 block that holds the surface.
// ---------------------------------------------------------------------------
// Spectra are stored frequency-blocked: spec[(fb * nn + node) * kFB + f % kFB]
// with fb = f / kFB, so one block of frequencies for every box (nn * 256 B)
// is contiguous and stays resident in L2 while the Hadamard kernel works on it.
constexpr int kFB = 32;
__host__ __device__ __forceinline__ size_t spec_index(int f, int node, int nn) {
  return ((size_t)(f / kFB) * nn + node) * kFB + (f % kFB);
}

struct FFTParams {
  int np, P, F, nn;
  int nboxes;           // entries of nodes
  const int* nodes;     // nodes to transform
  const int* depth;
  const int* surf_idx;  // np^3 -> surface index or -1, index (i*np + j)*np + k
  const int* surf_ijk;  // P x 3
  const double* cs;     // cos(2 pi m / n), m < n
  const double* sn;     // sin(2 pi m / n)
  const double* pln;    // uden (forward) or dchk target (inverse) base
  double* plnout;
  const void* specin;   // double2 (FP64 plans) or float2 (mixed plans)
  void* specout;
};

constexpr int kFFTThreads = 128;
constexpr int kMaxNP = 8;

// Multiplication by (-i)^e.
__device__ __forceinline__ double2 rot_mi(double2 v, int e) {
  switch (e & 3) {
    case 0: return v;
    case 1: return make_double2(v.y, -v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(-v.y, v.x);
  }
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}

// Pruned forward DFT of length N = 2 NP whose input is non-zero at positions
// H .. H + NP - 1 only (the surface block, H = NP / 2):
//   X[q] = sum_k v[k] w^(q (k + H)),  w = exp(-2 pi i / N),  q < N.
// Decimation in the output index: with Q = NP / 2 (NP even) and q = m + jQ,
// w^(jQ (k + H)) = (-i)^(j (k + H)) depends on k mod 4 only, so four partial
// sums per m over k of one residue mod 4 give all four outputs m + jQ:
// NP * NP / 2 complex multiply-adds instead of 2 NP^2.  For odd NP the split
// is on q = m + jNP, k mod 2: NP^2.  Twiddles come from the tables cs, sn
// (cos, sin of 2 pi m / N) at compile-time indices.
template <int NP>
__device__ __forceinline__ void dft_fwd_pruned(const double2 (&v)[NP], double2 (&X)[2 * NP],
                                               const double* cs, const double* sn) {
  constexpr int N = 2 * NP, H = NP / 2;
  constexpr int R = NP % 2 == 0 ? 4 : 2, Q = N / R;
#pragma unroll
  for (int m = 0; m < Q; ++m) {
    double2 S[R];
#pragma unroll
    for (int c = 0; c < R; ++c) S[c] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int e = (m * (k + H)) % N;
      double2& a = S[k % R];
      a.x = fma(v[k].x, cs[e], fma(v[k].y, sn[e], a.x));
      a.y = fma(v[k].y, cs[e], fma(-v[k].x, sn[e], a.y));
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
      double2 o = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < R; ++c) o = cadd(o, rot_mi(S[c], (4 / R) * j * (c + H)));
      X[m + j * Q] = o;
    }
  }
}

// Pruned inverse DFT of length N = 2 NP evaluated at positions H .. H+NP-1:
//   y[k] = sum_q X[q] w^(-q (k + H)),  k < NP.
// With q = m + jQ as above, the inner sum over j only depends on (k + H) mod
// R: R combinations of the X[m + jQ] per m, then NP * Q multiply-adds.
template <int NP>
__device__ __forceinline__ void dft_inv_pruned(const double2 (&X)[2 * NP], double2 (&y)[NP],
                                               const double* cs, const double* sn) {
  constexpr int N = 2 * NP, H = NP / 2;
  constexpr int R = NP % 2 == 0 ? 4 : 2, Q = N / R;
#pragma unroll
  for (int k = 0; k < NP; ++k) y[k] = make_double2(0.0, 0.0);
#pragma unroll
  for (int m = 0; m < Q; ++m) {
    double2 T[R];  // T[c] = sum_j X[m + jQ] (+i)^((4/R) j c), c = (k + H) mod R
#pragma unroll
    for (int c = 0; c < R; ++c) {
      double2 o = make_double2(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < R; ++j) o = cadd(o, rot_mi(X[m + j * Q], -(4 / R) * j * c));
      T[c] = o;
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int e = (m * (k + H)) % N;
      const double2 t = T[(k + H) % R];
      y[k].x = fma(t.x, cs[e], fma(-t.y, sn[e], y[k].x));
      y[k].y = fma(t.y, cs[e], fma(t.x, sn[e], y[k].y));
    }
  }
}

// Boxes per block: as many as fit in ~44 KB of static shared memory (at most
// 3), so that every pass keeps most of the block's threads busy.
template <int NP>
__host__ __device__ constexpr int fft_boxes_per_block() {
  constexpr int N = 2 * NP, NK = NP + 1;
  constexpr int fwd = NP * NP * NP * 8 + NP * NP * NK * 16 + NP * N * NK * 16;
  constexpr int b = 44000 / fwd;
  return b < 1 ? 1 : (b > 3 ? 3 : b);
}

// Pruned 3-D transforms, compiled per NP so every loop over the np^3 surface
// block unrolls and every twiddle index is a constant (the twiddle loads are
// then warp-wide broadcasts).  A block transforms fft_boxes_per_block<NP>()
// boxes.  Each pass gives one thread one line of one box's grid: the x pass a
// (z, y) row, the y pass a (z, kx) column, the z pass a (ky, kx) column, and
// each thread produces all outputs of its line from the <= np non-zero
// inputs.
// Five resident blocks per SM (shared memory allows five at NP = 6): with
// the next group's values held in registers the unbounded kernel takes 168
// registers and three blocks, measured slower on small and surface clouds.
template <int NP, class C>
__global__ void __launch_bounds__(kFFTThreads, 5) fft_src_np_kernel(FFTParams p) {
  constexpr int N = 2 * NP, H = NP / 2, NK = NP + 1, B = fft_boxes_per_block<NP>();
  __shared__ double den[B][NP * NP * NP];
  __shared__ double2 X[B][NP * NP * NK];
  __shared__ double2 Y[B][NP * N * NK];
  __shared__ double cs[N], sn[N];
  constexpr int P = NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2);
  constexpr int R = (B * P + kFFTThreads - 1) / kFFTThreads;  // surface values per thread
  __shared__ int node_s[B];
  __shared__ double scale_s[B];
  __shared__ int cell_s[P];  // surface point -> cell of the np^3 block
  const int tid = threadIdx.x;
  const int ngroups = (p.nboxes + B - 1) / B;
  if (tid < N) {
    cs[tid] = p.cs[tid];
    sn[tid] = p.sn[tid];
  }
  for (int q = tid; q < P; q += kFFTThreads)
    cell_s[q] = (p.surf_ijk[3 * q] * NP + p.surf_ijk[3 * q + 1]) * NP + p.surf_ijk[3 * q + 2];
  // Persistent: the block takes groups of B boxes in turn.  The P surface
  // values of the next group (consecutive threads, consecutive values) and
  // its nodes' scales are loaded into registers while this group is
  // transformed, so the passes do not wait for global memory.
  double pre[R];
  int nx_node = -1;
  double nx_scale = 0.0;
  auto fetch = [&](int grp) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = tid + r * kFFTThreads, bb = q / P, s = q % P, b = grp * B + bb;
      pre[r] = 0.0;
      if (q < B * P && grp < ngroups && b < p.nboxes) pre[r] = p.pln[(size_t)p.nodes[b] * p.P + s];
    }
    if (tid < B) {
      const int b = grp * B + tid;
      nx_node = grp < ngroups && b < p.nboxes ? p.nodes[b] : -1;
      nx_scale = nx_node >= 0 ? ldexp(1.0, p.depth[nx_node]) : 0.0;
    }
  };
  fetch(blockIdx.x);
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    __syncthreads();  // the previous group's passes are done with the shared arrays
    if (tid < B) {
      node_s[tid] = nx_node;
      scale_s[tid] = nx_scale;
    }
    for (int q = tid; q < B * NP * NP * NP; q += kFFTThreads) (&den[0][0])[q] = 0.0;
    __syncthreads();
    // the group's surface values into the boxes' np^3 blocks
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = tid + r * kFFTThreads, bb = q / P, s = q % P;
      if (q < B * P && node_s[bb] >= 0) den[bb][cell_s[s]] = pre[r] * scale_s[bb];
    }
    fetch(grp + gridDim.x);
    __syncthreads();
    // x: row (k = z, j = y), outputs kx
    for (int q = tid; q < B * NP * NP; q += kFFTThreads) {
      const int bb = q / (NP * NP), t = q % (NP * NP);
      const int k = t / NP, j = t % NP;
      double v[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) v[i] = den[bb][(i * NP + j) * NP + k];
#pragma unroll
      for (int kx = 0; kx < NK; ++kx) {
        double ar = 0, ai = 0;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const int m = (kx * (i + H)) % N;
          ar = fma(v[i], cs[m], ar);
          ai = fma(-v[i], sn[m], ai);
        }
        X[bb][(k * NP + j) * NK + kx] = make_double2(ar, ai);
      }
    }
    __syncthreads();
    // y: column (k, kx), outputs ky
    for (int q = tid; q < B * NP * NK; q += kFFTThreads) {
      const int bb = q / (NP * NK), t = q % (NP * NK);
      const int k = t / NK, kx = t % NK;
      double2 v[NP], o[N];
#pragma unroll
      for (int j = 0; j < NP; ++j) v[j] = X[bb][(k * NP + j) * NK + kx];
      dft_fwd_pruned<NP>(v, o, cs, sn);
#pragma unroll
      for (int ky = 0; ky < N; ++ky) Y[bb][(k * N + ky) * NK + kx] = o[ky];
    }
    __syncthreads();
    // z: column (ky, kx), outputs kz -> spectrum
    C* out = (C*)p.specout;
    for (int q = tid; q < B * N * NK; q += kFFTThreads) {
      const int bb = q / (N * NK), t = q % (N * NK);
      const int node = node_s[bb];
      if (node < 0) continue;
      const int ky = t / NK, kx = t % NK;
      double2 v[NP], o[N];
#pragma unroll
      for (int k = 0; k < NP; ++k) v[k] = Y[bb][(k * N + ky) * NK + kx];
      dft_fwd_pruned<NP>(v, o, cs, sn);
#pragma unroll
      for (int kz = 0; kz < N; ++kz) {
        C e;
        e.x = o[kz].x;
        e.y = o[kz].y;
        out[spec_index((kz * N + ky) * NK + kx, node, p.nn)] = e;
      }
    }
  }
}

// spectrum -> c2r -> gather at the DC surface, scaled by 1/(2np)^3
// (omp.cc:482-533, trans.cc:383-418).  Writes plnout[node*P + s].
template <int NP, class C>
__global__ void __launch_bounds__(kFFTThreads) ifft_trg_np_kernel(FFTParams p) {
  constexpr int N = 2 * NP, H = NP / 2, NK = NP + 1, B = fft_boxes_per_block<NP>();
  __shared__ double2 Z[B][NP * N * NK];
  __shared__ double2 W[B][NP * NP * NK];
  __shared__ double cs[N], sn[N];
  __shared__ int node_s[B];
  const int tid = threadIdx.x;
  const int b0 = blockIdx.x * B;
  if (tid < N) {
    cs[tid] = p.cs[tid];
    sn[tid] = p.sn[tid];
  }
  if (tid < B) node_s[tid] = b0 + tid < p.nboxes ? p.nodes[b0 + tid] : -1;
  __syncthreads();
  // z inverse: column (ky, kx), outputs z in the surface block; every
  // spectrum entry is read exactly once, straight from global memory
  // (consecutive threads, consecutive entries)
  const C* in = (const C*)p.specin;
  for (int q = tid; q < B * N * NK; q += kFFTThreads) {
    const int bb = q / (N * NK), t = q % (N * NK);
    const int node = node_s[bb];
    if (node < 0) continue;
    const int ky = t / NK, kx = t % NK;
    double2 v[N], acc[NP];
#pragma unroll
    for (int kz = 0; kz < N; ++kz) {
      const C e = in[spec_index((kz * N + ky) * NK + kx, node, p.nn)];
      v[kz] = make_double2(e.x, e.y);
    }
    dft_inv_pruned<NP>(v, acc, cs, sn);
#pragma unroll
    for (int k = 0; k < NP; ++k) Z[bb][(k * N + ky) * NK + kx] = acc[k];
  }
  __syncthreads();
  // y inverse: column (k, kx), outputs y in the surface block
  for (int q = tid; q < B * NP * NK; q += kFFTThreads) {
    const int bb = q / (NP * NK), t = q % (NP * NK);
    if (node_s[bb] < 0) continue;
    const int k = t / NK, kx = t % NK;
    double2 v[N], acc[NP];
#pragma unroll
    for (int ky = 0; ky < N; ++ky) v[ky] = Z[bb][(k * N + ky) * NK + kx];
    dft_inv_pruned<NP>(v, acc, cs, sn);
#pragma unroll
    for (int j = 0; j < NP; ++j) W[bb][(k * NP + j) * NK + kx] = acc[j];
  }
  __syncthreads();
  // x: Hermitian half -> real, at the surface points only
  constexpr double inv_g = 1.0 / (double)(N * N * N);
  constexpr int P = NP * NP * NP - (NP - 2) * (NP - 2) * (NP - 2);
  for (int q = tid; q < B * P; q += kFFTThreads) {
    const int bb = q / P, s = q % P;
    const int node = node_s[bb];
    if (node < 0) continue;
    const int i = p.surf_ijk[3 * s], j = p.surf_ijk[3 * s + 1], k = p.surf_ijk[3 * s + 2];
    const double2* w = &W[bb][(k * NP + j) * NK];
    const int x = i + H;
    double acc = w[0].x + ((x & 1) ? -w[NP].x : w[NP].x);
    int m = 0;
#pragma unroll
    for (int kx = 1; kx < NP; ++kx) {
      m += x;
      if (m >= N) m -= N;
      acc += 2.0 * (w[kx].x * cs[m] - w[kx].y * sn[m]);
    }
    p.plnout[(size_t)node * p.P + s] = acc * inv_g;
  }
}

// M2L Hadamard accumulation over sibling groups.  A group is the 8 children
// of one parent; their V lists all lie in the 6x6x6 window of same-depth
// positions 2*parent + [-2,3]^3 (fmm/input.cc:311-339), each member taking
// the window entries at Chebyshev distance >= 2 from itself.  Window entry w
// = (wx + 6 wy + 36 wz); member c = 4 cx + 2 cy + cz; offset delta = w - 2 -
// (cx,cy,cz) selects translation spectrum (dx+3) + 7 (dy+3) + 49 (dz+3)
// (fmm/omp_sse_block.cc:581-593).
struct HadamardParams {
  int nn, ngroups, groups_per_block;
  const int* win;      // ngroups x 216 node ids (-1 = absent)
  const int* members;  // ngroups x 8 node ids (-1 = no V list)
  // 343 x Fpad translation spectra, zero for |delta|_inf <= 1 and f >= F
  const double2* trans;
  int Fpad;
  const double2* spec;  // blocked layout
  double2* effv;        // blocked layout
};

constexpr int kHadThreads = 256;  // 8 warps, one group per warp, lane = frequency
constexpr int kHadGroupsInFlight = kHadThreads / 32;
constexpr int kHadGroupsPerBlock = 32;

// A row of the translation table at (dy, dz) with |dy| <= 1 and |dz| <= 1:
// its entries dx = -1, 0, 1 (k = 2, 3, 4 of the row) are adjacent offsets,
// whose spectra are zero (they are not V-list interactions), so the FP64
// window kernel skips those loads and multiply-adds: 27 of the 216 per member.
// (The FP32 kernels below are FMA-bound with their loads scheduled across the
// rows; there a branch per row costs more than the skipped work.)
__device__ __forceinline__ bool near_row(int dy, int dz) {
  return dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1;
}

__device__ __forceinline__ void cmac64(double& ar, double& ai, const double2 t, const double2 s) {
  ar = fma(t.x, s.x, ar);
  ar = fma(-t.y, s.y, ar);
  ai = fma(t.x, s.y, ai);
  ai = fma(t.y, s.x, ai);
}

// Plain FP64 form.  One block: one block of 32 frequencies (blockIdx.y) for
// groups_per_block groups.  Warp = one group, lane = one frequency, all 8
// members of the group in registers; every load of a warp is 32 distinct,
// contiguous values.  The translation spectra are read through L1 (the
// frequency block's FP64 tile, 176 KB, would leave room for one block per
// SM).  The window is walked row by row in x: a row of 6 source spectra
// meets, for each of the 4 (cy, cz) member pairs, one row of 7 translation
// spectra: 12 complex multiply-adds per 7 loads; the next row's source
// spectra are fetched while the current row is multiplied.
__global__ void __launch_bounds__(kHadThreads) hadamard_kernel(HadamardParams p) {
  __shared__ int win[kHadGroupsInFlight][216];
  __shared__ int mem[kHadGroupsInFlight][8];
  const int fb = blockIdx.y;
  const int f = threadIdx.x & 31, slot = threadIdx.x >> 5;
  const int g0 = blockIdx.x * p.groups_per_block;
  const int g1 = min(p.ngroups, g0 + p.groups_per_block);
  const size_t fbase = (size_t)fb * p.nn;
  for (int gb = g0; gb < g1; gb += kHadGroupsInFlight) {
    __syncthreads();
    for (int q = threadIdx.x; q < kHadGroupsInFlight * 216; q += kHadThreads) {
      const int g = gb + q / 216;
      win[q / 216][q % 216] = g < g1 ? p.win[(size_t)g * 216 + q % 216] : -1;
    }
    for (int q = threadIdx.x; q < kHadGroupsInFlight * 8; q += kHadThreads) {
      const int g = gb + q / 8;
      mem[q / 8][q % 8] = g < g1 ? p.members[(size_t)g * 8 + q % 8] : -1;
    }
    __syncthreads();
    if (gb + slot >= g1) continue;  // warp-uniform: no group for this warp
    const int* w = win[slot];
    double2 nxt[6];
#pragma unroll
    for (int wx = 0; wx < 6; ++wx) {
      const int sid = w[wx];
      nxt[wx] = sid >= 0 ? p.spec[(fbase + sid) * kFB + f] : make_double2(0.0, 0.0);
    }
    double ar[8], ai[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) ar[c] = ai[c] = 0.0;
    for (int row = 0; row < 36; ++row) {
      double2 srow[6];
#pragma unroll
      for (int wx = 0; wx < 6; ++wx) srow[wx] = nxt[wx];
      if (row + 1 < 36) {
#pragma unroll
        for (int wx = 0; wx < 6; ++wx) {
          const int sid = w[(row + 1) * 6 + wx];
          nxt[wx] = sid >= 0 ? p.spec[(fbase + sid) * kFB + f] : make_double2(0.0, 0.0);
        }
      }
      const int wy = row % 6, wz = row / 6;
#pragma unroll
      for (int cyz = 0; cyz < 4; ++cyz) {
        const int cy = cyz >> 1, cz = cyz & 1;
        const double2* trow =
            p.trans + (size_t)((wz - 2 - cz + 3) * 49 + (wy - 2 - cy + 3) * 7) * p.Fpad +
            fb * kFB + f;
        auto row_body = [&](auto near) {
          constexpr bool kNear = decltype(near)::value;
          double2 t[7];
#pragma unroll
          for (int k = 0; k < 7; ++k)
            t[k] = kNear && k >= 2 && k <= 4 ? make_double2(0.0, 0.0)
                                            : __ldg(trow + (size_t)k * p.Fpad);
#pragma unroll
          for (int wx = 0; wx < 6; ++wx)
#pragma unroll
            for (int cx = 0; cx < 2; ++cx) {
              const int c = cx * 4 + cy * 2 + cz, k = wx - cx + 1;
              if (kNear && k >= 2 && k <= 4) continue;
              cmac64(ar[c], ai[c], t[k], srow[wx]);
            }
        };
        if (near_row(wy - 2 - cy, wz - 2 - cz)) row_body(std::true_type{});
        else row_body(std::false_type{});
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int m = mem[slot][c];
      if (m >= 0) p.effv[(fbase + m) * kFB + f] = make_double2(ar[c], ai[c]);
    }
  }
}

// ---------------------------------------------------------------------------
// Mixed-form Hadamard, one CTA per SM.  The translation spectra of one block of
// 32 frequencies ([fb][343][32] complex FP32, 87,808 B) are brought into
// shared memory by bulk asynchronous copies (TMA, cp.async.bulk) that
// complete on an mbarrier.  A complex multiply-add is two packed FP32 FMAs on
// the translation value as loaded and the source value duplicated:
//   A += {tr, ti} * {sr, sr},  B += {tr, ti} * {si, si},
//   re = A.x - B.y,  im = A.y + B.x
// so a lane reads 8 B of shared memory per 12/7 multiply-adds and spends no
// instruction on rearranging it.  The products of each half of the window
// (z-planes 0-2 and 3-5, 108 per member of which up to 27 are zero) are
// summed in FP32 and the two half sums added in FP64.
// Warps are autonomous: each loads its own group's window into its slice of
// shared memory.
constexpr int kHad32Threads = 512;
constexpr int kHad32Warps = kHad32Threads / 32;
constexpr unsigned kHad32TileBytes = 343u * kFB * 8u;  // 87,808
constexpr int kHad32Copies = 7;                         // 49 offsets (12,544 B) each
constexpr long long kMbarSpinLimit = 1ll << 24;          // bounded waits

struct Had32Params {
  int nn, ngroups, groups_per_block;
  const int* win;
  const int* members;
  const unsigned long long* rows;  // per window: bit wy + 6 wz set if the row has an entry
  const float2* tile;  // [fb][343][32] translation spectra
  const float2* spec;
  float2* effv;
  int* error;  // set to 1 when the tile copy does not complete
  long long wait_limit;  // tries of the tile-copy wait (kMbarSpinLimit by default)
};

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity,
                                                  long long limit = kMbarSpinLimit) {
  for (long long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Bulk-copies the translation tile of frequency block fb into dst (one
// thread issues, all wait on the mbarrier with a bounded spin of `limit`
// tries).  Returns false in every thread of the block, after setting *error,
// if the copy did not complete; thread 0 then waits (with the full default
// bound) for the copy still in flight to land before the block exits.
__device__ __forceinline__ bool had32_load_tile(const float2* tile, int fb, unsigned char* dst,
                                                unsigned long long* bar, int* error,
                                                long long limit) {
  const unsigned b = smem_addr(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b),
                 "r"(kHad32TileBytes)
                 : "memory");
    const unsigned char* src = (const unsigned char*)(tile + (size_t)fb * 343 * kFB);
    constexpr unsigned chunk = kHad32TileBytes / kHad32Copies;
#pragma unroll 1
    for (int c = 0; c < kHad32Copies; ++c)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];\n" ::"r"(smem_addr(dst + c * chunk)),
          "l"(src + (size_t)c * chunk), "r"(chunk), "r"(b)
          : "memory");
  }
  const bool ready = mbar_wait_bounded(b, 0, limit);
  if (!__syncthreads_and(ready)) {
    if (threadIdx.x == 0) {
      atomicExch(error, 1);
      mbar_wait_bounded(b, 0);  // let copies still in flight land before exiting
    }
    return false;
  }
  return true;
}

__global__ void __launch_bounds__(kHad32Threads, 1) hadamard_fp32_kernel(Had32Params p) {
  extern __shared__ __align__(128) unsigned char had32_dyn[];
  __shared__ int win[kHad32Warps][216];
  __shared__ int mem[kHad32Warps][8];
  __shared__ __align__(8) unsigned long long bar;
  const unsigned long long* tsm = (const unsigned long long*)had32_dyn;
  const int fb = blockIdx.y;
  const int f = threadIdx.x & 31, slot = threadIdx.x >> 5;
  const int g0 = blockIdx.x * p.groups_per_block;
  const int g1 = min(p.ngroups, g0 + p.groups_per_block);
  const size_t fbase = (size_t)fb * p.nn;
  if (!had32_load_tile(p.tile, fb, had32_dyn, &bar, p.error, p.wait_limit)) return;
  for (int g = g0 + slot; g < g1; g += kHad32Warps) {
    for (int q = f; q < 216; q += 32) win[slot][q] = p.win[(size_t)g * 216 + q];
    if (f < 8) mem[slot][f] = p.members[(size_t)g * 8 + f];
    __syncwarp();
    const int* w = win[slot];
    const unsigned long long* spec = (const unsigned long long*)p.spec + fbase * kFB + f;
    unsigned long long rows = p.rows[g];  // rows with no entry are not visited
    unsigned long long A[8], B[8];
    double ar[8], ai[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      A[c] = B[c] = 0ull;
      ar[c] = ai[c] = 0.0;
    }
    auto fold = [&]() {  // the half window's FP32 sums into FP64
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        ar[c] += (double)lo_of(A[c]) - (double)hi_of(B[c]);
        ai[c] += (double)hi_of(A[c]) + (double)lo_of(B[c]);
        A[c] = B[c] = 0ull;
      }
    };
    int row = rows ? __ffsll((long long)rows) - 1 : 36;
    unsigned long long nxt[6];
    if (row < 36) {
#pragma unroll
      for (int wx = 0; wx < 6; ++wx) {
        const int sid = w[row * 6 + wx];
        nxt[wx] = sid >= 0 ? spec[(size_t)sid * kFB] : 0ull;
      }
    }
    bool folded = false;
    while (row < 36) {
      rows &= rows - 1;
      const int next = rows ? __ffsll((long long)rows) - 1 : 36;
      unsigned long long sr[6], si[6];  // {sr, sr}, {si, si}
#pragma unroll
      for (int wx = 0; wx < 6; ++wx) {
        sr[wx] = pack2(lo_of(nxt[wx]), lo_of(nxt[wx]));
        si[wx] = pack2(hi_of(nxt[wx]), hi_of(nxt[wx]));
      }
      if (next < 36) {
#pragma unroll
        for (int wx = 0; wx < 6; ++wx) {
          const int sid = w[next * 6 + wx];
          nxt[wx] = sid >= 0 ? spec[(size_t)sid * kFB] : 0ull;
        }
      }
      const int wy = row % 6, wz = row / 6;
      if (!folded && wz >= 3) {  // end of z-planes 0-2 of the window
        fold();
        folded = true;
      }
#pragma unroll
      for (int cyz = 0; cyz < 4; ++cyz) {
        const int cy = cyz >> 1, cz = cyz & 1;
        const unsigned long long* trow =
            tsm + ((wz - 2 - cz + 3) * 49 + (wy - 2 - cy + 3) * 7) * kFB + f;
        unsigned long long t[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) t[k] = trow[k * kFB];
#pragma unroll
        for (int wx = 0; wx < 6; ++wx)
#pragma unroll
          for (int cx = 0; cx < 2; ++cx) {
            const int c = cx * 4 + cy * 2 + cz;
            const unsigned long long tk = t[wx - cx + 1];
            asm("fma.rn.f32x2 %0, %2, %3, %0;\n"
                "fma.rn.f32x2 %1, %2, %4, %1;\n"
                : "+l"(A[c]), "+l"(B[c])
                : "l"(tk), "l"(sr[wx]), "l"(si[wx]));
          }
      }
      row = next;
    }
    fold();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int m = mem[slot][c];
      if (m >= 0) p.effv[(fbase + m) * kFB + f] = make_float2((float)ar[c], (float)ai[c]);
    }
    __syncwarp();
  }
}

// Pairs of sibling groups whose parents are x-neighbours (parent x even and
// x + 1) share one 8 x 6 x 6 window: a row of 8 source spectra meets each
// row of 7 translation values for both groups, 24 multiply-adds per 7 shared
// loads, which halves the shared-memory traffic per multiply-add.  The 16
// members' FP32 sums of the first half-window are kept in FP64 in the warp's
// slice of shared memory and added to the second half's at the end.  12 warps
// per CTA (up to 168 registers a thread).
//
// Rows whose 8 entries are all absent (windows at the domain's faces, and
// the many empty boxes around clouds on surfaces) are not visited: the plan
// gives each window a mask of its rows that hold an entry (4M points on the
// ellipsoid surface: 1.19 -> 0.65 ms; uniform cube: -2%).  The four centre
// rows, where every member pair meets the zero translation values of the
// adjacent offsets, run as separate runs of a body that skips them (1.527
// -> 1.510 ms at 4M, NP=6); elsewhere they are multiplied like the others:
// row bodies specialised on which member pairs meet an adjacent row (ten
// variants, dispatched per row) were measured 14% slower on the uniform cube.
constexpr int kHadPairThreads = 384;
constexpr int kHadPairWarps = kHadPairThreads / 32;
constexpr size_t kHadPairSumBytes = sizeof(double) * kHadPairWarps * 16 * 2 * 32;
constexpr size_t kHadPairSmemBytes = kHad32TileBytes + kHadPairSumBytes;

struct HadPairParams {
  int nn, npairs, pairs_per_block;
  const int* win;      // npairs x 288: x8 + 8 * (wy + 6 * wz), -1 = absent
  const int* members;  // npairs x 16: group 0 members, then group 1
  const unsigned long long* rows;  // npairs: bit wy + 6 wz set if the row has an entry
  const float2* tile;
  const float2* spec;
  float2* effv;
  int* error;
  long long wait_limit;
};

// One window row for the 4 (cy, cz) member pairs.  trow0 points at the
// translation row of offset (dy, dz) = (wy - 2, wz - 2) for lane f; member
// pair (cy, cz) uses the row cz * 49 + cy * 7 spectra lower.
__device__ __forceinline__ void had_pair_row(unsigned long long (&A)[16],
                                             unsigned long long (&B)[16],
                                             const unsigned long long (&sr)[8],
                                             const unsigned long long (&si)[8],
                                             const unsigned long long* trow0) {
#pragma unroll
  for (int cyz = 0; cyz < 4; ++cyz) {
    const int cy = cyz >> 1, cz = cyz & 1;
    const unsigned long long* trow = trow0 - (cz * 49 + cy * 7) * kFB;
    unsigned long long t[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) t[k] = trow[k * kFB];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int wx = 0; wx < 6; ++wx)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int k = wx - cx + 1;
          const int c = h * 8 + cx * 4 + cy * 2 + cz;
          asm("fma.rn.f32x2 %0, %2, %3, %0;\n"
              "fma.rn.f32x2 %1, %2, %4, %1;\n"
              : "+l"(A[c]), "+l"(B[c])
              : "l"(t[k]), "l"(sr[wx + 2 * h]), "l"(si[wx + 2 * h]));
        }
  }
}

// A centre row of the window (wy and wz in {2, 3}): every member pair (cy, cz)
// meets it at |dy|, |dz| <= 1, so its translation values k = 2..4 (dx = -1,
// 0, 1: adjacent offsets, zero spectra) are neither loaded nor multiplied.
__device__ __forceinline__ void had_pair_row_centre(unsigned long long (&A)[16],
                                                    unsigned long long (&B)[16],
                                                    const unsigned long long (&sr)[8],
                                                    const unsigned long long (&si)[8],
                                                    const unsigned long long* trow0) {
#pragma unroll
  for (int cyz = 0; cyz < 4; ++cyz) {
    const int cy = cyz >> 1, cz = cyz & 1;
    const unsigned long long* trow = trow0 - (cz * 49 + cy * 7) * kFB;
    unsigned long long t[7];
#pragma unroll
    for (int k = 0; k < 7; ++k)
      if (k < 2 || k > 4) t[k] = trow[k * kFB];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int wx = 0; wx < 6; ++wx)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int k = wx - cx + 1;
          if (k >= 2 && k <= 4) continue;
          const int c = h * 8 + cx * 4 + cy * 2 + cz;
          asm("fma.rn.f32x2 %0, %2, %3, %0;\n"
              "fma.rn.f32x2 %1, %2, %4, %1;\n"
              : "+l"(A[c]), "+l"(B[c])
              : "l"(t[k]), "l"(sr[wx + 2 * h]), "l"(si[wx + 2 * h]));
        }
  }
}

__global__ void __launch_bounds__(kHadPairThreads, 1) hadamard_fp32_pair_kernel(HadPairParams p) {
  extern __shared__ __align__(128) unsigned char had32_dyn[];
  __shared__ int win[kHadPairWarps][288];
  __shared__ int mem[kHadPairWarps][16];
  __shared__ __align__(8) unsigned long long bar;
  const unsigned long long* tsm = (const unsigned long long*)had32_dyn;
  const int fb = blockIdx.y;
  const int f = threadIdx.x & 31, slot = threadIdx.x >> 5;
  double* sums = (double*)(had32_dyn + kHad32TileBytes) + (size_t)slot * 16 * 2 * 32 + f;
  const int g0 = blockIdx.x * p.pairs_per_block;
  const int g1 = min(p.npairs, g0 + p.pairs_per_block);
  const size_t fbase = (size_t)fb * p.nn;
  const unsigned long long* spec = (const unsigned long long*)p.spec + fbase * kFB + f;
  if (!had32_load_tile(p.tile, fb, had32_dyn, &bar, p.error, p.wait_limit)) return;
  for (int g = g0 + slot; g < g1; g += kHadPairWarps) {
    for (int q = f; q < 288; q += 32) win[slot][q] = p.win[(size_t)g * 288 + q];
    if (f < 16) mem[slot][f] = p.members[(size_t)g * 16 + f];
    __syncwarp();
    const int* w = win[slot];
    unsigned long long rows = p.rows[g];
    unsigned long long A[16], B[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) A[c] = B[c] = 0ull;
    // the first half-window's sums go to shared memory (FP64) once its rows
    // are done
    auto flush = [&]() {
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        sums[(2 * c) * 32] = (double)lo_of(A[c]) - (double)hi_of(B[c]);
        sums[(2 * c + 1) * 32] = (double)hi_of(A[c]) + (double)lo_of(B[c]);
        A[c] = B[c] = 0ull;
      }
    };
    // Rows in four runs: the first half-window's other rows, its centre rows
    // (14, 15), the flush, the second half's centre rows (20, 21), then its
    // other rows; the centre rows skip the zero adjacent offsets.
    constexpr unsigned long long kLow = (1ull << 18) - 1;  // z-planes 0-2
    constexpr unsigned long long kCentre = (1ull << 14) | (1ull << 15) | (1ull << 20) | (1ull << 21);
    auto run_rows = [&](int run) {
      return rows & (run < 2 ? kLow : ~kLow) & (run == 1 || run == 2 ? kCentre : ~kCentre);
    };
    auto first_after = [&](int run) {  // first row of the runs after `run`, 36 if none
      for (int q = run + 1; q < 4; ++q) {
        const unsigned long long mm = run_rows(q);
        if (mm) return __ffsll((long long)mm) - 1;
      }
      return 36;
    };
    // the next row's source spectra are loaded while the current row is
    // multiplied, across the runs' boundaries too
    unsigned long long nxt[8];
    auto fetch = [&](int r) {
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const int sid = w[r * 8 + x];
        nxt[x] = sid >= 0 ? spec[(size_t)sid * kFB] : 0ull;
      }
    };
    {
      const int r0 = first_after(-1);
      if (r0 < 36) fetch(r0);
    }
#pragma unroll 1
    for (int run = 0; run < 4; ++run) {
      if (run == 2) flush();
      unsigned long long m = run_rows(run);
      int row = m ? __ffsll((long long)m) - 1 : 36;
      auto walk = [&](auto centre) {
        while (row < 36) {
          m &= m - 1;
          const int next = m ? __ffsll((long long)m) - 1 : 36;
          const int ahead = next < 36 ? next : first_after(run);
          unsigned long long sr[8], si[8];  // {sr, sr}, {si, si}
#pragma unroll
          for (int x = 0; x < 8; ++x) {
            sr[x] = pack2(lo_of(nxt[x]), lo_of(nxt[x]));
            si[x] = pack2(hi_of(nxt[x]), hi_of(nxt[x]));
          }
          if (ahead < 36) fetch(ahead);
          const int wy = row % 6, wz = row / 6;
          const unsigned long long* trow0 = tsm + ((wz + 1) * 49 + (wy + 1) * 7) * kFB + f;
          if constexpr (decltype(centre)::value) had_pair_row_centre(A, B, sr, si, trow0);
          else had_pair_row(A, B, sr, si, trow0);
          row = next;
        }
      };
      if (run == 1 || run == 2) walk(std::true_type{});
      else walk(std::false_type{});
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int m = mem[slot][c];
      if (m >= 0)
        p.effv[(fbase + m) * kFB + f] =
            make_float2((float)(sums[(2 * c) * 32] + ((double)lo_of(A[c]) - (double)hi_of(B[c]))),
                        (float)(sums[(2 * c + 1) * 32] + ((double)hi_of(A[c]) + (double)lo_of(B[c]))));
    }
    __syncwarp();
  }
}

#include "hadamard_tc.cuh"

// ---------------------------------------------------------------------------
// Point reordering (fmm/evaluate.cc:14-52 on the host in the reference) and
// the final scatter to original order (copy_trg_val, fmm/cuda.cu:2543-2565).
// ---------------------------------------------------------------------------
// Points to leaf order, driven from the original order: point k (read
// coalesced) goes to leaf-order position inv[k], one full 32-byte record
// (and, for mixed plans, a 16-byte record of FP32 offsets from the point's
// leaf centre, leaf[i]) per store; gathering instead reads 8 bytes from four
// random places per point (measured 0.21 ms against ... at 4M points).
__global__ void scatter_points_kernel(int n, const int* inv, const double* x, const double* y,
                                      const double* z, const double* w, double4* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[inv[k]] = make_double4(x[k], y[k], z[k], w ? w[k] : 0.0);
}

// Mixed plans keep only the FP32 offsets (src4f); leaf[k]: source k's leaf.
__global__ void scatter_sources_mixed_kernel(int n, const int* inv, const int* leaf,
                                             const double* x, const double* y, const double* z,
                                             const double* w, const double4* ctr, float4* outf) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double4 c = ctr[leaf[k]];
    outf[inv[k]] =
        make_float4((float)(x[k] - c.x), (float)(y[k] - c.y), (float)(z[k] - c.z), (float)w[k]);
  }
}

// Leaf-order view of original-order potentials (introspection).
__global__ void gather_pot_kernel(int n, const int* perm, const double* pot_orig,
                                  double* pot_leaf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pot_leaf[i] = pot_orig[perm[i]];
}

__global__ void scatter_pot_kernel(int n, const int* perm, const double* pot_leaf,
                                   double* pot_orig) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pot_orig[perm[i]] = pot_leaf[i];
}

// error[1] |= error[0]: the per-solve flag of a bounded wait folded into the
// flag kfmm_evaluate_wait reports for every solve queued since the last wait.
__global__ void error_fold_kernel(int* error) {
  if (error[0]) error[1] = 1;
}

// Plain direct sum (ulist__direct_evaluation) over SoA device arrays.
__global__ void __launch_bounds__(128) direct_fp64_kernel(int nt, const double* tx,
                                                          const double* ty, const double* tz,
                                                          double* pot, int ns, const double* sx,
                                                          const double* sy, const double* sz,
                                                          const double* den) {
  __shared__ double4 stage[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double x = 0, y = 0, z = 0, acc = 0;
  if (i < nt) {
    x = tx[i];
    y = ty[i];
    z = tz[i];
  }
  for (int b = 0; b < ns; b += 256) {
    const int m = min(256, ns - b);
    for (int k = threadIdx.x; k < m; k += blockDim.x)
      stage[k] = make_double4(sx[b + k], sy[b + k], sz[b + k], den[b + k]);
    __syncthreads();
    for (int j = 0; j < m; ++j) {
      const double4 s = stage[j];
      const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      acc = fma(s.w, r2 > 0.0 ? rsqrt(r2) : 0.0, acc);
    }
    __syncthreads();
  }
  if (i < nt) pot[i] += kOOFP * acc;
}

}  // namespace kfmm
