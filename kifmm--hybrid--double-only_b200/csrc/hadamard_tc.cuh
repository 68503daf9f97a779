// Mixed-form V-list Hadamard on the fifth-generation tensor cores (tcgen05,
// kind::tf32), for tree levels whose boxes are all present.  Included by
// kernels.cuh.
//
// The products.  Per frequency f, the 8 children of a parent (a sibling
// group) receive E_c[f] = sum_w T[w - c][f] * S_w[f] over the 6 x 6 x 6
// window w of same-depth boxes around them (their V lists; the translation
// spectra T are zero at the 27 adjacent offsets; fmm/omp_sse_block.cc:537-658,
// fmm/cuda.cu:1200-1240).  With the complex numbers in real form this is a
// matrix product per frequency,
//     D[g][n] = sum_k A[g][k] B[k][n],  g = group, n = (member, re|im) (16),
//     k = (window box, re|im of S) (432),
// B[k][n] the translation spectra arranged per member, shared by all groups.
//
// The A operand without a gather.  A tile is 8 groups along x by 16 along y
// at one z (M = 128 rows).  Shared memory holds the tile's neighbourhood as
// z-planes of 20 x 36 boxes, each box one complex FP32 value (8 bytes, re
// then im) at frequency f.  A K-major core matrix of the MMA is 8 rows of 16
// bytes at a 16-byte row stride: rows = 8 consecutive groups along x, whose
// windows start 2 boxes (16 bytes) apart, so the 16-byte K chunk {re, im} of
// boxes (wx, wx + 1) of every group's window is read in place from one plane
// row; successive groups along y (row blocks) are 2 plane rows (320 bytes)
// apart; the two K chunks of one MMA (K = 8) sit at a free leading-byte
// offset, so one MMA covers window boxes wx 0..3 of a row, the next wx 4..5
// of that row and 0..1 of the next (LBO = one plane row - 32 bytes), the
// third wx 2..5 of the second row: 3 MMAs per pair of window rows, 54 per
// pass, no padding.  Every group thus reads its 216 window values straight
// from the shared planes: nothing is duplicated.
//
// Precision: FP32 spectra are split into TF32 hi = rn(x), lo = rn(x - hi);
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi (three passes; the products keep ~22
// of FP32's 24 mantissa bits).  The tensor cores' FP32 accumulation rounds
// toward zero, so a long chain of MMAs into one accumulator drifts: one
// accumulator for all 162 MMAs of a tile measured 4.8e-6 of max |E| on
// random spectra.  The hi x hi pass therefore goes to six accumulators (one
// per window plane, 9 MMAs each) and both correction passes to a seventh
// (their terms are 2^-11 smaller); the epilogue adds the seven in FP64.
//
// Schedule.  A CTA per SM takes work units (frequency, tile column: the
// tiles at every z of one (x, y) tile position of one level) from a counter,
// frequency-major (one block of 32 frequencies of every box stays in L2).
// The unit's translation matrix (hi and lo, 55 KB, precomputed in the
// shared-memory layout per frequency) arrives by one bulk copy into one of two
// buffers while the previous unit runs.  Along z a tile needs 6 planes, of
// which 4 are the previous tile's: a ring of 8 planes takes the 2 new ones,
// filled by all threads (gathered from the frequency-blocked spectra, split
// hi/lo) while the tensor cores work on the current tile.  Thread 0 issues
// the MMAs (seven 16-column accumulators per tile, in two tile buffers of
// tensor memory) and commits them to an mbarrier; warps 0-3 read the
// finished accumulators of the previous tile (tcgen05.ld, one lane per
// group) and store the members' target spectra while the next tile's MMAs
// run.
//
// Every wait is bounded: a wait that runs out sets *error, the CTA waits
// (bounded) for its own copies and MMAs still in flight, frees its tensor
// memory and returns.
#pragma once

// (inside namespace kfmm: kernels.cuh includes this file within it)

constexpr int kTcThreads = 256;
constexpr int kTcGX = 8, kTcGY = 16;                      // groups per tile along x, y
constexpr int kTcPX = 2 * kTcGX + 4, kTcPY = 2 * kTcGY + 4;  // 20 x 36 boxes per plane
constexpr int kTcRowBytes = kTcPX * 8;                    // 160
constexpr int kTcPlaneBytes = kTcRowBytes * kTcPY;        // 5,760
constexpr int kTcRing = 8;
constexpr int kTcRingBytes = kTcRing * kTcPlaneBytes;     // 46,080 (hi or lo)
constexpr int kTcMma = 54;                                // MMAs (K = 8) per pass
constexpr int kTcBPartBytes = kTcMma * 512;               // 27,648: B hi or B lo
constexpr int kTcBBytes = 2 * kTcBPartBytes;              // 55,296 per frequency
constexpr size_t kTcSmemBytes = 2 * (size_t)kTcBBytes + 2 * (size_t)kTcRingBytes;  // 202,752
constexpr int kTcMaxLevels = 8;
constexpr int kTcAcc = 7;             // accumulators per tile: hi x hi per plane, corrections
constexpr int kTcBufCols = 128;       // tensor-memory columns per tile buffer (7 x 16 used)
constexpr int kTcCols = 2 * kTcBufCols;  // allocated: two tile buffers
constexpr int kTcFillPerThread = (2 * kTcPX * kTcPY + kTcThreads - 1) / kTcThreads;  // 6
// instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N = 16 (bits 17-22 = N/8), M = 128
// (bits 24-28 = M/16)
constexpr unsigned kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) |
                              ((128u >> 4) << 24);

struct TcLevel {
  int n;            // boxes per dimension (2^depth)
  int ntx, nty;     // tiles along x and y
  int col0;         // first tile column of this level in a frequency's unit range
  const int* srcmap;  // n^3, index (z n + y) n + x: node holding the box's source spectrum, or -1
  const int* trgmap;  // n^3: node whose target spectrum the box receives, or -1
};

struct HadTcParams {
  int nn, F;
  int nlevels, cols;  // tile columns per frequency (all levels)
  TcLevel lv[kTcMaxLevels];
  const unsigned char* btab;  // [F][hi, lo][54][512 B], the MMAs' B operands
  const float2* spec;
  float2* effv;
  int* next_unit;  // zero before the launch
  int* error;
  long long wait_limit;
};

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major: start address,
// leading (K) and stride (M/N) byte offsets in 16-byte units, version 1.
__device__ __forceinline__ unsigned long long tc_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3fff) |
         ((unsigned long long)((lbo >> 4) & 0x3fff) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(unsigned tmem_d, unsigned long long adesc,
                                       unsigned long long bdesc, unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %3, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(kTcIdesc)
      : "memory");
}

__device__ __forceinline__ void tc_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ float tf32_rn(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

// One thread: bulk copies of `bytes` (a multiple of 64, 16-byte aligned
// addresses) into dst in four pieces, completing on bar.
__device__ __forceinline__ void tc_bulk_load(unsigned dst, const unsigned char* src,
                                             unsigned bytes, unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
  const unsigned piece = bytes / 4;
#pragma unroll
  for (int c = 0; c < 4; ++c)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];\n" ::"r"(dst + c * piece),
        "l"(src + (size_t)c * piece), "r"(piece), "r"(bar)
        : "memory");
}

// Where unit u lies: frequency, level, tile position.
struct TcUnit {
  int f, l, tx, ty;
};
__device__ __forceinline__ TcUnit tc_unit(const HadTcParams& p, int u) {
  TcUnit r;
  r.f = u / p.cols;
  int c = u - r.f * p.cols;
  r.l = 0;
  while (r.l + 1 < p.nlevels && c >= p.lv[r.l + 1].col0) ++r.l;
  c -= p.lv[r.l].col0;
  r.ty = c / p.lv[r.l].ntx;
  r.tx = c - r.ty * p.lv[r.l].ntx;
  return r;
}

// Fill ring planes z0 and z0 + 1 (global box z) of unit U into their slots:
// each box's source spectrum at frequency f (zero outside the domain or for
// boxes without one), split into TF32 hi and lo.
__device__ __forceinline__ void tc_fill2(const HadTcParams& p, const TcUnit& U, int z0,
                                         unsigned char* ring_hi, unsigned char* ring_lo) {
  const TcLevel& L = p.lv[U.l];
  const int n = L.n;
  const int bx0 = 2 * kTcGX * U.tx - 2, by0 = 2 * kTcGY * U.ty - 2;
  constexpr int kPlane = kTcPX * kTcPY;
  int node[kTcFillPerThread];
#pragma unroll
  for (int k = 0; k < kTcFillPerThread; ++k) {
    const int q = threadIdx.x + k * kTcThreads;
    node[k] = -1;
    if (q < 2 * kPlane) {
      const int h = q >= kPlane, r = q - h * kPlane;
      const int iy = r / kTcPX, ix = r - iy * kTcPX;
      const int x = bx0 + ix, y = by0 + iy, z = z0 + h;
      if (x >= 0 && y >= 0 && z >= 0 && x < n && y < n && z < n)
        node[k] = __ldg(&L.srcmap[((size_t)z * n + y) * n + x]);
    }
  }
  float2 v[kTcFillPerThread];
#pragma unroll
  for (int k = 0; k < kTcFillPerThread; ++k)
    v[k] = node[k] >= 0 ? __ldg(&p.spec[spec_index(U.f, node[k], p.nn)]) : make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < kTcFillPerThread; ++k) {
    const int q = threadIdx.x + k * kTcThreads;
    if (q < 2 * kPlane) {
      const int h = q >= kPlane, r = q - h * kPlane;
      const int slot = (z0 + h + 2) & (kTcRing - 1);
      const size_t off = (size_t)slot * kTcPlaneBytes + (size_t)r * 8;
      const float hx = tf32_rn(v[k].x), hy = tf32_rn(v[k].y);
      *(float2*)(ring_hi + off) = make_float2(hx, hy);
      *(float2*)(ring_lo + off) = make_float2(tf32_rn(v[k].x - hx), tf32_rn(v[k].y - hy));
    }
  }
}

// The 162 MMAs of tile gz (3 passes x 54) into the tile buffer at
// tensor-memory column tmem_d: pass 0 (hi x hi) of plane wz into accumulator
// wz, passes 1 and 2 into accumulator 6 (16 columns each).
__device__ __forceinline__ void tc_issue_tile(int gz, unsigned ring_hi, unsigned ring_lo,
                                              unsigned bbuf, unsigned tmem_d) {
#pragma unroll 1
  for (int pass = 0; pass < 3; ++pass) {
    const unsigned abase = pass == 2 ? ring_lo : ring_hi;
    const unsigned bb = bbuf + (pass == 1 ? kTcBPartBytes : 0);
#pragma unroll 1
    for (int wz = 0; wz < 6; ++wz) {
      const unsigned plane = abase + ((2 * gz + wz) & (kTcRing - 1)) * kTcPlaneBytes;
      const unsigned acc = tmem_d + 16 * (pass == 0 ? wz : 6);
      const unsigned first = pass == 0 ? 0u : (pass == 1 && wz == 0 ? 0u : 1u);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const unsigned row0 = plane + 2 * q * kTcRowBytes;
        const int j = wz * 9 + q * 3;
        tc_mma(acc, tc_desc(row0, 16, 2 * kTcRowBytes), tc_desc(bb + j * 512, 128, 256),
               q ? 1u : first);
        tc_mma(acc, tc_desc(row0 + 32, kTcRowBytes - 32, 2 * kTcRowBytes),
               tc_desc(bb + (j + 1) * 512, 128, 256), 1u);
        tc_mma(acc, tc_desc(row0 + kTcRowBytes + 16, 16, 2 * kTcRowBytes),
               tc_desc(bb + (j + 2) * 512, 128, 256), 1u);
      }
    }
  }
}

// Warps 0-3: the accumulators of tile gz (tile buffer at tensor-memory
// column taddr) to the members' target spectra.  Lane m of the 128 is group
// (8 tx + m % 8, 16 ty + m / 8); each accumulator's 16 columns are
// (member c, re | im); the seven are added in FP64.
__device__ __forceinline__ void tc_epilogue(const HadTcParams& p, const TcUnit& U, int gz,
                                            unsigned taddr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double e[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) e[k] = 0.0;
#pragma unroll 1
  for (int a = 0; a < kTcAcc; ++a) {
    unsigned d[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];\n"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
          "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
          "=r"(d[14]), "=r"(d[15])
        : "r"(taddr + 16 * a + ((unsigned)(32 * warp) << 16)));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] += (double)__uint_as_float(d[k]);
  }
  const TcLevel& L = p.lv[U.l];
  const int G = L.n >> 1, m = 32 * warp + lane;
  const int gx = kTcGX * U.tx + (m & 7), gy = kTcGY * U.ty + (m >> 3);
  if (gx >= G || gy >= G) return;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int x = 2 * gx + (c >> 2), y = 2 * gy + ((c >> 1) & 1), z = 2 * gz + (c & 1);
    const int node = __ldg(&L.trgmap[((size_t)z * L.n + y) * L.n + x]);
    if (node >= 0)
      p.effv[spec_index(U.f, node, p.nn)] = make_float2((float)e[2 * c], (float)e[2 * c + 1]);
  }
}

__global__ void __launch_bounds__(kTcThreads, 1) hadamard_tc_kernel(HadTcParams p) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long bar_b[2], bar_m[2];
  __shared__ unsigned tmem_base;
  __shared__ int unit_at[2];
  unsigned char* ring_hi = tc_smem + 2 * kTcBBytes;
  unsigned char* ring_lo = ring_hi + kTcRingBytes;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int nunits = p.F * p.cols;
  const unsigned sb = smem_addr(tc_smem), shi = smem_addr(ring_hi), slo = smem_addr(ring_lo);
  const unsigned bb[2] = {smem_addr(&bar_b[0]), smem_addr(&bar_b[1])};
  const unsigned bm[2] = {smem_addr(&bar_m[0]), smem_addr(&bar_m[1])};
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(bb[i], 1);
      mbar_init(bm[i], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    const int u0 = atomicAdd(p.next_unit, 1);
    unit_at[1] = u0;
    if (u0 < nunits) tc_bulk_load(sb, p.btab + (size_t)(u0 / p.cols) * kTcBBytes, kTcBBytes, bb[0]);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(&tmem_base)),
                 "n"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_base;
  // mbarrier phases waited for (the same in every thread), and issued (kept
  // by thread 0, the only thread that issues)
  int b_issued[2] = {0, 0}, b_waited[2] = {0, 0}, m_issued[2] = {0, 0}, m_waited[2] = {0, 0};
  int u = unit_at[1];
  if (u < nunits) b_issued[0] = 1;
  bool ok = true;
  for (int k = 0; u < nunits && ok; ++k) {
    const int b = k & 1;
    if (tid == 0) {  // the next unit, and its translation matrix into the other buffer
      const int un = atomicAdd(p.next_unit, 1);
      unit_at[b] = un;
      if (un < nunits) {
        tc_bulk_load(sb + (b ^ 1) * kTcBBytes, p.btab + (size_t)(un / p.cols) * kTcBBytes,
                     kTcBBytes, bb[b ^ 1]);
        ++b_issued[b ^ 1];
      }
    }
    const TcUnit U = tc_unit(p, u);
    const int G = p.lv[U.l].n >> 1;
    const unsigned bbuf = sb + b * kTcBBytes;
    tc_fill2(p, U, -2, ring_hi, ring_lo);  // planes -2 .. 3 for tile 0
    tc_fill2(p, U, 0, ring_hi, ring_lo);
    tc_fill2(p, U, 2, ring_hi, ring_lo);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    ok = __syncthreads_and(mbar_wait_bounded(bb[b], b_waited[b] & 1, p.wait_limit));
    if (!ok) break;
    ++b_waited[b];
    const int un = unit_at[b];
    if (tid == 0) {
      tc_fence_after();
      tc_issue_tile(0, shi, slo, bbuf, tmem);
      tc_commit(bm[0]);
      ++m_issued[0];
    }
    for (int gz = 0; gz < G; ++gz) {
      const int tb = gz & 1;
      if (gz + 1 < G) tc_fill2(p, U, 2 * gz + 4, ring_hi, ring_lo);  // tile gz + 1's new planes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      tc_fence_before();
      __syncthreads();
      if (gz + 1 < G) {
        if (tid == 0) {
          tc_fence_after();
          tc_issue_tile(gz + 1, shi, slo, bbuf, tmem + kTcBufCols * (tb ^ 1));
          tc_commit(bm[tb ^ 1]);
          ++m_issued[tb ^ 1];
        }
      }
      ok = __syncthreads_and(mbar_wait_bounded(bm[tb], m_waited[tb] & 1, p.wait_limit));
      if (!ok) break;
      ++m_waited[tb];
      tc_fence_after();
      if (warp < 4) tc_epilogue(p, U, gz, tmem + kTcBufCols * tb);
      tc_fence_before();
    }
    if (!ok) break;
    __syncthreads();
    u = un;
  }
  if (!ok) {
    // a wait ran out: report it, let this CTA's copies and MMAs still in
    // flight land (bounded), then free the tensor memory and leave
    if (tid == 0) {
      atomicExch(p.error, 1);
      for (int i = 0; i < 2; ++i) {
        for (; b_waited[i] < b_issued[i]; ++b_waited[i])
          mbar_wait_bounded(bb[i], b_waited[i] & 1);
        for (; m_waited[i] < m_issued[i]; ++m_waited[i])
          mbar_wait_bounded(bm[i], m_waited[i] & 1);
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "n"(kTcCols)
                 : "memory");
}

