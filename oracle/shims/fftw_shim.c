/*
 * Test infrastructure (oracle build only).  Separable discrete Fourier
 * transforms that stand in for FFTW 3.2.2's r2c / c2r plans (double, and
 * single precision for the reference's USE_FLOAT build) in the reference
 * CPU build.  Each 1-D pass is a direct DFT with twiddles exp(+-2*pi*i*m/n)
 * tabulated once per plan from libm cos/sin; the 3-D transform is the usual
 * row-column composition (last dimension first for r2c, last dimension last
 * for c2r), exactly as the DFT definition FFTW documents.
 *
 * Execution is re-entrant: omp_sse_block.cc calls fftw_execute_dft_r2c on one
 * plan from many OpenMP threads at once, so all scratch lives on the stack.
 *
 * KFMM_SHIM_SUM_ORDER=1 in the environment sums every 1-D DFT in reverse
 * order.  FFTW does not fix its summation order (it depends on the plan it
 * picks), so the reference's potentials legitimately vary by that much; tests
 * use the switch to measure the reference's own rounding floor.
 */
#include <assert.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

/* One source, two instances: FFTW's double API (fftw_*) by default, its
   single-precision API (fftwf_*, arithmetic in float) with -DSHIM_FLOAT. */
#ifdef SHIM_FLOAT
#define SR float
#define SC fftwf_complex
#define SP fftwf_plan
#define PLAN_S kfmm_shim_fftwf_plan_s
#define SNAME(x) fftwf_##x
#else
#define SR double
#define SC fftw_complex
#define SP fftw_plan
#define PLAN_S kfmm_shim_fftw_plan_s
#define SNAME(x) fftw_##x
#endif

#define SHIM_MAXN 32

#ifndef KFMM_SHIM_ORDER_DEFINED
#define KFMM_SHIM_ORDER_DEFINED
static int shim_reverse(void) {
  static int order = -1; /* read once; concurrent first reads store the same value */
  if (order < 0) {
    const char* e = getenv("KFMM_SHIM_SUM_ORDER");
    order = (e && e[0] == '1') ? 1 : 0;
  }
  return order;
}
#endif

struct PLAN_S {
  int dir; /* -1: r2c forward, +1: c2r backward */
  int n0, n1, n2, h2; /* h2 = n2/2 + 1 */
  SR* rbuf;       /* real array bound at plan time */
  SC* cbuf; /* complex array bound at plan time */
  SR cs[3][SHIM_MAXN]; /* cos(2 pi m / n_d) */
  SR sn[3][SHIM_MAXN]; /* sin(2 pi m / n_d) */
};

static struct PLAN_S* make_plan(int rank, const int* n, int howmany,
                                               int istride, int idist, int ostride,
                                               int odist, int dir) {
  assert(rank == 3 && howmany == 1 && istride == 1 && ostride == 1);
  (void)idist;
  (void)odist;
  struct PLAN_S* p =
      (struct PLAN_S*)calloc(1, sizeof(*p));
  assert(p);
  p->dir = dir;
  p->n0 = n[0];
  p->n1 = n[1];
  p->n2 = n[2];
  p->h2 = n[2] / 2 + 1;
  assert(p->n0 <= SHIM_MAXN && p->n1 <= SHIM_MAXN && p->n2 <= SHIM_MAXN);
  int dims[3] = {p->n0, p->n1, p->n2};
  for (int d = 0; d < 3; ++d)
    for (int m = 0; m < dims[d]; ++m) {
      double a = 2.0 * M_PI * (double)m / (double)dims[d];
      p->cs[d][m] = cos(a);
      p->sn[d][m] = sin(a);
    }
  return p;
}

SP SNAME(plan_many_dft_r2c)(int rank, const int* n, int howmany, SR* in,
                                 const int* inembed, int istride, int idist,
                                 SC* out, const int* onembed, int ostride,
                                 int odist, unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)flags;
  struct PLAN_S* p =
      make_plan(rank, n, howmany, istride, idist, ostride, odist, -1);
  p->rbuf = in;
  p->cbuf = out;
  return p;
}

SP SNAME(plan_many_dft_c2r)(int rank, const int* n, int howmany, SC* in,
                                 const int* inembed, int istride, int idist, SR* out,
                                 const int* onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)flags;
  struct PLAN_S* p =
      make_plan(rank, n, howmany, istride, idist, ostride, odist, +1);
  p->cbuf = in;
  p->rbuf = out;
  return p;
}

/* complex 1-D DFT of length n along a strided line, in place via scratch */
static void cdft_line(SR* re, SR* im, int stride, int n, const SR* cs,
                      const SR* sn, int sign) {
  SR tr[SHIM_MAXN], ti[SHIM_MAXN];
  const int rev = shim_reverse();
  for (int k = 0; k < n; ++k) {
    SR ar = 0.0, ai = 0.0;
    for (int xs = 0; xs < n; ++xs) {
      const int x = rev ? n - 1 - xs : xs;
      int m = (k * x) % n;
      SR c = cs[m], s = sign * sn[m];
      SR xr = re[x * stride], xi = im[x * stride];
      ar += xr * c - xi * s;
      ai += xr * s + xi * c;
    }
    tr[k] = ar;
    ti[k] = ai;
  }
  for (int k = 0; k < n; ++k) {
    re[k * stride] = tr[k];
    im[k * stride] = ti[k];
  }
}

void SNAME(execute_dft_r2c)(const SP p, SR* in, SC* out) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = p->h2;
  const int nc = n0 * n1 * h2;
  SR* re = (SR*)malloc(sizeof(SR) * (size_t)nc);
  SR* im = (SR*)malloc(sizeof(SR) * (size_t)nc);
  assert(re && im);
  /* last dimension: real -> half complex, sign -1 */
  const int rev = shim_reverse();
  for (int a = 0; a < n0; ++a)
    for (int b = 0; b < n1; ++b) {
      const SR* row = in + ((size_t)a * n1 + b) * n2;
      for (int k = 0; k < h2; ++k) {
        SR ar = 0.0, ai = 0.0;
        for (int xs = 0; xs < n2; ++xs) {
          const int x = rev ? n2 - 1 - xs : xs;
          int m = (k * x) % n2;
          ar += row[x] * p->cs[2][m];
          ai -= row[x] * p->sn[2][m];
        }
        re[((size_t)a * n1 + b) * h2 + k] = ar;
        im[((size_t)a * n1 + b) * h2 + k] = ai;
      }
    }
  /* middle dimension */
  for (int a = 0; a < n0; ++a)
    for (int k = 0; k < h2; ++k)
      cdft_line(re + (size_t)a * n1 * h2 + k, im + (size_t)a * n1 * h2 + k, h2, n1,
                p->cs[1], p->sn[1], -1);
  /* first dimension */
  for (int b = 0; b < n1; ++b)
    for (int k = 0; k < h2; ++k)
      cdft_line(re + (size_t)b * h2 + k, im + (size_t)b * h2 + k, n1 * h2, n0, p->cs[0],
                p->sn[0], -1);
  for (int i = 0; i < nc; ++i) {
    out[i][0] = re[i];
    out[i][1] = im[i];
  }
  free(re);
  free(im);
}

void SNAME(execute_dft_c2r)(const SP p, SC* in, SR* out) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = p->h2;
  const int nc = n0 * n1 * h2;
  SR* re = (SR*)malloc(sizeof(SR) * (size_t)nc);
  SR* im = (SR*)malloc(sizeof(SR) * (size_t)nc);
  assert(re && im);
  for (int i = 0; i < nc; ++i) {
    re[i] = in[i][0];
    im[i] = in[i][1];
  }
  /* first and middle dimensions: complex inverse, sign +1 */
  for (int b = 0; b < n1; ++b)
    for (int k = 0; k < h2; ++k)
      cdft_line(re + (size_t)b * h2 + k, im + (size_t)b * h2 + k, n1 * h2, n0, p->cs[0],
                p->sn[0], +1);
  for (int a = 0; a < n0; ++a)
    for (int k = 0; k < h2; ++k)
      cdft_line(re + (size_t)a * n1 * h2 + k, im + (size_t)a * n1 * h2 + k, h2, n1,
                p->cs[1], p->sn[1], +1);
  /* last dimension: Hermitian half complex -> real */
  for (int a = 0; a < n0; ++a)
    for (int b = 0; b < n1; ++b) {
      const SR* yr = re + ((size_t)a * n1 + b) * h2;
      const SR* yi = im + ((size_t)a * n1 + b) * h2;
      SR* row = out + ((size_t)a * n1 + b) * n2;
      for (int x = 0; x < n2; ++x) {
        int kmax = (n2 % 2 == 0) ? n2 / 2 - 1 : n2 / 2;
        SR acc;
        if (!shim_reverse()) {
          acc = yr[0];
          for (int k = 1; k <= kmax; ++k) {
            int m = (k * x) % n2;
            acc += 2.0 * (yr[k] * p->cs[2][m] - yi[k] * p->sn[2][m]);
          }
          if (n2 % 2 == 0) acc += (x % 2 ? -yr[n2 / 2] : yr[n2 / 2]);
        } else {
          acc = (n2 % 2 == 0) ? (x % 2 ? -yr[n2 / 2] : yr[n2 / 2]) : 0.0;
          for (int k = kmax; k >= 1; --k) {
            int m = (k * x) % n2;
            acc += 2.0 * (yr[k] * p->cs[2][m] - yi[k] * p->sn[2][m]);
          }
          acc += yr[0];
        }
        row[x] = acc;
      }
    }
  free(re);
  free(im);
}

void SNAME(execute)(const SP p) {
  if (p->dir < 0)
    SNAME(execute_dft_r2c)(p, p->rbuf, p->cbuf);
  else
    SNAME(execute_dft_c2r)(p, p->cbuf, p->rbuf);
}

void SNAME(destroy_plan)(SP p) { free(p); }
