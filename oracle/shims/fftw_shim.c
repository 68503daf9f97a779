/*
 * Test infrastructure (oracle build only).  Separable discrete Fourier
 * transforms that stand in for FFTW 3.2.2's r2c / c2r plans in the reference
 * CPU build.  Each 1-D pass is a direct DFT with twiddles exp(+-2*pi*i*m/n)
 * tabulated once per plan from libm cos/sin; the 3-D transform is the usual
 * row-column composition (last dimension first for r2c, last dimension last
 * for c2r), exactly as the DFT definition FFTW documents.
 *
 * Execution is re-entrant: omp_sse_block.cc calls fftw_execute_dft_r2c on one
 * plan from many OpenMP threads at once, so all scratch lives on the stack.
 */
#include <assert.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#define SHIM_MAXN 32

struct kfmm_shim_fftw_plan_s {
  int dir; /* -1: r2c forward, +1: c2r backward */
  int n0, n1, n2, h2; /* h2 = n2/2 + 1 */
  double* rbuf;       /* real array bound at plan time */
  fftw_complex* cbuf; /* complex array bound at plan time */
  double cs[3][SHIM_MAXN]; /* cos(2 pi m / n_d) */
  double sn[3][SHIM_MAXN]; /* sin(2 pi m / n_d) */
};

static struct kfmm_shim_fftw_plan_s* make_plan(int rank, const int* n, int howmany,
                                               int istride, int idist, int ostride,
                                               int odist, int dir) {
  assert(rank == 3 && howmany == 1 && istride == 1 && ostride == 1);
  (void)idist;
  (void)odist;
  struct kfmm_shim_fftw_plan_s* p =
      (struct kfmm_shim_fftw_plan_s*)calloc(1, sizeof(*p));
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

fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in,
                                 const int* inembed, int istride, int idist,
                                 fftw_complex* out, const int* onembed, int ostride,
                                 int odist, unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)flags;
  struct kfmm_shim_fftw_plan_s* p =
      make_plan(rank, n, howmany, istride, idist, ostride, odist, -1);
  p->rbuf = in;
  p->cbuf = out;
  return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in,
                                 const int* inembed, int istride, int idist, double* out,
                                 const int* onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)flags;
  struct kfmm_shim_fftw_plan_s* p =
      make_plan(rank, n, howmany, istride, idist, ostride, odist, +1);
  p->cbuf = in;
  p->rbuf = out;
  return p;
}

/* complex 1-D DFT of length n along a strided line, in place via scratch */
static void cdft_line(double* re, double* im, int stride, int n, const double* cs,
                      const double* sn, int sign) {
  double tr[SHIM_MAXN], ti[SHIM_MAXN];
  for (int k = 0; k < n; ++k) {
    double ar = 0.0, ai = 0.0;
    for (int x = 0; x < n; ++x) {
      int m = (k * x) % n;
      double c = cs[m], s = sign * sn[m];
      double xr = re[x * stride], xi = im[x * stride];
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

void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = p->h2;
  const int nc = n0 * n1 * h2;
  double* re = (double*)malloc(sizeof(double) * (size_t)nc);
  double* im = (double*)malloc(sizeof(double) * (size_t)nc);
  assert(re && im);
  /* last dimension: real -> half complex, sign -1 */
  for (int a = 0; a < n0; ++a)
    for (int b = 0; b < n1; ++b) {
      const double* row = in + ((size_t)a * n1 + b) * n2;
      for (int k = 0; k < h2; ++k) {
        double ar = 0.0, ai = 0.0;
        for (int x = 0; x < n2; ++x) {
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

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h2 = p->h2;
  const int nc = n0 * n1 * h2;
  double* re = (double*)malloc(sizeof(double) * (size_t)nc);
  double* im = (double*)malloc(sizeof(double) * (size_t)nc);
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
      const double* yr = re + ((size_t)a * n1 + b) * h2;
      const double* yi = im + ((size_t)a * n1 + b) * h2;
      double* row = out + ((size_t)a * n1 + b) * n2;
      for (int x = 0; x < n2; ++x) {
        double acc = yr[0];
        int kmax = (n2 % 2 == 0) ? n2 / 2 - 1 : n2 / 2;
        for (int k = 1; k <= kmax; ++k) {
          int m = (k * x) % n2;
          acc += 2.0 * (yr[k] * p->cs[2][m] - yi[k] * p->sn[2][m]);
        }
        if (n2 % 2 == 0) acc += (x % 2 ? -yr[n2 / 2] : yr[n2 / 2]);
        row[x] = acc;
      }
    }
  free(re);
  free(im);
}

void fftw_execute(const fftw_plan p) {
  if (p->dir < 0)
    fftw_execute_dft_r2c(p, p->rbuf, p->cbuf);
  else
    fftw_execute_dft_c2r(p, p->cbuf, p->rbuf);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
