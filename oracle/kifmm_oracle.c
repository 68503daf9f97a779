/*
 * TEST INFRASTRUCTURE — the oracle (see kifmm_oracle.h).
 *
 * Restates the exact-FP64 evaluator fmm/omp.cc phase by phase, each function
 * citing the lines it follows.  Operators come in as inputs (the reference's
 * own, dumped by oracle/ref_harness.cc, or any other set) so the evaluation is
 * checked independently of the SVD.  Every node's work is done by one thread
 * in the reference's order, so results do not depend on the thread count.
 */
#include "kifmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OOFP_R (1.0 / (4.0 * M_PI)) /* fmm/evaluate.h:10 */
#define SRC_TAG 1
#define TRG_TAG 2

typedef struct {
  int np, P, Q, n, F;
  double *ue, *uc, *de, *dc; /* 3 per point */
} surf_t;

/* compute_sampos, fmm/trans.cc:35-63 */
static double* sampos(int np, double R, int* count) {
  int n = np * np * np - (np - 2) * (np - 2) * (np - 2), c = 0;
  double* out = (double*)malloc(sizeof(double) * 3 * n);
  double step = 2.0 / (np - 1), init = -1.0;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++)
      for (int k = 0; k < np; k++)
        if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
          double x = init + i * step, y = init + j * step, z = init + k * step;
          out[3 * c] = R * x;
          out[3 * c + 1] = R * y;
          out[3 * c + 2] = R * z;
          c++;
        }
  *count = n;
  return out;
}

static double center(const oracle_tree* t, int node, int d) {
  /* fmm/input.cc:122-135 */
  return -1.0 + (2.0 * 1.0) * (t->path[3 * node + d] + 0.5) / (double)(1 << t->depth[node]);
}
static double radius(const oracle_tree* t, int node) {
  return 1.0 / (double)(1 << t->depth[node]); /* fmm/input.cc:113-117 */
}

/* Summation order: 0 = the reference's (ascending), 1 = every sum of the
 * direct evaluations and matrix-vector products taken in descending order.
 * Order 1 is an equally valid FP64 evaluation; the spread between the two
 * measures the algorithm's own rounding floor. */
static int g_reverse = 0;
void oracle_set_order(int reverse) { g_reverse = reverse; }

/* ulist__direct_evaluation, fmm/omp.cc:259-283 (SoA targets/sources) */
static void direct(int nt, const double* tx, const double* ty, const double* tz, double* pot,
                   int ns, const double* sx, const double* sy, const double* sz,
                   const double* w) {
  for (int i = 0; i < nt; i++) {
    double td = 0.0;
    for (int jj = 0; jj < ns; jj++) {
      int j = g_reverse ? ns - 1 - jj : jj;
      double x = tx[i] - sx[j], y = ty[i] - sy[j], z = tz[i] - sz[j];
      double r = sqrt(x * x + y * y + z * z);
      if (r != 0) td += w[j] / r;
    }
    pot[i] += OOFP_R * td;
  }
}

/* compute_localpos, fmm/trans.cc:92-100 */
static void localpos(const oracle_tree* t, int node, const double* sp, int n, double* x,
                     double* y, double* z) {
  double c0 = center(t, node, 0), c1 = center(t, node, 1), c2 = center(t, node, 2);
  double r = radius(t, node);
  for (int i = 0; i < n; i++) {
    x[i] = c0 + r * sp[3 * i];
    y[i] = c1 + r * sp[3 * i + 1];
    z[i] = c2 + r * sp[3 * i + 2];
  }
}

/* Precision of the operator products (matrix-vector products with the
 * translation operators): 0 FP64 (the reference), 1 FP32 inputs and FP32
 * accumulation, 2 split-TF32 three-pass products (hi*hi + hi*lo + lo*hi,
 * 10-bit mantissas) accumulated in FP32.  Modes 1 and 2 exist to measure what
 * reduced-precision level products would do to the potentials. */
static int g_prod = 0;
void oracle_set_product_precision(int mode) { g_prod = mode; }

static float round_tf32(float x) {
  unsigned u;
  memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xffffe000u; /* round to 10 explicit mantissa bits */
  float r;
  memcpy(&r, &u, 4);
  return r;
}

static void gemv_reduced(int m, int n, const double* A, const double* x, double* y) {
  float* acc = (float*)calloc(m, sizeof(float));
  for (int j = 0; j < n; j++) {
    float xj = (float)x[j];
    const double* a = A + (size_t)j * m;
    for (int i = 0; i < m; i++) {
      float ai = (float)a[i];
      if (g_prod == 1) {
        acc[i] = fmaf(xj, ai, acc[i]);
      } else {
        float ah = round_tf32(ai), al = round_tf32(ai - ah);
        float xh = round_tf32(xj), xl = round_tf32(xj - xh);
        acc[i] += ah * xh + (ah * xl + al * xh);
      }
    }
  }
  for (int i = 0; i < m; i++) y[i] += acc[i];
  free(acc);
}

/* y += A x, A m x n column-major (dgemv, fmm/vecmatop.cc:15-22) */
static void gemv(int m, int n, const double* A, const double* x, double* y) {
  if (g_prod) {
    gemv_reduced(m, n, A, x, y);
    return;
  }
  for (int jj = 0; jj < n; jj++) {
    int j = g_reverse ? n - 1 - jj : jj;
    double xj = x[j];
    const double* a = A + (size_t)j * m;
    for (int i = 0; i < m; i++) y[i] += xj * a[i];
  }
}

/* ---- r2c / c2r over the (2np)^3 grid (FFTW semantics) ---- */
static void dft_r2c(int n, const double* in, double* re, double* im, const double* cs,
                    const double* sn) {
  int h = n / 2 + 1;
  double tr[32], ti[32];
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++)
      for (int k = 0; k < h; k++) {
        double ar = 0, ai = 0;
        for (int x = 0; x < n; x++) {
          int m = (k * x) % n;
          ar += in[(a * n + b) * n + x] * cs[m];
          ai -= in[(a * n + b) * n + x] * sn[m];
        }
        re[(a * n + b) * h + k] = ar;
        im[(a * n + b) * h + k] = ai;
      }
  for (int pass = 0; pass < 2; pass++)
    for (int u = 0; u < n; u++)
      for (int k = 0; k < h; k++) {
        size_t base = pass == 0 ? (size_t)u * n * h + k : (size_t)u * h + k;
        size_t stride = pass == 0 ? (size_t)h : (size_t)n * h;
        for (int q = 0; q < n; q++) {
          double ar = 0, ai = 0;
          for (int x = 0; x < n; x++) {
            int m = (q * x) % n;
            double xr = re[base + x * stride], xi = im[base + x * stride];
            ar += xr * cs[m] + xi * sn[m];
            ai += xi * cs[m] - xr * sn[m];
          }
          tr[q] = ar;
          ti[q] = ai;
        }
        for (int q = 0; q < n; q++) {
          re[base + q * stride] = tr[q];
          im[base + q * stride] = ti[q];
        }
      }
}

static void dft_c2r(int n, double* re, double* im, double* out, const double* cs,
                    const double* sn) {
  int h = n / 2 + 1;
  double tr[32], ti[32];
  for (int pass = 0; pass < 2; pass++)
    for (int u = 0; u < n; u++)
      for (int k = 0; k < h; k++) {
        size_t base = pass == 0 ? (size_t)u * h + k : (size_t)u * n * h + k;
        size_t stride = pass == 0 ? (size_t)n * h : (size_t)h;
        for (int q = 0; q < n; q++) {
          double ar = 0, ai = 0;
          for (int x = 0; x < n; x++) {
            int m = (q * x) % n;
            double xr = re[base + x * stride], xi = im[base + x * stride];
            ar += xr * cs[m] - xi * sn[m];
            ai += xi * cs[m] + xr * sn[m];
          }
          tr[q] = ar;
          ti[q] = ai;
        }
        for (int q = 0; q < n; q++) {
          re[base + q * stride] = tr[q];
          im[base + q * stride] = ti[q];
        }
      }
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++) {
      const double* yr = re + (a * n + b) * h;
      const double* yi = im + (a * n + b) * h;
      for (int x = 0; x < n; x++) {
        double acc = yr[0];
        for (int k = 1; k < n / 2; k++) {
          int m = (k * x) % n;
          acc += 2.0 * (yr[k] * cs[m] - yi[k] * sn[m]);
        }
        acc += (x % 2 ? -yr[n / 2] : yr[n / 2]);
        out[(a * n + b) * n + x] = acc;
      }
    }
}

int oracle_evaluate(const oracle_tree* t, int np, const oracle_ops* ops, const double* sx,
                    const double* sy, const double* sz, const double* den, const double* tx,
                    const double* ty, const double* tz, double* pot_orig, double* uden_out,
                    double* dchk_out, double* dden_out) {
  const int nn = t->num_nodes, ns = t->num_src, nt = t->num_trg;
  surf_t S;
  S.np = np;
  S.ue = sampos(np, 1.0, &S.P);
  S.uc = sampos(np + 2, 3.0, &S.Q);
  S.de = sampos(np, 3.0, &S.P);
  S.dc = sampos(np, 1.0, &S.P);
  S.n = 2 * np;
  S.F = (np + 1) * S.n * S.n;
  const int P = S.P, Q = S.Q, n = S.n, G = n * n * n, h = n / 2 + 1, F = S.F;
  double cs[32], sn[32];
  for (int m = 0; m < n; m++) {
    cs[m] = cos(2.0 * M_PI * m / n);
    sn[m] = sin(2.0 * M_PI * m / n);
  }
  /* leaf-ordered points: get_input, fmm/evaluate.cc:14-52 */
  double* lsx = (double*)malloc(sizeof(double) * ns);
  double* lsy = (double*)malloc(sizeof(double) * ns);
  double* lsz = (double*)malloc(sizeof(double) * ns);
  double* lsw = (double*)malloc(sizeof(double) * ns);
  double* ltx = (double*)malloc(sizeof(double) * nt);
  double* lty = (double*)malloc(sizeof(double) * nt);
  double* ltz = (double*)malloc(sizeof(double) * nt);
  double* lpot = (double*)calloc(nt, sizeof(double));
  for (int i = 0; i < ns; i++) {
    int k = t->src_perm[i];
    lsx[i] = sx[k];
    lsy[i] = sy[k];
    lsz[i] = sz[k];
    lsw[i] = den[k];
  }
  for (int i = 0; i < nt; i++) {
    int k = t->trg_perm[i];
    ltx[i] = tx[k];
    lty[i] = ty[k];
    ltz[i] = tz[k];
  }
  double* uden = (double*)calloc((size_t)nn * P, sizeof(double));
  double* dchk = (double*)calloc((size_t)nn * P, sizeof(double));
  double* dden = (double*)calloc((size_t)nn * P, sizeof(double));
  double* effd = (double*)calloc((size_t)nn * 2 * F, sizeof(double));
  const int nlev = t->num_levels;

  /* ---- up_calc__cpu / up_compute, fmm/omp.cc:61-227: deepest level first */
  for (int lev = nlev - 1; lev >= 0; lev--) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = t->node_level[lev]; i < t->node_level[lev + 1]; i++) {
      if (!(t->tag[i] & SRC_TAG)) continue;
      double* chk = (double*)calloc(Q, sizeof(double));
      double* tmp = (double*)calloc(P, sizeof(double));
      if (t->child[i] == -1) {
        double* x = (double*)malloc(sizeof(double) * 3 * Q);
        localpos(t, i, S.uc, Q, x, x + Q, x + 2 * Q);
        direct(Q, x, x + Q, x + 2 * Q, chk, t->src_num[i], lsx + t->src_beg[i],
               lsy + t->src_beg[i], lsz + t->src_beg[i], lsw + t->src_beg[i]);
        free(x);
      } else {
        double* td = (double*)malloc(sizeof(double) * P);
        for (int c = 0; c < 8; c++) {
          int ch = t->child[i] + c;
          if (!(t->tag[ch] & SRC_TAG)) continue;
          double sc = pow(2.0, t->depth[ch]);
          for (int k = 0; k < P; k++) td[k] = uden[(size_t)ch * P + k] * sc;
          gemv(Q, P, ops->ue2uc + (size_t)c * Q * P, td, chk);
        }
        free(td);
      }
      gemv(P, Q, ops->uc2ue, chk, tmp);
      double sc = pow(2.0, -t->depth[i]);
      for (int k = 0; k < P; k++) uden[(size_t)i * P + k] += tmp[k] * sc;
      free(chk);
      free(tmp);
    }
  }

  /* ---- U list, fmm/omp.cc:232-256 */
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nn; i++)
    for (int k = t->u_ptr[i]; k < t->u_ptr[i + 1]; k++) {
      int s = t->u_idx[k];
      direct(t->trg_num[i], ltx + t->trg_beg[i], lty + t->trg_beg[i], ltz + t->trg_beg[i],
             lpot + t->trg_beg[i], t->src_num[s], lsx + t->src_beg[s], lsy + t->src_beg[s],
             lsz + t->src_beg[s], lsw + t->src_beg[s]);
    }

  /* ---- V list, fmm/omp.cc:386-573 with trans.cc:309-418 */
  {
    const int hh = np / 2;
    /* compute_fft_src: 2^depth scale, samDen2RegDen, r2c */
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < nn; i++) {
      if (!(t->tag[i] & SRC_TAG)) continue;
      double* reg = (double*)calloc(G, sizeof(double));
      double* re = (double*)malloc(sizeof(double) * n * n * h);
      double* im = (double*)malloc(sizeof(double) * n * n * h);
      double sc = pow(2.0, t->depth[i]);
      int cnt = 0;
      for (int a = 0; a < np; a++)
        for (int b = 0; b < np; b++)
          for (int c = 0; c < np; c++)
            if (a == 0 || a == np - 1 || b == 0 || b == np - 1 || c == 0 || c == np - 1) {
              reg[(c + hh) * n * n + (b + hh) * n + (a + hh)] = uden[(size_t)i * P + cnt] * sc;
              cnt++;
            }
      dft_r2c(n, reg, re, im, cs, sn);
      for (int f = 0; f < F; f++) {
        effd[(size_t)i * 2 * F + 2 * f] = re[f];
        effd[(size_t)i * 2 * F + 2 * f + 1] = im[f];
      }
      free(reg);
      free(re);
      free(im);
    }
    /* pointwise products and compute_ifft_trg */
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < nn; i++) {
      if (!(t->tag[i] & TRG_TAG) || t->v_ptr[i + 1] == t->v_ptr[i]) continue;
      double* re = (double*)calloc((size_t)n * n * h, sizeof(double));
      double* im = (double*)calloc((size_t)n * n * h, sizeof(double));
      for (int k = t->v_ptr[i]; k < t->v_ptr[i + 1]; k++) {
        int s = t->v_idx[k];
        int d0 = t->path[3 * s] - t->path[3 * i], d1 = t->path[3 * s + 1] - t->path[3 * i + 1],
            d2 = t->path[3 * s + 2] - t->path[3 * i + 2];
        const double* T = ops->ue2dc + (size_t)((d0 + 3) + (d1 + 3) * 7 + (d2 + 3) * 49) * 2 * F;
        const double* Sp = effd + (size_t)s * 2 * F;
        for (int f = 0; f < F; f++) {
          re[f] += (T[2 * f] * Sp[2 * f] - T[2 * f + 1] * Sp[2 * f + 1]);
          im[f] += (T[2 * f] * Sp[2 * f + 1] + T[2 * f + 1] * Sp[2 * f]);
        }
      }
      double nrm = 1.0 / (double)G;
      for (int f = 0; f < F; f++) {
        re[f] *= nrm;
        im[f] *= nrm;
      }
      double* reg = (double*)malloc(sizeof(double) * G);
      dft_c2r(n, re, im, reg, cs, sn);
      int cnt = 0;
      for (int a = 0; a < np; a++)
        for (int b = 0; b < np; b++)
          for (int c = 0; c < np; c++)
            if (a == 0 || a == np - 1 || b == 0 || b == np - 1 || c == 0 || c == np - 1) {
              dchk[(size_t)i * P + cnt] += reg[(c + hh) * n * n + (b + hh) * n + (a + hh)];
              cnt++;
            }
      free(reg);
      free(re);
      free(im);
    }
  }

  /* ---- W list, fmm/omp.cc:663-707 */
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nn; i++) {
    if (!(t->tag[i] & TRG_TAG) || t->child[i] != -1) continue;
    double* x = (double*)malloc(sizeof(double) * 3 * P);
    for (int k = t->w_ptr[i]; k < t->w_ptr[i + 1]; k++) {
      int s = t->w_idx[k];
      if (t->child[s] == -1 && t->src_num[s] < P) {
        direct(t->trg_num[i], ltx + t->trg_beg[i], lty + t->trg_beg[i], ltz + t->trg_beg[i],
               lpot + t->trg_beg[i], t->src_num[s], lsx + t->src_beg[s], lsy + t->src_beg[s],
               lsz + t->src_beg[s], lsw + t->src_beg[s]);
      } else {
        localpos(t, s, S.ue, P, x, x + P, x + 2 * P);
        direct(t->trg_num[i], ltx + t->trg_beg[i], lty + t->trg_beg[i], ltz + t->trg_beg[i],
               lpot + t->trg_beg[i], P, x, x + P, x + 2 * P, uden + (size_t)s * P);
      }
    }
    free(x);
  }

  /* ---- X list, fmm/omp.cc:712-756 */
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < nn; i++) {
    if (!(t->tag[i] & TRG_TAG)) continue;
    double* x = (double*)malloc(sizeof(double) * 3 * P);
    for (int k = t->x_ptr[i]; k < t->x_ptr[i + 1]; k++) {
      int s = t->x_idx[k];
      if (t->child[i] == -1 && t->trg_num[i] < P) {
        direct(t->trg_num[i], ltx + t->trg_beg[i], lty + t->trg_beg[i], ltz + t->trg_beg[i],
               lpot + t->trg_beg[i], t->src_num[s], lsx + t->src_beg[s], lsy + t->src_beg[s],
               lsz + t->src_beg[s], lsw + t->src_beg[s]);
      } else {
        localpos(t, i, S.dc, P, x, x + P, x + 2 * P);
        direct(P, x, x + P, x + 2 * P, dchk + (size_t)i * P, t->src_num[s], lsx + t->src_beg[s],
               lsy + t->src_beg[s], lsz + t->src_beg[s], lsw + t->src_beg[s]);
      }
    }
    free(x);
  }

  /* ---- down_calc__cpu, fmm/omp.cc:762-868: shallowest level first */
  for (int lev = 0; lev < nlev; lev++) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = t->node_level[lev]; i < t->node_level[lev + 1]; i++) {
      if (!(t->tag[i] & TRG_TAG)) continue;
      double* tmp = (double*)malloc(sizeof(double) * P);
      if (t->depth[i] >= 3) {
        int par = t->parent[i];
        int c = (t->path[3 * i] - 2 * t->path[3 * par]) * 4 +
                (t->path[3 * i + 1] - 2 * t->path[3 * par + 1]) * 2 +
                (t->path[3 * i + 2] - 2 * t->path[3 * par + 2]);
        double sc = pow(2.0, t->depth[par]);
        for (int k = 0; k < P; k++) tmp[k] = dden[(size_t)par * P + k] * sc;
        gemv(P, P, ops->de2dc + (size_t)c * P * P, tmp, dchk + (size_t)i * P);
      }
      if (t->depth[i] >= 2) {
        memset(tmp, 0, sizeof(double) * P);
        gemv(P, P, ops->dc2de, dchk + (size_t)i * P, tmp);
        double sc = pow(2.0, -t->depth[i]);
        for (int k = 0; k < P; k++) dden[(size_t)i * P + k] += tmp[k] * sc;
      }
      if (t->child[i] == -1) {
        double* x = (double*)malloc(sizeof(double) * 3 * P);
        localpos(t, i, S.de, P, x, x + P, x + 2 * P);
        direct(t->trg_num[i], ltx + t->trg_beg[i], lty + t->trg_beg[i], ltz + t->trg_beg[i],
               lpot + t->trg_beg[i], P, x, x + P, x + 2 * P, dden + (size_t)i * P);
        free(x);
      }
      free(tmp);
    }
  }

  /* ---- copy_trg_val__cpu, fmm/omp.cc:873-887 */
  for (int i = 0; i < nt; i++) pot_orig[t->trg_perm[i]] = lpot[i];
  if (uden_out) memcpy(uden_out, uden, sizeof(double) * (size_t)nn * P);
  if (dchk_out) memcpy(dchk_out, dchk, sizeof(double) * (size_t)nn * P);
  if (dden_out) memcpy(dden_out, dden, sizeof(double) * (size_t)nn * P);
  free(lsx);
  free(lsy);
  free(lsz);
  free(lsw);
  free(ltx);
  free(lty);
  free(ltz);
  free(lpot);
  free(uden);
  free(dchk);
  free(dden);
  free(effd);
  free(S.ue);
  free(S.uc);
  free(S.de);
  free(S.dc);
  return 0;
}

void oracle_direct(int nt, const double* tx, const double* ty, const double* tz, int ns,
                   const double* sx, const double* sy, const double* sz, const double* den,
                   double* pot) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    pot[i] = 0.0;
    direct(1, tx + i, ty + i, tz + i, pot + i, ns, sx, sy, sz, den);
  }
}
