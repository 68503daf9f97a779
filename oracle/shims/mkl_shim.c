/*
 * Test infrastructure (oracle build only): see mkl.h.
 *
 * KFMM_SHIM_SUM_ORDER=1 in the environment makes the matrix-vector products
 * (DGEMV/SGEMV, the reference's M2M, L2L and check-to-equivalent products,
 * fmm/vecmatop.cc:14-21) sum their columns in reverse order.  MKL does not
 * fix that order either (it depends on the build, the CPU and the thread
 * count), so tests use the switch to measure how far the reference's own
 * potentials move under a legal reordering.
 */
#include <assert.h>
#include <stddef.h>
#include <stdlib.h>

#include "mkl.h"

static int shim_reverse(void) {
  static int order = -1; /* read once; concurrent first reads store the same value */
  if (order < 0) {
    const char* e = getenv("KFMM_SHIM_SUM_ORDER");
    order = (e && e[0] == '1') ? 1 : 0;
  }
  return order;
}

/* OpenBLAS (gfortran ABI: hidden string lengths after the argument list) */
extern void scipy_dgesvd_(const char*, const char*, const int*, const int*, double*,
                          const int*, double*, double*, const int*, double*,
                          const int*, double*, const int*, int*, size_t, size_t);
extern void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*,
                         const double*, const double*, const int*, const double*,
                         const int*, const double*, double*, const int*, size_t,
                         size_t);

void DGESVD(const char* jobu, const char* jobvt, const int* m, const int* n, double* a,
            const int* lda, double* s, double* u, const int* ldu, double* vt,
            const int* ldvt, double* work, const int* lwork, int* info) {
  scipy_dgesvd_(jobu, jobvt, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork, info, 1,
                1);
}

void DGEMM(const char* transa, const char* transb, const int* m, const int* n,
           const int* k, const double* alpha, const double* a, const int* lda,
           const double* b, const int* ldb, const double* beta, double* c,
           const int* ldc) {
  scipy_dgemm_(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}

void DGEMV(const char* trans, const int* m, const int* n, const double* alpha,
           const double* a, const int* lda, const double* x, const int* incx,
           const double* beta, double* y, const int* incy) {
  assert((*trans == 'N' || *trans == 'n') && *incx == 1 && *incy == 1);
  const int M = *m, N = *n, LD = *lda;
  const int rev = shim_reverse();
  for (int i = 0; i < M; ++i) y[i] *= *beta;
  for (int js = 0; js < N; ++js) {
    const int j = rev ? N - 1 - js : js;
    const double t = *alpha * x[j];
    const double* col = a + (size_t)j * LD;
    for (int i = 0; i < M; ++i) y[i] += t * col[i];
  }
}

void DAXPY(const int* n, const double* alpha, const double* x, const int* incx,
           double* y, const int* incy) {
  for (int i = 0; i < *n; ++i) y[(size_t)i * *incy] += *alpha * x[(size_t)i * *incx];
}

/* single precision (USE_FLOAT build) */
extern void scipy_sgesvd_(const char*, const char*, const int*, const int*, float*, const int*,
                          float*, float*, const int*, float*, const int*, float*, const int*,
                          int*, size_t, size_t);
extern void scipy_sgemm_(const char*, const char*, const int*, const int*, const int*,
                         const float*, const float*, const int*, const float*, const int*,
                         const float*, float*, const int*, size_t, size_t);

void SGESVD(const char* jobu, const char* jobvt, const int* m, const int* n, float* a,
            const int* lda, float* s, float* u, const int* ldu, float* vt, const int* ldvt,
            float* work, const int* lwork, int* info) {
  scipy_sgesvd_(jobu, jobvt, m, n, a, lda, s, u, ldu, vt, ldvt, work, lwork, info, 1, 1);
}

void SGEMM(const char* transa, const char* transb, const int* m, const int* n, const int* k,
           const float* alpha, const float* a, const int* lda, const float* b, const int* ldb,
           const float* beta, float* c, const int* ldc) {
  scipy_sgemm_(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}

void SGEMV(const char* trans, const int* m, const int* n, const float* alpha, const float* a,
           const int* lda, const float* x, const int* incx, const float* beta, float* y,
           const int* incy) {
  assert((*trans == 'N' || *trans == 'n') && *incx == 1 && *incy == 1);
  const int M = *m, N = *n, LD = *lda;
  const int rev = shim_reverse();
  for (int i = 0; i < M; ++i) y[i] *= *beta;
  for (int js = 0; js < N; ++js) {
    const int j = rev ? N - 1 - js : js;
    const float t = *alpha * x[j];
    const float* col = a + (size_t)j * LD;
    for (int i = 0; i < M; ++i) y[i] += t * col[i];
  }
}

void SAXPY(const int* n, const float* alpha, const float* x, const int* incx, float* y,
           const int* incy) {
  for (int i = 0; i < *n; ++i) y[(size_t)i * *incy] += *alpha * x[(size_t)i * *incx];
}
