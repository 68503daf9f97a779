/*
 * Test infrastructure (oracle build only): the four MKL 10.2.2.025 BLAS/LAPACK
 * entry points the reference calls (fmm/reals_aligned.h:84-87; call sites
 * fmm/svdrep.cc:29 and fmm/vecmatop.cc:11,20,73), with Fortran-style by-pointer
 * arguments, column-major storage.
 *
 * DGESVD and DGEMM forward to the LAPACK/BLAS bundled with the scipy wheel in
 * this image (OpenBLAS, symbols scipy_dgesvd_ / scipy_dgemm_): the same
 * published LAPACK DGESVD algorithm MKL ships.  DGEMV and DAXPY are plain
 * column-order loops (they run inside OpenMP regions of the reference).
 */
#ifndef KIFMM_ORACLE_MKL_SHIM_H
#define KIFMM_ORACLE_MKL_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

void DGESVD(const char* jobu, const char* jobvt, const int* m, const int* n, double* a,
            const int* lda, double* s, double* u, const int* ldu, double* vt,
            const int* ldvt, double* work, const int* lwork, int* info);
void DGEMM(const char* transa, const char* transb, const int* m, const int* n,
           const int* k, const double* alpha, const double* a, const int* lda,
           const double* b, const int* ldb, const double* beta, double* c,
           const int* ldc);
void DGEMV(const char* trans, const int* m, const int* n, const double* alpha,
           const double* a, const int* lda, const double* x, const int* incx,
           const double* beta, double* y, const int* incy);
void DAXPY(const int* n, const double* alpha, const double* x, const int* incx,
           double* y, const int* incy);

/* single precision, for the reference's USE_FLOAT build (fmm/reals_aligned.h:136-139) */
void SGESVD(const char* jobu, const char* jobvt, const int* m, const int* n, float* a,
            const int* lda, float* s, float* u, const int* ldu, float* vt, const int* ldvt,
            float* work, const int* lwork, int* info);
void SGEMM(const char* transa, const char* transb, const int* m, const int* n, const int* k,
           const float* alpha, const float* a, const int* lda, const float* b, const int* ldb,
           const float* beta, float* c, const int* ldc);
void SGEMV(const char* trans, const int* m, const int* n, const float* alpha, const float* a,
           const int* lda, const float* x, const int* incx, const float* beta, float* y,
           const int* incy);
void SAXPY(const int* n, const float* alpha, const float* x, const int* incx, float* y,
           const int* incy);

#ifdef __cplusplus
}
#endif

#endif
