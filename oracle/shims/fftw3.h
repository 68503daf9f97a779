/*
 * Test infrastructure (oracle build only): a stand-in for the FFTW 3.2.2 API
 * subset that the reference KIFMM CPU path calls.  It is never linked into the
 * product library.
 *
 * The reference names FFTW 3.2.2 (fmm/Makefile:28-31); it is not installed here.
 * Symbols bound through fmm/reals_aligned.h:71-81, called at
 *   fmm/trans.cc:299-300,328,371-372,385 and fmm/omp_sse_block.cc:474.
 * Only the shapes the reference uses are supported: rank-3, howmany=1, unit
 * strides, contiguous C-order arrays, out-of-place.  The transforms follow the
 * published FFTW definitions (unnormalised; r2c keeps the last dimension's
 * n/2+1 non-negative frequencies; c2r assumes Hermitian input and uses only
 * the real parts of the k=0 and k=n/2 bins of the halved dimension).
 */
#ifndef KIFMM_ORACLE_FFTW3_SHIM_H
#define KIFMM_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct kfmm_shim_fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                 double* in, const int* inembed, int istride, int idist,
                                 fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                 fftw_complex* in, const int* inembed, int istride, int idist,
                                 double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);

/* single precision (the reference's USE_FLOAT build, fmm/reals_aligned.h:123-134) */
typedef float fftwf_complex[2];
typedef struct kfmm_shim_fftwf_plan_s* fftwf_plan;
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                   float* in, const int* inembed, int istride, int idist,
                                   fftwf_complex* out, const int* onembed, int ostride,
                                   int odist, unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed, int istride,
                                   int idist, float* out, const int* onembed, int ostride,
                                   int odist, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif

#endif
