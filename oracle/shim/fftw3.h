/*
 * TEST INFRASTRUCTURE ONLY -- API shim used to compile the reference's own
 * sources into oracle/_ref (FFTW3 is not installed in this image).
 *
 * Declares the subset of the documented FFTW3 interface that the reference
 * calls (src/step.cc:15-16,41,50; src/strFunc.cc:15,39; src/fts_cpu.cc:33-34,67).
 * The transforms are implemented in oracle/fft_core.c from the DFT
 * definition (unnormalised, forward sign -1), with FFTW's real-data layout.
 * Only rank-3, unit-stride, packed (NULL embed) plans are supported.
 */
#ifndef LFTS_SHIM_FFTW3_H
#define LFTS_SHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif
#endif
