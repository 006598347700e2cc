/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.  Nothing on the product
 * path may link or call this file; only tests/, the smoke check and the CPU
 * baseline leg of bench.py use it, as the oracle.
 *
 * Double-precision discrete Fourier transforms written from the DFT definition:
 *   forward  X[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   backward x[j] = sum_k X[k] exp(+2 pi i j k / n)      (both unnormalised)
 * This is the convention FFTW3 documents for fftw_plan_dft_* / r2c / c2r,
 * which the reference calls at src/step.cc:15-16,41,50 and
 * src/strFunc.cc:15,39 (FFTW 3.3.10 per tests/valgrind/valgrind.supp:10;
 * FFTW itself is absent from the reference tree).
 *
 * Multi-dimensional real transforms follow FFTW's documented layout: a real
 * row-major n0 x n1 x n2 array maps to a row-major n0 x n1 x (n2/2+1) complex
 * half spectrum; c2r takes the complex transforms over the leading dimensions
 * first and then a 1-D complex-to-real transform along the last one, using
 * only the real parts of the k=0 and k=n/2 (n even) coefficients.
 */
#ifndef LFTS_ORACLE_FFT_CORE_H
#define LFTS_ORACLE_FFT_CORE_H

#ifdef __cplusplus
extern "C" {
#endif

/* 1-D complex plan: mixed radix (factors 4, 2, 3, 5, then any prime). */
typedef struct fc_plan1d {
    int n;
    int nfac;
    int fac[40];
    double *tw;      /* 2n doubles: exp(-2 pi i t / n), t = 0..n-1 */
} fc_plan1d;

int  fc_plan1d_init(fc_plan1d *p, int n);
void fc_plan1d_free(fc_plan1d *p);
/* In-place transform of n interleaved complex values; sign -1 forward, +1 backward.
 * work must hold 2n doubles. */
void fc_exec1d(const fc_plan1d *p, double *x, double *work, int sign);

/* 3-D real <-> half-complex transforms of one row-major array. */
typedef struct fc_plan3d {
    int m[3];
    int M, Mk, Kz;
    fc_plan1d px, py, pz;
    int nthreads;    /* >1: OpenMP over lines when compiled with -fopenmp */
} fc_plan3d;

int  fc_plan3d_init(fc_plan3d *p, const int m[3]);
void fc_plan3d_free(fc_plan3d *p);
/* in: M reals, out: Mk complex (2*Mk doubles).  in is not modified. */
void fc_r2c3d(const fc_plan3d *p, const double *in, double *out);
/* in: Mk complex (destroyed), out: M reals. */
void fc_c2r3d(const fc_plan3d *p, double *in, double *out);
void fc_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
