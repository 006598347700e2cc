/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle.  See fft_core.h for the conventions.
 *
 * Recursive decimation-in-time mixed-radix FFT (Cooley-Tukey), written from the
 * DFT definition.  Twiddles come from a per-length table of exp(-2 pi i t/n)
 * evaluated in long double and rounded once to double.
 */
#include "fft_core.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

void fc_set_threads(int nthreads) { g_threads = nthreads > 0 ? nthreads : 1; }

int fc_plan1d_init(fc_plan1d *p, int n)
{
    const long double two_pi = 6.283185307179586476925286766559005768L;
    int r = n, f;
    memset(p, 0, sizeof(*p));
    if (n < 1) return -1;
    p->n = n;
    /* factor order: 4s first, then 2, 3, 5, then remaining primes */
    while (r % 4 == 0) { p->fac[p->nfac++] = 4; r /= 4; }
    while (r % 2 == 0) { p->fac[p->nfac++] = 2; r /= 2; }
    for (f = 3; r > 1; f += 2) {
        while (r % f == 0) { p->fac[p->nfac++] = f; r /= f; }
    }
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (!p->tw) return -1;
    for (int t = 0; t < n; t++) {
        long double a = -two_pi * (long double)t / (long double)n;
        p->tw[2 * t] = (double)cosl(a);
        p->tw[2 * t + 1] = (double)sinl(a);
    }
    return 0;
}

void fc_plan1d_free(fc_plan1d *p)
{
    free(p->tw);
    p->tw = NULL;
}

/* DFT of length n of in[0], in[s], ... into contiguous out[0..n).  The
 * twiddle exp(-2 pi i t / n) is tw[t * tstep] with tstep = N / n. */
static void dit(const fc_plan1d *p, int fi, int n, const double *in, int s,
                double *out, int tstep, int sign)
{
    const int N = p->n;
    const double *tw = p->tw;
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    const int r = p->fac[fi], m = n / r;
    for (int q = 0; q < r; q++)
        dit(p, fi + 1, m, in + 2 * (size_t)q * s, s * r, out + 2 * (size_t)q * m, tstep * r, sign);

    double t[2 * 64];
    double *tt = t;
    double *heap = NULL;
    if (r > 64) {
        heap = (double *)malloc(sizeof(double) * 2 * (size_t)r);
        tt = heap;
    }
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < r; q++) {
            const double *v = out + 2 * ((size_t)q * m + k);
            long idx = ((long)q * k * tstep) % N;
            double wr = tw[2 * idx], wi = -sign * tw[2 * idx + 1];
            tt[2 * q] = v[0] * wr - v[1] * wi;
            tt[2 * q + 1] = v[0] * wi + v[1] * wr;
        }
        if (r == 2) {
            double *o0 = out + 2 * (size_t)k, *o1 = out + 2 * ((size_t)k + m);
            o0[0] = tt[0] + tt[2]; o0[1] = tt[1] + tt[3];
            o1[0] = tt[0] - tt[2]; o1[1] = tt[1] - tt[3];
        } else if (r == 4) {
            /* multiply by (-i) forward, (+i) backward */
            double a0r = tt[0] + tt[4], a0i = tt[1] + tt[5];
            double a1r = tt[0] - tt[4], a1i = tt[1] - tt[5];
            double b0r = tt[2] + tt[6], b0i = tt[3] + tt[7];
            double dr = tt[2] - tt[6], di = tt[3] - tt[7];
            /* (dr + i di) * (sign * i) */
            double b1r = -(double)sign * di, b1i = (double)sign * dr;
            double *o0 = out + 2 * (size_t)k, *o1 = out + 2 * ((size_t)k + m);
            double *o2 = out + 2 * ((size_t)k + 2 * m), *o3 = out + 2 * ((size_t)k + 3 * m);
            o0[0] = a0r + b0r; o0[1] = a0i + b0i;
            o2[0] = a0r - b0r; o2[1] = a0i - b0i;
            o1[0] = a1r + b1r; o1[1] = a1i + b1i;
            o3[0] = a1r - b1r; o3[1] = a1i - b1i;
        } else {
            /* direct DFT of length r: out[k + m u] = sum_q tt[q] w_r^{q u} */
            const int rstep = N / r;
            for (int u = 0; u < r; u++) {
                double sr = 0.0, si = 0.0;
                for (int q = 0; q < r; q++) {
                    long idx = ((long)(q * u) % r) * rstep;
                    double wr = tw[2 * idx], wi = -sign * tw[2 * idx + 1];
                    sr += tt[2 * q] * wr - tt[2 * q + 1] * wi;
                    si += tt[2 * q] * wi + tt[2 * q + 1] * wr;
                }
                double *o = out + 2 * ((size_t)k + (size_t)u * m);
                o[0] = sr;
                o[1] = si;
            }
        }
    }
    free(heap);
}

void fc_exec1d(const fc_plan1d *p, double *x, double *work, int sign)
{
    memcpy(work, x, sizeof(double) * 2 * (size_t)p->n);
    dit(p, 0, p->n, work, 1, x, 1, sign);
}

int fc_plan3d_init(fc_plan3d *p, const int m[3])
{
    memset(p, 0, sizeof(*p));
    for (int d = 0; d < 3; d++) p->m[d] = m[d];
    p->M = m[0] * m[1] * m[2];
    p->Kz = m[2] / 2 + 1;
    p->Mk = m[0] * m[1] * p->Kz;
    if (fc_plan1d_init(&p->px, m[0]) || fc_plan1d_init(&p->py, m[1]) || fc_plan1d_init(&p->pz, m[2]))
        return -1;
    return 0;
}

void fc_plan3d_free(fc_plan3d *p)
{
    fc_plan1d_free(&p->px);
    fc_plan1d_free(&p->py);
    fc_plan1d_free(&p->pz);
}

/* complex transforms along x (stride n1*Kz) and y (stride Kz) of a half spectrum */
static void xy_pass(const fc_plan3d *p, double *spec, int sign)
{
    const int n0 = p->m[0], n1 = p->m[1], Kz = p->Kz;
    const int nmax = n0 > n1 ? n0 : n1;
    /* y columns: for each (i0, kz) */
#pragma omp parallel num_threads(g_threads)
    {
        double *buf = (double *)malloc(sizeof(double) * 4 * (size_t)nmax);
        double *work = buf + 2 * (size_t)nmax;
#pragma omp for schedule(static)
        for (long c = 0; c < (long)n0 * Kz; c++) {
            long i0 = c / Kz, kz = c % Kz;
            double *base = spec + 2 * ((size_t)i0 * n1 * Kz + kz);
            for (int j = 0; j < n1; j++) {
                buf[2 * j] = base[2 * (size_t)j * Kz];
                buf[2 * j + 1] = base[2 * (size_t)j * Kz + 1];
            }
            fc_exec1d(&p->py, buf, work, sign);
            for (int j = 0; j < n1; j++) {
                base[2 * (size_t)j * Kz] = buf[2 * j];
                base[2 * (size_t)j * Kz + 1] = buf[2 * j + 1];
            }
        }
#pragma omp for schedule(static)
        for (long c = 0; c < (long)n1 * Kz; c++) {
            double *base = spec + 2 * (size_t)c;
            const size_t st = (size_t)n1 * Kz;
            for (int j = 0; j < n0; j++) {
                buf[2 * j] = base[2 * j * st];
                buf[2 * j + 1] = base[2 * j * st + 1];
            }
            fc_exec1d(&p->px, buf, work, sign);
            for (int j = 0; j < n0; j++) {
                base[2 * j * st] = buf[2 * j];
                base[2 * j * st + 1] = buf[2 * j + 1];
            }
        }
        free(buf);
    }
}

void fc_r2c3d(const fc_plan3d *p, const double *in, double *out)
{
    const int n2 = p->m[2], Kz = p->Kz;
    const long nlines = (long)p->m[0] * p->m[1];
    /* real lines along z, two at a time packed as a + i b */
#pragma omp parallel num_threads(g_threads)
    {
        double *z = (double *)malloc(sizeof(double) * 4 * (size_t)n2);
        double *work = z + 2 * (size_t)n2;
#pragma omp for schedule(static)
        for (long lp = 0; lp < (nlines + 1) / 2; lp++) {
            long la = 2 * lp, lb = la + 1;
            const double *a = in + (size_t)la * n2;
            const double *b = lb < nlines ? in + (size_t)lb * n2 : NULL;
            for (int j = 0; j < n2; j++) {
                z[2 * j] = a[j];
                z[2 * j + 1] = b ? b[j] : 0.0;
            }
            fc_exec1d(&p->pz, z, work, -1);
            double *A = out + 2 * (size_t)la * Kz;
            double *B = b ? out + 2 * (size_t)lb * Kz : NULL;
            for (int k = 0; k < Kz; k++) {
                int nk = (n2 - k) % n2;
                double zr = z[2 * k], zi = z[2 * k + 1];
                double cr = z[2 * nk], ci = -z[2 * nk + 1]; /* conj(Z[n-k]) */
                A[2 * k] = 0.5 * (zr + cr);
                A[2 * k + 1] = 0.5 * (zi + ci);
                if (B) {
                    /* (Z - conj Z') / (2i) */
                    double dr = zr - cr, di = zi - ci;
                    B[2 * k] = 0.5 * di;
                    B[2 * k + 1] = -0.5 * dr;
                }
            }
        }
        free(z);
    }
    xy_pass(p, out, -1);
}

void fc_c2r3d(const fc_plan3d *p, double *in, double *out)
{
    const int n2 = p->m[2], Kz = p->Kz;
    const long nlines = (long)p->m[0] * p->m[1];
    xy_pass(p, in, +1);
#pragma omp parallel num_threads(g_threads)
    {
        double *z = (double *)malloc(sizeof(double) * 4 * (size_t)n2);
        double *work = z + 2 * (size_t)n2;
#pragma omp for schedule(static)
        for (long lp = 0; lp < (nlines + 1) / 2; lp++) {
            long la = 2 * lp, lb = la + 1;
            const double *A = in + 2 * (size_t)la * Kz;
            const double *B = lb < nlines ? in + 2 * (size_t)lb * Kz : NULL;
            for (int k = 0; k < n2; k++) {
                double ar, ai, br = 0.0, bi = 0.0;
                if (k < Kz) {
                    ar = A[2 * k]; ai = A[2 * k + 1];
                    if (B) { br = B[2 * k]; bi = B[2 * k + 1]; }
                    if (k == 0 || 2 * k == n2) { ai = 0.0; bi = 0.0; }
                } else {
                    int nk = n2 - k;
                    ar = A[2 * nk]; ai = -A[2 * nk + 1];
                    if (B) { br = B[2 * nk]; bi = -B[2 * nk + 1]; }
                }
                /* Z = A + i B */
                z[2 * k] = ar - bi;
                z[2 * k + 1] = ai + br;
            }
            fc_exec1d(&p->pz, z, work, +1);
            double *a = out + (size_t)la * n2;
            double *b = B ? out + (size_t)lb * n2 : NULL;
            for (int j = 0; j < n2; j++) {
                a[j] = z[2 * j];
                if (b) b[j] = z[2 * j + 1];
            }
        }
        free(z);
    }
}
