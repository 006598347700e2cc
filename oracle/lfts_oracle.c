/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle (see lfts_oracle.h).  Restates the
 * reference's algorithm in plain C; the FFTs come from fft_core.c.
 */
#include "lfts_oracle.h"
#include "fft_core.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct orc_sys {
    int NA, NB, N, M, Mk;
    int m[3];
    double L[3];
    double *g;     /* Mk */
    double *qr;    /* 2(N+1)M propagators, slot i = [q_i | q^_{N+1-i}] (src/diblock.cc:19-24) */
    double *h;     /* 2M = [hA | hB] */
    double *work;  /* 2M real scratch */
    double *qk;    /* 2 Mk complex scratch */
    fc_plan3d plan;
};

static int g_orc_threads = 1;
void orc_set_threads(int nthreads)
{
    g_orc_threads = nthreads > 0 ? nthreads : 1;
    fc_set_threads(g_orc_threads);
}

/* src/step.cc:69-89 */
void orc_g_lookup(const orc_sys *s, double *g)
{
    const int *m = s->m;
    const double *L = s->L;
    for (int k0 = -(m[0] - 1) / 2; k0 <= m[0] / 2; k0++) {
        int K0 = (k0 < 0) ? (k0 + m[0]) : k0;
        double kx_sq = k0 * k0 / (L[0] * L[0]);
        for (int k1 = -(m[1] - 1) / 2; k1 <= m[1] / 2; k1++) {
            int K1 = (k1 < 0) ? (k1 + m[1]) : k1;
            double ky_sq = k1 * k1 / (L[1] * L[1]);
            for (int k2 = 0; k2 <= m[2] / 2; k2++) {
                double kz_sq = k2 * k2 / (L[2] * L[2]);
                int k = k2 + (m[2] / 2 + 1) * (K1 + m[1] * K0);
                double K = 2 * M_PI * pow(kx_sq + ky_sq + kz_sq, 0.5);
                g[k] = exp(-K * K / (6.0 * s->N)) / s->M;
            }
        }
    }
}

orc_sys *orc_create(int NA, int NB, const int m[3], const double L[3])
{
    orc_sys *s = (orc_sys *)calloc(1, sizeof(*s));
    s->NA = NA;
    s->NB = NB;
    s->N = NA + NB;
    for (int d = 0; d < 3; d++) { s->m[d] = m[d]; s->L[d] = L[d]; }
    s->M = m[0] * m[1] * m[2];
    s->Mk = m[0] * m[1] * (m[2] / 2 + 1);
    s->g = (double *)malloc(sizeof(double) * s->Mk);
    s->qr = (double *)calloc((size_t)2 * (s->N + 1) * s->M, sizeof(double));
    s->h = (double *)malloc(sizeof(double) * 2 * (size_t)s->M);
    s->work = (double *)malloc(sizeof(double) * 2 * (size_t)s->M);
    s->qk = (double *)malloc(sizeof(double) * 4 * (size_t)s->Mk);
    if (!s->g || !s->qr || !s->h || !s->work || !s->qk || fc_plan3d_init(&s->plan, m)) {
        orc_destroy(s);
        return NULL;
    }
    orc_g_lookup(s, s->g);
    return s;
}

void orc_destroy(orc_sys *s)
{
    if (!s) return;
    fc_plan3d_free(&s->plan);
    free(s->g); free(s->qr); free(s->h); free(s->work); free(s->qk);
    free(s);
}

const double *orc_propagators(const orc_sys *s) { return s->qr; }

/* src/step.cc:35-65 */
void orc_step_fwd(orc_sys *s, const double *q_in, double *q_out, const double *h, int i)
{
    const int M = s->M, Mk = s->Mk;
    memcpy(s->work, q_in, sizeof(double) * 2 * (size_t)M);
    fc_r2c3d(&s->plan, s->work, s->qk);
    fc_r2c3d(&s->plan, s->work + M, s->qk + 2 * (size_t)Mk);
    for (int r = 0; r < Mk; r++) {
        s->qk[2 * r] *= s->g[r];
        s->qk[2 * r + 1] *= s->g[r];
        s->qk[2 * (r + Mk)] *= s->g[r];
        s->qk[2 * (r + Mk) + 1] *= s->g[r];
    }
    fc_c2r3d(&s->plan, s->qk, s->work);
    fc_c2r3d(&s->plan, s->qk + 2 * (size_t)Mk, s->work + M);
    const double *h1 = (i < s->NA) ? h : h + M;       /* chain 1: hA while i < NA */
    const double *h2 = (i < s->NB) ? h + M : h;       /* chain 2: hB while i < NB */
    for (int r = 0; r < M; r++) q_out[r] = s->work[r] * h1[r];
    for (int r = 0; r < M; r++) q_out[r + M] = s->work[r + M] * h2[r];
}

/* src/diblock.cc:30-60, with prepare_h (:64-72), sum_phi (:76-80), normalize_phi (:85-95) */
double orc_calc_concs(orc_sys *s, double *w)
{
    const int M = s->M, N = s->N, NA = s->NA;
    double *phiA = w + 2 * (size_t)M, *phiB = w + 3 * (size_t)M;
    const double *wm = w, *wp = w + M;
    double *hA = s->h, *hB = s->h + M;
    for (int r = 0; r < M; r++) {
        hA[r] = exp(-(wm[r] + wp[r]) / N);
        hB[r] = exp(-(-wm[r] + wp[r]) / N);
    }
    double *slot1 = s->qr + 2 * (size_t)M;
    memcpy(slot1, s->h, sizeof(double) * 2 * (size_t)M);
    for (int i = 1; i < N; i++)
        orc_step_fwd(s, s->qr + 2 * (size_t)i * M, s->qr + 2 * (size_t)(i + 1) * M, s->h, i);

    double Q = 0.0;
    const double *qN = s->qr + 2 * (size_t)N * M;
    for (int r = 0; r < M; r++) Q += qN[r];
    Q /= M;

    for (int r = 0; r < 2 * M; r++) phiA[r] = 0.0;
    for (int i = 1; i <= N; i++) {
        const double *q1 = s->qr + 2 * (size_t)i * M;                 /* q_i      */
        const double *q2 = s->qr + (2 * (size_t)(N + 1 - i) + 1) * M; /* q^_i     */
        double *phi = (i <= NA) ? phiA : phiB;
        for (int r = 0; r < M; r++) phi[r] += q1[r] * q2[r];
    }
    for (int r = 0; r < M; r++) {
        double a = phiA[r] / (N * Q * hA[r]);
        double b = phiB[r] / (N * Q * hB[r]);
        phiA[r] = a - b;
        phiB[r] = a + b;
    }
    return log(Q);
}

/* ------------------------------------------------------------ Anderson --- */
struct orc_anderson {
    int M, nhMax;
    double *DD;        /* (nhMax+1)^2 */
    double *U, *V, *C, *Acpy, *Ycpy;
    double *Dh, *wh;   /* (nhMax+1) x M */
};

orc_anderson *orc_anderson_create(int M, int maxHist)
{
    orc_anderson *a = (orc_anderson *)calloc(1, sizeof(*a));
    int D = maxHist + 1;
    a->M = M;
    a->nhMax = maxHist;
    a->DD = (double *)calloc((size_t)D * D, sizeof(double));
    a->U = (double *)calloc((size_t)maxHist * maxHist + 1, sizeof(double));
    a->V = (double *)calloc((size_t)maxHist + 1, sizeof(double));
    a->C = (double *)calloc((size_t)maxHist + 1, sizeof(double));
    a->Acpy = (double *)calloc((size_t)maxHist * maxHist + 1, sizeof(double));
    a->Ycpy = (double *)calloc((size_t)maxHist + 1, sizeof(double));
    a->Dh = (double *)calloc((size_t)D * M, sizeof(double));
    a->wh = (double *)calloc((size_t)D * M, sizeof(double));
    return a;
}

void orc_anderson_destroy(orc_anderson *a)
{
    if (!a) return;
    free(a->DD); free(a->U); free(a->V); free(a->C); free(a->Acpy); free(a->Ycpy);
    free(a->Dh); free(a->wh);
    free(a);
}

/* Solve A x = y (n x n, row-major) by LU with partial pivoting, the GSL
 * routines the reference calls at src/anderson.cc:106-127 (gsl_linalg_LU_decomp
 * + gsl_linalg_LU_solve; GSL version unpinned).  Unblocked right-looking
 * elimination, first maximal |pivot|, reciprocal scaling of the sub-column. */
static int lu_solve(double *A, double *y, double *x, int n)
{
    int perm[64];
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int j = 0; j < n; j++) {
        int piv = j;
        double amax = fabs(A[j * n + j]);
        for (int i = j + 1; i < n; i++) {
            double v = fabs(A[i * n + j]);
            if (v > amax) { amax = v; piv = i; }
        }
        if (piv != j) {
            for (int k = 0; k < n; k++) {
                double t = A[j * n + k]; A[j * n + k] = A[piv * n + k]; A[piv * n + k] = t;
            }
            int t = perm[j]; perm[j] = perm[piv]; perm[piv] = t;
        }
        if (j + 1 < n) {
            double ajj = A[j * n + j];
            if (fabs(ajj) >= DBL_MIN) {
                double inv = 1.0 / ajj;
                for (int i = j + 1; i < n; i++) A[i * n + j] *= inv;
            } else {
                for (int i = j + 1; i < n; i++) A[i * n + j] /= ajj;
            }
            for (int i = j + 1; i < n; i++) {
                double lij = A[i * n + j];
                for (int k = j + 1; k < n; k++) A[i * n + k] -= lij * A[j * n + k];
            }
        }
    }
    for (int i = 0; i < n; i++)
        if (A[i * n + i] == 0.0) return -1;
    for (int i = 0; i < n; i++) x[i] = y[perm[i]];
    for (int i = 0; i < n; i++) {
        double t = x[i];
        for (int j = 0; j < i; j++) t -= A[i * n + j] * x[j];
        x[i] = t;
    }
    for (int i = n - 1; i >= 0; i--) {
        double t = x[i];
        for (int j = i + 1; j < n; j++) t -= A[i * n + j] * x[j];
        x[i] = t / A[i * n + i];
    }
    return 0;
}

/* src/anderson.cc:24-93 */
int orc_anderson_mix(orc_anderson *a, orc_sys *s, int maxIter, double errTol, double *w)
{
    const int M = a->M, nhMax = a->nhMax, D = nhMax + 1;
    double err = 1.0;
    int k;
#define DDm(i, j) a->DD[(i) * D + (j)]
#define DH(i) (a->Dh + (size_t)(i) * M)
#define WH(i) (a->wh + (size_t)(i) * M)
    for (k = 1; k < maxIter && err > errTol; k++) {
        orc_calc_concs(s, w);
        for (int r = 0; r < M; r++) {
            DH(0)[r] = w[r + 3 * (size_t)M] - 1.0;
            WH(0)[r] = w[r + (size_t)M];
        }
        double S1 = 0.0;
        for (int r = 0; r < M; r++) S1 += DH(0)[r] * DH(0)[r];
        err = sqrt(S1 / M);
        double lambda = 1.0 - pow(0.9, (double)k);
        int nh = (k < nhMax + 1) ? k - 1 : nhMax;
        for (int m = 0; m <= nh; m++) {
            double acc = 0.0;
            for (int r = 0; r < M; r++) acc += DH(0)[r] * DH(m)[r];
            DDm(0, m) = acc;
        }
        if (k < 2) {
            for (int r = 0; r < M; r++) w[r + M] += lambda * DH(0)[r];
        } else {
            for (int m = 1; m <= nh; m++) {
                a->V[m - 1] = DDm(0, 0) - DDm(0, m);
                for (int n = 1; n <= m; n++) {
                    double u = DDm(0, 0) - DDm(0, m) - DDm(0, n) + DDm(n, m);
                    a->U[(m - 1) * nh + n - 1] = u;
                    a->U[(n - 1) * nh + m - 1] = u;
                }
            }
            for (int i = 0; i < nh; i++) {
                a->Ycpy[i] = a->V[i];
                for (int j = 0; j < nh; j++) a->Acpy[i * nh + j] = a->U[i * nh + j];
            }
            if (lu_solve(a->Acpy, a->Ycpy, a->C, nh)) {
                fprintf(stderr, "oracle: Anderson matrix is singular\n");
                abort();
            }
            for (int r = 0; r < M; r++) w[r + M] += lambda * DH(0)[r];
            for (int n = 1; n <= nh; n++) {
                const double c = a->C[n - 1];
                for (int r = 0; r < M; r++)
                    w[r + M] += c * ((WH(n)[r] + lambda * DH(n)[r]) - (WH(0)[r] + lambda * DH(0)[r]));
            }
        }
        int n = 1 + (k - 1) % nhMax;
        memcpy(DH(n), DH(0), sizeof(double) * M);
        memcpy(WH(n), WH(0), sizeof(double) * M);
        DDm(n, n) = DDm(0, 0);
        for (int m = 1; m < n; m++) DDm(m, n) = DDm(0, m);
        for (int m = n + 1; m <= nh; m++) DDm(n, m) = DDm(0, m);
    }
#undef DDm
#undef DH
#undef WH
    return k;
}

/* src/langevin.cc:31 */
void orc_langevin_update(double *w, const double *noise_prev, const double *noise_new,
                         double XbN, double dt, int M)
{
    for (int r = 0; r < M; r++)
        w[r] += -(w[r + 2 * (size_t)M] + 2 * w[r] / XbN) * dt + 0.5 * (noise_prev[r] + noise_new[r]);
}

/* src/strFunc.cc:36-46 */
void orc_sk_sample(orc_sys *s, const double *w, double *S)
{
    fc_r2c3d(&s->plan, w, s->qk);
    for (int k = 0; k < s->Mk; k++) {
        double re = s->qk[2 * k], im = s->qk[2 * k + 1];
        S[k] += re * re + im * im;
    }
}

/* stable merge sort of idx[] by key[] ascending */
static void msort(int *idx, int *tmp, const double *key, int n)
{
    if (n < 2) return;
    int h = n / 2;
    msort(idx, tmp, key, h);
    msort(idx + h, tmp, key, n - h);
    int i = 0, j = h, o = 0;
    while (i < h && j < n) tmp[o++] = (key[idx[j]] < key[idx[i]]) ? idx[j++] : idx[i++];
    while (i < h) tmp[o++] = idx[i++];
    while (j < n) tmp[o++] = idx[j++];
    memcpy(idx, tmp, sizeof(int) * n);
}

/* src/strFunc.cc:9-32 (constructor), 50-76 (save), 80-103 (calcK) */
int orc_sk_bin(const int m[3], const double L[3], const double *S, int nsamples,
               double CV, double chi_b, double dK, double *Kout, double *Sout)
{
    const int M = m[0] * m[1] * m[2];
    const int Mk = m[0] * m[1] * (m[2] / 2 + 1);
    double *K = (double *)malloc(sizeof(double) * Mk);
    int *wt = (int *)malloc(sizeof(int) * Mk);
    int *P = (int *)malloc(sizeof(int) * Mk);
    int *tmp = (int *)malloc(sizeof(int) * Mk);
    const double coeff = CV / (chi_b * chi_b * M * M);
    for (int k = 0; k < Mk; k++) wt[k] = 2;
    for (int k0 = -(m[0] - 1) / 2; k0 <= m[0] / 2; k0++) {
        int K0 = (k0 < 0) ? (k0 + m[0]) : k0;
        double kx_sq = k0 * k0 / (L[0] * L[0]);
        for (int k1 = -(m[1] - 1) / 2; k1 <= m[1] / 2; k1++) {
            int K1 = (k1 < 0) ? (k1 + m[1]) : k1;
            double ky_sq = k1 * k1 / (L[1] * L[1]);
            for (int k2 = 0; k2 <= m[2] / 2; k2++) {
                double kz_sq = k2 * k2 / (L[2] * L[2]);
                int k = k2 + (m[2] / 2 + 1) * (K1 + m[1] * K0);
                K[k] = 2 * M_PI * pow(kx_sq + ky_sq + kz_sq, 0.5);
                if ((k2 == 0) || (k2 == m[2] / 2)) wt[k] = 1;
            }
        }
    }
    for (int k = 0; k < Mk; k++) P[k] = k;
    msort(P, tmp, K, Mk);
    double S_sum = 0.0;
    int n_same = 0, nout = 0;
    for (int k = 0; k < Mk; k++) {
        S_sum += wt[P[k]] * ((coeff / nsamples) * S[P[k]] - 0.5 / chi_b);
        n_same += wt[P[k]];
        if ((k == Mk - 1) || (fabs(K[P[k + 1]] - K[P[k]]) > dK)) {
            Kout[nout] = K[P[k]];
            Sout[nout] = S_sum / n_same;
            nout++;
            S_sum = 0.0;
            n_same = 0;
        }
    }
    free(K); free(wt); free(P); free(tmp);
    return nout;
}

/* src/lfts_simulation.cc:122-135 */
double orc_getH(orc_sys *s, double *w, double XbN)
{
    const int M = s->M;
    double lnQ = orc_calc_concs(s, w);
    double wp_sum = 0.0, wm2_sum = 0.0;
    for (int r = 0; r < M; r++) wp_sum += w[r + M];
    for (int r = 0; r < M; r++) wm2_sum += w[r] * w[r];
    return -lnQ + (wm2_sum / XbN - wp_sum) / M;
}

/* src/lfts_params.cc:122-142 */
double orc_z_inf_discrete(const double L[3], const int m[3], int N, double Nbar, int tmax)
{
    double sum = 0.5, prod = 1.0, X, ell, R0, R0dL[3];
    R0 = sqrt((double)N);
    for (int i = 0; i < 3; i++) {
        R0dL[i] = R0 * L[i] / m[i];
        prod *= R0dL[i];
    }
    ell = pow(prod, 1.0 / 3.0);
    for (int t = 1; t <= tmax; t++) {
        X = (M_PI / ell) * sqrt(t / 6.0);
        prod = 1.0;
        for (int i = 0; i < 3; i++) prod *= erf(X * ell / R0dL[i]);
        sum += pow(sqrt(M_PI) / (2 * X), 3.0) * prod;
    }
    sum *= 2 * R0 / (pow(ell, 3.0) * sqrt(Nbar));
    X = (M_PI / ell) * sqrt((0.5 + tmax) / 6.0);
    return 1.0 - sum - 3 * R0 / (ell * sqrt(M_PI * Nbar) * X);
}
