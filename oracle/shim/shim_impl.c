/*
 * TEST INFRASTRUCTURE ONLY -- implementations behind oracle/shim/fftw3.h and
 * oracle/shim/gsl/gsl_linalg.h, written from the documented semantics of those
 * interfaces, so that the reference's unmodified sources link into oracle/_ref.
 */
#include "fftw3.h"
#include "gsl/gsl_linalg.h"
#include "../fft_core.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- FFTW ---- */
enum { K_R2C = 1, K_C2R = 2 };

struct fftw_plan_s {
    int kind, howmany, idist, odist;
    double *in, *out;
    fc_plan3d p3;
};

static fftw_plan make_plan(int kind, int rank, const int *n, int howmany, double *in,
                           const int *inembed, int istride, int idist, double *out,
                           const int *onembed, int ostride, int odist)
{
    if (rank != 3 || inembed || onembed || istride != 1 || ostride != 1) {
        fprintf(stderr, "fftw shim: only packed unit-stride rank-3 plans are supported\n");
        abort();
    }
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->kind = kind;
    p->howmany = howmany;
    p->idist = idist;
    p->odist = odist;
    p->in = in;
    p->out = out;
    if (fc_plan3d_init(&p->p3, n)) abort();
    return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist, unsigned flags)
{
    (void)flags;
    return make_plan(K_R2C, rank, n, howmany, in, inembed, istride, idist, (double *)out,
                     onembed, ostride, odist);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *inembed, int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist, unsigned flags)
{
    (void)flags;
    return make_plan(K_C2R, rank, n, howmany, (double *)in, inembed, istride, idist, out,
                     onembed, ostride, odist);
}

fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    int M = n[0] * n[1] * n[2];
    int Mk = n[0] * n[1] * (n[2] / 2 + 1);
    return make_plan(K_R2C, rank, n, 1, in, NULL, 1, M, (double *)out, NULL, 1, Mk);
}

void fftw_execute(const fftw_plan p)
{
    for (int b = 0; b < p->howmany; b++) {
        if (p->kind == K_R2C)
            fc_r2c3d(&p->p3, p->in + (size_t)b * p->idist, p->out + 2 * (size_t)b * p->odist);
        else
            fc_c2r3d(&p->p3, p->in + 2 * (size_t)b * p->idist, p->out + (size_t)b * p->odist);
    }
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    fc_plan3d_free(&p->p3);
    free(p);
}

void fftw_cleanup(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { fc_set_threads(nthreads); }
void fftw_cleanup_threads(void) {}

/* ----------------------------------------------------------------- GSL ---- */
gsl_matrix_view gsl_matrix_view_array(double *base, const size_t n1, const size_t n2)
{
    gsl_matrix_view v;
    memset(&v, 0, sizeof(v));
    v.matrix.size1 = n1;
    v.matrix.size2 = n2;
    v.matrix.tda = n2;
    v.matrix.data = base;
    return v;
}

gsl_vector_view gsl_vector_view_array(double *base, size_t n)
{
    gsl_vector_view v;
    memset(&v, 0, sizeof(v));
    v.vector.size = n;
    v.vector.stride = 1;
    v.vector.data = base;
    return v;
}

gsl_permutation *gsl_permutation_alloc(const size_t n)
{
    gsl_permutation *p = (gsl_permutation *)malloc(sizeof(*p));
    p->size = n;
    p->data = (size_t *)malloc(sizeof(size_t) * (n ? n : 1));
    for (size_t i = 0; i < n; i++) p->data[i] = i;
    return p;
}

void gsl_permutation_free(gsl_permutation *p)
{
    if (!p) return;
    free(p->data);
    free(p);
}

#define A_(i, j) (A->data[(i) * A->tda + (j)])

/* Gaussian elimination with partial pivoting (Golub & Van Loan, Alg. 3.4.1),
 * unblocked, right-looking: pivot = first row of largest |a_ij| in column j,
 * the sub-column is scaled by the reciprocal of the pivot, then a rank-1
 * update of the trailing block.  P A = L U with L unit lower triangular. */
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum)
{
    const size_t n = A->size1;
    *signum = 1;
    for (size_t i = 0; i < n; i++) p->data[i] = i;
    for (size_t j = 0; j < n; j++) {
        size_t piv = j;
        double amax = fabs(A_(j, j));
        for (size_t i = j + 1; i < n; i++) {
            double a = fabs(A_(i, j));
            if (a > amax) { amax = a; piv = i; }
        }
        if (piv != j) {
            for (size_t k = 0; k < n; k++) {
                double t = A_(j, k); A_(j, k) = A_(piv, k); A_(piv, k) = t;
            }
            size_t t = p->data[j]; p->data[j] = p->data[piv]; p->data[piv] = t;
            *signum = -*signum;
        }
        if (j + 1 < n) {
            double ajj = A_(j, j);
            if (fabs(ajj) >= DBL_MIN) {
                double inv = 1.0 / ajj;
                for (size_t i = j + 1; i < n; i++) A_(i, j) *= inv;
            } else {
                for (size_t i = j + 1; i < n; i++) A_(i, j) /= ajj;
            }
            for (size_t i = j + 1; i < n; i++) {
                double lij = A_(i, j);
                for (size_t k = j + 1; k < n; k++) A_(i, k) -= lij * A_(j, k);
            }
        }
    }
    return 0;
}

int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b,
                        gsl_vector *x)
{
    const gsl_matrix *A = LU;
    const size_t n = A->size1;
    for (size_t i = 0; i < n; i++) {
        if (A_(i, i) == 0.0) {
            fprintf(stderr, "gsl: matrix is singular\n");
            abort();
        }
    }
    for (size_t i = 0; i < n; i++) x->data[i * x->stride] = b->data[p->data[i] * b->stride];
    for (size_t i = 0; i < n; i++) {
        double t = x->data[i * x->stride];
        for (size_t j = 0; j < i; j++) t -= A_(i, j) * x->data[j * x->stride];
        x->data[i * x->stride] = t;
    }
    for (size_t ii = n; ii-- > 0;) {
        double t = x->data[ii * x->stride];
        for (size_t j = ii + 1; j < n; j++) t -= A_(ii, j) * x->data[j * x->stride];
        x->data[ii * x->stride] = t / A_(ii, ii);
    }
    return 0;
}
