/*
 * TEST INFRASTRUCTURE ONLY -- API shim used to compile the reference's own
 * sources into oracle/_ref (GSL is not installed in this image).
 *
 * Declares the subset of the documented GSL interface called at
 * src/anderson.cc:118-126: matrix/vector views over caller arrays, permutations,
 * and LU decomposition with partial (row) pivoting plus the matching solve.
 * Implemented in oracle/shim/shim_impl.c.
 */
#ifndef LFTS_SHIM_GSL_LINALG_H
#define LFTS_SHIM_GSL_LINALG_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    size_t size1, size2, tda;
    double *data;
    void *block;
    int owner;
} gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;

typedef struct {
    size_t size, stride;
    double *data;
    void *block;
    int owner;
} gsl_vector;
typedef struct { gsl_vector vector; } gsl_vector_view;

typedef struct {
    size_t size;
    size_t *data;
} gsl_permutation;

gsl_matrix_view gsl_matrix_view_array(double *base, const size_t n1, const size_t n2);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);
gsl_permutation *gsl_permutation_alloc(const size_t n);
void gsl_permutation_free(gsl_permutation *p);
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p,
                        const gsl_vector *b, gsl_vector *x);

#ifdef __cplusplus
}
#endif
#endif
