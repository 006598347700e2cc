/* TEST INFRASTRUCTURE ONLY -- the reference includes this header
 * (src/anderson.h:8) but calls nothing from it beyond gsl_linalg.h. */
#ifndef LFTS_SHIM_GSL_BLAS_H
#define LFTS_SHIM_GSL_BLAS_H
#include "gsl_linalg.h"
#endif
