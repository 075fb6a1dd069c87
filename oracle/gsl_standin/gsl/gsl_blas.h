/* Project-written stand-in for gsl_blas_dgemm (see gsl_matrix.h in this folder for why it
 * exists). Test infrastructure only. */
#ifndef SDC_GSL_STANDIN_BLAS_H
#define SDC_GSL_STANDIN_BLAS_H

#include "gsl_matrix.h"

typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE_t;

/* C = alpha op(A) op(B) + beta C */
static inline int gsl_blas_dgemm(CBLAS_TRANSPOSE_t ta, CBLAS_TRANSPOSE_t tb, double alpha, const gsl_matrix* A,
                                 const gsl_matrix* B, double beta, gsl_matrix* C)
{
    const size_t M = C->size1, N = C->size2;
    const size_t K = ta == CblasNoTrans ? A->size2 : A->size1;
    for (size_t i = 0; i < M; ++i)
        for (size_t j = 0; j < N; ++j) {
            double s = 0.0;
            for (size_t k = 0; k < K; ++k) {
                const double a = ta == CblasNoTrans ? gsl_matrix_get(A, i, k) : gsl_matrix_get(A, k, i);
                const double b = tb == CblasNoTrans ? gsl_matrix_get(B, k, j) : gsl_matrix_get(B, j, k);
                s += a * b;
            }
            gsl_matrix_set(C, i, j, alpha * s + (beta == 0.0 ? 0.0 : beta * gsl_matrix_get(C, i, j)));
        }
    return 0;
}

#endif
