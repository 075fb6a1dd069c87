/* Project-written stand-in for gsl_linalg_LU_decomp / gsl_linalg_LU_invert (see
 * gsl_matrix.h in this folder for why it exists). Test infrastructure only. */
#ifndef SDC_GSL_STANDIN_LINALG_H
#define SDC_GSL_STANDIN_LINALG_H

#include "gsl_matrix.h"

/* In place A = P^T L U: unit lower L below the diagonal, U on and above it. Column j
 * pivots on the row (j..n-1) of largest |a_ij|; p records the row order, signum the
 * parity of the swaps. */
static inline int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum)
{
    const size_t n = A->size1;
    for (size_t i = 0; i < n; ++i) p->data[i] = i;
    *signum = 1;
    for (size_t j = 0; j < n; ++j) {
        size_t piv = j;
        double best = std::fabs(gsl_matrix_get(A, j, j));
        for (size_t i = j + 1; i < n; ++i) {
            const double v = std::fabs(gsl_matrix_get(A, i, j));
            if (v > best) {
                best = v;
                piv = i;
            }
        }
        if (piv != j) {
            for (size_t c = 0; c < n; ++c) {
                const double t = gsl_matrix_get(A, j, c);
                gsl_matrix_set(A, j, c, gsl_matrix_get(A, piv, c));
                gsl_matrix_set(A, piv, c, t);
            }
            const size_t t = p->data[j];
            p->data[j] = p->data[piv];
            p->data[piv] = t;
            *signum = -*signum;
        }
        const double d = gsl_matrix_get(A, j, j);
        if (d != 0.0) {
            for (size_t i = j + 1; i < n; ++i) {
                const double l = gsl_matrix_get(A, i, j) / d;
                gsl_matrix_set(A, i, j, l);
                for (size_t c = j + 1; c < n; ++c)
                    gsl_matrix_set(A, i, c, gsl_matrix_get(A, i, c) - l * gsl_matrix_get(A, j, c));
            }
        }
    }
    return 0;
}

/* inverse = A^-1 from the decomposition: column e_k of P is solved by forward then
 * back substitution. */
static inline int gsl_linalg_LU_invert(const gsl_matrix* LU, const gsl_permutation* p, gsl_matrix* inverse)
{
    const size_t n = LU->size1;
    double* x = (double*)std::malloc((n > 0 ? n : 1) * sizeof(double));
    for (size_t k = 0; k < n; ++k) {
        // row i of P b is b[p[i]]: b = e_k
        for (size_t i = 0; i < n; ++i) x[i] = p->data[i] == k ? 1.0 : 0.0;
        for (size_t i = 0; i < n; ++i) {
            double s = x[i];
            for (size_t c = 0; c < i; ++c) s -= gsl_matrix_get(LU, i, c) * x[c];
            x[i] = s;
        }
        for (size_t ii = n; ii-- > 0;) {
            double s = x[ii];
            for (size_t c = ii + 1; c < n; ++c) s -= gsl_matrix_get(LU, ii, c) * x[c];
            x[ii] = s / gsl_matrix_get(LU, ii, ii);
        }
        for (size_t i = 0; i < n; ++i) gsl_matrix_set(inverse, i, k, x[i]);
    }
    std::free(x);
    return 0;
}

#endif
