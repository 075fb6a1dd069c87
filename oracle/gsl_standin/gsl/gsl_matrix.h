/* Project-written stand-in for the few GSL matrix calls the reference's operator
 * constructors make (gpu_flow/code/operator/linear_implicit_operator.cu:63-173,
 * operator/inverse_B_matrix.cu:100-148): dense row-major matrices, permutations, an LU
 * decomposition with partial pivoting (largest magnitude in the column, as
 * gsl_linalg_LU_decomp documents), the inverse from it, and a plain DGEMM. Only the API
 * names and argument meanings follow GSL; the code is this project's own.
 *
 * Test infrastructure: used only to build the reference's own FP64 step into
 * oracle/_ref/ (build_ref_step.sh), never by the library. GSL itself is not installed
 * here; results agree with it to rounding (the bar the tests use is 1e-10). */
#ifndef SDC_GSL_STANDIN_MATRIX_H
#define SDC_GSL_STANDIN_MATRIX_H

#include <cmath>
#include <cstddef>
#include <cstdlib>

typedef struct {
    size_t size1, size2, tda;
    double* data;
} gsl_matrix;

typedef struct {
    size_t size;
    size_t* data;
} gsl_permutation;

static inline gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2)
{
    gsl_matrix* m = (gsl_matrix*)std::malloc(sizeof(gsl_matrix));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double*)std::calloc(n1 * n2 > 0 ? n1 * n2 : 1, sizeof(double));
    return m;
}
static inline void gsl_matrix_free(gsl_matrix* m)
{
    if (!m) return;
    std::free(m->data);
    std::free(m);
}
static inline double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
static inline void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
static inline void gsl_matrix_set_zero(gsl_matrix* m)
{
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = 0; j < m->size2; ++j) m->data[i * m->tda + j] = 0.0;
}
static inline void gsl_matrix_set_identity(gsl_matrix* m)
{
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = 0; j < m->size2; ++j) m->data[i * m->tda + j] = i == j ? 1.0 : 0.0;
}
/* a += b (same shape) */
static inline int gsl_matrix_add(gsl_matrix* a, const gsl_matrix* b)
{
    for (size_t i = 0; i < a->size1; ++i)
        for (size_t j = 0; j < a->size2; ++j) a->data[i * a->tda + j] += b->data[i * b->tda + j];
    return 0;
}

static inline gsl_permutation* gsl_permutation_alloc(size_t n)
{
    gsl_permutation* p = (gsl_permutation*)std::malloc(sizeof(gsl_permutation));
    p->size = n;
    p->data = (size_t*)std::malloc((n > 0 ? n : 1) * sizeof(size_t));
    for (size_t i = 0; i < n; ++i) p->data[i] = i;
    return p;
}
static inline void gsl_permutation_free(gsl_permutation* p)
{
    if (!p) return;
    std::free(p->data);
    std::free(p);
}

#endif
