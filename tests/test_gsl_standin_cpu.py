"""CPU test of the project-written GSL stand-in (oracle/gsl_standin) that lets the
reference's own FP64 step build here: the LU decomposition with partial pivoting, the inverse
from it and the DGEMM, against numpy on random and ill-ordered matrices (the pivoting is
exercised by a zero leading entry), in the shapes the reference's operator constructors use
(2 L x 2 L and L x L, L up to 12)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include <cstdio>
#include <gsl/gsl_blas.h>
#include <gsl/gsl_linalg.h>
#include <gsl/gsl_matrix.h>
int main() {
    int n;
    while (std::scanf("%d", &n) == 1) {
        gsl_matrix* a = gsl_matrix_alloc(n, n);
        gsl_matrix* b = gsl_matrix_alloc(n, n);
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) { double v; std::scanf("%lf", &v); gsl_matrix_set(a, i, j, v); gsl_matrix_set(b, i, j, v); }
        gsl_permutation* p = gsl_permutation_alloc(n);
        int sg = 0;
        gsl_linalg_LU_decomp(a, p, &sg);
        gsl_matrix* inv = gsl_matrix_alloc(n, n);
        gsl_linalg_LU_invert(a, p, inv);
        gsl_matrix* c = gsl_matrix_alloc(n, n);
        gsl_matrix_set_identity(c);
        gsl_blas_dgemm(CblasNoTrans, CblasNoTrans, -0.5, b, inv, 0.0, c);   // c = -0.5 b inv
        gsl_matrix* id = gsl_matrix_alloc(n, n);
        gsl_matrix_set_identity(id);
        gsl_matrix_add(c, id);                                                // c = id - 0.5 b inv
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) std::printf("%.17g %.17g\n", gsl_matrix_get(inv, i, j), gsl_matrix_get(c, i, j));
        gsl_matrix_free(a); gsl_matrix_free(b); gsl_matrix_free(inv); gsl_matrix_free(c); gsl_matrix_free(id);
        gsl_permutation_free(p);
    }
    return 0;
}
'''


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("gsl")
    src = d / "t.cpp"
    src.write_text(SRC)
    out = d / "t"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I" + os.path.join(ROOT, "oracle", "gsl_standin"), str(src),
                           "-o", str(out)])
    return str(out)


@pytest.mark.parametrize("n", [2, 3, 8, 16, 24])
def test_lu_inverse_and_dgemm_match_numpy(exe, n):
    rng = np.random.default_rng(n)
    mats = [rng.standard_normal((n, n)) + n * np.eye(n), rng.standard_normal((n, n))]
    m = rng.standard_normal((n, n))
    m[0, 0] = 0.0  # the first pivot must come from another row
    mats.append(m)
    inp = "".join(f"{n}\n" + " ".join(f"{v:.17g}" for v in a.ravel()) + "\n" for a in mats)
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split()
    vals = np.array(out, dtype=np.float64).reshape(len(mats), n * n, 2)
    for a, v in zip(mats, vals):
        inv = v[:, 0].reshape(n, n)
        ref = np.linalg.inv(a)
        assert np.abs(inv - ref).max() <= 1e-10 * np.abs(ref).max() * np.linalg.cond(a) / 1e2 + 1e-13
        c = v[:, 1].reshape(n, n)
        assert np.allclose(c, np.eye(n) - 0.5 * a @ ref, atol=1e-9 * max(1.0, np.abs(a @ ref).max()))
