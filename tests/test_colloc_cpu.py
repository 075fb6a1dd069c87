"""CPU checks of the collocation form (RBC_FORM_COLLOC): its product program, derived at
compile time from the exact contraction's units (colloc_prog.h), and its level tables
reproduce the exact contraction evaluated with the level rule's tensors; the oracle's
collocation tensors converge to the exact integrals as the levels grow."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests.helpers import random_state, rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "sdc_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("colloc") / "colloc_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "colloc_check.cpp"), os.path.join(CSRC, "galerkin.cpp"), "-o", exe],
                   check=True)
    return exe


@pytest.mark.parametrize("L,Q", [(2, 8), (3, 8), (4, 8), (6, 16), (8, 16), (8, 24), (8, 32), (12, 24), (12, 32)])
def test_level_products_equal_exact_program_with_level_tensors(checker, L, Q):
    out = subprocess.run([checker, str(L), str(Q)], capture_output=True, text=True, check=True).stdout
    assert float(out) < 1e-12, (L, Q, out)


def test_oracle_collocation_tensors_converge_to_the_integrals():
    case = (32, 32, 8, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    st = random_state(32, 32, 8, seed=3)
    o = oracle.Oracle(*case, threads=2)
    o.set_state(*st)
    exact = o.nonlinear()
    errs = []
    for q in (16, 24, 32):
        o.set_colloc(q)
        o.set_state(*st)
        got = o.nonlinear()
        errs.append(max(rel_err(a, b) for a, b in zip(got, exact)))
    o.set_colloc(0)
    o.set_state(*st)
    back = o.nonlinear()
    assert max(rel_err(a, b) for a, b in zip(back, exact)) == 0.0
    # 4 L levels integrate the triple products of the L-mode basis to rounding
    assert errs[2] < 1e-9 and errs[0] > errs[1] > errs[2], errs
