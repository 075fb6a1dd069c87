"""The reference's OWN FP64 step as the anchor: fixtures made by running the reference's
step, nonlinear operator and operator constructors, compiled from its sources
(oracle/build_ref_step.sh: implicit_explicit_step::step_time + make_real_signal per
iteration, gpu_flow/code/main.cu:612-616; nonlinear_operator_rayleigh_noslip::
calculate_operator, operator/nonlinear_operator_rayleigh_noslip.cu:83-1394), on a B200
(tests/golden/make_ref_step_golden.py). The inputs are rebuilt here from their seeds.

CPU tests hold the oracle to those fixtures; GPU tests hold the library to them directly.
Bars: 1e-10 relative for states after steps (the 64^2 x 4 run to its full 1000 steps),
1e-12 for the operator; a field that is zero by symmetry (the mean flow from a theta-only
start) is measured against 1e-6 of the output's scale."""
import os
import sys

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_step_golden as gold  # noqa: E402

THREADS = os.cpu_count() or 1
FAST = ["c1_seeded", "c1_random", "op_64x64x4", "op_64x64x8", "op_48x32x3"]
LARGE = ["c2_seeded", "c2_random", "op_512x512x12"]


def fixture(name):
    return np.load(os.path.join(HERE, "golden", f"ref_step_{name}.npz"))


def outputs(name, advance):
    """(tag, state) for every output of a case: `advance(n)` steps n more and returns the
    state, advance(None) returns the operator of the input."""
    prm, inp, mode, marks, full = gold.CASES[name]
    if mode == "operator":
        yield "op", 0, advance(None), "op" in full
        return
    done = 0
    for i, m in enumerate(marks):
        st = advance(m - done)
        done = m
        yield str(m), i, st, m in full


def compare(name, fx, tag, i, state, full, tol):
    prm = gold.CASES[name][0]
    nx, ny, L = prm[:3]
    mine = gold.summarize(state, nx, ny, L, f"s{tag}", full, seed=1000 + i)
    vals = [k for k in fx.files if k.startswith(f"s{tag}_") and not k.endswith("norm2")]
    scale = max(np.abs(fx[k]).max() for k in vals)
    assert set(mine) <= set(fx.files), sorted(set(mine) - set(fx.files))
    for k in mine:
        a, b = np.asarray(mine[k]), fx[k]
        den = max(np.abs(b).max(), 1e-6 * scale) if not k.endswith("norm2") else max(np.abs(b).max(), 1e-300)
        e = np.abs(a - b).max() / den
        assert e < tol, (name, k, e)


def _oracle_run(name):
    prm = gold.CASES[name][0]
    o = oracle.Oracle(*prm, threads=THREADS)
    o.set_state(*gold.case_input(name))

    def advance(n):
        if n is None:
            return o.nonlinear()
        o.step(n)
        return o.get_state()
    return advance


@pytest.mark.parametrize("name", FAST + LARGE)
def test_oracle_matches_reference_step(name):
    fx = fixture(name)
    tol = 1e-12 if gold.CASES[name][2] == "operator" else 1e-10
    for tag, i, st, full in outputs(name, _oracle_run(name)):
        compare(name, fx, tag, i, st, full, tol)


def test_fixture_params_match_cases():
    for name in FAST + LARGE:
        assert np.array_equal(fixture(name)["params"], np.array(gold.CASES[name][0], dtype=np.float64)), name


@pytest.mark.gpu
@pytest.mark.parametrize("name", FAST + LARGE)
def test_library_matches_reference_step(name):
    import sdc_b200
    prm = gold.CASES[name][0]
    fx = fixture(name)
    s = sdc_b200.Solver(*prm)
    inp = gold.case_input(name)
    s.set_state(*inp)

    def advance(n):
        if n is None:
            return s.nonlinear(*inp)
        s.step(n)
        return s.get_state()
    tol = 1e-12 if gold.CASES[name][2] == "operator" else 1e-10
    for tag, i, st, full in outputs(name, advance):
        compare(name, fx, tag, i, st, full, tol)
    s.close()
