"""GPU tests of the collocation form (RBC_FORM_COLLOC): the nonlinear term with the
products formed on Q Gauss-Legendre levels, the mode -> level products on the tensor cores
(tcgen05 kind::tf32, split operands) and the level -> mode sums in FP32, against the FP64
oracle switched to the same level rule (Oracle.set_colloc), and with 4 L levels against the
exact Galerkin oracle. Bars: FP32-level agreement (the form computes in FP32 like the mixed
form); steps keep the FP64 implicit solve, so the state after 20 steps is held at 3e-6 of
its scale."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    ((64, 64, 8, 8.0, 8.0, 2000.0, 1.0, 1e-3), 16),
    ((64, 64, 8, 8.0, 8.0, 2000.0, 1.0, 1e-3), 24),
    ((64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3), 8),
    ((48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3), 8),
    ((64, 48, 6, 8.0, 6.0, 2000.0, 1.0, 1e-3), 16),
    ((64, 64, 12, 8.0, 8.0, 2000.0, 1.0, 1e-3), 24),
    ((32, 32, 2, 8.0, 8.0, 2000.0, 1.0, 1e-3), 8),
    ((48, 36, 5, 12.0, 9.0, 2000.0, 1.0, 1e-3), 16),
]


@pytest.mark.parametrize("case,q", CASES)
def test_collocation_operator_matches_oracle_with_the_level_rule(case, q):
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=11, amp=1.0)
    o = oracle.Oracle(*case, threads=8)
    o.set_colloc(q)
    o.set_state(*st)
    ref = o.nonlinear()
    s = sdc_b200.Solver(*case, form="colloc", colloc_nq=q)
    got = s.nonlinear(*st)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert rel_err(a, b) < 1e-5, (name, rel_err(a, b))


def test_four_levels_per_mode_reproduce_the_exact_operator():
    case = (64, 64, 8, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    st = random_state(64, 64, 8, seed=12, amp=1.0)
    o = oracle.Oracle(*case, threads=8)
    o.set_state(*st)
    ref = o.nonlinear()
    got = sdc_b200.Solver(*case, form="colloc", colloc_nq=32).nonlinear(*st)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert rel_err(a, b) < 1e-5, (name, rel_err(a, b))


@pytest.mark.parametrize("case,q", [CASES[0], CASES[3], CASES[5]])
def test_collocation_steps_match_oracle(case, q):
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=13, amp=0.05)
    o = oracle.Oracle(*case, threads=8)
    o.set_colloc(q)
    o.set_state(*st)
    s = sdc_b200.Solver(*case, form="colloc", colloc_nq=q)
    s.set_state(*st)
    s.step(20)
    o.step(20)
    got, ref = s.get_state(), o.get_state()
    scale = max(np.abs(b).max() for b in ref[:3])
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert np.abs(a - b).max() / scale < 3e-6, (name, np.abs(a - b).max() / scale)


def test_collocation_form_with_tracers_and_graphs_matches_oracle():
    """40 graph-replayed steps with 4,096 tracers: the tracer node records come from the
    collocation kernel (FP32 records, FP64 RK4 positions)."""
    case = (64, 64, 8, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    q, n = 16, 4096
    o = oracle.Oracle(*case, threads=8)
    o.set_colloc(q)
    s = sdc_b200.Solver(*case, form="colloc", colloc_nq=q, n_tracers=n)
    st = random_state(64, 64, 8, seed=43, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(3, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(40)
    o.step(40)
    got, ref = s.get_state(), o.get_state()
    scale = max(np.abs(b).max() for b in ref[:3])
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert np.abs(a - b).max() / scale < 3e-6, (name, np.abs(a - b).max() / scale)
    # FP32 node records (as the mixed form's): positions agree to 1e-5 after 40 steps
    assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-5
    assert np.abs(s.tracers_get() - xyz).max() > 1e-6  # they moved


def test_collocation_levels_are_validated():
    case = (64, 64, 8, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    for q in (4, 12, 40):   # below nz, not a multiple of 8, above the tile
        with pytest.raises(sdc_b200.RBCError):
            sdc_b200.Solver(*case, form="colloc", colloc_nq=q)


@pytest.mark.parametrize("kind", ["rectangle", "circle"])
def test_collocation_form_with_penalization_matches_oracle(kind):
    """The penalized operator of the PENALIZED builds adds its terms to the contracted
    groups the collocation kernel writes; steps against the oracle with the same level rule
    and the same penalization."""
    case = (64, 48, 6, 16.0, 12.0, 4500.0, 1.0, 5e-4)
    q = 16
    s = sdc_b200.Solver(*case, form="colloc", colloc_nq=q, penalization=(0.02, kind))
    o = oracle.Oracle(*case, threads=8)
    o.set_colloc(q)
    o.set_penalization(0.02, kind)
    st = random_state(64, 48, 6, seed=44, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.step(10)
    o.step(10)
    got, ref = s.get_state(), o.get_state()
    scale = max(np.abs(b).max() for b in ref[:3])
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert np.abs(a - b).max() / scale < 3e-6, (name, np.abs(a - b).max() / scale)
