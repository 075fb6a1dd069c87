"""GPU parity at the workload sizes themselves: the library (through its C ABI) against
the FP64 oracle on the production grid (256 x 256 x 8 with 65,536 tracers) and on the
spiral-defect-chaos grid (512 x 512 x 12), in FP64 and in the mixed form.

Bars (written in each test): FP64 spectral coefficients 1e-10 relative after 20 and 100
steps and tracer positions 1e-9 absolute (the reference step's own run lengths are longer;
these are the sizes at which the oracle finishes in minutes: about 1 s per step at
256^2 x 8 and 20-30 s per step at 512^2 x 12 on 8-16 host cores); the nonlinear operator
1e-12; the mixed form (FP32 synthesis, products and transforms, FP64 solve) against the
FP64 oracle itself, with the error stated per diagnostic.

Reference: timestepping/implicit_explicit_stepping.cu:32-97 (the step),
operator/nonlinear_operator_rayleigh_noslip.cu:83-1394 (the operator),
particle/particle_tracer.cu:141-212 (the tracer advance)."""
import os

import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state

pytestmark = pytest.mark.gpu

# (nx, ny, L, lx, ly, ra, pr, dt)
PROD = (256, 256, 8, 32.0, 32.0, 5000.0, 0.9, 5e-4)      # plain FP64 + tracers
SDC = (512, 512, 12, 64.0, 64.0, 6000.0, 1.0, 2.5e-4)    # spiral-defect-chaos grid
NTR = 65536
NAMES = ("theta", "f", "g", "F", "G")
THREADS = os.cpu_count() or 1


def _check_state(got, ref, tol, what, floor=1e-6):
    """Relative error per field; a field that is (nearly) zero by symmetry -- the mean flow
    F, G from a theta-only start holds rounding residue only -- is measured against
    `floor` times the state's largest coefficient instead of its own size."""
    scale = max(np.abs(b).max() for b in ref)
    for name, a, b in zip(NAMES, got, ref):
        den = max(np.abs(b).max(), floor * scale)
        e = np.abs(np.asarray(a) - np.asarray(b)).max() / den
        assert e < tol, (what, name, e)


@pytest.fixture(scope="module")
def prod_seeded():
    """Seeded production run (theta N(0, 1e-3^2) on |k| <= 8 of the lowest mode, seed 2;
    65,536 tracers uniform, seed 2): library and oracle states after 20 and 100 steps."""
    s = sdc_b200.Solver(*PROD, n_tracers=NTR)
    o = oracle.Oracle(*PROD, threads=THREADS)
    s.init_fields(2, 1e-3, 8.0)
    o.init_theta(2, 1e-3, 8.0)
    s.tracers_seed(2)
    xyz = oracle.tracer_positions(2, NTR, PROD[3], PROD[4])
    o.tracers_set(xyz)
    start_equal = all(np.array_equal(a, b) for a, b in zip(s.get_state(), o.get_state())) and \
        np.array_equal(s.tracers_get(), xyz)
    out = {"start_equal": start_equal, "xyz0": xyz}
    for n, upto in ((20, 20), (80, 100)):
        s.step(n)
        o.step(n)
        out[upto] = (s.get_state(), o.get_state(), s.tracers_get(), o.tracers_get(), s.diagnostics(),
                     o.diagnostics())
    s.close()
    return out


def test_production_grid_seeded_start_is_identical(prod_seeded):
    assert prod_seeded["start_equal"]


@pytest.mark.parametrize("nsteps", [20, 100])
def test_production_grid_step_and_tracers_match_oracle(prod_seeded, nsteps):
    got, ref, tg, tr, dg, dr = prod_seeded[nsteps]
    _check_state(got, ref, 1e-10, f"{nsteps} steps")
    assert np.abs(tg - tr).max() < 1e-9
    assert np.abs(tg - prod_seeded["xyz0"]).max() > 1e-9   # the tracers moved
    for k in ("nu_wall", "nu_vol", "ke"):
        assert abs(dg[k] - dr[k]) <= 1e-10 * abs(dr[k]), (k, dg[k], dr[k])


def test_production_grid_nonlinear_state_and_tracers_match_oracle():
    """A state far from the linear regime (random, O(5e-2) per mode) on the production
    grid: 20 steps with 65,536 tracers."""
    s = sdc_b200.Solver(*PROD, n_tracers=NTR)
    o = oracle.Oracle(*PROD, threads=THREADS)
    st = random_state(256, 256, 8, seed=21, amp=0.05, decay=0.08)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(5, NTR, PROD[3], PROD[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(20)
    o.step(20)
    _check_state(s.get_state(), o.get_state(), 1e-10, "random state, 20 steps")
    got, ref = s.tracers_get(), o.tracers_get()
    assert np.abs(got - ref).max() < 1e-9, np.abs(got - ref).max()
    assert np.abs(got - xyz).max() > 1e-4


def test_production_grid_operator_matches_oracle():
    s = sdc_b200.Solver(*PROD)
    o = oracle.Oracle(*PROD, threads=THREADS)
    st = random_state(256, 256, 8, seed=22, amp=1.0, decay=0.05)
    o.set_state(*st)
    _check_state(s.nonlinear(*st), o.nonlinear(), 1e-12, "operator")


@pytest.fixture(scope="module")
def sdc_oracle_run():
    """Oracle: the operator of a random state and 5 steps from the seeded start (seed 3,
    |k| <= 8) on the 512^2 x 12 grid."""
    o = oracle.Oracle(*SDC, threads=THREADS)
    st = random_state(512, 512, 12, seed=31, amp=1.0, decay=0.05)
    o.set_state(*st)
    op = o.nonlinear()
    o.init_theta(3, 1e-3, 8.0)
    o.step(5)
    return {"st": st, "op": op, "state5": o.get_state(), "diag5": o.diagnostics()}


def test_sdc_grid_operator_matches_oracle(sdc_oracle_run):
    s = sdc_b200.Solver(*SDC)
    _check_state(s.nonlinear(*sdc_oracle_run["st"]), sdc_oracle_run["op"], 1e-12, "operator 512^2 x 12")


def test_sdc_grid_five_steps_match_oracle(sdc_oracle_run):
    s = sdc_b200.Solver(*SDC)
    s.init_fields(3, 1e-3, 8.0)
    s.step(5)
    _check_state(s.get_state(), sdc_oracle_run["state5"], 1e-10, "5 steps 512^2 x 12")


def test_mixed_form_against_oracle_on_sdc_grid(sdc_oracle_run):
    """Mixed form on the spiral-defect-chaos grid against the FP64 oracle itself: the
    operator (FP32 synthesis, products, transforms) and 5 steps; per-diagnostic error."""
    m = sdc_b200.Solver(*SDC, form="mixed")
    # against the operator's largest coefficient: the F, G entries are grid means of
    # products, small beside the products themselves, and carry FP32 cancellation
    # (measured on a B200: 2.6e-5 for f, the largest)
    _check_state(m.nonlinear(*sdc_oracle_run["st"]), sdc_oracle_run["op"], 1e-4, "mixed operator", floor=1.0)
    m.init_fields(3, 1e-3, 8.0)
    m.step(5)
    _check_state(m.get_state(), sdc_oracle_run["state5"], 1e-7, "mixed, 5 steps", floor=1.0)
    d, dr = m.diagnostics(), sdc_oracle_run["diag5"]
    for k in ("nu_wall", "nu_vol", "ke"):
        assert abs(d[k] - dr[k]) <= 1e-7 * abs(dr[k]), (k, d[k], dr[k])


def test_mixed_form_against_oracle_on_production_grid(prod_seeded):
    """Mixed form on the production grid against the FP64 oracle's 20- and 100-step states
    of the seeded run, with its 65,536 tracers."""
    m = sdc_b200.Solver(*PROD, n_tracers=NTR, form="mixed")
    m.init_fields(2, 1e-3, 8.0)
    m.tracers_seed(2)
    m.step(20)
    got, ref, _, tr, _, dr = prod_seeded[20]
    _check_state(m.get_state(), ref, 1e-7, "mixed, 20 steps", floor=1.0)
    # tracer positions through the FP32 node records: error ~ FP32 rounding of the velocity
    assert np.abs(m.tracers_get() - tr).max() < 1e-6
    m.step(80)
    got, ref, _, _, _, dr = prod_seeded[100]
    _check_state(m.get_state(), ref, 1e-7, "mixed, 100 steps", floor=1.0)
    d = m.diagnostics()
    for k in ("nu_wall", "nu_vol", "ke"):
        assert abs(d[k] - dr[k]) <= 1e-7 * abs(dr[k]), (k, d[k], dr[k])
