"""GPU parity of the penalized nonlinear operator (rbc_params.penalization_eta > 0; the
reference's PENALIZED builds) with the oracle: the operator alone, steps with each mask,
and the mixed form."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state, rel_err

pytestmark = pytest.mark.gpu

NAMES = ("theta", "f", "g", "F", "G")
CASES = [
    (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3),
    (48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3),
    (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3),
    (32, 64, 5, 4.0, 8.0, 4000.0, 7.0, 5e-4),
    (64, 48, 6, 16.0, 12.0, 4500.0, 1.0, 5e-4),
    (64, 64, 8, 8.0, 8.0, 5000.0, 0.9, 5e-4),
    (48, 48, 12, 8.0, 8.0, 5000.0, 1.0, 2e-4),
]
KINDS = ["rectangle", "circle", "disk_array", "everywhere"]


def make_pair(case, eta, kind, form="fp64"):
    s = sdc_b200.Solver(*case, form=form, penalization=(eta, kind))
    o = oracle.Oracle(*case, threads=8)
    o.set_penalization(eta, kind)
    return s, o


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("kind", KINDS)
def test_penalized_operator_matches_oracle(case, kind):
    nx, ny, L = case[:3]
    s, o = make_pair(case, 0.01, kind)
    st = random_state(nx, ny, L, seed=41, amp=0.05)
    o.set_state(*st)
    got = s.nonlinear(*st)
    ref = o.nonlinear()
    for name, a, b in zip(NAMES, got, ref):
        assert rel_err(a, b) < 1e-11, (name, rel_err(a, b))


@pytest.mark.parametrize("case", CASES[:4])
@pytest.mark.parametrize("kind", KINDS)
def test_penalized_steps_match_oracle(case, kind):
    nx, ny, L = case[:3]
    s, o = make_pair(case, 0.05, kind)
    st = random_state(nx, ny, L, seed=43, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.step(30)
    o.step(30)
    for name, a, b in zip(NAMES, s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, rel_err(a, b))


def test_penalized_steps_with_tracers_and_graph_replay_match_oracle():
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    n = 2048
    s = sdc_b200.Solver(*case, n_tracers=n, penalization=(0.02, "circle"))
    o = oracle.Oracle(*case, threads=8)
    o.set_penalization(0.02, "circle")
    st = random_state(nx, ny, L, seed=47, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(7, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(40)
    o.step(40)
    for name, a, b in zip(NAMES, s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, rel_err(a, b))
    assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-9


def test_penalized_mixed_form_close_to_fp64():
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    a = sdc_b200.Solver(*case, penalization=(0.02, "rectangle"))
    b = sdc_b200.Solver(*case, form="mixed", penalization=(0.02, "rectangle"))
    st = random_state(nx, ny, L, seed=53, amp=0.05)
    for x in (a, b):
        x.set_state(*st)
        x.step(20)
    for name, u, v in zip(NAMES, a.get_state(), b.get_state()):
        assert rel_err(u, v) < 1e-5, (name, rel_err(u, v))


def test_invalid_penalization_rejected():
    case = CASES[0]
    with pytest.raises(sdc_b200.RBCError):
        sdc_b200.Solver(*case, penalization=(-1.0, "rectangle"))
    with pytest.raises(sdc_b200.RBCError):
        sdc_b200.Solver(*case, penalization=(float("nan"), "rectangle"))


def test_cli_driver_penalized_matches_library(tmp_path):
    """rbc_run -penalized circle -eta 0.05 against the library with the same parameters."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    cmd = [exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1", "-dt", "1e-3",
           "-t", "0.01", "-nfiles", "1", "-seed", "5", "-init_amp", "1e-2", "-init_kmax", "3",
           "-real_bytes", "8", "-penalized", "circle", "-eta", "0.05", "-dir", str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "eta(penalization): 0.05" in open(tmp_path / "simulation.log").read()
    s = sdc_b200.Solver(32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3, penalization=(0.05, "circle"))
    s.init_fields(5, 1e-2, 3.0)
    s.step(10)
    for name, w in zip(NAMES, s.get_state()):
        got = sdc_b200.dump_read(tmp_path / f"{name}_{10:08d}.bin")
        assert np.array_equal(got.reshape(w.shape), w), name
