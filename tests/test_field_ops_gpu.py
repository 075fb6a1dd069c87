"""GPU parity of the freeze and heating operators (rbc_freeze_*, rbc_heat_*) with the
oracle's restatement of freeze_operator.cu and masktemp.cu, alone and inside the
iteration order of main.cu:569-616 (freeze, heating, step)."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import kept_mask, random_state, rel_err

pytestmark = pytest.mark.gpu

NAMES = ("theta", "f", "g", "F", "G")
CASES = [
    (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3),
    (48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3),   # radix 3, non-square
    (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3),
    (64, 48, 6, 16.0, 12.0, 4500.0, 1.0, 5e-4),
    (256, 256, 8, 16.0, 16.0, 5000.0, 1.0, 5e-4),
]


def make_pair(case, form="fp64", **kw):
    s = sdc_b200.Solver(*case, form=form, field_ops=("freeze", "heat"), **kw)
    o = oracle.Oracle(*case, threads=8)
    return s, o


def dealiased(state, nx, ny):
    keep = kept_mask(nx, ny)
    return [a * keep for a in state[:3]] + list(state[3:])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("shape,size", [("circle", 0.8), ("rectangle", 0.1)])
def test_freeze_apply_matches_oracle(case, shape, size):
    nx, ny, L = case[:3]
    s, o = make_pair(case)
    st = random_state(nx, ny, L, seed=11, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.freeze_mask(shape, size)
    o.freeze_mask(shape, size)
    st2 = random_state(nx, ny, L, seed=12, amp=0.05)
    s.set_state(*st2)
    o.set_state(*st2)
    s.freeze_apply()
    o.freeze_apply()
    got = s.get_state()
    ref = dealiased(o.get_state(), nx, ny)
    for name, a, b in zip(NAMES, got, ref):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("shape,size,inc", [("rectangle", 0.1, 1.5 / 100), ("circle", 0.8, -0.3)])
def test_heat_apply_matches_oracle(case, shape, size, inc):
    nx, ny, L = case[:3]
    s, o = make_pair(case)
    st = random_state(nx, ny, L, seed=13, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.heat_apply()  # no mask yet: nothing
    assert all(np.array_equal(a, b) for a, b in zip(s.get_state(), dealiased(st, nx, ny)))
    s.heat_mask(shape, size, inc)
    o.heat_mask(shape, size, inc)
    s.heat_apply()
    o.heat_apply()
    for name, a, b in zip(NAMES, s.get_state(), dealiased(o.get_state(), nx, ny)):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))


@pytest.mark.parametrize("case", CASES[:4])
def test_iteration_loop_with_freeze_and_heating_matches_oracle(case):
    """main.cu's loop with -freeze_circle 4 -temp_circle 6: at iteration i the freeze
    (from the iteration after it was taken), the freeze taken at i == 4, the heating, its
    mask set at i == 6, then the step. 30 iterations, parity after every tenth."""
    nx, ny, L = case[:3]
    s, o = make_pair(case)
    st = random_state(nx, ny, L, seed=17, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    for i in range(1, 31):
        for x in (s, o):
            x.freeze_apply()
            if i == 4:
                x.freeze_mask("circle", 0.8)
            x.heat_apply()
            if i == 6:
                x.heat_mask("rectangle", 0.1)
            x.step(1)
        if i % 10 == 0:
            for name, a, b in zip(NAMES, s.get_state(), o.get_state()):
                assert rel_err(a, b) < 1e-10, (i, name, rel_err(a, b))


def test_freeze_keeps_the_ab2_history_and_tracers_match():
    """The operators run between AB2 steps without restarting the stepper, and a pending
    tracer advance uses the state before the freeze changes it (the reference advances
    the tracers after step_time, before the next iteration's freeze)."""
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    n = 2048
    s, o = make_pair(case, n_tracers=n)
    st = random_state(nx, ny, L, seed=19, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(5, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    for x in (s, o):
        x.step(3)
        x.freeze_mask("circle", 0.6)
        x.heat_mask("circle", 0.5, 0.05)
    for _ in range(12):
        for x in (s, o):
            x.freeze_apply()
            x.heat_apply()
            x.step(1)
    for name, a, b in zip(NAMES, s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, rel_err(a, b))
    assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-9


def test_reset_and_missing_buffers():
    case = CASES[0]
    nx, ny, L = case[:3]
    s, _ = make_pair(case)
    st = random_state(nx, ny, L, seed=23, amp=0.05)
    s.set_state(*st)
    s.freeze_mask("circle", 0.8)
    s.heat_mask("rectangle", 0.1)
    s.field_ops_reset()
    s.freeze_apply()
    s.heat_apply()
    assert all(np.array_equal(a, b) for a, b in zip(s.get_state(), dealiased(st, nx, ny)))
    plain = sdc_b200.Solver(*case)
    with pytest.raises(sdc_b200.RBCError):
        plain.freeze_mask("circle", 0.8)
    with pytest.raises(sdc_b200.RBCError):
        plain.heat_mask("rectangle", 0.1)
    only_heat = sdc_b200.Solver(*case, field_ops=("heat",))
    only_heat.heat_mask("rectangle", 0.1)
    with pytest.raises(sdc_b200.RBCError):
        only_heat.freeze_mask("circle", 0.8)


def test_mixed_form_freeze_close_to_fp64():
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    a = sdc_b200.Solver(*case, field_ops=("freeze",))
    b = sdc_b200.Solver(*case, form="mixed", field_ops=("freeze",))
    st = random_state(nx, ny, L, seed=29, amp=0.05)
    for x in (a, b):
        x.set_state(*st)
        x.step(2)
        x.freeze_mask("rectangle", 0.2)
        for _ in range(10):
            x.freeze_apply()
            x.step(1)
    for name, u, v in zip(NAMES, a.get_state(), b.get_state()):
        assert rel_err(u, v) < 1e-5, (name, rel_err(u, v))


def test_cli_driver_field_operators_match_library(tmp_path):
    """rbc_run -freeze_circle 3 -temp_circle 5 against the same iteration loop through the
    library (freeze circle 0.8, heating frame 0.1 by 1.5/100, as main.cu fixes them)."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    cmd = [exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1", "-dt", "1e-3",
           "-t", "0.012", "-nfiles", "1", "-seed", "5", "-init_amp", "1e-2", "-init_kmax", "3",
           "-real_bytes", "8", "-freeze_circle", "3", "-temp_circle", "5", "-dir", str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    s = sdc_b200.Solver(32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3, field_ops=("freeze", "heat"))
    s.init_fields(5, 1e-2, 3.0)
    for i in range(1, 13):
        s.freeze_apply()
        if i == 3:
            s.freeze_mask("circle", 0.8)
        s.heat_apply()
        if i == 5:
            s.heat_mask("rectangle", 0.1, 1.5 / 100)
        s.step(1)
    for name, w in zip(NAMES, s.get_state()):
        got = sdc_b200.dump_read(tmp_path / f"{name}_{12:08d}.bin")
        assert np.array_equal(got.reshape(w.shape), w), name


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("x,y,radius,factor", [(0.5, 0.5, 0.15, 1.1), (0.3, 0.7, 0.4, 0.5)])
def test_masker_matches_oracle(case, x, y, radius, factor):
    nx, ny, L = case[:3]
    s = sdc_b200.Solver(*case, field_ops=("scale",))
    o = oracle.Oracle(*case, threads=8)
    st = random_state(nx, ny, L, seed=31, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.masker(x, y, radius, factor)
    o.masker(x, y, radius, factor)
    for name, a, b in zip(NAMES, s.get_state(), dealiased(o.get_state(), nx, ny)):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))
    with pytest.raises(sdc_b200.RBCError):
        sdc_b200.Solver(*case).masker()
