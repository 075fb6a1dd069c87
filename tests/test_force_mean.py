"""The reference's -mean_F (force_mean, gpu_flow/code/util/util.cu:74-81, called before every
step at main.cu:566-568): F of the lowest vertical mode is set to (mean_F, 0)."""
import os

import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state, rel_err

CASE = (32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3)
NAMES = ("theta", "f", "g", "F", "G")


def test_oracle_forces_f0_before_each_step():
    nx, ny, L = CASE[:3]
    st = random_state(nx, ny, L, seed=61, amp=0.05)
    a = oracle.Oracle(*CASE, threads=2)
    a.set_state(*st)
    a.set_force_mean(0.3)
    a.step(1)
    b = oracle.Oracle(*CASE, threads=2)
    st2 = [x.copy() for x in st]
    st2[3][0] = 0.3
    b.set_state(*st2)
    b.step(1)
    assert all(np.array_equal(x, y) for x, y in zip(a.get_state(), b.get_state()))
    # later steps start from F_0 = 0.3 again, whatever the step made of it
    a.step(1)
    s_after = a.get_state()
    c = oracle.Oracle(*CASE, threads=2)
    c.set_state(*st)
    c.set_force_mean(0.3)
    c.step(2)
    assert all(np.array_equal(x, y) for x, y in zip(s_after, c.get_state()))
    assert s_after[3][0] != 0.3


@pytest.mark.gpu
@pytest.mark.parametrize("ntr", [0, 2048])
def test_force_mean_matches_oracle(ntr):
    nx, ny, L = CASE[:3]
    s = sdc_b200.Solver(*CASE, n_tracers=ntr, mean_F=0.2)
    o = oracle.Oracle(*CASE, threads=8)
    o.set_force_mean(0.2)
    st = random_state(nx, ny, L, seed=63, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    if ntr:
        xyz = oracle.tracer_positions(9, ntr, CASE[3], CASE[4])
        s.tracers_set(xyz)
        o.tracers_set(xyz)
    s.step(3)
    s.step(17)      # graph-replayed steps, chained for tracers
    o.step(20)
    for name, a, b in zip(NAMES, s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, rel_err(a, b))
    if ntr:
        assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-9


@pytest.mark.gpu
def test_cli_driver_mean_F_matches_library(tmp_path):
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    cmd = [exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1", "-dt", "1e-3",
           "-t", "0.01", "-nfiles", "1", "-seed", "5", "-init_amp", "1e-2", "-init_kmax", "3",
           "-real_bytes", "8", "-mean_F", "0.25", "-dir", str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    s = sdc_b200.Solver(*CASE, mean_F=0.25)
    s.init_fields(5, 1e-2, 3.0)
    s.step(10)
    for name, w in zip(NAMES, s.get_state()):
        got = sdc_b200.dump_read(tmp_path / f"{name}_{10:08d}.bin")
        assert np.array_equal(got.reshape(w.shape), w), name
