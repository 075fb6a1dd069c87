"""Batched ensemble (rbc_ensemble_*) and the launch autotuner: both reorganise launches
only, so results must equal those of independent, untuned handles bit for bit."""
import numpy as np
import pytest

import sdc_b200
from tests.helpers import random_state

pytestmark = pytest.mark.gpu

MEMBERS = [
    (64, 64, 4, 8.0, 8.0, 2500.0, 0.7, 5e-4),
    (128, 128, 6, 16.0, 16.0, 6100.0, 1.0, 5e-4),
    (64, 64, 8, 8.0, 8.0, 7900.0, 7.0, 5e-4),
    (192, 192, 4, 24.0, 24.0, 3300.0, 1.0, 5e-4),
    (128, 128, 4, 16.0, 16.0, 2000.0, 0.7, 5e-4),
    (64, 64, 6, 8.0, 8.0, 4400.0, 1.0, 5e-4),
]


def test_ensemble_members_match_independent_runs():
    ens = sdc_b200.Ensemble(MEMBERS, nstreams=4)
    refs = []
    for i, (m, c) in enumerate(zip(ens.members, MEMBERS)):
        st = random_state(c[0], c[1], c[2], seed=100 + i, amp=0.02)
        m.set_state(*st)
        r = sdc_b200.Solver(*c)
        r.set_state(*st)
        refs.append(r)
    ens.step(3)      # first step is an Euler step, then graph replays
    ms = ens.timed_step(17)
    assert ms > 0.0  # device time of the 17 replayed steps (CUDA events on the root stream)
    for m, r in zip(ens.members, refs):
        r.step(20)
        for a, b in zip(m.get_state(), r.get_state()):
            assert np.array_equal(a, b)
        assert m.diagnostics()["step"] == 20


def test_autotuned_launches_give_identical_results():
    c = (128, 192, 6, 16.0, 24.0, 4000.0, 1.0, 5e-4)
    st = random_state(128, 192, 6, seed=3, amp=0.02)
    a = sdc_b200.Solver(*c)
    b = sdc_b200.Solver(*c, tune=True)
    W, NP = b.launch_config
    assert W in (1, 2, 4) and NP >= 1 and (192 // 2) % NP == 0
    for s in (a, b):
        s.set_state(*st)
        s.step(10)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
