"""Pattern initial conditions through the C ABI against the oracle, and the steps that
follow them."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import kept_mask

pytestmark = pytest.mark.gpu

CASE = (64, 48, 4, 8.0, 6.0, 2500.0, 1.0, 1e-3)
KINDS = {"isr": 1, "dislocation": 2, "rectangle": 3, "sv": 4, "cr": 5, "giantspiral": 6, "test": 7}


@pytest.mark.parametrize("name", list(KINDS))
def test_pattern_matches_oracle(name):
    s = sdc_b200.Solver(*CASE)
    o = oracle.Oracle(*CASE, threads=8)
    s.init_pattern(name, mode=4.7, amplitude=1e-6, seed=21, noise=1e-7)
    o.init_pattern(KINDS[name], 4.7, 1e-6, 21, 1e-7)
    ref = o.get_state()
    # the library uploads through the 2/3 dealias of the first step (set_state)
    m = kept_mask(CASE[0], CASE[1])[None]
    got = s.get_state()
    scale = max(np.abs(r).max() for r in ref)
    for a, b in zip(got[:3], ref[:3]):
        assert np.abs(a - b * m).max() <= 1e-12 * scale
    for a, b in zip(got[3:], ref[3:]):
        assert np.abs(a - b).max() <= 1e-12 * scale
    s.step(5)
    o.step(5)
    ref = o.get_state()
    # fields that a pattern leaves at rounding level (g of the x-only test pattern, ~1e-47)
    # are measured against the scale of the whole state
    scale = max(np.abs(r).max() for r in ref[:3])
    for a, b in zip(s.get_state()[:3], ref[:3]):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-6 * scale)
