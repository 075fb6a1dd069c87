"""GPU test of rbc_nonlinear_noalloc, the nonlinear operator for callers that cannot
allocate device memory (all its scratch is a fixed static device array).

It is compared, through the C ABI, with the regular rbc_nonlinear on the same inputs,
with the tolerance of the other operator parity tests, on consecutive calls (the static
scratch keeps the previous call's contents, so later calls must not depend on them).
This file is collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

import sdc_b200
from tests.helpers import random_state, rel_err

pytestmark = pytest.mark.gpu

RBC_ERR_INVALID_ARG = 1


def _device_copy(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128).view(np.float64).copy()).cuda()


def call_noalloc(case, state, use_stream=False):
    """Runs the no-allocation operator on device copies of `state` (torch owns the
    input and output buffers; the entry point itself allocates nothing). With
    use_stream the work goes to a torch side stream, which is then waited for."""
    import torch
    nx, ny, L, lx, ly, ra, pr, dt = case
    ins = [_device_copy(torch, a) for a in state]
    outs = [torch.zeros_like(t) for t in ins]
    err = ctypes.create_string_buffer(256)
    ptrs = [ctypes.c_void_p(t.data_ptr()) for t in ins + outs]
    torch.cuda.synchronize()
    stream = torch.cuda.Stream() if use_stream else None
    handle = ctypes.c_void_p(stream.cuda_stream) if use_stream else None
    st = sdc_b200.lib().rbc_nonlinear_noalloc(0, nx, ny, L, lx, ly, pr, *ptrs, handle, err, 256)
    if use_stream:
        stream.synchronize()
    torch.cuda.synchronize()
    shapes = [a.shape for a in state]
    res = [o.cpu().numpy().view(np.complex128).reshape(s) for o, s in zip(outs, shapes)]
    return st, res, err.value.decode()


def check_against_regular(case, seed, use_stream=False):
    nx, ny, L = case[:3]
    state = random_state(nx, ny, L, seed=seed, amp=1.0)
    ref = sdc_b200.Solver(*case).nonlinear(*state)
    st, got, msg = call_noalloc(case, state, use_stream)
    assert st == 0, msg
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))


def test_noalloc_matches_regular_operator_on_consecutive_calls():
    c1 = (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3)
    c2 = (32, 48, 3, 8.0, 12.0, 2500.0, 0.7, 1e-3)
    check_against_regular(c1, seed=3)
    check_against_regular(c1, seed=4)   # same size again: no stale scratch is used
    check_against_regular(c2, seed=5)   # another size and L over the same scratch
    check_against_regular(c1, seed=6)


def test_noalloc_two_modes_and_a_side_stream():
    c = (48, 32, 2, 12.0, 8.0, 2000.0, 1.3, 1e-3)
    check_against_regular(c, seed=7, use_stream=True)
    check_against_regular(c, seed=8, use_stream=True)   # tables of this size already in place
    check_against_regular((64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3), seed=9, use_stream=True)


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    case = (128, 64, 4, 16.0, 8.0, 2000.0, 1.0, 1e-3)
    state = random_state(128, 64, 4, seed=1)
    st, _, msg = call_noalloc(case, state)
    assert st == RBC_ERR_INVALID_ARG
    assert "static scratch limit" in msg
    st, _, msg = call_noalloc((64, 64, 5, 8.0, 8.0, 2000.0, 1.0, 1e-3), random_state(64, 64, 5, seed=1))
    assert st == RBC_ERR_INVALID_ARG and "static scratch limit" in msg
