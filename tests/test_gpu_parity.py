"""GPU parity tests: the CUDA library (through its C ABI) against the FP64 oracle on
the same seeded inputs. FP64 form: bit-level agreement is not expected (summation order
and FFT algorithm differ), the bar is the north-star tolerance written in each test."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import hermitian_fix, kept_mask, random_state, rel_err

pytestmark = pytest.mark.gpu

# (nx, ny, L, lx, ly, ra, pr, dt)
C1 = (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3)
SMALL_CASES = [
    (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3),
    (48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3),   # radix 3, non-square, odd L
    (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3),
    (32, 64, 5, 4.0, 8.0, 4000.0, 7.0, 5e-4),
    (64, 48, 6, 16.0, 12.0, 4500.0, 1.0, 5e-4),
    (64, 64, 8, 8.0, 8.0, 5000.0, 0.9, 5e-4),
]


def make_pair(case, threads=8, **kw):
    nx, ny, L, lx, ly, ra, pr, dt = case
    s = sdc_b200.Solver(nx, ny, L, lx, ly, ra, pr, dt, **kw)
    o = oracle.Oracle(nx, ny, L, lx, ly, ra, pr, dt, threads=threads)
    return s, o


@pytest.mark.parametrize("case", SMALL_CASES)
def test_nonlinear_operator_matches_oracle(case):
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=11 + L, amp=1.0)
    o.set_state(*st)
    ref = o.nonlinear()
    got = s.nonlinear(*st)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))


# longer FFT lengths, each in x (row kernels) and in y (column kernels): register forms
# 128 = 8 lanes x 16, 192 = 16 lanes x 12, 256 = 16 x 16, 512 = 32 lanes x 16; Stockham
# passes for 96 = 16*2*3
FFT_CASES = [
    (128, 192, 2, 16.0, 24.0, 3000.0, 1.0, 1e-3),
    (192, 128, 3, 24.0, 16.0, 3000.0, 1.0, 1e-3),
    (256, 96, 2, 32.0, 12.0, 3000.0, 1.0, 1e-3),
    (512, 64, 2, 64.0, 8.0, 3000.0, 1.0, 1e-3),
    (64, 512, 3, 8.0, 64.0, 3000.0, 1.0, 1e-3),
]


@pytest.mark.parametrize("case", FFT_CASES)
def test_nonlinear_operator_fft_lengths(case):
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=7, amp=1.0, decay=0.05)
    o.set_state(*st)
    ref = o.nonlinear()
    got = s.nonlinear(*st)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, ref):
        assert rel_err(a, b) < 1e-12, (name, rel_err(a, b))


@pytest.mark.parametrize("case", SMALL_CASES[:3])
def test_synthesis_matches_oracle(case):
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=3, amp=1.0)
    o.set_state(*st)
    s.set_state(*st)
    got = s.synthesis()
    ref = o.synthesis()
    for fld in range(8):
        assert rel_err(got[fld], ref[fld]) < 1e-13, fld


def test_set_get_state_roundtrip_applies_dealias():
    s, _ = make_pair(C1)
    nx, ny, L = C1[:3]
    rng = np.random.default_rng(0)
    full = [rng.standard_normal((L, ny, nx // 2 + 1)) + 1j * rng.standard_normal((L, ny, nx // 2 + 1)) for _ in range(3)]
    F = rng.standard_normal(L) + 0j
    G = rng.standard_normal(L) + 0j
    s.set_state(full[0], full[1], full[2], F, G)
    back = s.get_state()
    m = kept_mask(nx, ny)
    for a, b in zip(back[:3], full):
        assert np.array_equal(a[:, m], b[:, m])
        assert np.all(a[:, ~m] == 0)
    assert np.array_equal(back[3], F) and np.array_equal(back[4], G)


@pytest.mark.parametrize("nsteps", [1, 10, 100])
def test_step_matches_oracle_c1(nsteps):
    # plain FP64 64x64x4, Lx=Ly=8, Ra=2000, Pr=1, dt=1e-3 from the seeded theta (|k| <= 4)
    s, o = make_pair(C1)
    s.init_fields(1, 1e-3, 4.0)
    o.init_theta(1, 1e-3, 4.0)
    assert all(np.array_equal(a, b) for a, b in zip(s.get_state(), o.get_state()))
    s.step(nsteps)
    o.step(nsteps)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, nsteps, rel_err(a, b))


@pytest.mark.parametrize("case", SMALL_CASES)
def test_step_matches_oracle_random_state(case):
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=5, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.step(20)
    o.step(20)
    for name, a, b in zip(("theta", "f", "g", "F", "G"), s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10, (name, rel_err(a, b))


def test_step_chunking_is_irrelevant():
    s1, _ = make_pair(C1)
    s2, _ = make_pair(C1)
    for s in (s1, s2):
        s.init_fields(4, 1e-3, 4.0)
    s1.step(12)
    for _ in range(4):
        s2.step(3)
    for a, b in zip(s1.get_state(), s2.get_state()):
        assert np.array_equal(a, b)


def test_hermitian_and_band_invariants_after_steps():
    s, _ = make_pair(SMALL_CASES[2])
    nx, ny, L = SMALL_CASES[2][:3]
    s.set_state(*random_state(nx, ny, L, seed=9, amp=0.05))
    s.step(7)
    th, f, g, F, G = s.get_state()
    m = kept_mask(nx, ny)
    for a in (th, f, g):
        assert np.all(a[:, ~m] == 0)
        for r in range(1, ny // 2):
            assert np.array_equal(a[:, r, 0], np.conj(a[:, ny - r, 0]))
        assert np.all(a[:, 0, 0].imag == 0)
    assert np.all(F.imag == 0) and np.all(G.imag == 0)


def test_diagnostics_match_oracle():
    case = SMALL_CASES[2]
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=21, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.step(5)
    o.step(5)
    d = s.diagnostics()
    r = o.diagnostics()
    assert d["step"] == 5
    assert abs(d["nu_wall"] - r["nu_wall"]) < 1e-12 * abs(r["nu_wall"])
    assert abs(d["nu_vol"] - r["nu_vol"]) < 1e-11 * abs(r["nu_vol"])
    assert abs(d["ke"] - r["ke"]) < 1e-10 * abs(r["ke"])
    hist = s.diag_history(10)
    assert hist.shape == (5, 4) and list(hist[:, 3]) == [1, 2, 3, 4, 5]


def test_diag_history_ring_wraps():
    """With a ring of 8 entries and 21 steps the history returns the newest 8 in step
    order across the wrap, and the last equals rbc_diagnostics; before any step the
    diagnostics hold only Nu_wall of the current state."""
    case = SMALL_CASES[2]
    s = sdc_b200.Solver(*case, diag_capacity=8)
    nx, ny, L = case[:3]
    s.set_state(*random_state(nx, ny, L, seed=22, amp=0.05))
    d0 = s.diagnostics()
    assert d0["step"] == 0 and np.isfinite(d0["nu_wall"]) and np.isnan(d0["ke"])
    s.step(21)
    hist = s.diag_history(20)
    assert hist.shape == (8, 4) and list(hist[:, 3]) == list(range(14, 22))
    d = s.diagnostics()
    assert d["step"] == 21 and d["nu_wall"] == hist[-1, 0] and d["ke"] == hist[-1, 2]
    assert s.diag_history(3).shape == (3, 4)


def test_pipelined_diagnostics_match_history():
    """rbc_diagnostics_async / _get: each ticket returns the entry of the step it was
    enqueued after, read while later steps are queued; stale tickets are rejected."""
    case = SMALL_CASES[2]
    s = sdc_b200.Solver(*case)
    nx, ny, L = case[:3]
    s.set_state(*random_state(nx, ny, L, seed=24, amp=0.05))
    t_init = s.diagnostics_async()
    d = s.diagnostics_get(t_init)
    assert d["step"] == 0 and np.isnan(d["nu_wall"])
    got = []
    prev = None
    for _ in range(20):
        s.step_async(1)
        t = s.diagnostics_async()
        if prev is not None:
            got.append(s.diagnostics_get(prev))
        prev = t
    got.append(s.diagnostics_get(prev))
    hist = s.diag_history(20)
    assert [g["step"] for g in got] == list(range(1, 21))
    for g, h in zip(got, hist):
        assert (g["nu_wall"], g["nu_vol"], g["ke"]) == (h[0], h[1], h[2])
    with pytest.raises(sdc_b200.RBCError):
        s.diagnostics_get(prev - 8)
    with pytest.raises(sdc_b200.RBCError):
        s.diagnostics_get(prev + 1)
    # a non-finite state is reported through the pipelined read too
    st = random_state(nx, ny, L, seed=1, amp=0.01)
    st[0][0, 3, 2] = np.nan
    s2 = sdc_b200.Solver(*case)
    s2.set_state(*st)
    s2.step_async(2)
    t = s2.diagnostics_async()
    with pytest.raises(sdc_b200.RBCError) as e:
        s2.diagnostics_get(t)
    assert e.value.status == 3


@pytest.mark.parametrize("z", [0.0, 0.23])
def test_spectrum_matches_oracle(z):
    case = SMALL_CASES[4]
    s, o = make_pair(case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=31, amp=1.0)
    s.set_state(*st)
    o.set_state(*st)
    nb = nx // 2 + 1
    a = s.spectrum(nb, z)
    b = o.spectrum(nb, z)
    assert rel_err(a, b) < 1e-12


@pytest.mark.parametrize("field", ["theta", "u1", "u2"])
@pytest.mark.parametrize("direction", ["x", "y"])
def test_structure_function_matches_oracle(field, direction):
    """The spectral sum of the library against the reference's FFT round trip (oracle)."""
    from oracle.structure import structure_function
    case = (64, 48, 4, 8.0, 6.0, 3000.0, 1.0, 1e-3)
    s = sdc_b200.Solver(*case)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=51, amp=1.0)
    s.set_state(*st)
    got = s.structure_function(field, direction, 0.1, 3.1, 12)
    ref = structure_function(st[0], st[1], st[2], field, direction, 0.1, 3.1, 12, nx, case[3], case[4])
    assert rel_err(got, ref) < 1e-12, rel_err(got, ref)


def test_tracers_match_oracle():
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    n = 4096
    s, o = make_pair(case, n_tracers=n)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=41, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(2, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(10)
    o.step(10)
    got = s.tracers_get()
    ref = o.tracers_get()
    assert np.abs(got - ref).max() < 1e-9
    assert np.abs(got - xyz).max() > 1e-6  # they moved
    for name, a, b in zip(("theta", "f", "g", "F", "G"), s.get_state(), o.get_state()):
        assert rel_err(a, b) < 1e-10


def test_tracers_match_oracle_over_40_steps():
    """Tracer positions after 40 steps (graph-replayed steps with the advance on the side
    stream) still match the oracle."""
    case = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    n = 4096
    s, o = make_pair(case, n_tracers=n)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=43, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    xyz = oracle.tracer_positions(3, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(40)
    o.step(40)
    assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-9


def test_tracer_seed_matches_oracle_generator():
    case = (32, 32, 2, 32.0, 32.0, 3000.0, 1.0, 1e-3)
    s, _ = make_pair(case, n_tracers=1000)
    s.tracers_seed(2)
    assert np.array_equal(s.tracers_get(), oracle.tracer_positions(2, 1000, 32.0, 32.0))


def test_mixed_form_close_to_fp64():
    case = SMALL_CASES[5]
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=8, amp=0.05)
    a = sdc_b200.Solver(*case, form="fp64")
    b = sdc_b200.Solver(*case, form="mixed")
    a.set_state(*st)
    b.set_state(*st)
    a.step(20)
    b.step(20)
    for x, y in zip(a.get_state()[:3], b.get_state()[:3]):
        assert rel_err(y, x) < 1e-4
    da, db = a.diagnostics(), b.diagnostics()
    assert abs(da["nu_wall"] - db["nu_wall"]) < 1e-6


def test_nan_in_state_reported():
    s, _ = make_pair(C1)
    nx, ny, L = C1[:3]
    st = random_state(nx, ny, L, seed=1, amp=0.01)
    st[0][0, 3, 2] = np.nan
    s.set_state(*st)
    with pytest.raises(sdc_b200.RBCError) as e:
        s.step(2)
    assert e.value.status == 3
    # the one-wait pattern (enqueue, then read the diagnostics) reports it as well
    s2, _ = make_pair(C1)
    s2.set_state(*st)
    s2.step_async(2)
    with pytest.raises(sdc_b200.RBCError) as e2:
        s2.diagnostics()
    assert e2.value.status == 3


def test_kernel_launch_count():
    s, _ = make_pair(C1)
    s.init_fields(1)
    s.step(3)
    assert s.kernel_launches == 3 * 6
