"""Tracer consumers on the GPU against the oracle: start patterns, the diffusion step,
moments, recorded tracks (the reference's position buffer and track writer) and the
refusal to overrun the track ring."""
import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state

pytestmark = pytest.mark.gpu

CASE = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)


def _pair(n, **kw):
    s = sdc_b200.Solver(*CASE, n_tracers=n, **kw)
    o = oracle.Oracle(*CASE, threads=8)
    st = random_state(*CASE[:3], seed=41, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    return s, o


@pytest.mark.parametrize("pattern,kind", [("random", 0), ("center", 1), ("center_sigma", 2), ("diagonal", 3),
                                          ("pairs", 4), ("coord_sigma", 5)])
def test_start_patterns_match_oracle(pattern, kind):
    n = 1000
    s = sdc_b200.Solver(*CASE, n_tracers=n)
    s.tracers_init(pattern, seed=13, coord=(1.5, 2.5, -0.2), sigma=0.01)
    ref = oracle.tracer_pattern(kind, 13, n, CASE[3], CASE[4], coord=(1.5, 2.5, -0.2), sigma=0.01)
    assert np.array_equal(s.tracers_get(), ref)


def test_pairs_need_an_even_count():
    s = sdc_b200.Solver(*CASE, n_tracers=7)
    with pytest.raises(sdc_b200.RBCError):
        s.tracers_init("pairs", seed=1)


def test_diffusion_matches_oracle():
    n, D, seed = 4096, 0.01, 1234
    s, o = _pair(n, tracer_diffusivity=D, noise_seed=seed)
    o.set_diffusion(D, seed)
    xyz = oracle.tracer_positions(2, n, CASE[3], CASE[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(12)
    o.step(12)
    got, ref = s.tracers_get(), o.tracers_get()
    assert np.abs(got - ref).max() < 1e-9
    # without diffusion the same run ends elsewhere: the noise was applied
    s2, _ = _pair(n)
    s2.tracers_set(xyz)
    s2.step(12)
    assert np.abs(s2.tracers_get() - got).max() > 1e-3


def test_moments_match_oracle():
    """Pairs start on one point; advection alone moves both alike, diffusion separates them."""
    n = 4096
    s, o = _pair(n, tracer_diffusivity=0.02, noise_seed=4)
    o.set_diffusion(0.02, 4)
    s.tracers_init("pairs", seed=3)
    xyz = s.tracers_get()
    o.tracers_set(xyz)
    s.step(5)
    o.step(5)
    got = s.tracer_moments()
    ref = oracle.tracer_moments(o.tracers_get(), CASE[3], CASE[4])
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-14)
    assert got[3] > 0   # the pairs separated


def test_tracks_record_every_period():
    n, period = 2048, 3
    s, _ = _pair(n, track_frames=8, track_period=period)
    s.tracers_seed(5)
    ref = {0: s.tracers_get()}
    for m in range(1, 13):
        s.step(1)
        if m % period == 0:
            ref[m] = s.tracers_get()
    frames, times = s.tracks_read()
    assert list(times) == [0, 3, 6, 9, 12]
    for f, t in zip(frames, times):
        assert np.array_equal(f, ref[int(t)].reshape(3, n).astype(np.float32))
    # everything was read; the next frames continue from step 15
    s.step(3)
    frames, times = s.tracks_read()
    assert list(times) == [15]


def test_track_ring_full_refuses_steps(tmp_path):
    n = 256
    s, _ = _pair(n, track_frames=3)
    s.tracers_seed(5)                      # frame 0
    s.step(2)                              # frames 1, 2: the ring is full
    with pytest.raises(sdc_b200.RBCError) as e:
        s.step(1)
    assert e.value.status == 1
    frames, times = s.tracks_read(max_frames=2)
    assert list(times) == [0, 1]
    s.step(2)
    frames, times = s.tracks_read()
    assert list(times) == [2, 3, 4]
    p = tmp_path / "tr.trkss"
    sdc_b200.track_write(p, frames, times, "Particle tracks")
    t = oracle.read_trkss(p)
    assert np.array_equal(t["frames"], frames) and list(t["times"]) == [2, 3, 4]


def test_tracks_identical_with_graph_replay():
    """Steps replayed from the CUDA graph (the tracer on its side stream) record the same
    frames as single steps."""
    n = 1024
    a, _ = _pair(n, track_frames=40)
    b, _ = _pair(n, track_frames=40)
    for s in (a, b):
        s.tracers_seed(9)
    a.step(30)
    for _ in range(30):
        b.step(1)
    fa, ta = a.tracks_read()
    fb, tb = b.tracks_read()
    assert np.array_equal(ta, tb) and np.array_equal(fa, fb)


def test_tracer_sets_match_oracle():
    """Two tracer sets with their own diffusivities (one particle_tracer per Lewis number
    in the reference) against the oracle's per-set diffusion."""
    case = (32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    n = 1024
    s = sdc_b200.Solver(*case, n_tracers=n, tracer_sets=2, noise_seed=11)
    o = oracle.Oracle(*case, threads=8)
    st = random_state(nx, ny, L, seed=71, amp=0.05)
    s.set_state(*st)
    o.set_state(*st)
    s.tracer_set_diffusivity(0, 1e-3)
    s.tracer_set_diffusivity(1, 0.0)
    o.set_diffusion(0.0, 11)
    o.set_tracer_sets([1e-3, 0.0])
    xyz = oracle.tracer_positions(4, n, case[3], case[4])
    s.tracers_set(xyz)
    o.tracers_set(xyz)
    s.step(12)
    o.step(12)
    assert np.abs(s.tracers_get() - o.tracers_get()).max() < 1e-9
    m = [s.tracer_moments_set(k) for k in range(2)]
    pos = o.tracers_get().reshape(3, n)
    for k in range(2):
        x, y = pos[0, 512 * k:512 * (k + 1)], pos[1, 512 * k:512 * (k + 1)]
        assert abs(m[k][0] - x.mean()) < 1e-12 and abs(m[k][1] - y.mean()) < 1e-12
