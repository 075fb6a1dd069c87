"""Tracer consumers on the host: start patterns and the diffusion noise of the oracle,
the moment definitions, and the TRKSS track file writer of the library (no GPU)."""
import numpy as np
import pytest

import oracle
import sdc_b200

LX, LY = 16.0, 8.0


def test_patterns_follow_the_reference_definitions():
    n = 10
    c = oracle.tracer_pattern(1, 5, n, LX, LY).reshape(3, n)
    assert np.all(c[0] == LX / 2) and np.all(c[1] == LY / 2) and np.all(c[2] == 0)
    d = oracle.tracer_pattern(3, 5, n, LX, LY).reshape(3, n)
    assert np.array_equal(d[0], LX * np.arange(n) / n) and np.array_equal(d[1], LY * np.arange(n) / n)
    p = oracle.tracer_pattern(4, 5, n, LX, LY).reshape(3, n)
    assert np.array_equal(p[:, 0::2], p[:, 1::2]) and np.all(p[2] == 0)
    assert np.all((p[0] >= 0) & (p[0] < LX) & (p[1] >= 0) & (p[1] < LY))
    r = oracle.tracer_pattern(0, 5, n, LX, LY)
    assert np.array_equal(r, oracle.tracer_positions(5, n, LX, LY))


def test_sigma_patterns_are_normal():
    n = 20000
    cs = oracle.tracer_pattern(5, 9, n, LX, LY, coord=(3.0, 2.0, 0.1), sigma=0.05).reshape(3, n)
    for v, m in zip(cs, (3.0, 2.0, 0.1)):
        assert abs(v.mean() - m) < 4 * 0.05 / np.sqrt(n)
        assert abs(v.std() / 0.05 - 1) < 0.03
    c0 = oracle.tracer_pattern(2, 9, n, LX, LY, sigma=0.0).reshape(3, n)
    assert np.all(c0[0] == LX / 2)


def test_moments_definition_on_a_small_case():
    # two pairs; the second pair straddles the periodic x boundary
    x = np.array([1.0, 2.0, 0.5, 15.5])
    y = np.array([1.0, 1.0, 3.0, 3.0])
    xyz = np.concatenate([x, y, np.zeros(4)])
    m = oracle.tracer_moments(xyz, LX, LY)
    assert m[0] == pytest.approx(x.mean()) and m[1] == pytest.approx(y.mean())
    assert m[2] == pytest.approx((x * x + y * y).mean() - x.mean() ** 2 - y.mean() ** 2)
    assert m[3] == pytest.approx((1.0 + 1.0) / 2)          # |dx| = 15 > 8 -> 16 - 15 = 1


def test_diffusion_moves_tracers_in_a_fluid_at_rest():
    """With zero velocity the advance is pure diffusion: after m steps every coordinate
    is the start plus sigma times a sum of the counter-based normals."""
    case = (16, 16, 2, LX, LY, 1000.0, 1.0, 1e-3)
    n, D, seed = 4000, 0.2, 77
    o = oracle.Oracle(*case, threads=2)
    xyz = oracle.tracer_pattern(1, 0, n, LX, LY)
    o.tracers_set(xyz)
    o.set_diffusion(D, seed)
    o.step(4)
    got = o.tracers_get().reshape(3, n)
    sig = np.sqrt(2 * D * case[7])
    dx = (got[0] - LX / 2) / sig
    assert abs(dx.mean()) < 0.1 and abs(dx.var() / 4 - 1) < 0.1
    # z starts at 0 and stays well inside the lids: no reflection happened
    dz = got[2] / sig
    assert abs(dz.var() / 4 - 1) < 0.1


def test_trkss_writer_round_trip(tmp_path):
    n, nf = 5, 3
    rng = np.random.default_rng(0)
    frames = rng.standard_normal((nf, 3, n)).astype(np.float32)
    times = np.array([0, 4, 8], np.uint32)
    p = tmp_path / "t.trkss"
    sdc_b200.track_write(p, frames, times, "Particle tracks.  Simulation: Ra=5000.0")
    t = oracle.read_trkss(p)
    assert t["version"] == b"a" and t["tracks"] == n and t["fs"] == 1
    assert t["description"] == "Particle tracks.  Simulation: Ra=5000.0"
    assert (t["time_min"], t["time_max"]) == (0, 8)
    assert np.array_equal(t["times"], times) and np.array_equal(t["frames"], frames)
    # header size: 5 + 1 + 3*4 + len(desc) + 3*4; per frame 4 + 12 n bytes
    assert p.stat().st_size == 5 + 1 + 12 + len(t["description"]) + 12 + nf * (4 + 12 * n)


def test_trkss_writer_rejects_bad_arguments(tmp_path):
    with pytest.raises(sdc_b200.RBCError):
        sdc_b200.track_write(tmp_path / "missing_dir" / "t.trkss", np.zeros((1, 3, 2), np.float32), [0])


def test_oracle_tracer_sets_pinned_by_uniform_runs():
    """Sets [D, 0]: the first half moves exactly as with D for every tracer, the second half
    exactly as without diffusion (the noise is indexed by the global tracer number, and the
    tracers do not act on the flow)."""
    from tests.helpers import random_state
    case = (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    n = 256
    st = random_state(nx, ny, L, seed=81, amp=0.05)
    xyz = oracle.tracer_positions(6, n, case[3], case[4])
    runs = {}
    for name, D, sets in (("sets", 0.0, [1e-3, 0.0]), ("all", 1e-3, None), ("none", 0.0, None)):
        o = oracle.Oracle(*case, threads=2)
        o.set_state(*st)
        o.set_diffusion(D, 13)
        if sets is not None:
            o.set_tracer_sets(sets)
        o.tracers_set(xyz)
        o.step(6)
        runs[name] = o.tracers_get().reshape(3, n)
    h = n // 2
    assert np.array_equal(runs["sets"][:, :h], runs["all"][:, :h])
    assert np.array_equal(runs["sets"][:, h:], runs["none"][:, h:])
    assert not np.array_equal(runs["all"][:, h:], runs["none"][:, h:])
