"""rbc_run's tracer options, as main.cu names them (-npart with one -le value, start patterns,
-write_tracks_every, -calc_secondmoment, -no_step_time), against the same run through the
library."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import sdc_b200

pytestmark = pytest.mark.gpu

CASE = (32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3)
BASE = ["-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1", "-dt", "1e-3",
        "-nfiles", "1", "-seed", "5", "-init_amp", "1e-2", "-init_kmax", "3", "-real_bytes", "8"]


def run(tmp_path, *extra):
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    r = subprocess.run([exe] + BASE + list(extra) + ["-dir", str(tmp_path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    return r


def test_tracks_and_second_moment_match_library(tmp_path):
    run(tmp_path, "-t", "0.02", "-npart", "512", "-le", "1e-3", "-part_pairs", "-write_tracks_every", "2",
        "-calc_secondmoment")
    s = sdc_b200.Solver(*CASE, n_tracers=512, tracer_diffusivity=1e-3, track_frames=256, track_period=2)
    s.init_fields(5, 1e-2, 3.0)
    s.tracers_init("pairs", seed=5)
    m2 = []
    for i in range(20):
        s.step(1)
        m2.append(s.tracer_moments()[2])
    fr, times = s.tracks_read()
    trk = oracle.read_trkss(tmp_path / f"particles_le{'1e-03'}_{20:08d}.trkss")
    assert np.array_equal(trk["times"], times)
    assert np.array_equal(trk["frames"], fr)
    assert "Tracks: Le=1e-03" in trk["description"]
    lines = open(tmp_path / "secondmoment_0.dat").read().splitlines()
    assert lines[0] == "# Data point writer" and lines[1].startswith("# Le 0.001") and lines[2] == "# Data ordering: t, val"
    data = np.array([[float(v) for v in ln.split("\t")] for ln in lines[3:]])
    assert data.shape == (20, 2)
    assert np.allclose(data[:, 0], 1e-3 * np.arange(1, 21))
    assert np.allclose(data[:, 1], m2, rtol=1e-5, atol=0)


def test_no_step_time_advances_only_the_tracers(tmp_path):
    run(tmp_path, "-t", "0.005", "-npart", "256", "-le", "0", "-part_center_sigma", "-part_sigma", "0.3",
        "-write_tracks_every", "1", "-no_step_time")
    s = sdc_b200.Solver(*CASE, n_tracers=256, track_frames=256, track_period=1)
    s.init_fields(5, 1e-2, 3.0)
    init = s.get_state()
    s.tracers_init("center_sigma", seed=5, sigma=0.3)
    for _ in range(5):
        s.tracers_advance()
    fr, times = s.tracks_read()
    trk = oracle.read_trkss(tmp_path / f"particles_le{'0e+00'}_{5:08d}.trkss")
    assert np.array_equal(trk["frames"], fr) and np.array_equal(trk["times"], times)
    for name, w in zip(("theta", "f", "g", "F", "G"), init):
        got = sdc_b200.dump_read(tmp_path / f"{name}_{5:08d}.bin")
        assert np.array_equal(got.reshape(w.shape), w), name


def test_npart_without_le_has_no_tracers(tmp_path):
    """The reference makes one tracer set per -le value: -npart alone gives none."""
    run(tmp_path, "-t", "0.003", "-npart", "128", "-write_tracks_every", "1")
    assert not any(f.endswith(".trkss") for f in os.listdir(tmp_path))


def test_several_lewis_numbers_give_one_set_each(tmp_path):
    """-le_count 2 -le D1 D2: two sets of -npart tracers (one particle_tracer per Lewis
    number), each with its tracks file and second-moment file."""
    run(tmp_path, "-t", "0.006", "-npart", "128", "-le_count", "2", "-le", "1e-3", "1e-1",
        "-write_tracks_every", "1", "-calc_secondmoment")
    s = sdc_b200.Solver(*CASE, n_tracers=256, tracer_sets=2, track_frames=256, track_period=1)
    s.init_fields(5, 1e-2, 3.0)
    for k, D in enumerate((1e-3, 1e-1)):
        s.tracer_set_diffusivity(k, D)
        s.tracers_init_set(k, "random", seed=5 + k)
    m2 = [[], []]
    for _ in range(6):
        s.step(1)
        for k in range(2):
            m2[k].append(s.tracer_moments_set(k)[2])
    fr, times = s.tracks_read()
    for k, tag in enumerate(("1e-03", "1e-01")):
        trk = oracle.read_trkss(tmp_path / f"particles_le{tag}_{6:08d}.trkss")
        assert trk["tracks"] == 128
        assert np.array_equal(trk["frames"], fr[:, :, 128 * k:128 * (k + 1)])
        lines = open(tmp_path / f"secondmoment_{k}.dat").read().splitlines()
        data = np.array([[float(v) for v in ln.split("\t")] for ln in lines[3:]])
        assert np.allclose(data[:, 1], m2[k], rtol=1e-5, atol=0)
    assert m2[1][-1] > m2[0][-1]  # the more diffusive set spreads faster


def test_multitracer_defaults_give_ten_sets(tmp_path):
    """-multitracer without -le: the ten Lewis numbers of the reference's MULTITRACER builds."""
    run(tmp_path, "-t", "0.003", "-npart", "64", "-multitracer", "-calc_secondmoment", "-write_tracks_every", "1")
    les = [1e1, 3e0, 1e0, 3e-1, 1e-1, 3e-2, 1e-2, 1e-3, 1e-4, 1e-5]
    for k, le in enumerate(les):
        lines = open(tmp_path / f"secondmoment_{k}.dat").read().splitlines()
        assert lines[1] == "# Le %.9f" % le and len(lines) == 3 + 3
        trk = oracle.read_trkss(tmp_path / ("particles_le%.0e_%08d.trkss" % (le, 3)))
        assert trk["tracks"] == 64
