"""Reference dump format (gpu_flow/code/output/matrix_folder_writer.cu:3-101): host
reader/writer round trips, the reference's own FP32 snapshots, and exact restart with
the AB2 history file (GPU)."""
import os

import numpy as np
import pytest

import oracle
import sdc_b200
from tests.helpers import random_state, rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("real_bytes", [4, 8])
def test_dump_roundtrip(tmp_path, real_bytes):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((3, 16, 9)) + 1j * rng.standard_normal((3, 16, 9))
    p = tmp_path / "m.bin"
    sdc_b200.dump_write(p, a, real_bytes)
    # header: nmat, ndim, dims (x fastest), then complex data
    assert os.path.getsize(p) == 4 * 5 + a.size * 2 * real_bytes
    b = sdc_b200.dump_read(p)
    assert b.shape == a.shape
    if real_bytes == 8:
        assert np.array_equal(a, b)
    else:
        assert np.array_equal(b, a.astype(np.complex64).astype(np.complex128))


def test_dump_rejects_truncated_file(tmp_path):
    a = np.ones((2, 4, 3), np.complex128)
    p = tmp_path / "m.bin"
    sdc_b200.dump_write(p, a)
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-5])
    with pytest.raises(sdc_b200.RBCError) as e:
        sdc_b200.dump_read(p)
    assert e.value.status == 5


def _rebuild_snapshot(tmp_path, snap, name):
    """A file with the reference snapshot's header and size; theta carries its kx = 0 column."""
    hdr = snap[f"{name}_header"]
    dims = [int(d) for d in hdr[2:]]
    vals = np.zeros(dims[::-1] + [2], np.float32)                 # [L][Ny][mox][re, im]
    if name == "theta":
        vals[:, :, 0, :] = snap["theta_col0"]
    if name == "F":
        vals.reshape(-1)[:] = snap["F_values"]
    p = tmp_path / f"{name}.bin"
    p.write_bytes(hdr.astype("<i4").tobytes() + vals.astype("<f4").tobytes())
    assert os.path.getsize(p) == int(snap[f"{name}_size"])
    return p


def test_reads_reference_snapshot_layout(tmp_path):
    """Header words, sizes and the kx = 0 column of the reference's FP32 snapshots
    gpu_flow/data/*_00030000.bin (fixture made by tests/golden/make_snapshot_golden.py)."""
    snap = np.load(os.path.join(GOLDEN, "snapshot_00030000.npz"))
    th = sdc_b200.dump_read(_rebuild_snapshot(tmp_path, snap, "theta"))
    F = sdc_b200.dump_read(_rebuild_snapshot(tmp_path, snap, "F"))
    for n in ("f", "g", "G"):
        assert sdc_b200.dump_read(_rebuild_snapshot(tmp_path, snap, n)).shape == \
            tuple(int(d) for d in snap[f"{n}_header"][2:][::-1])
    assert th.shape == (2, 512, 257)          # [L][Ny][Nx/2+1] of a 512 x 512 x 2 run
    assert F.shape == (2, 1, 1)
    assert np.array_equal(F.reshape(-1), snap["F_values"].astype(np.float64).view(np.complex128))
    col = th[:, :, 0]
    assert np.array_equal(col, snap["theta_col0"].astype(np.float64).view(np.complex128)[..., 0])
    assert np.all(np.isfinite(col)) and np.abs(col).max() > 0
    # the kx = 0 column of a saved state is Hermitian (make_real ran before the dump)
    ny = th.shape[1]
    for r in range(1, ny // 2):
        assert np.array_equal(col[:, r], np.conj(col[:, ny - r]))


CASE = (64, 64, 4, 8.0, 8.0, 3000.0, 1.0, 1e-3)


@pytest.mark.gpu
def test_restart_with_history_is_exact(tmp_path):
    st = random_state(64, 64, 4, seed=12, amp=0.05)
    a = sdc_b200.Solver(*CASE)
    a.set_state(*st)
    a.step(12)
    b = sdc_b200.Solver(*CASE)
    b.set_state(*st)
    b.step(7)
    b.save_state(str(tmp_path), 7, real_bytes=8)
    b.save_history(str(tmp_path / "hist.bin"))
    c = sdc_b200.Solver(*CASE)
    names = [str(tmp_path / f"{n}_{7:08d}.bin") for n in ("theta", "f", "g", "F", "G")]
    c.load_state(*names)
    c.load_history(str(tmp_path / "hist.bin"))
    c.step(5)
    for x, y in zip(a.get_state(), c.get_state()):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_restart_without_history_takes_an_euler_step(tmp_path):
    # the reference's restart from dump files (main.cu:355-385) starts with Euler
    st = random_state(64, 64, 4, seed=13, amp=0.05)
    b = sdc_b200.Solver(*CASE)
    b.set_state(*st)
    b.step(3)
    b.save_state(str(tmp_path), 3, real_bytes=8)
    c = sdc_b200.Solver(*CASE)
    names = [str(tmp_path / f"{n}_{3:08d}.bin") for n in ("theta", "f", "g", "F", "G")]
    c.load_state(*names)
    o = oracle.Oracle(*CASE, threads=8)
    o.set_state(*b.get_state())
    c.step(4)
    o.step(4)
    for x, y in zip(c.get_state(), o.get_state()):
        assert rel_err(x, y) < 1e-10


@pytest.mark.gpu
def test_load_rejects_wrong_dimensions(tmp_path):
    c = sdc_b200.Solver(*CASE)
    bad = tmp_path / "bad.bin"
    sdc_b200.dump_write(bad, np.zeros((4, 32, 33), np.complex128))
    with pytest.raises(sdc_b200.RBCError) as e:
        c.load_state(str(bad), str(bad), str(bad), str(bad), str(bad))
    assert e.value.status == 1


@pytest.mark.gpu
def test_cli_driver_matches_library(tmp_path):
    import subprocess
    exe = os.path.join(os.path.dirname(sdc_b200.LIB_PATH), "rbc_run")
    cmd = [exe, "-nmodes", "32", "32", "3", "-clength", "8", "8", "-ra", "3000", "-pr", "1", "-dt", "1e-3",
           "-t", "0.01", "-nfiles", "1", "-seed", "5", "-init_amp", "1e-2", "-init_kmax", "3",
           "-real_bytes", "8", "-diag", "5", "-dir", str(tmp_path)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Nu_wall" in r.stdout and os.path.exists(tmp_path / "simulation.log")
    s = sdc_b200.Solver(32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    s.init_fields(5, 1e-2, 3.0)
    s.step(10)
    want = s.get_state()
    for name, w in zip(("theta", "f", "g", "F", "G"), want):
        got = sdc_b200.dump_read(tmp_path / f"{name}_{10:08d}.bin")
        assert np.array_equal(got.reshape(w.shape), w), name
