"""CPU tests of the oracle: pinned to the reference's own Galerkin tables (golden
vectors from gpu_flow/code/util/coeff.cu, tests/golden/make_golden.py), its known-answer
comments, numpy/scipy for FFT and LU, and physics checks of the assembled step."""
import os

import numpy as np
import pytest
import scipy.linalg

import oracle
from tests.helpers import random_state, rel_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["Iac", "Ia1", "Ia2", "Ibbb", "Ibb1", "Ib11", "I111", "Iabc", "Iac1", "Iaab", "Iaa1", "Iab2", "Ia12", "lambda"]


@pytest.mark.parametrize("L", [4, 8, 12])
@pytest.mark.parametrize("name", NAMES)
def test_oracle_tables_match_reference_golden(L, name):
    ref = np.load(os.path.join(GOLD, f"coeff_L{L}.npz"))[name]
    got = oracle.table(L, name)
    assert got.shape == ref.shape
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-13 * scale, name


@pytest.mark.parametrize("L", [4, 8, 12])
def test_linear_tables_couple_equal_parities_only(L):
    """The update kernel keeps only the same-parity half of each row of B_ff^-1 and of the
    implicit operator (built from Iac and Ia1): in the reference's own tables every entry
    whose row and column parities differ is an exact zero."""
    ref = np.load(os.path.join(GOLD, f"coeff_L{L}.npz"))
    i, j = np.meshgrid(np.arange(L), np.arange(L), indexing="ij")
    odd = ((i + j) % 2).ravel() == 1
    for name in ("Iac", "Ia1"):
        t = ref[name].ravel()
        assert np.all(t[odd] == 0.0), name
        assert np.all(np.diag(t.reshape(L, L)) != 0.0), name  # the diagonal is not


def test_known_answer_comments():
    # gpu_flow/code/operator/linear_implicit_operator.cu:3-9
    ia1 = oracle.table(2, "Ia1")
    iac = oracle.table(2, "Iac")
    lam = oracle.table(2, "lambda")
    assert abs(ia1[0] - 0.6973) < 1e-4
    assert abs(ia1[3] - (-0.6904)) < 1e-4
    assert abs(iac[0] - (-12.30)) < 1e-2
    assert abs(iac[3] - (-46.05)) < 1e-2
    assert abs(lam[0] - 4.73) < 1e-2 and abs(lam[1] - 7.85) < 1e-2


@pytest.mark.parametrize("n", [8, 12, 48, 64, 96, 192, 256, 512])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.abs(oracle.fft(x, -1) - np.fft.fft(x)).max() < 1e-13 * n
    assert np.abs(oracle.fft(x, +1) - n * np.fft.ifft(x)).max() < 1e-13 * n


def test_rfft2_conventions():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((48, 64))
    A = oracle.rfft2(a)
    assert np.abs(A - np.fft.rfft2(a)).max() < 1e-11
    # cuFFT C2R is unnormalised
    assert np.abs(oracle.irfft2(A, 64) - a * a.size).max() < 1e-9


@pytest.mark.parametrize("n", [2, 5, 8, 16])
def test_lu_matches_scipy(n):
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n)) + n * np.eye(n)
    assert np.abs(oracle.lu_invert(m) - scipy.linalg.inv(m)).max() < 1e-12


def test_below_onset_decays_above_grows():
    res = {}
    for ra in (1500.0, 2500.0):
        o = oracle.Oracle(32, 32, 4, 8.0, 8.0, ra, 1.0, 1e-2, threads=4)
        o.init_theta(1, 1e-3, 4.0)
        n0 = np.linalg.norm(o.get_state()[0])
        o.step(200)
        res[ra] = np.linalg.norm(o.get_state()[0]) / n0
    assert res[1500.0] < 0.1
    assert res[2500.0] > 2.0


def test_nusselt_forms_agree_at_steady_state():
    # Ra = 2500 relaxes to steady rolls. In steady state the q = 0 temperature balance
    # makes sum_k (k pi) theta_k the L-term cosine series of <w theta>(z) at the wall, so
    # Nu_wall and Nu_vol agree up to that series' truncation tail: the gap must be small
    # and shrink as L grows.
    gaps = []
    for L in (4, 6):
        o = oracle.Oracle(24, 24, L, 6.0, 6.0, 2500.0, 1.0, 2e-2, threads=4)
        o.init_theta(7, 1e-2, 3.0)
        o.step(1500)
        d = o.diagnostics()
        assert d["nu_wall"] > 1.05
        gaps.append(abs(d["nu_wall"] - d["nu_vol"]) / d["nu_wall"])
    assert gaps[0] < 0.02
    assert gaps[1] < gaps[0]


def test_hermitian_symmetry_preserved():
    o = oracle.Oracle(32, 32, 3, 8.0, 8.0, 3000.0, 1.0, 1e-2, threads=4)
    o.set_state(*random_state(32, 32, 3, 5, amp=1e-2))
    o.step(5)
    th, f, g, F, G = o.get_state()
    ny = th.shape[1]
    for a in (th, f, g):
        for r in range(1, ny // 2):
            assert np.array_equal(a[:, r, 0], np.conj(a[:, ny - r, 0]))
        assert np.all(a[:, 0, 0].imag == 0)
    assert np.all(F.imag == 0) and np.all(G.imag == 0)


def test_seeded_init_is_reproducible_and_banded():
    o = oracle.Oracle(64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3, threads=1)
    o.init_theta(1, 1e-3, 4.0)
    th = o.get_state()[0]
    o.init_theta(1, 1e-3, 4.0)
    assert np.array_equal(th, o.get_state()[0])
    ny, mox = th.shape[1], th.shape[2]
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    ry = np.where(r > ny // 2, r - ny, r)
    outside = (c * c + ry * ry) > 16
    assert np.all(th[0][outside] == 0) and np.all(th[1:] == 0)
    assert np.abs(th[0]).max() > 1e-4


def test_tracer_positions_uniform():
    xyz = oracle.tracer_positions(2, 20000, 32.0, 32.0)
    x, y, z = xyz[:20000], xyz[20000:40000], xyz[40000:]
    assert x.min() >= 0 and x.max() < 32 and y.min() >= 0 and y.max() < 32
    assert z.min() > -0.5 and z.max() < 0.5
    assert abs(x.mean() - 16) < 0.3 and abs(z.mean()) < 0.01
