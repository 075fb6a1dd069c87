"""Pattern initial conditions (gpu_flow/code/util/init.cu:22-310) in the oracle against a
separate numpy evaluation of the same formulas and numpy's FFT (no GPU)."""
import numpy as np
import pytest

import oracle

NX, NY, L, LX, LY = 64, 48, 4, 8.0, 6.0


def _numpy_pattern(kind, mode, amp):
    m = int(mode)
    i = np.arange(NX)[None, :]
    j = np.arange(NY)[:, None]
    x, y = i / NX, j / NY
    if kind == 2:      # dislocation: defects at (1/2 + dx/2, 1/4 + dy/2) and (1/2 + dx/2, 3/4 + dy/2)
        x1, y1, y2 = 0.5 + 0.5 / NX, 0.25 + 0.5 / NY, 0.75 + 0.5 / NY
        return amp * np.cos(m * 2 * np.pi * x - np.arctan2(y - y1, x - x1) + np.arctan2(y - y2, x - x1))
    if kind == 4:      # sv, x_frac 0.2
        lo, hi = 0.4, 0.6
        ph = -0.5 * np.sin(2 * np.pi * y) - x * x
        ph = ph + np.where(x > hi, 1.0, np.where(x > lo, 0.5 * (1 - np.cos(np.pi * (x - lo) / 0.2)), 0.0))
        return amp * np.cos(2 * np.pi * (j * (m / NY) + ph))
    if kind == 5:      # cr, x_frac 0.8
        x1 = 0.5 * (0.2 * NX + 1) / NX
        cy = 0.5 * (NY + 1) / NY
        return amp * np.cos(m * 2 * np.pi * y - np.arctan2(y - cy, x - x1) + np.arctan2(y - cy, x - (1 - x1)))
    if kind == 6:      # giantspiral
        r = np.hypot(x - 0.5, y - 0.5)
        return amp * np.cos(2 * np.pi * m * r - np.arctan2(y - 0.5, x - 0.5) + np.arctan2(y - 0.5, x - 0.8))
    raise ValueError(kind)


def _hermitian(a):
    a = a.copy()
    ny = a.shape[0]
    for r in range(ny):
        if r == 0 or r == ny // 2:
            a[r, 0] = a[r, 0].real
        elif r < ny // 2:
            a[r, 0] = np.conj(a[ny - r, 0])
    return a


@pytest.mark.parametrize("kind", [2, 4, 5, 6])
def test_deterministic_patterns_match_numpy(kind):
    o = oracle.Oracle(NX, NY, L, LX, LY, 2000.0, 1.0, 1e-3, threads=2)
    o.init_pattern(kind, 4.7, 1e-6, seed=0, noise=0.0)
    th = o.get_state()[0]
    ref = _hermitian(np.fft.rfft2(_numpy_pattern(kind, 4.7, 1e-6)))
    assert np.abs(th[0] - ref).max() < 1e-12 * np.abs(ref).max()
    assert np.all(th[1:] == 0)


def test_isr_is_one_fourier_mode():
    o = oracle.Oracle(NX, NY, L, LX, LY, 2000.0, 1.0, 1e-3, threads=2)
    o.init_pattern(1, 4.0, 1e-6, seed=11, noise=0.0)
    th = o.get_state()[0][0]
    # amp cos(2 pi 4 x + phase): the unnormalised R2C has P amp / 2 at column 4, row 0
    assert abs(abs(th[0, 4]) - NX * NY * 1e-6 / 2) < 1e-15
    th[0, 4] = 0
    assert np.abs(th).max() < 1e-17


def test_rectangle_and_noise_draws():
    o = oracle.Oracle(NX, NY, L, LX, LY, 2000.0, 1.0, 1e-3, threads=2)
    o.init_pattern(3, 0.0, 1e-6, seed=5, noise=2e-7)
    th = o.get_state()[0]
    parts = np.concatenate([th[1:].real.ravel(), th[1:].imag.ravel()])
    assert np.abs(parts).max() <= 2e-7 and np.abs(parts).max() > 1.9e-7
    o2 = oracle.Oracle(NX, NY, L, LX, LY, 2000.0, 1.0, 1e-3, threads=2)
    o2.init_pattern(3, 0.0, 1e-6, seed=5, noise=2e-7)
    assert np.array_equal(o2.get_state()[0], th)


def test_init_test_pattern():
    o = oracle.Oracle(NX, NY, L, LX, LY, 2000.0, 1.0, 1e-3, threads=2)
    o.init_pattern(7, 0.0, 1e-6)
    th, f, g, F, G = o.get_state()
    c = np.arange(NX // 2 + 1)
    for k in range(L):
        assert np.array_equal(th[k, 0, 1:], 1e-6 * np.sin(c[1:]) + 0j)
        assert np.array_equal(f[k, 0, 1:], 1e-6 * np.sin(c[1:]) + 0j)
    assert th[:, 1:].max() == 0 and np.all(g == 0) and np.all(G == 0)
    assert np.allclose(F.real, 1e-6 * np.cos(np.arange(L)), rtol=0, atol=0)
