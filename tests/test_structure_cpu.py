"""CPU tests of the structure-function oracle (oracle/structure.py): the reference's FFT
round trip on a single Fourier mode against its closed form."""
import numpy as np

from oracle.structure import structure_function


def test_single_mode_closed_form():
    """theta_0 with one mode (kx index 3, ky index 2) and its Hermitian partner absent
    (kx > 0): the half-spectrum sum is (2 - 2 cos(k.r)) |a|^2."""
    nx, ny, L, lx, ly = 32, 24, 3, 8.0, 6.0
    mox = nx // 2 + 1
    th = np.zeros((L, ny, mox), complex)
    f = np.zeros_like(th)
    g = np.zeros_like(th)
    a = 0.3 - 0.7j
    th[0, 2, 3] = a
    th[1, 5, 4] = 5.0  # higher modes do not enter the mid-plane field
    for direction, k in (("x", 3 * 2 * np.pi / lx), ("y", 2 * 2 * np.pi / ly)):
        got = structure_function(th, f, g, "theta", direction, 0.1, 2.1, 10, nx, lx, ly)
        rr = 0.1 + np.arange(10) * 0.2
        ref = (2 - 2 * np.cos(k * rr)) * abs(a) ** 2
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-15)


def test_velocity_uses_the_reference_z_values():
    """u1 of a single f mode of vertical mode 1: |i kx z_1 f|^2 with z_1 = C'_2(0) from the
    reference's literal lambda."""
    nx, ny, L, lx, ly = 32, 24, 2, 8.0, 6.0
    mox = nx // 2 + 1
    th = np.zeros((L, ny, mox), complex)
    f = np.zeros_like(th)
    g = np.zeros_like(th)
    f[1, 0, 2] = 1.5
    lb = 7.85320462
    z1 = lb * (1 / np.sinh(lb / 2) - 1 / np.sin(lb / 2))
    kx = 2 * 2 * np.pi / lx
    got = structure_function(th, f, g, "u1", "x", 0.5, 0.5 + 5 * 0.3, 5, nx, lx, ly)
    rr = 0.5 + np.arange(5) * 0.3
    ref = (2 - 2 * np.cos(kx * rr)) * (kx * z1 * 1.5) ** 2
    assert np.allclose(got, ref, rtol=1e-12)
