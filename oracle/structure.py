"""CPU oracle of the second-order structure functions (test infrastructure only).

Restates structure_function_2d (gpu_flow/code/postProcessing/structure_function_2d.cu)
step by step, with the oracle's own FFT in place of cuFFT: for every displacement r the
spectrum of the shifted difference (twiddle_by_shift_*, :444-656), the C2R transform to
the physical plane (:146-158), the power order/2 (abs_and_square, :434-441), the R2C
transform back and the 1/P scaling (:162-171), and the sum over the half spectrum of
part_1 * conj(part_2) (mult_conj_pointwise_on_device, reduce: :174-178, 324-352); the
reference computes part_1 and part_2 the same way, so the sum is of |.|^2.
"""
import numpy as np

from oracle import irfft2, rfft2

LAMBDA_A, LAMBDA_B = 4.73004074, 7.85320462  # the literal lambdas of twiddle_by_shift_u_*


def midplane_field(theta, f, g, field, nx, lx, ly):
    """The reference's mid-plane spectrum A(k) [Ny][Nx/2+1] of field 'theta', 'u1', 'u2'."""
    L, ny, mox = theta.shape
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    kx = c * 2 * np.pi / lx
    ky = np.where(r < ny // 2 + 1, r, r - ny) * 2 * np.pi / ly
    if field == "theta":
        return theta[0].astype(complex)  # the second ansatz function vanishes at z = 0
    la, lb = LAMBDA_A, LAMBDA_B
    z = [la * np.sinh(la * 0) / np.cosh(la * 0.5) + la * np.sin(la * 0) / np.cos(la * 0.5),
         lb * np.cosh(lb * 0) / np.sinh(lb * 0.5) - lb * np.cos(lb * 0) / np.sin(lb * 0.5)]
    fz = sum(z[m] * f[m] for m in range(min(L, 2)))
    if field == "u1":
        return 1j * kx * fz + 1j * ky * g[0]
    return 1j * ky * fz - 1j * kx * g[0]


def structure_function(theta, f, g, field, direction, r_min, r_max, nsamples, nx, lx, ly, order=2):
    """S(r_i), i < nsamples, r_i = r_min + i (r_max - r_min) / nsamples along 'x' or 'y'."""
    ny = theta.shape[1]
    mox = nx // 2 + 1
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    kx = c * 2 * np.pi / lx
    ky = np.where(r < ny // 2 + 1, r, r - ny) * 2 * np.pi / ly
    a = midplane_field(theta, f, g, field, nx, lx, ly)
    inc = (r_max - r_min) / nsamples
    out = np.zeros(nsamples)
    for i in range(nsamples):
        rd = r_min + i * inc
        r1, r2 = (rd, 0.0) if direction == "x" else (0.0, rd)
        arg = r1 * kx + r2 * ky
        tw = (np.cos(arg) - 1.0) + 1j * np.sin(arg)
        d = a * tw
        phys = irfft2(d, nx) ** (order / 2.0)
        part = rfft2(phys) / (nx * ny)
        out[i] = np.sum(part * np.conj(part)).real
    return out
