"""CPU tests of the surrogate's oracle (oracle/fno.py): its BF16 rounding against torch's,
its truncated DFT matrices against numpy.fft, and its hand-written gradient against
central finite differences."""
import numpy as np
import pytest
import torch

from oracle.fno import FNOOracle, round_bf16


def test_round_bf16_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=4096) * 10.0 ** rng.integers(-8, 8, size=4096),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(round_bf16(x), ref)


def test_spectral_conv_is_truncated_fft_filter():
    """With R = identity per mode the spectral part is the low-pass filter
    irfft2(rfft2(h) on kx < m, ky in [0, m) U [-m, 0))."""
    nx, ny, m, W = 16, 12, 4, 3
    o = FNOOracle(nx, ny, 4, W, m, 1, 8, bf16=False)
    rng = np.random.default_rng(1)
    h = rng.normal(size=(2, ny, nx, W))
    Rc = np.zeros((2 * m, m, W, W), complex)
    Rc[:, :, np.arange(W), np.arange(W)] = 1.0
    got = o.spectral_conv(h, Rc)
    sp = np.fft.rfft2(h, axes=(1, 2))
    mask = np.zeros((ny, nx // 2 + 1), bool)
    ky = np.fft.fftfreq(ny, 1.0 / ny)
    mask[(ky >= -m) & (ky < m), :m] = True
    ref = np.fft.irfft2(sp * mask[None, :, :, None], s=(ny, nx), axes=(1, 2))
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


def test_oracle_gradient_matches_finite_differences():
    nx, ny, C, W, m, nl, H, B = 12, 10, 8, 8, 3, 2, 8, 2
    o = FNOOracle(nx, ny, C, W, m, nl, H, bf16=False)
    rng = np.random.default_rng(2)
    v = rng.normal(size=o.nparam) * 0.3
    # spectral weights of the size that makes the spectral part matter
    p = o.unpack(v)
    for l in range(nl):
        p[f"R{l}"] *= 0.5
    v = o.pack(p)
    x = rng.normal(size=(B, ny, nx, C))
    t = rng.normal(size=(B, ny, nx, C))
    loss, g = o.loss_grad(v, x, t)
    idx = rng.choice(o.nparam, 60, replace=False)
    # include every block
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in o.shapes])
    idx = np.unique(np.concatenate([idx, offs[:-1], offs[1:] - 1]))
    eps = 1e-6
    for i in idx:
        vp, vm = v.copy(), v.copy()
        vp[i] += eps
        vm[i] -= eps
        fd = (o.loss_grad(vp, x, t)[0] - o.loss_grad(vm, x, t)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7 * np.abs(g).max(), (i, fd, g[i])
