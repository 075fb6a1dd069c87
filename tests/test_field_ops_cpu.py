"""The oracle's freeze and heating operators (freeze_operator.cu, masktemp.cu of
gpu_flow/code/operator) against an independent numpy restatement: masks from the
reference's formulas evaluated on index grids, C2R / R2C as numpy's irfft2 * P / rfft2
(cuFFT's unnormalised conventions)."""
import numpy as np
import pytest

import oracle
from tests.helpers import kept_mask, random_state, rel_err


def np_mask(nx, ny, shape, cx, cy, size):
    """init_mask_physical_space_circle / _rectangle (freeze_operator.cu:261-308,
    masktemp.cu:211-259) on [Ny][Nx]: 1 keeps the current value."""
    row, col = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    if shape == "circle":
        d2 = (col - cx * nx) * (col - cx * nx) + (row - cy * ny) * (row - cy * ny)
        dmax = size * 0.5 * min(nx, ny)
        return (d2 > dmax * dmax).astype(np.int32)
    m = (col < size * nx) | (col > (1 - size) * nx) | (row < size * ny) | (row > (1 - size) * ny)
    return m.astype(np.int32)


def c2r(plane, nx):
    ny = plane.shape[0]
    return np.fft.irfft2(plane, s=(ny, nx)) * (nx * ny)


def r2c(x):
    return np.fft.rfft2(x)


@pytest.mark.parametrize("nx,ny", [(256, 256), (64, 48), (48, 96), (32, 32)])
@pytest.mark.parametrize("shape,cx,cy,size", [
    ("circle", 0.5, 0.5, 0.8),      # main.cu's freeze_circle(0.8)
    ("circle", 0.2, 0.3, 0.8),      # masktemp's centre
    ("circle", 0.5, 0.5, 0.33),
    ("rectangle", 0.5, 0.5, 0.1),   # main.cu's temp_rectangle(0.1)
    ("rectangle", 0.5, 0.5, 0.25),
])
def test_masks_match_reference_formulas(nx, ny, shape, cx, cy, size):
    got = oracle.field_mask(nx, ny, shape, cx, cy, size)
    assert np.array_equal(got, np_mask(nx, ny, shape, cx, cy, size))
    assert 0 < got.sum() < nx * ny


CASES = [(32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3), (48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3)]


def make(case, seed):
    nx, ny, L = case[:3]
    o = oracle.Oracle(*case, threads=2)
    st = random_state(nx, ny, L, seed=seed, amp=0.05)
    o.set_state(*st)
    return o, st


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("shape,size", [("circle", 0.8), ("rectangle", 0.2)])
def test_freeze_matches_numpy(case, shape, size):
    nx, ny, L = case[:3]
    o, st = make(case, 3)
    o.freeze_mask(shape, size)
    assert all(np.array_equal(a, b) for a, b in zip(o.get_state(), st))  # the freeze leaves the state
    frozen = [[c2r(st[fi][k], nx) for k in range(L)] for fi in range(3)]
    st2 = random_state(nx, ny, L, seed=4, amp=0.05)
    o.set_state(*st2)
    o.freeze_apply()
    got = o.get_state()
    m = np_mask(nx, ny, shape, 0.5, 0.5, size)
    for fi in range(3):
        for k in range(L):
            x = c2r(st2[fi][k], nx)
            ref = r2c(np.where(m == 1, x, frozen[fi][k]) * (1.0 / (nx * ny)))
            assert rel_err(got[fi][k], ref) < 1e-13, (fi, k)
    assert np.array_equal(got[3], st2[3]) and np.array_equal(got[4], st2[4])  # F, G untouched


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("shape,size", [("rectangle", 0.1), ("circle", 0.5)])
def test_heat_matches_numpy(case, shape, size):
    nx, ny, L = case[:3]
    o, st = make(case, 5)
    o.heat_apply()  # before the mask: nothing
    assert all(np.array_equal(a, b) for a, b in zip(o.get_state(), st))
    o.heat_mask(shape, size)
    o.heat_apply()
    got = o.get_state()
    m = np_mask(nx, ny, shape, 0.2, 0.3, size)
    for k in range(L):
        x = c2r(st[0][k], nx)
        ref = r2c(np.where(m == 1, x, x + 1.5 / 100) * (1.0 / (nx * ny)))
        assert rel_err(got[0][k], ref) < 1e-13, k
        # the mean of every vertical mode grows by increment x (heated fraction)
        assert abs((got[0][k][0, 0] - st[0][k][0, 0]).real - 0.015 * (m == 0).mean()) < 1e-15
    for a, b in zip(got[1:], st[1:]):
        assert np.array_equal(a, b)


def test_freeze_right_after_the_mask_keeps_the_state():
    case = CASES[0]
    nx, ny = case[:2]
    o, st = make(case, 7)
    o.freeze_mask("circle", 0.8)
    o.freeze_apply()
    keep = kept_mask(nx, ny)
    for a, b in zip(o.get_state()[:3], st[:3]):
        assert rel_err(a * keep, b) < 1e-14


def test_freeze_holds_the_inside_of_the_circle_over_steps():
    """With the freeze applied before every step (main.cu:571-577) the field inside the
    circle stays at its frozen values up to the step's one-step change."""
    case = (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    o, st = make(case, 9)
    o.step(3)
    o.freeze_mask("circle", 0.8)
    th0 = c2r(o.get_state()[0][0], nx)
    o.step(1)
    one = np.abs(c2r(o.get_state()[0][0], nx) - th0).max()
    for _ in range(20):
        o.freeze_apply()
        o.step(1)
    m = np_mask(nx, ny, "circle", 0.5, 0.5, 0.8)
    drift_free = np.abs(c2r(o.get_state()[0][0], nx) - th0)
    o2, _ = make(case, 9)
    o2.step(24)
    drift_plain = np.abs(c2r(o2.get_state()[0][0], nx) - th0)
    inside = m == 0
    assert drift_free[inside].mean() < 0.5 * drift_plain[inside].mean()
    assert one > 0


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("x,y,radius,factor", [(0.5, 0.5, 0.15, 1.1), (0.3, 0.7, 0.4, 0.5)])
def test_masker_matches_numpy(case, x, y, radius, factor):
    """masking::masker: theta scaled by factor inside the circle whose centre is column
    y Nx, row x Ny (the reference's kernel takes c_y for the columns)."""
    nx, ny, L = case[:3]
    o, st = make(case, 8)
    o.masker(x, y, radius, factor)
    got = o.get_state()
    m = np_mask(nx, ny, "circle", y, x, radius)
    for k in range(L):
        xk = c2r(st[0][k], nx)
        ref = r2c(np.where(m == 0, (1.0 / (nx * ny)) * xk * factor, xk * (1.0 / (nx * ny))))
        assert rel_err(got[0][k], ref) < 1e-13, k
    for a, b in zip(got[1:], st[1:]):
        assert np.array_equal(a, b)
