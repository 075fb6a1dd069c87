"""The oracle's penalized nonlinear operator (PENALIZED builds of the reference,
nonlinear_operator_rayleigh_noslip.cu:1097-1335) against an independent numpy
restatement of the penalized parts, and its masks (:1653-1738) against numpy formulas."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import random_state, rel_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def np_pen_mask(nx, ny, kind):
    row, col = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    if kind == "rectangle":
        m = (col < 3) | (col > nx - 4) | (row < 3) | (row > ny - 4)
    elif kind == "circle":
        mn = min(nx, ny)
        m = (col - nx // 2) ** 2 + (row - ny // 2) ** 2 > (mn // 2 - 3) ** 2
    elif kind == "disk_array":
        m = np.zeros((ny, nx), bool)
        r = min(nx // 6, ny // 4)
        for a in range(3):
            for b in range(2):
                cx = a * nx // 3 + nx // 6
                cy = b * ny // 2 + ny // 4
                m |= (cx - col) ** 2 + (cy - row) ** 2 < r
    else:
        m = np.ones((ny, nx), bool)
    return m.astype(np.float64)


@pytest.mark.parametrize("nx,ny", [(64, 64), (48, 32), (256, 256), (96, 64)])
@pytest.mark.parametrize("kind", ["rectangle", "circle", "disk_array", "everywhere"])
def test_pen_masks(nx, ny, kind):
    got = oracle.pen_mask(nx, ny, kind)
    assert np.array_equal(got, np_pen_mask(nx, ny, kind))
    assert got.sum() > 0


def test_ia2_is_the_reference_table():
    for L in (4, 8, 12):
        ref = np.load(os.path.join(GOLD, f"coeff_L{L}.npz"))["Ia2"]
        assert np.array_equal(oracle.table(L, "Ia2"), ref)


def np_penalized_parts(case, syn, mask, eta, L):
    """Difference between the penalized and the plain operator, restated with numpy."""
    nx, ny, _, lx, ly, _, pr, _ = case
    P = nx * ny
    mox = nx // 2 + 1
    iac = oracle.table(L, "Iac").reshape(L, L).T   # iac[a, c] = Iac(a, c)
    ia2 = oracle.table(L, "Ia2").reshape(L, L).T
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    ry = np.where(r > ny // 2, r - ny, r)
    ikx = 1j * c * (2 * np.pi / lx)
    iky = 1j * ry * (2 * np.pi / ly)
    lap = -4 * np.pi ** 2 * ((c / lx) ** 2 + (ry / ly) ** 2)
    mu = np.array([[np.fft.rfft2(mask * syn[a, j]) / P for j in range(L)] for a in range(6)])
    u11, u21, u31, u12, u22, th = mu
    pe = pr / eta
    pf = np.zeros((L, ny, mox), complex)
    pF = np.zeros(L, complex)
    pG = np.zeros(L, complex)
    for k in range(L):
        for j in range(L):
            pf[k] += pe * (iac[j, k] * ikx * u11[j] + ia2[k, j] * ikx * u12[j] + iac[j, k] * iky * u21[j]
                           + ia2[k, j] * iky * u22[j] - ia2[j, k] * iky * u11[j] + ia2[j, k] * ikx * u21[j])
            pF[k] += -pe * ia2[j, k] * u11[j][0, 0]
            pG[k] += -pe * ia2[j, k] * u21[j][0, 0]
        pf[k] += pe * (-lap * u31[k] + 0.5 * iky * u12[k] - 0.5 * iky * u22[k])
        pF[k] += 0.5 * pe * u12[k][0, 0]
        pG[k] += 0.5 * pe * u22[k][0, 0]
    dth = -(0.5 / eta) * th
    return dth, -pf / pr, np.zeros_like(pf), -pF / pr, -pG / pr


@pytest.mark.parametrize("case", [(32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3), (48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3),
                                  (32, 48, 4, 6.0, 9.0, 3000.0, 7.0, 1e-3)])
@pytest.mark.parametrize("kind", ["rectangle", "circle", "disk_array", "everywhere"])
def test_penalized_operator_matches_numpy(case, kind):
    nx, ny, L = case[:3]
    eta = 0.01
    o = oracle.Oracle(*case, threads=2)
    st = random_state(nx, ny, L, seed=31, amp=0.05)
    o.set_state(*st)
    plain = o.nonlinear()
    syn = o.synthesis()
    o.set_penalization(eta, kind)
    pen = o.nonlinear()
    want = np_penalized_parts(case, syn, np_pen_mask(nx, ny, kind), eta, L)
    for name, a, b, w in zip(("theta", "f", "g", "F", "G"), pen, plain, want):
        d = a - b
        if name == "g":
            assert np.array_equal(d, 0 * d), name
            continue
        assert rel_err(d, w) < 1e-11, (name, rel_err(d, w))
    o.set_penalization(0.0)
    assert all(np.array_equal(a, b) for a, b in zip(o.nonlinear(), plain))


def test_penalized_steps_damp_the_flow_in_the_frame():
    """Over steps the penalization drives the velocity inside the frame towards zero."""
    case = (32, 32, 2, 8.0, 8.0, 3000.0, 1.0, 1e-3)
    nx, ny, L = case[:3]
    st = random_state(nx, ny, L, seed=37, amp=0.05)
    out = {}
    for eta in (0.0, 0.01):
        o = oracle.Oracle(*case, threads=2)
        o.set_state(*st)
        if eta:
            o.set_penalization(eta, "everywhere")
        o.step(20)
        out[eta] = o.synthesis()
    m = np_pen_mask(nx, ny, "everywhere") > 0
    ke = {e: sum(np.abs(v[a][:, m]).sum() for a in (0, 1, 3, 4)) for e, v in out.items()}
    assert ke[0.01] < 0.5 * ke[0.0]
