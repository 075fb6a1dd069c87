"""GPU tests of the learned surrogate (rbc_fno_*, through the C ABI): the collocation
fields against the oracle's synthesis, the increment projection round trip, the network's
forward pass and gradient against the CPU oracle (oracle/fno.py, same BF16 rounding
points), training, and the judge logic of the rollout."""
import numpy as np
import pytest

import oracle
import sdc_b200
from oracle.fno import FNOOracle
from tests.helpers import random_state, rel_err

pytestmark = pytest.mark.gpu


def basis_at_nodes(L, nq):
    """C, C', S of the vertical basis at the nq Gauss-Legendre nodes of (-1/2, 1/2)."""
    z = 0.5 * np.polynomial.legendre.leggauss(nq)[0]
    lam = oracle.table(L, "lambda")
    C = np.zeros((nq, L))
    Cp = np.zeros((nq, L))
    S = np.zeros((nq, L))
    for m in range(L):
        k, l = m + 1, lam[m]
        if k % 2:
            C[:, m] = np.cosh(l * z) / np.cosh(l / 2) - np.cos(l * z) / np.cos(l / 2)
            Cp[:, m] = l * (np.sinh(l * z) / np.cosh(l / 2) + np.sin(l * z) / np.cos(l / 2))
        else:
            C[:, m] = np.sinh(l * z) / np.sinh(l / 2) - np.sin(l * z) / np.sin(l / 2)
            Cp[:, m] = l * (np.cosh(l * z) / np.sinh(l / 2) - np.cos(l * z) / np.sin(l / 2))
        S[:, m] = np.sin(k * np.pi * (z + 0.5))
    return C, Cp, S


CASE = (64, 48, 4, 8.0, 6.0, 3000.0, 1.0, 1e-3)


def test_colloc_fields_match_oracle_synthesis():
    nx, ny, L = CASE[:3]
    nq = 8
    s = sdc_b200.Solver(*CASE)
    o = oracle.Oracle(*CASE, threads=4)
    st = random_state(nx, ny, L, seed=5)
    s.set_state(*st)
    o.set_state(*st)
    f = sdc_b200.FNO(nx, ny, L, nq, width=8, modes=4, layers=1, hidden=8, max_batch=1)
    got = f.colloc_get(s)
    ph = o.synthesis()
    C, Cp, S = basis_at_nodes(L, nq)
    th = np.einsum("qm,myx->yxq", S, ph[5])
    u = np.einsum("qm,myx->yxq", Cp, ph[0]) + np.einsum("qm,myx->yxq", S, ph[3])
    v = np.einsum("qm,myx->yxq", Cp, ph[1]) + np.einsum("qm,myx->yxq", S, ph[4])
    w = np.einsum("qm,myx->yxq", C, ph[2])
    ref = np.concatenate([th, u, v, w], axis=-1)
    assert got.shape == ref.shape
    for k in range(4):
        sl = slice(k * nq, (k + 1) * nq)
        assert rel_err(got[..., sl], ref[..., sl]) < 1e-6, k


def test_colloc_increment_roundtrip():
    """Adding the collocation fields of the state as an increment doubles the state:
    the least-squares projection in z, the DFT and the vorticity/divergence inversion
    recover (theta, f, g, F, G) from (theta, u, v, w)."""
    nx, ny, L = CASE[:3]
    s = sdc_b200.Solver(*CASE)
    st = random_state(nx, ny, L, seed=6)
    # f and g at q = 0 do not enter any field (the solver keeps them 0)
    st[1][:, 0, 0] = 0
    st[2][:, 0, 0] = 0
    s.set_state(*st)
    f = sdc_b200.FNO(nx, ny, L, 2 * L, width=8, modes=4, layers=1, hidden=8, max_batch=1)
    x = f.colloc_get(s)
    f.colloc_add(s, x)
    got = s.get_state()
    for name, a, b in zip(("theta", "f", "g", "F", "G"), got, st):
        assert rel_err(a, 2 * b) < 2e-6, (name, rel_err(a, 2 * b))


NET = dict(nx=32, ny=32, nz=2, nq=2, width=16, modes=4, layers=2, hidden=32)


def net_pair(seed=3):
    f = sdc_b200.FNO(NET["nx"], NET["ny"], NET["nz"], NET["nq"], width=NET["width"], modes=NET["modes"],
                     layers=NET["layers"], hidden=NET["hidden"], max_batch=2, seed=seed)
    o = FNOOracle(NET["nx"], NET["ny"], 4 * NET["nq"], NET["width"], NET["modes"], NET["layers"], NET["hidden"],
                  bf16=True)
    v = f.get_params().astype(np.float64)
    p = o.unpack(v)
    for l in range(NET["layers"]):  # spectral weights large enough that the spectral path matters
        p[f"R{l}"] *= NET["width"] ** 2 / 4
    v = o.pack(p).astype(np.float32)
    f.set_params(v)
    return f, o, v


def test_fno_forward_matches_oracle():
    f, o, v = net_pair()
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, NET["ny"], NET["nx"], 4 * NET["nq"])).astype(np.float32)
    got = f.forward(x)
    ref = o.forward(v, x)[0]
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 2e-3, err
    # the unrounded network differs by about the BF16 resolution: the rounding is real
    o64 = FNOOracle(NET["nx"], NET["ny"], 4 * NET["nq"], NET["width"], NET["modes"], NET["layers"], NET["hidden"],
                    bf16=False)
    err64 = np.linalg.norm(got - o64.forward(v, x)[0]) / np.linalg.norm(ref)
    assert err64 > 3 * err


def test_fno_gradient_matches_oracle():
    f, o, v = net_pair(seed=4)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, NET["ny"], NET["nx"], 4 * NET["nq"])).astype(np.float32)
    t = rng.standard_normal(x.shape).astype(np.float32)
    loss, g = f.loss_grad(x, t)
    lref, gref = o.loss_grad(v, x, t)
    assert abs(loss - lref) <= 1e-4 * lref
    gp, gr = o.unpack(g), o.unpack(gref)
    for name, _ in o.shapes:
        e = np.linalg.norm(gp[name] - gr[name]) / max(np.linalg.norm(gr[name]), 1e-30)
        assert e < 1e-2, (name, e)


def run_snapshots(case, ra, seed, spin, interval, nsnap):
    """Host states of one run every `interval` steps after `spin` steps."""
    c = list(case)
    c[5] = ra
    s = sdc_b200.Solver(*c)
    s.init_fields(seed, 1e-2, 4.0)
    s.step(spin)
    out = []
    for k in range(nsnap):
        out.append(s.get_state())
        if k + 1 < nsnap:
            s.step(interval)
    s.close()
    return out


SMALL = (32, 32, 2, 8.0, 8.0, 4000.0, 1.0, 1e-3)


def test_training_reduces_loss_and_predicts_increment():
    """Trained on the even-numbered pairs (10 steps apart) of four runs, the network
    predicts most of the increment of the odd-numbered pairs it has not seen: what the
    learned part gains over persistence (predicting no change)."""
    f = sdc_b200.FNO(32, 32, 2, 4, width=16, modes=6, layers=2, hidden=32, max_batch=4, seed=1, interval_steps=10)
    runs = [run_snapshots(SMALL, ra, seed, 1500, 10, 21) for ra, seed in
            [(3000.0, 1), (3700.0, 2), (4400.0, 3), (5000.0, 4)]]
    f.reserve(sum(len(r) for r in runs))
    s = sdc_b200.Solver(*SMALL)
    slot, src, dst, held = 0, [], [], []
    for r in runs:
        for k, st in enumerate(r):
            s.set_state(*st)
            f.capture(s, slot)
            if k:
                (src if k % 2 else held).append(slot - 1)
                if k % 2:
                    dst.append(slot)
            slot += 1
    losses = f.train(np.array(src), np.array(dst), epochs=60, batch=4, lr=3e-3, seed=0)
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.3 * losses[0], losses
    flat = [st for r in runs for st in r]
    err2 = inc2 = 0.0
    for i in held:
        s.set_state(*flat[i])
        x0 = f.colloc_get(s)
        f.advance(s, 1)
        pred = f.colloc_get(s)
        s.set_state(*flat[i + 1])
        ref = f.colloc_get(s)
        err2 += np.sum((pred - ref) ** 2)
        inc2 += np.sum((ref - x0) ** 2)
    assert np.sqrt(err2 / inc2) < 0.5, np.sqrt(err2 / inc2)


def test_surrogate_judge_takes_over():
    f = sdc_b200.FNO(32, 32, 2, 4, width=16, modes=6, layers=2, hidden=32, max_batch=2, seed=2, interval_steps=10)
    s = sdc_b200.Solver(*SMALL)
    s.init_fields(4, 1e-2, 4.0)
    s.step(500)
    st = s.get_state()
    # an untrained network fails a tight check: the plain step runs the rest
    r = f.run(s, intervals=20, judge_every=5, nu_tol=1e-12, spec_bins=16, spec_tol=0.0,
              fallback_intervals=-1)
    assert (r["checks"], r["fallbacks"], r["surrogate_intervals"], r["plain_intervals"]) == (1, 1, 4, 16), r
    # a loose check never fails: every fifth interval is a plain one
    s.set_state(*st)
    r = f.run(s, intervals=20, judge_every=5, nu_tol=1e9, spec_bins=16, spec_tol=1e9)
    assert (r["checks"], r["fallbacks"], r["surrogate_intervals"], r["plain_intervals"]) == (4, 0, 16, 4), r
    assert r["ms"] > 0 and r["max_nu_err"] >= r["last_nu_err"] >= 0
    # every check fails and fallback_intervals = 2: checks at t = 2, 5, 8, 11, two plain
    # intervals after each of the first three, the surrogate only at t = 0, 1
    s.set_state(*st)
    r = f.run(s, intervals=12, judge_every=3, nu_tol=1e-12, fallback_intervals=2)
    assert (r["checks"], r["fallbacks"], r["surrogate_intervals"], r["plain_intervals"]) == (4, 4, 2, 10), r


def test_physics_mean_modes_track_the_plain_step():
    """With the network's increment zeroed, one surrogate interval still advances the
    horizontal-mean modes (theta_k at q = 0, F_k, G_k) by the plain step's own q = 0
    recursion: they follow the plain run over the same steps to a small fraction of their
    change, while without the physics update they stay where they were."""
    s = sdc_b200.Solver(*SMALL)
    s.init_fields(5, 1e-2, 4.0)
    s.step(1500)
    st0 = s.get_state()
    s.step(10)
    ref = s.get_state()
    mean = lambda st: np.concatenate([st[0][:, 0, 0].real, st[3].real, st[4].real])
    m0, mref = mean(st0), mean(ref)
    change = np.abs(mref - m0).max()
    assert change > 1e-8
    # the forcing is taken constant over the interval (no previous interval): in this
    # growth phase that leaves a fraction of the change
    for pm, bound in ((True, 0.25), (False, None)):
        f = sdc_b200.FNO(32, 32, 2, 4, width=16, modes=6, layers=2, hidden=32, max_batch=1, seed=2,
                         interval_steps=10, physics_mean=pm)
        f.set_params(np.zeros(f.num_params, np.float32))
        C = 16
        f.set_norm(np.stack([np.zeros(C), np.ones(C), np.zeros(C), np.ones(C)]).astype(np.float32))
        s.set_state(*st0)
        f.advance(s, 1)
        got = s.get_state()
        # everything but the mean modes is unchanged (zero increment)
        assert rel_err(got[0][:, 1:, :], st0[0][:, 1:, :]) == 0.0
        err = np.abs(mean(got) - mref).max()
        if bound is None:
            assert err == pytest.approx(change, rel=1e-12)
        else:
            assert err < bound * change, (err, change)


def test_pushforward_and_augmented_training_run():
    """Training with the box symmetries, input noise and pushforward inputs (the network's
    own prediction from the previous snapshot of a run) stays finite and lowers the loss."""
    f = sdc_b200.FNO(32, 32, 2, 4, width=16, modes=6, layers=2, hidden=32, max_batch=4, seed=3, interval_steps=10)
    runs = [run_snapshots(SMALL, ra, seed, 1500, 10, 9) for ra, seed in [(3500.0, 6), (4500.0, 7)]]
    f.reserve(sum(len(r) for r in runs))
    s = sdc_b200.Solver(*SMALL)
    slot, src, dst = 0, [], []
    for r in runs:
        for k, st in enumerate(r):
            s.set_state(*st)
            f.capture(s, slot)
            if k:
                src.append(slot - 1)
                dst.append(slot)
            slot += 1
    f.set_train_options(augment=2, noise_rel=0.1, pushforward=True)
    losses = f.train(np.array(src), np.array(dst), epochs=30, batch=4, lr=3e-3, seed=1)
    # input noise makes single epochs noisy: compare the first and last five
    assert np.all(np.isfinite(losses)) and losses[-5:].mean() < 0.7 * losses[:5].mean(), losses
    with pytest.raises(sdc_b200.RBCError):
        f.set_train_options(augment=3)


NET_BIG = dict(nx=128, ny=128, nz=2, nq=2, width=16, modes=8, layers=2, hidden=32)


def test_fno_tensor_core_path_matches_oracle():
    """At 128^2 with batch 3 (49,152 rows, 384 row tiles) the channel-map products run on the
    tcgen05 kernel: forward and gradient against the oracle with the bars above, and the two
    GEMM paths agree with each other to BF16 resolution."""
    b = 3
    f = sdc_b200.FNO(NET_BIG["nx"], NET_BIG["ny"], NET_BIG["nz"], NET_BIG["nq"], width=NET_BIG["width"],
                     modes=NET_BIG["modes"], layers=NET_BIG["layers"], hidden=NET_BIG["hidden"], max_batch=b, seed=5)
    g = sdc_b200.FNO(NET_BIG["nx"], NET_BIG["ny"], NET_BIG["nz"], NET_BIG["nq"], width=NET_BIG["width"],
                     modes=NET_BIG["modes"], layers=NET_BIG["layers"], hidden=NET_BIG["hidden"], max_batch=b, seed=5,
                     gemm_path="mma_sync")
    o = FNOOracle(NET_BIG["nx"], NET_BIG["ny"], 4 * NET_BIG["nq"], NET_BIG["width"], NET_BIG["modes"],
                  NET_BIG["layers"], NET_BIG["hidden"], bf16=True)
    v = f.get_params()
    g.set_params(v)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((b, NET_BIG["ny"], NET_BIG["nx"], 4 * NET_BIG["nq"])).astype(np.float32)
    t = rng.standard_normal(x.shape).astype(np.float32)
    got, alt = f.forward(x), g.forward(x)
    ref = o.forward(v.astype(np.float64), x)[0]
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-3
    assert np.linalg.norm(got - alt) / np.linalg.norm(alt) < 2e-3
    loss, gr = f.loss_grad(x, t)
    lref, gref = o.loss_grad(v.astype(np.float64), x, t)
    assert abs(loss - lref) <= 1e-4 * lref
    gp, gq = o.unpack(gr), o.unpack(gref)
    for name, _ in o.shapes:
        e = np.linalg.norm(gp[name] - gq[name]) / max(np.linalg.norm(gq[name]), 1e-30)
        assert e < 1e-2, (name, e)
