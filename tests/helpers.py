"""Shared helpers for the tests: seeded spectral states in the reference layout."""
import numpy as np


def kept_mask(nx, ny):
    """2/3-rule mask of dealias_implicit (implicit_explicit_stepping.cu:173-180)."""
    mox = nx // 2 + 1
    c = np.arange(mox)
    r = np.arange(ny)
    keep_c = ~(mox - c <= (1.0 / 3.0) * mox)
    keep_r = ~(np.abs(0.5 * ny - r) <= (1.0 / 3.0) * 0.5 * ny)
    return keep_r[:, None] & keep_c[None, :]


def hermitian_fix(a):
    """make_real (util.cu:184-209) on [L][Ny][mox] arrays, in place."""
    ny = a.shape[1]
    for r in range(ny):
        if r == 0 or r == ny // 2:
            a[:, r, 0] = a[:, r, 0].real
        elif r < ny // 2:
            a[:, r, 0] = np.conj(a[:, ny - r, 0])
    return a


def random_state(nx, ny, L, seed, amp=1.0, decay=0.15):
    """Seeded smooth random state: kept band only, Hermitian kx=0 column, real F, G."""
    rng = np.random.default_rng(seed)
    mox = nx // 2 + 1
    m = kept_mask(nx, ny)
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    ry = np.where(r > ny // 2, r - ny, r)
    env = np.exp(-decay * np.sqrt(c * c + ry * ry))
    out = []
    for _ in range(3):
        a = (rng.standard_normal((L, ny, mox)) + 1j * rng.standard_normal((L, ny, mox))) * amp
        a *= (env * m)[None]
        a /= (1.0 + np.arange(L))[:, None, None] ** 2
        out.append(hermitian_fix(a))
    out.append(rng.standard_normal(L) * 0.1 * amp + 0j)
    out.append(rng.standard_normal(L) * 0.1 * amp + 0j)
    return out


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max()
    num = np.abs(a - b).max()
    if den == 0:
        return float(num)
    return float(num / den)


_GOLD = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(seed, n):
    """n outputs of SplitMix64 (Steele, Lea & Flood 2014) started at `seed`: integer
    arithmetic only, so the stream is the same on every machine and numpy version."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + _GOLD * (np.arange(1, n + 1, dtype=np.uint64))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def splitmix_uniform(seed, n):
    """n doubles uniform in [-1, 1) from splitmix64 (53-bit mantissas)."""
    u = (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def splitmix_state(nx, ny, L, seed, amp=1.0, decay=0.15):
    """Reproducible smooth random state (same role as random_state, but from SplitMix64 so
    that committed fixtures can rebuild their inputs exactly): uniform [-amp, amp) real and
    imaginary parts in the kept band, an exp(-decay |k|) envelope, 1/(k+1)^2 per vertical
    mode, Hermitian kx = 0 column, real F, G."""
    mox = nx // 2 + 1
    m = kept_mask(nx, ny)
    c = np.arange(mox)[None, :]
    r = np.arange(ny)[:, None]
    ry = np.where(r > ny // 2, r - ny, r)
    env = np.exp(-decay * np.sqrt(c * c + ry * ry))
    n = L * ny * mox
    u = splitmix_uniform(seed, 6 * n + 2 * L)
    out = []
    for i in range(3):
        re = u[2 * i * n:(2 * i + 1) * n].reshape(L, ny, mox)
        im = u[(2 * i + 1) * n:(2 * i + 2) * n].reshape(L, ny, mox)
        a = (re + 1j * im) * amp
        a *= (env * m)[None]
        a /= (1.0 + np.arange(L))[:, None, None] ** 2
        out.append(hermitian_fix(a))
    out.append(u[6 * n:6 * n + L] * 0.1 * amp + 0j)
    out.append(u[6 * n + L:6 * n + 2 * L] * 0.1 * amp + 0j)
    return out
