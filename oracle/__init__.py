"""ctypes wrapper around the CPU FP64 oracle (oracle/rbc_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py, as the checker. The sdc_b200 package never imports it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    assert a.dtype in (np.float64, np.complex128) and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            _build.build()
        L = ctypes.CDLL(path)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 5 + [ctypes.c_int]
        for name in ("oracle_destroy", "oracle_step", "oracle_set_threads", "oracle_tracers_advance"):
            getattr(L, name).restype = None
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_tracers_advance.argtypes = [ctypes.c_void_p]
        for name in ("oracle_set_state", "oracle_get_state", "oracle_nonlinear"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [ctypes.c_void_p] + [_dp] * 5
        L.oracle_synthesis.argtypes = [ctypes.c_void_p, _dp]
        L.oracle_synthesis.restype = None
        L.oracle_tracers_set.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int]
        L.oracle_tracers_set.restype = None
        L.oracle_tracers_get.argtypes = [ctypes.c_void_p, _dp]
        L.oracle_tracers_get.restype = None
        L.oracle_velocity_grid.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.oracle_velocity_grid.restype = None
        L.oracle_diagnostics.argtypes = [ctypes.c_void_p, _dp]
        L.oracle_diagnostics.restype = None
        L.oracle_nu_wall.argtypes = [ctypes.c_void_p]
        L.oracle_nu_wall.restype = ctypes.c_double
        L.oracle_spectrum.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, ctypes.c_int]
        L.oracle_spectrum.restype = None
        L.oracle_table.argtypes = [ctypes.c_int, ctypes.c_char_p, _dp]
        L.oracle_table.restype = ctypes.c_int
        L.oracle_operator_table.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.oracle_operator_table.restype = None
        L.oracle_fft.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.oracle_set_colloc.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_set_colloc.restype = None
        L.oracle_fft.restype = None
        L.oracle_rfft2.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.oracle_rfft2.restype = None
        L.oracle_irfft2.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.oracle_irfft2.restype = None
        L.oracle_lu_invert.argtypes = [ctypes.c_int, _dp, _dp]
        L.oracle_lu_invert.restype = ctypes.c_int
        L.oracle_init_theta.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]
        L.oracle_init_theta.restype = None
        L.oracle_tracer_positions.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_tracer_positions.restype = None
        L.oracle_init_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_uint64, ctypes.c_double]
        L.oracle_init_pattern.restype = None
        L.oracle_set_diffusion.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_uint64]
        L.oracle_set_diffusion.restype = None
        L.oracle_tracer_pattern.argtypes = ([ctypes.c_int, ctypes.c_uint64, ctypes.c_int] + [ctypes.c_double] * 6 +
                                            [_dp])
        L.oracle_tracer_pattern.restype = None
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_field_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 3 + [ip]
        L.oracle_field_mask.restype = None
        L.oracle_freeze_mask.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.oracle_freeze_mask.restype = None
        L.oracle_heat_mask.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.oracle_heat_mask.restype = None
        L.oracle_pen_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_pen_mask.restype = None
        L.oracle_set_penalization.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.oracle_set_penalization.restype = None
        L.oracle_set_tracer_sets.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.oracle_set_tracer_sets.restype = None
        L.oracle_set_force_mean.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.oracle_set_force_mean.restype = None
        L.oracle_masker.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4
        L.oracle_masker.restype = None
        for name in ("oracle_freeze_apply", "oracle_heat_apply"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
            getattr(L, name).restype = None
        _LIB = L
    return _LIB


def table(L, name):
    n = L if name == "lambda" else (L * L if name in ("Iac", "Ia1") else L ** 3)
    out = np.zeros(n)
    m = lib().oracle_table(L, name.encode(), _ptr(out))
    if m < 0:
        raise KeyError(name)
    return out[:m]


def fft(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.zeros_like(x)
    lib().oracle_fft(x.size, _ptr(x), _ptr(out), sign)
    return out


def rfft2(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    ny, nx = a.shape
    out = np.zeros((ny, nx // 2 + 1), np.complex128)
    lib().oracle_rfft2(nx, ny, _ptr(a), _ptr(out))
    return out


def irfft2(a, nx):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    ny = a.shape[0]
    out = np.zeros((ny, nx))
    lib().oracle_irfft2(nx, ny, _ptr(a), _ptr(out))
    return out


MASK_SHAPES = {"circle": 0, "rectangle": 1}


def field_mask(nx, ny, shape, cx, cy, size):
    """Mask [Ny][Nx] of the freeze / heating operators (1 keeps the current value)."""
    out = np.zeros((ny, nx), np.int32)
    lib().oracle_field_mask(nx, ny, MASK_SHAPES[shape], cx, cy, size,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return out


PEN_MASKS = {"rectangle": 0, "circle": 1, "disk_array": 2, "everywhere": 3}


def pen_mask(nx, ny, kind):
    """Penalization mask [Ny][Nx] of the PENALIZED builds (1 inside the penalized region)."""
    out = np.zeros((ny, nx))
    lib().oracle_pen_mask(nx, ny, PEN_MASKS[kind], _ptr(out))
    return out


def lu_invert(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros_like(a)
    if lib().oracle_lu_invert(a.shape[0], _ptr(a), _ptr(out)) != 0:
        raise np.linalg.LinAlgError("singular")
    return out


def tracer_positions(seed, n, lx, ly):
    out = np.zeros(3 * n)
    lib().oracle_tracer_positions(seed, n, lx, ly, _ptr(out))
    return out


def tracer_pattern(kind, seed, n, lx, ly, coord=(0.0, 0.0, 0.0), sigma=0.0):
    """Start positions of particle_tracer::init_positions (0 random ... 5 coord_sigma)."""
    out = np.zeros(3 * n)
    lib().oracle_tracer_pattern(kind, seed, n, lx, ly, *coord, sigma, _ptr(out))
    return out


def tracer_moments(xyz, lx, ly):
    """calc_moments_on_GPU and calc_pair_secondmoment_on_GPU (particle_tracer.cu:771-870)
    restated in FP64: <x>, <y>, <x^2+y^2> - <x>^2 - <y>^2, and the mean over pairs
    (2i, 2i+1) of the squared separation with the PERIODIC minimum image, divided by n/2."""
    n = xyz.size // 3
    x, y = xyz[:n], xyz[n:2 * n]
    mx, my = x.mean(), y.mean()
    m2 = (x * x + y * y).mean() - mx * mx - my * my
    m = (n // 2) * 2 if n % 2 == 0 else n - 1
    dx = np.abs(x[1:m:2] - x[0:m:2])
    dy = np.abs(y[1:m:2] - y[0:m:2])
    dx = np.where(dx > 0.5 * lx, lx - dx, dx)
    dy = np.where(dy > 0.5 * ly, ly - dy, dy)
    return np.array([mx, my, m2, (dx * dx + dy * dy).sum() / (n // 2)])


def read_trkss(path):
    """Parses a TRKSS version 'a' track file (track_movie::Write,
    gpu_flow/code/output/track_movie.cpp:256-325) into a dict."""
    import struct
    b = open(path, "rb").read()
    assert b[:5] == b"TRKSS"
    version = b[5:6]
    ntr, fs, dl = struct.unpack_from("<3I", b, 6)
    o = 18
    desc = b[o:o + dl].decode()
    o += dl
    tmin, tmax, nfr = struct.unpack_from("<3I", b, o)
    o += 12
    times, frames = [], []
    for _ in range(nfr):
        times.append(struct.unpack_from("<I", b, o)[0])
        o += 4
        xyz = np.frombuffer(b, "<f4", 3 * ntr, o).reshape(ntr, 3)
        o += 12 * ntr
        frames.append(xyz.T.copy())
    assert o == len(b)
    return {"version": version, "tracks": ntr, "fs": fs, "description": desc, "time_min": tmin,
            "time_max": tmax, "times": np.array(times, np.uint32),
            "frames": np.array(frames, np.float32).reshape(nfr, 3, ntr)}


class Oracle:
    """FP64 CPU restatement of the reference step (see rbc_oracle.cpp header)."""

    def __init__(self, nx, ny, L, lx, ly, ra, pr, dt, threads=None):
        if threads is None:
            threads = os.cpu_count() or 1
        self.nx, self.ny, self.L = nx, ny, L
        self.mox = nx // 2 + 1
        self.h = lib().oracle_create(nx, ny, L, lx, ly, ra, pr, dt, threads)
        if not self.h:
            raise ValueError("invalid oracle parameters")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def set_threads(self, n):
        lib().oracle_set_threads(self.h, n)

    def set_colloc(self, nq):
        """Nonlinear term of the library's collocation form on nq Gauss-Legendre levels (the
        3-index tensors become nq-point sums; not a reference method); 0: exact integrals."""
        lib().oracle_set_colloc(self.h, nq)

    def _bufs(self):
        shp = (self.L, self.ny, self.mox)
        return [np.zeros(shp, np.complex128) for _ in range(3)] + [np.zeros(self.L, np.complex128) for _ in range(2)]

    def set_state(self, th, f, g, F, G):
        arrs = [np.ascontiguousarray(a, dtype=np.complex128) for a in (th, f, g, F, G)]
        lib().oracle_set_state(self.h, *[_ptr(a) for a in arrs])

    def get_state(self):
        b = self._bufs()
        lib().oracle_get_state(self.h, *[_ptr(a) for a in b])
        return b

    def step(self, n=1):
        lib().oracle_step(self.h, n)

    def set_tracer_sets(self, diffusivities):
        """Equal consecutive tracer sets with their own diffusivities."""
        d = np.ascontiguousarray(diffusivities, dtype=np.float64)
        lib().oracle_set_tracer_sets(self.h, d.size, _ptr(d))

    def set_force_mean(self, mean_F):
        """F of the lowest mode set to mean_F before every step (0: off)."""
        lib().oracle_set_force_mean(self.h, mean_F)

    def set_penalization(self, eta, kind="rectangle"):
        """Penalized nonlinear operator (eta > 0) with the named mask; eta = 0 turns it off."""
        lib().oracle_set_penalization(self.h, eta, PEN_MASKS[kind])

    # freeze_operator / masktemp of the reference's iteration loop
    def freeze_mask(self, shape, size):
        lib().oracle_freeze_mask(self.h, MASK_SHAPES[shape], size)

    def freeze_apply(self):
        lib().oracle_freeze_apply(self.h)

    def heat_mask(self, shape, size, increment=1.5 / 100):
        lib().oracle_heat_mask(self.h, MASK_SHAPES[shape], size, increment)

    def heat_apply(self):
        lib().oracle_heat_apply(self.h)

    def masker(self, x=0.5, y=0.5, radius=0.15, factor=1.1):
        lib().oracle_masker(self.h, x, y, radius, factor)

    def nonlinear(self):
        b = self._bufs()
        lib().oracle_nonlinear(self.h, *[_ptr(a) for a in b])
        return b

    def synthesis(self):
        out = np.zeros((8, self.L, self.ny, self.nx))
        lib().oracle_synthesis(self.h, _ptr(out))
        return out

    def init_theta(self, seed, amp, kmax):
        lib().oracle_init_theta(self.h, seed, amp, kmax)

    def tracers_set(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.ntr = xyz.size // 3
        lib().oracle_tracers_set(self.h, _ptr(xyz), self.ntr)

    def tracers_get(self):
        out = np.zeros(3 * self.ntr)
        lib().oracle_tracers_get(self.h, _ptr(out))
        return out

    def tracers_advance(self):
        lib().oracle_tracers_advance(self.h)

    def init_pattern(self, kind, mode, amp=1e-6, seed=0, noise=0.0):
        """Pattern initial condition (1 isr ... 6 giantspiral, 7 test), see oracle_init_pattern."""
        lib().oracle_init_pattern(self.h, kind, mode, amp, seed, noise)

    def set_diffusion(self, D, seed):
        lib().oracle_set_diffusion(self.h, D, seed)

    def velocity_grid(self):
        shp = (128, self.ny, self.nx)
        u = [np.zeros(shp) for _ in range(3)]
        lib().oracle_velocity_grid(self.h, *[_ptr(a) for a in u])
        return u

    def diagnostics(self):
        d = np.zeros(3)
        lib().oracle_diagnostics(self.h, _ptr(d))
        return {"nu_wall": d[0], "nu_vol": d[1], "ke": d[2]}

    def nu_wall(self):
        return lib().oracle_nu_wall(self.h)

    def spectrum(self, nbins, z=0.0):
        out = np.zeros(nbins)
        lib().oracle_spectrum(self.h, z, _ptr(out), nbins)
        return out

    def operator_table(self, which):
        out = np.zeros((self.L * self.L, self.ny, self.mox))
        lib().oracle_operator_table(self.h, which, _ptr(out))
        return out
