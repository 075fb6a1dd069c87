"""sdc_b200 -- B200-native (sm_100a) Boussinesq Rayleigh-Benard step.

Python access to libsdc_b200.so through its C ABI (include/rbc.h). The library is the
only compute path: if it is missing this package raises on import of `Solver` use, it
never falls back to another implementation.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SDC_B200_LIB") or os.path.join(_HERE, "_lib", "libsdc_b200.so")
_LIB = None

RBC_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite value", 4: "timeout",
          5: "I/O error", 6: "unsupported", 7: "out of device memory"}
FORMS = {"fp64": 0, "mixed": 1, "colloc": 2}


class RBCError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class _Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("ra", ctypes.c_double),
                ("pr", ctypes.c_double), ("dt", ctypes.c_double), ("form", ctypes.c_int),
                ("n_tracers", ctypes.c_int), ("device", ctypes.c_int), ("diag_capacity", ctypes.c_int),
                ("tune", ctypes.c_int), ("tracer_diffusivity", ctypes.c_double), ("noise_seed", ctypes.c_ulonglong),
                ("track_frames", ctypes.c_int), ("track_period", ctypes.c_int), ("field_ops", ctypes.c_int),
                ("penalization_eta", ctypes.c_double), ("penalization_mask", ctypes.c_int),
                ("tracer_sets", ctypes.c_int), ("mean_F", ctypes.c_double), ("colloc_nq", ctypes.c_int)]


class _Diag(ctypes.Structure):
    _fields_ = [("nu_wall", ctypes.c_double), ("nu_vol", ctypes.c_double), ("ke", ctypes.c_double),
                ("step", ctypes.c_longlong)]


class _FnoParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nq", ctypes.c_int),
                ("width", ctypes.c_int), ("modes", ctypes.c_int), ("layers", ctypes.c_int),
                ("hidden", ctypes.c_int), ("max_batch", ctypes.c_int), ("device", ctypes.c_int),
                ("seed", ctypes.c_ulonglong), ("interval_steps", ctypes.c_int), ("physics_mean", ctypes.c_int),
                ("gemm_path", ctypes.c_int)]


class _SurrogateParams(ctypes.Structure):
    _fields_ = [("intervals", ctypes.c_int), ("judge_every", ctypes.c_int),
                ("nu_tol", ctypes.c_double), ("spec_tol", ctypes.c_double), ("spec_bins", ctypes.c_int),
                ("fallback_intervals", ctypes.c_int)]


class _SurrogateReport(ctypes.Structure):
    _fields_ = [("surrogate_intervals", ctypes.c_int), ("plain_intervals", ctypes.c_int), ("checks", ctypes.c_int),
                ("fallbacks", ctypes.c_int), ("max_nu_err", ctypes.c_double), ("max_spec_err", ctypes.c_double),
                ("last_nu_err", ctypes.c_double), ("last_spec_err", ctypes.c_double), ("ms", ctypes.c_double)]


class _State(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_void_p), ("f", ctypes.c_void_p), ("g", ctypes.c_void_p),
                ("F", ctypes.c_void_p), ("G", ctypes.c_void_p)]


_dp = ctypes.POINTER(ctypes.c_double)
EXPORTS = ["rbc_create", "rbc_destroy", "rbc_last_error", "rbc_status_string", "rbc_set_stream",
           "rbc_init_fields", "rbc_set_state", "rbc_get_state", "rbc_step", "rbc_step_async",
           "rbc_synchronize", "rbc_nonlinear", "rbc_tracers_set", "rbc_tracers_get", "rbc_tracers_seed",
           "rbc_tracers_advance", "rbc_diagnostics", "rbc_diag_history", "rbc_spectrum", "rbc_synthesis",
           "rbc_table", "rbc_galerkin_table", "rbc_stage_times", "rbc_measure_fp64_peak", "rbc_nonlinear_noalloc", "rbc_dump_read", "rbc_dump_write",
           "rbc_save_state", "rbc_load_state", "rbc_save_history", "rbc_load_history", "rbc_ensemble_create",
           "rbc_ensemble_destroy", "rbc_ensemble_member", "rbc_ensemble_step", "rbc_ensemble_last_error",
           "rbc_ensemble_elapsed", "rbc_launch_config",
           "rbc_kernel_launches", "rbc_tracers_init", "rbc_tracer_moments", "rbc_tracks_read", "rbc_track_write",
           "rbc_init_pattern", "rbc_fno_create", "rbc_gemm_bf16", "rbc_fno_destroy", "rbc_fno_last_error", "rbc_fno_num_params",
           "rbc_fno_get_params", "rbc_fno_set_params", "rbc_fno_get_norm", "rbc_fno_set_norm", "rbc_fno_forward",
           "rbc_fno_loss_grad", "rbc_fno_colloc_get", "rbc_fno_colloc_add", "rbc_fno_dataset_reserve",
           "rbc_fno_dataset_capture", "rbc_fno_train", "rbc_fno_advance", "rbc_surrogate_run",
           "rbc_fno_set_train_options", "rbc_structure_function", "rbc_freeze_mask", "rbc_freeze_apply",
           "rbc_heat_mask", "rbc_heat_apply", "rbc_field_ops_reset", "rbc_masker",
           "rbc_diagnostics_async", "rbc_diagnostics_get",
           "rbc_tracer_set_diffusivity", "rbc_tracers_init_set", "rbc_tracer_moments_set"]
FIELD_OPS = {"freeze": 1, "heat": 2, "scale": 4}
MASK_SHAPES = {"circle": 0, "rectangle": 1}
PEN_MASKS = {"rectangle": 0, "circle": 1, "disk_array": 2, "everywhere": 3}
INIT_PATTERNS = {"isr": 1, "dislocation": 2, "rectangle": 3, "sv": 4, "cr": 5, "giantspiral": 6, "test": 7}
GEMM_PATHS = {"tcgen05": 0, "mma_sync": 1}
TRACER_PATTERNS = {"random": 0, "center": 1, "center_sigma": 2, "diagonal": 3, "pairs": 4, "coord_sigma": 5}


def lib():
    """Loads libsdc_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not built: run python -c 'import __graft_entry__ as g; g.build()'")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.rbc_create.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(vp)]
    L.rbc_destroy.argtypes = [vp]
    L.rbc_destroy.restype = None
    L.rbc_last_error.argtypes = [vp]
    L.rbc_last_error.restype = ctypes.c_char_p
    L.rbc_status_string.argtypes = [ctypes.c_int]
    L.rbc_status_string.restype = ctypes.c_char_p
    L.rbc_set_stream.argtypes = [vp, vp]
    L.rbc_init_fields.argtypes = [vp, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double]
    L.rbc_set_state.argtypes = [vp] + [_dp] * 5
    L.rbc_get_state.argtypes = [vp] + [_dp] * 5
    L.rbc_step.argtypes = [vp, ctypes.c_int]
    L.rbc_step_async.argtypes = [vp, ctypes.c_int]
    L.rbc_synchronize.argtypes = [vp]
    L.rbc_nonlinear.argtypes = [vp, ctypes.POINTER(_State), ctypes.POINTER(_State)]
    L.rbc_tracers_set.argtypes = [vp, _dp, ctypes.c_int]
    L.rbc_tracers_get.argtypes = [vp, _dp, ctypes.c_int]
    L.rbc_tracers_seed.argtypes = [vp, ctypes.c_ulonglong]
    L.rbc_tracers_advance.argtypes = [vp]
    L.rbc_init_pattern.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong,
                                   ctypes.c_double]
    L.rbc_tracers_init.argtypes = [vp, ctypes.c_int, ctypes.c_ulonglong] + [ctypes.c_double] * 4
    L.rbc_tracer_moments.argtypes = [vp, _dp]
    fp = ctypes.POINTER(ctypes.c_float)
    up = ctypes.POINTER(ctypes.c_uint)
    L.rbc_tracks_read.argtypes = [vp, fp, up, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.rbc_track_write.argtypes = [ctypes.c_char_p, ctypes.c_char_p, fp, up, ctypes.c_int, ctypes.c_int]
    L.rbc_diagnostics.argtypes = [vp, ctypes.POINTER(_Diag)]
    L.rbc_diag_history.argtypes = [vp, ctypes.POINTER(_Diag), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.rbc_spectrum.argtypes = [vp, ctypes.c_double, _dp, ctypes.c_int]
    L.rbc_synthesis.argtypes = [vp, _dp]
    L.rbc_table.argtypes = [vp, ctypes.c_char_p, _dp, ctypes.POINTER(ctypes.c_int)]
    L.rbc_galerkin_table.argtypes = [ctypes.c_int, ctypes.c_char_p, _dp, ctypes.POINTER(ctypes.c_int)]
    L.rbc_stage_times.argtypes = [vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]
    L.rbc_measure_fp64_peak.argtypes = [ctypes.c_int, _dp]
    L.rbc_nonlinear_noalloc.argtypes = ([ctypes.c_int] * 4 + [ctypes.c_double] * 3 + [ctypes.c_void_p] * 10 +
                                        [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int])
    cp = ctypes.c_char_p
    ip = ctypes.POINTER(ctypes.c_int)
    L.rbc_dump_read.argtypes = [cp, ctypes.c_int, ip, ctypes.c_int, ip, _dp, ctypes.c_longlong]
    L.rbc_dump_write.argtypes = [cp, ip, ctypes.c_int, _dp, ctypes.c_int]
    L.rbc_save_state.argtypes = [vp, cp, ctypes.c_longlong, ctypes.c_int]
    L.rbc_load_state.argtypes = [vp, cp, cp, cp, cp, cp]
    L.rbc_save_history.argtypes = [vp, cp]
    L.rbc_load_history.argtypes = [vp, cp]
    L.rbc_ensemble_create.argtypes = [ctypes.POINTER(_Params), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.rbc_ensemble_destroy.argtypes = [vp]
    L.rbc_ensemble_destroy.restype = None
    L.rbc_ensemble_member.argtypes = [vp, ctypes.c_int]
    L.rbc_ensemble_member.restype = vp
    L.rbc_ensemble_step.argtypes = [vp, ctypes.c_int]
    L.rbc_ensemble_elapsed.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.rbc_ensemble_last_error.argtypes = [vp]
    L.rbc_ensemble_last_error.restype = ctypes.c_char_p
    L.rbc_launch_config.argtypes = [vp, ip, ip]
    L.rbc_kernel_launches.argtypes = [vp]
    L.rbc_kernel_launches.restype = ctypes.c_longlong
    L.rbc_structure_function.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, _dp]
    L.rbc_freeze_mask.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.rbc_freeze_apply.argtypes = [vp]
    L.rbc_heat_mask.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.rbc_heat_apply.argtypes = [vp]
    L.rbc_field_ops_reset.argtypes = [vp]
    L.rbc_masker.argtypes = [vp] + [ctypes.c_double] * 4
    L.rbc_diagnostics_async.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.rbc_tracer_set_diffusivity.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.rbc_tracers_init_set.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong] + [ctypes.c_double] * 4
    L.rbc_tracer_moments_set.argtypes = [vp, ctypes.c_int, _dp]
    L.rbc_diagnostics_get.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(_Diag)]
    L.rbc_fno_create.argtypes = [ctypes.POINTER(_FnoParams), ctypes.POINTER(vp)]
    L.rbc_gemm_bf16.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    L.rbc_fno_destroy.argtypes = [vp]
    L.rbc_fno_destroy.restype = None
    L.rbc_fno_last_error.argtypes = [vp]
    L.rbc_fno_last_error.restype = ctypes.c_char_p
    L.rbc_fno_num_params.argtypes = [vp]
    L.rbc_fno_num_params.restype = ctypes.c_longlong
    L.rbc_fno_get_params.argtypes = [vp, fp, ctypes.c_longlong]
    L.rbc_fno_set_params.argtypes = [vp, fp, ctypes.c_longlong]
    L.rbc_fno_get_norm.argtypes = [vp, fp]
    L.rbc_fno_set_norm.argtypes = [vp, fp]
    L.rbc_fno_forward.argtypes = [vp, fp, ctypes.c_int, fp]
    L.rbc_fno_loss_grad.argtypes = [vp, fp, fp, ctypes.c_int, _dp, fp]
    L.rbc_fno_colloc_get.argtypes = [vp, vp, fp]
    L.rbc_fno_colloc_add.argtypes = [vp, vp, fp]
    L.rbc_fno_dataset_reserve.argtypes = [vp, ctypes.c_int]
    L.rbc_fno_dataset_capture.argtypes = [vp, vp, ctypes.c_int]
    L.rbc_fno_train.argtypes = [vp, ip, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                ctypes.c_ulonglong, ctypes.c_int, _dp]
    L.rbc_fno_advance.argtypes = [vp, vp, ctypes.c_int]
    L.rbc_fno_set_train_options.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.rbc_surrogate_run.argtypes = [vp, vp, ctypes.POINTER(_SurrogateParams), ctypes.POINTER(_SurrogateReport), _dp]
    _LIB = L
    return L


def galerkin_table(nz, name):
    """Galerkin table of the library (host computation; no GPU needed)."""
    out = np.zeros(max(nz ** 3, 1))
    cnt = ctypes.c_int(0)
    st = lib().rbc_galerkin_table(nz, name.encode(), out.ctypes.data_as(_dp), ctypes.byref(cnt))
    if st != RBC_OK:
        raise RBCError(st, f"rbc_galerkin_table({nz}, {name})")
    return out[:cnt.value]


def fp64_peak_tflops(device=0):
    """Measured FP64 FMA throughput of the device (TFLOP/s)."""
    v = ctypes.c_double(0)
    st = lib().rbc_measure_fp64_peak(device, ctypes.byref(v))
    if st != RBC_OK:
        raise RBCError(st, "rbc_measure_fp64_peak")
    return v.value


def dump_read(path, index=0):
    """One matrix of a reference dump file as a complex array shaped [dims reversed]."""
    dims = (ctypes.c_int * 8)()
    nd = ctypes.c_int(0)
    st = lib().rbc_dump_read(os.fsencode(path), index, dims, 8, ctypes.byref(nd), None, 0)
    if st != RBC_OK:
        raise RBCError(st, f"rbc_dump_read({path})")
    d = [dims[i] for i in range(nd.value)]
    n = int(np.prod(d))
    out = np.zeros(2 * n)
    st = lib().rbc_dump_read(os.fsencode(path), index, dims, 8, ctypes.byref(nd), out.ctypes.data_as(_dp), n)
    if st != RBC_OK:
        raise RBCError(st, f"rbc_dump_read({path})")
    return out.view(np.complex128).reshape(d[::-1])


def dump_write(path, arr, real_bytes=8):
    """Writes a complex array (shape [dims reversed]) as a one-matrix dump file."""
    a = np.ascontiguousarray(arr, dtype=np.complex128)
    d = (ctypes.c_int * a.ndim)(*a.shape[::-1])
    st = lib().rbc_dump_write(os.fsencode(path), d, a.ndim, a.view(np.float64).ctypes.data_as(_dp), real_bytes)
    if st != RBC_OK:
        raise RBCError(st, f"rbc_dump_write({path})")


def make_params(nx, ny, nz, lx, ly, ra, pr, dt, form="fp64", n_tracers=0, device=0, diag_capacity=0, tune=False,
                tracer_diffusivity=0.0, noise_seed=0, track_frames=0, track_period=1, field_ops=(),
                penalization=None, mean_F=0.0, tracer_sets=1, colloc_nq=0):
    """penalization: None, or (eta, mask) with mask one of PEN_MASKS."""
    ops = 0
    for name in field_ops:
        ops |= FIELD_OPS[name]
    eta, kind = penalization if penalization else (0.0, "rectangle")
    return _Params(nx, ny, nz, lx, ly, ra, pr, dt, FORMS[form], n_tracers, device, diag_capacity, int(bool(tune)),
                   tracer_diffusivity, noise_seed, track_frames, track_period, ops, eta, PEN_MASKS[kind], tracer_sets, mean_F,
                   colloc_nq)


def track_write(path, frames, times, description=""):
    """Writes FP32 frames [nframes][3][n] with their step numbers as a TRKSS track file."""
    fr = np.ascontiguousarray(frames, dtype=np.float32)
    tm = np.ascontiguousarray(times, dtype=np.uint32)
    nf = fr.shape[0]
    n = fr.shape[2] if nf else 0
    st = lib().rbc_track_write(os.fsencode(path), description.encode(),
                               fr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                               tm.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), nf, n)
    if st != RBC_OK:
        raise RBCError(st, f"rbc_track_write({path})")


class Ensemble:
    """n independent runs advanced together, one CUDA graph per step (rbc_ensemble_*)."""

    def __init__(self, configs, nstreams=16, device=0, tune=False):
        arr = (_Params * len(configs))(*[make_params(*c[:8], form=c[8] if len(c) > 8 else "fp64", device=device,
                                                     tune=tune) for c in configs])
        e = ctypes.c_void_p()
        st = lib().rbc_ensemble_create(arr, len(configs), nstreams, ctypes.byref(e))
        if st != RBC_OK:
            raise RBCError(st, "rbc_ensemble_create failed")
        self.e = e
        self.members = [Solver(*c[:8], _handle=ctypes.c_void_p(lib().rbc_ensemble_member(e, i)))
                        for i, c in enumerate(configs)]

    def step(self, n=1):
        st = lib().rbc_ensemble_step(self.e, n)
        if st != RBC_OK:
            raise RBCError(st, "rbc_ensemble_step: " + lib().rbc_ensemble_last_error(self.e).decode())

    def timed_step(self, n):
        """step(n) and the device time in ms of its graph-replayed steps (CUDA events on the
        ensemble's root stream)."""
        self.step(n)
        ms = ctypes.c_float()
        st = lib().rbc_ensemble_elapsed(self.e, ctypes.byref(ms))
        if st != RBC_OK:
            raise RBCError(st, "rbc_ensemble_elapsed")
        return ms.value

    def close(self):
        if getattr(self, "e", None):
            for m in self.members:
                m.h = None
            lib().rbc_ensemble_destroy(self.e)
            self.e = None

    __del__ = close


def _p(a):
    assert a.flags["C_CONTIGUOUS"] and a.dtype in (np.float64, np.complex128)
    return a.ctypes.data_as(_dp)


class Solver:
    """One RBC run on one GPU (mirrors the reference's operator set, see include/rbc.h)."""

    def __init__(self, nx, ny, nz, lx, ly, ra, pr, dt, form="fp64", n_tracers=0, device=0, diag_capacity=0,
                 tune=False, tracer_diffusivity=0.0, noise_seed=0, track_frames=0, track_period=1, field_ops=(),
                 penalization=None, mean_F=0.0, tracer_sets=1, colloc_nq=0, _handle=None):
        self.nx, self.ny, self.L = nx, ny, nz
        self.mox = nx // 2 + 1
        self.n_tracers = n_tracers
        self.track_frames = track_frames
        self.params = dict(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, ra=ra, pr=pr, dt=dt, form=form)
        self._owned = _handle is None
        if _handle is not None:
            self.h = _handle
            return
        p = make_params(nx, ny, nz, lx, ly, ra, pr, dt, form, n_tracers, device, diag_capacity, tune,
                        tracer_diffusivity, noise_seed, track_frames, track_period, field_ops, penalization, mean_F, tracer_sets,
                        colloc_nq)
        h = ctypes.c_void_p()
        st = lib().rbc_create(ctypes.byref(p), ctypes.byref(h))
        if st != RBC_OK:
            raise RBCError(st, "rbc_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and getattr(self, "_owned", True):
            try:
                lib().rbc_destroy(self.h)
            except TypeError:  # interpreter shutdown: module globals are gone
                pass
        self.h = None

    @property
    def launch_config(self):
        W, NP = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().rbc_launch_config(self.h, ctypes.byref(W), ctypes.byref(NP)))
        return W.value, NP.value

    __del__ = close

    def _check(self, st):
        if st != RBC_OK:
            raise RBCError(st, lib().rbc_last_error(self.h).decode())

    def _bufs(self):
        shp = (self.L, self.ny, self.mox)
        return [np.zeros(shp, np.complex128) for _ in range(3)] + [np.zeros(self.L, np.complex128) for _ in range(2)]

    # fields
    def init_fields(self, seed, amplitude=1e-3, kmax=4.0):
        self._check(lib().rbc_init_fields(self.h, seed, amplitude, kmax))

    def init_pattern(self, pattern, mode=None, amplitude=1e-6, seed=0, noise=0.0):
        """Pattern initial condition of the reference (-init_isr, -init_sv, ...); mode defaults
        to Lx/2 as main.cu's -init_mode does."""
        if mode is None:
            mode = self.params["lx"] / 2.0
        self._check(lib().rbc_init_pattern(self.h, INIT_PATTERNS[pattern], mode, amplitude, seed, noise))

    def set_state(self, theta, f, g, F, G):
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (theta, f, g, F, G)]
        self._check(lib().rbc_set_state(self.h, *[_p(x) for x in a]))

    def get_state(self, out=None):
        """The state in the reference layout; `out` (five C-contiguous complex128 arrays of
        the state's shapes, e.g. views of pinned host memory) is filled and returned."""
        b = self._bufs() if out is None else out
        self._check(lib().rbc_get_state(self.h, *[_p(x) for x in b]))
        return b

    # files (reference dump format)
    def save_state(self, directory, step, real_bytes=8):
        self._check(lib().rbc_save_state(self.h, os.fsencode(directory), step, real_bytes))

    def load_state(self, theta, f, g, F, G):
        self._check(lib().rbc_load_state(self.h, *[os.fsencode(p) for p in (theta, f, g, F, G)]))

    def save_history(self, path):
        self._check(lib().rbc_save_history(self.h, os.fsencode(path)))

    def load_history(self, path):
        self._check(lib().rbc_load_history(self.h, os.fsencode(path)))

    # step
    def step(self, n=1):
        self._check(lib().rbc_step(self.h, n))

    def step_async(self, n=1):
        self._check(lib().rbc_step_async(self.h, n))

    def synchronize(self):
        self._check(lib().rbc_synchronize(self.h))

    def set_stream(self, stream_ptr):
        self._check(lib().rbc_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    @property
    def kernel_launches(self):
        return lib().rbc_kernel_launches(self.h)

    STAGES = ("synth_columns", "rows_c2r", "tracers", "contract", "rows_r2c", "columns_combine", "update")

    def stage_times(self, nsteps):
        """Runs nsteps steps with CUDA events around each kernel; mean ms per launch."""
        ms = np.zeros(7)
        cnt = (ctypes.c_int * 7)()
        self._check(lib().rbc_stage_times(self.h, nsteps, _p(ms), cnt))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.STAGES)}

    # operator
    def nonlinear(self, theta, f, g, F, G):
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (theta, f, g, F, G)]
        out = self._bufs()
        si = _State(*[x.ctypes.data for x in a])
        so = _State(*[x.ctypes.data for x in out])
        self._check(lib().rbc_nonlinear(self.h, ctypes.byref(si), ctypes.byref(so)))
        return out

    def synthesis(self):
        out = np.zeros((8, self.L, self.ny, self.nx))
        self._check(lib().rbc_synthesis(self.h, _p(out)))
        return out

    # tracers
    def tracers_set(self, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self._check(lib().rbc_tracers_set(self.h, _p(xyz), xyz.size // 3))

    def tracers_get(self, out=None):
        out = np.zeros(3 * self.n_tracers) if out is None else out
        self._check(lib().rbc_tracers_get(self.h, _p(out), self.n_tracers))
        return out

    def tracers_seed(self, seed):
        self._check(lib().rbc_tracers_seed(self.h, seed))

    def tracers_advance(self):
        self._check(lib().rbc_tracers_advance(self.h))

    def tracers_init(self, pattern, seed=0, coord=(0.0, 0.0, 0.0), sigma=0.0):
        """Start positions by pattern (random, center, center_sigma, diagonal, pairs, coord_sigma)."""
        self._check(lib().rbc_tracers_init(self.h, TRACER_PATTERNS[pattern], seed, *coord, sigma))

    def tracer_set_diffusivity(self, set_index, D):
        self._check(lib().rbc_tracer_set_diffusivity(self.h, set_index, D))

    def tracers_init_set(self, set_index, pattern, seed=0, coord=(0.0, 0.0, 0.0), sigma=0.0):
        self._check(lib().rbc_tracers_init_set(self.h, set_index, TRACER_PATTERNS[pattern], seed, *coord, sigma))

    def tracer_moments_set(self, set_index):
        out = np.zeros(4)
        self._check(lib().rbc_tracer_moments_set(self.h, set_index, _p(out)))
        return out

    def tracer_moments(self):
        """(<x>, <y>, second moment, pair second moment) of the current positions."""
        out = np.zeros(4)
        self._check(lib().rbc_tracer_moments(self.h, _p(out)))
        return out

    def tracks_read(self, max_frames=1 << 30):
        """Unread recorded frames as (FP32 [nframes][3][n], step numbers)."""
        k = ctypes.c_int(0)
        ring = max(1, self.track_frames)
        cap = min(max_frames, ring)
        frames, times = [], []
        while True:
            fr = np.zeros((cap, 3, self.n_tracers), np.float32)
            tm = np.zeros(cap, np.uint32)
            self._check(lib().rbc_tracks_read(self.h, fr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              tm.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), cap, ctypes.byref(k)))
            frames.append(fr[:k.value])
            times.append(tm[:k.value])
            max_frames -= k.value
            if k.value < cap or max_frames <= 0:
                break
            cap = min(max_frames, ring)
        return np.concatenate(frames), np.concatenate(times)

    # diagnostics
    def diagnostics(self):
        d = _Diag()
        self._check(lib().rbc_diagnostics(self.h, ctypes.byref(d)))
        return {"nu_wall": d.nu_wall, "nu_vol": d.nu_vol, "ke": d.ke, "step": d.step}

    def diagnostics_async(self):
        """Enqueues a read of the newest diagnostics entry; returns its ticket."""
        t = ctypes.c_longlong(0)
        self._check(lib().rbc_diagnostics_async(self.h, ctypes.byref(t)))
        return t.value

    def diagnostics_get(self, ticket):
        """Waits for the read of `ticket` only and returns its entry."""
        d = _Diag()
        self._check(lib().rbc_diagnostics_get(self.h, ticket, ctypes.byref(d)))
        return {"nu_wall": d.nu_wall, "nu_vol": d.nu_vol, "ke": d.ke, "step": d.step}

    def diag_history(self, n):
        arr = (_Diag * max(1, n))()
        cnt = ctypes.c_int(0)
        self._check(lib().rbc_diag_history(self.h, arr, n, ctypes.byref(cnt)))
        return np.array([(d.nu_wall, d.nu_vol, d.ke, d.step) for d in arr[:cnt.value]]).reshape(-1, 4)

    def structure_function(self, field, direction, r_min, r_max, nsamples):
        """Second-order structure function of the mid-plane field ("theta", "u1", "u2")
        along "x" or "y" (rbc_structure_function)."""
        out = np.zeros(nsamples)
        fi = {"theta": 0, "u1": 1, "u2": 2}[field]
        di = {"x": 0, "y": 1}[direction]
        self._check(lib().rbc_structure_function(self.h, fi, di, r_min, r_max, nsamples, out.ctypes.data_as(_dp)))
        return out

    # field operators of the iteration loop (freeze, heating); field_ops at construction
    # names the buffers ("freeze", "heat")
    def freeze_mask(self, shape="circle", size=0.8):
        """Mask and frozen planes of the current state (freeze_circle / freeze_rectangle)."""
        self._check(lib().rbc_freeze_mask(self.h, MASK_SHAPES[shape], size))

    def freeze_apply(self):
        self._check(lib().rbc_freeze_apply(self.h))

    def heat_mask(self, shape="rectangle", size=0.1, increment=1.5 / 100):
        """Heating mask and increment (temp_rectangle / temp_circle)."""
        self._check(lib().rbc_heat_mask(self.h, MASK_SHAPES[shape], size, increment))

    def heat_apply(self):
        self._check(lib().rbc_heat_apply(self.h))

    def masker(self, x=0.5, y=0.5, radius=0.15, factor=1.1):
        """Scales theta by factor inside a circle (masking::masker; field_ops "scale")."""
        self._check(lib().rbc_masker(self.h, x, y, radius, factor))

    def field_ops_reset(self):
        self._check(lib().rbc_field_ops_reset(self.h))

    def spectrum(self, nbins, z=0.0):
        out = np.zeros(nbins)
        self._check(lib().rbc_spectrum(self.h, z, _p(out), nbins))
        return out

    def table(self, name):
        L = self.L
        out = np.zeros(L ** 3)
        cnt = ctypes.c_int(0)
        self._check(lib().rbc_table(self.h, name.encode(), _p(out), ctypes.byref(cnt)))
        return out[:cnt.value]


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class FNO:
    """Fourier neural operator surrogate of a solver grid (rbc_fno_*, include/rbc.h).

    Channels are theta, u, v, w at nq collocation levels (C = 4 nq); arrays are float32
    [batch][ny][nx][C]."""

    def __init__(self, nx, ny, nz, nq, width=32, modes=16, layers=4, hidden=128, max_batch=8, device=0, seed=0,
                 interval_steps=40, physics_mean=True, gemm_path="tcgen05"):
        self.nx, self.ny, self.nz, self.nq = nx, ny, nz, nq
        self.C = 4 * nq
        self.interval_steps = interval_steps
        p = _FnoParams(nx, ny, nz, nq, width, modes, layers, hidden, max_batch, device, seed, interval_steps,
                       int(physics_mean), GEMM_PATHS[gemm_path])
        m = ctypes.c_void_p()
        st = lib().rbc_fno_create(ctypes.byref(p), ctypes.byref(m))
        if st != RBC_OK:
            raise RBCError(st, "rbc_fno_create failed")
        self.m = m

    def close(self):
        if getattr(self, "m", None):
            try:
                lib().rbc_fno_destroy(self.m)
            except TypeError:  # interpreter shutdown: module globals are gone
                pass
        self.m = None

    __del__ = close

    def _check(self, st):
        if st != RBC_OK:
            raise RBCError(st, lib().rbc_fno_last_error(self.m).decode())

    @property
    def num_params(self):
        return lib().rbc_fno_num_params(self.m)

    def get_params(self):
        out = np.empty(self.num_params, np.float32)
        self._check(lib().rbc_fno_get_params(self.m, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), out.size))
        return out

    def set_params(self, v):
        v, ptr = _f32(v)
        self._check(lib().rbc_fno_set_params(self.m, ptr, v.size))

    def get_norm(self):
        out = np.empty((4, self.C), np.float32)
        self._check(lib().rbc_fno_get_norm(self.m, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_norm(self, v):
        v, ptr = _f32(v)
        self._check(lib().rbc_fno_set_norm(self.m, ptr))

    def forward(self, x):
        x, px = _f32(x)
        y = np.empty_like(x)
        self._check(lib().rbc_fno_forward(self.m, px, x.shape[0], y.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return y

    def loss_grad(self, x, target):
        x, px = _f32(x)
        t, pt = _f32(target)
        loss = ctypes.c_double(0)
        g = np.empty(self.num_params, np.float32)
        self._check(lib().rbc_fno_loss_grad(self.m, px, pt, x.shape[0], ctypes.byref(loss),
                                            g.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return loss.value, g

    def colloc_get(self, solver):
        out = np.empty((self.ny, self.nx, self.C), np.float32)
        self._check(lib().rbc_fno_colloc_get(self.m, solver.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def colloc_add(self, solver, delta):
        d, pd = _f32(delta)
        self._check(lib().rbc_fno_colloc_add(self.m, solver.h, pd))

    def reserve(self, nslots):
        self._check(lib().rbc_fno_dataset_reserve(self.m, nslots))

    def capture(self, solver, slot):
        self._check(lib().rbc_fno_dataset_capture(self.m, solver.h, slot))

    def train(self, src, dst, epochs, batch, lr=1e-3, seed=0, fit_norm=True):
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        loss = np.zeros(max(epochs, 1), np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(lib().rbc_fno_train(self.m, src.ctypes.data_as(ip), dst.ctypes.data_as(ip), len(src), epochs,
                                        batch, lr, seed, int(fit_norm), loss.ctypes.data_as(_dp)))
        return loss[:epochs]

    def set_train_options(self, augment=0, noise_rel=0.0, pushforward=False):
        """augment: 0 none, 1 reflections, 2 reflections + transpose (square boxes);
        pushforward: every other iteration trains on the network's own predictions."""
        self._check(lib().rbc_fno_set_train_options(self.m, augment, noise_rel, int(pushforward)))

    def advance(self, solver, n=1):
        self._check(lib().rbc_fno_advance(self.m, solver.h, n))

    def run(self, solver, intervals, judge_every=10, nu_tol=1e-3, spec_tol=0.0, spec_bins=0, fallback_intervals=-1,
            trace=False):
        """Judged rollout (rbc_surrogate_run); with trace=True the report's "nu_trace" is
        Nu_wall after every interval."""
        p = _SurrogateParams(intervals, judge_every, nu_tol, spec_tol, spec_bins, fallback_intervals)
        r = _SurrogateReport()
        tr = np.zeros(max(intervals, 1)) if trace else None
        self._check(lib().rbc_surrogate_run(self.m, solver.h, ctypes.byref(p), ctypes.byref(r),
                                            tr.ctypes.data_as(_dp) if trace else None))
        out = {k: getattr(r, k) for k, _ in _SurrogateReport._fields_}
        if trace:
            out["nu_trace"] = tr[:intervals]
        return out
