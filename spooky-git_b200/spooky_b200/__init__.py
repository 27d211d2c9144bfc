"""Python binding of libspooky_b200.so (the C ABI in include/spooky_b200.h).

The objects mirror the reference's host interface for the hot path
(LorenzoLMP/spooky-git): ``Supervisor`` owns ``Parameters``, ``Fields``,
``TimeStepping`` and ``RKLegendre``; ``TimeStepping.compute_dt``,
``compute_dfield``, ``HydroMHDAdvance`` and ``RKLegendre.compute_cycle``
keep the reference's names and meaning.  Device memory is owned by the
context; torch tensors (CUDA) or numpy arrays (host) may be passed where a
state array is expected.

The library is required: importing works without it, but creating a context
raises ``RuntimeError`` if ``lib/libspooky_b200.so`` is missing -- there is no
CPU fallback.
"""
import ctypes
import os

import numpy as np

from .params import (SPK_FORM_FP32, SPK_FORM_PLAIN, SPK_INT_EULER, SPK_INT_RK3, SPK_STS_RKL1, SPK_STS_RKL2, SPK_STS_STS, Params,
                     check_parameters, default_params, num_fields, var_list)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libspooky_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "spooky_b200.h")

SPK_OK = 0
ERRORS = {1: "SPK_ERR_ARG", 2: "SPK_ERR_UNSUPPORTED", 3: "SPK_ERR_CUDA", 4: "SPK_ERR_ALLOC",
          5: "SPK_ERR_NONFINITE", 6: "SPK_ERR_CONFIG"}

EXPORTED = ["spk_params_default", "spk_ctx_create", "spk_ctx_destroy", "spk_sizes", "spk_set_state",
            "spk_get_state", "spk_set_time", "spk_get_time", "spk_clean_divergence", "spk_compute_dt",
            "spk_compute_dfield", "spk_advance", "spk_rkl_cycle", "spk_to_real", "spk_synchronize",
            "spk_budgets", "spk_step_info", "spk_profile_passes", "spk_last_error",
            "spk_compute_dfield_noalloc", "spk_params_from_file", "spk_params_from_string",
            "spk_ensemble_create", "spk_ensemble_destroy", "spk_ensemble_size", "spk_ensemble_set_state",
            "spk_ensemble_get_state", "spk_ensemble_get_time", "spk_ensemble_budgets", "spk_ensemble_advance",
            "spk_ensemble_synchronize", "spk_ensemble_kernels_per_step",
            "spk_closure_set", "spk_products", "spk_closure_samples_size", "spk_closure_samples",
            "spk_trainer_create", "spk_trainer_destroy", "spk_trainer_set_params", "spk_trainer_get_params",
            "spk_trainer_set_samples", "spk_trainer_loss_grad", "spk_trainer_train", "spk_spectrum",
            "spk_autotune", "spk_ensemble_autotune", "spk_advance_fields", "spk_compute_dt_fields",
            "spk_rk3_fields", "spk_rkl_cycle_fields", "spk_get_state_real", "spk_set_state_real",
            "spk_write_snapshot", "spk_read_snapshot", "spk_h5_write", "spk_h5_read", "spk_diagnostics",
            "spk_cfg_lookup_int", "spk_cfg_lookup_bool", "spk_cfg_lookup_float", "spk_cfg_lookup_string",
            "spk_cfg_setting_length", "spk_transfer_spectra", "spk_trainer_create_variant",
            "spk_closure_nparam", "spk_closure_rows", "spk_get_schedule", "spk_set_schedule"]

DIAGNOSTICS = ("w2", "hv", "j2", "hm", "hc", "thetaB", "bz2", "phiB", "dissgradT", "pv")


class Diagnostics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in DIAGNOSTICS]

# learned closure (include/spooky_b200.h, SPK_CLOSURE_*)
CLOSURE_NPARAM = 32 * 8 + 32 + 32 * 32 + 32 + 2 * 32 + 2
CLOSURE_ROWS = 33
# variant 3, the tensor network (SPK_CLOSURE3_*)
CLOSURE3_NPARAM = 64 * 18 + 64 + 2 * (64 * 64 + 64) + 12 * 64 + 12
CLOSURE3_ROWS = 51


def closure_nparam(variant):
    """Parameters of a closure variant's network."""
    return CLOSURE3_NPARAM if variant == 3 else CLOSURE_NPARAM


def closure_rows(variant):
    """Sample rows of a closure variant."""
    return CLOSURE3_ROWS if variant == 3 else CLOSURE_ROWS


class Budgets(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double * 8), ("dissipation", ctypes.c_double * 8)]


class PassStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 24), ("ms", ctypes.c_double), ("bytes", ctypes.c_double),
                ("launches_per_step", ctypes.c_int)]


class SpookyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def lib():
    """Load the CUDA library (raises if it is not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libspooky_b200.so not built at {LIB_PATH} (run `make -C spooky-git_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip, sp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_size_t
        L.spk_params_default.argtypes = [ctypes.POINTER(Params)]
        L.spk_params_default.restype = None
        L.spk_ctx_create.argtypes = [ctypes.POINTER(Params), vp, ctypes.POINTER(vp)]
        L.spk_ctx_destroy.argtypes = [vp]
        L.spk_sizes.argtypes = [vp, ip, ctypes.POINTER(sp)]
        L.spk_set_state.argtypes = [vp, vp, ctypes.c_int]
        L.spk_get_state.argtypes = [vp, vp, ctypes.c_int]
        L.spk_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.spk_get_time.argtypes = [vp, dp, dp, ip]
        L.spk_clean_divergence.argtypes = [vp]
        L.spk_compute_dt.argtypes = [vp, dp, dp, dp, dp]
        L.spk_compute_dfield.argtypes = [vp, vp, vp]
        L.spk_advance.argtypes = [vp, ctypes.c_int]
        L.spk_rkl_cycle.argtypes = [vp, ip]
        L.spk_to_real.argtypes = [vp, vp]
        L.spk_synchronize.argtypes = [vp]
        L.spk_budgets.argtypes = [vp, ctypes.POINTER(Budgets)]
        L.spk_step_info.argtypes = [vp, ip, dp]
        L.spk_profile_passes.argtypes = [vp, ctypes.c_int, ctypes.POINTER(PassStat), ctypes.c_int, ip]
        L.spk_last_error.argtypes = [vp]
        L.spk_compute_dfield_noalloc.argtypes = [ctypes.POINTER(Params), vp, vp, vp]
        L.spk_params_from_file.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params)]
        L.spk_params_from_string.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params)]
        L.spk_ensemble_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, vp, ctypes.POINTER(vp)]
        L.spk_ensemble_destroy.argtypes = [vp]
        L.spk_ensemble_size.argtypes = [vp, ip, ip]
        L.spk_ensemble_set_state.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int]
        L.spk_ensemble_get_state.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int]
        L.spk_ensemble_get_time.argtypes = [vp, ctypes.c_int, dp, dp, ip]
        L.spk_ensemble_budgets.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Budgets)]
        L.spk_ensemble_advance.argtypes = [vp, ctypes.c_int]
        L.spk_ensemble_synchronize.argtypes = [vp]
        L.spk_ensemble_kernels_per_step.argtypes = [vp, ip]
        fp = ctypes.POINTER(ctypes.c_float)
        L.spk_closure_set.argtypes = [vp, fp]
        L.spk_products.argtypes = [vp, vp, vp, ip]
        L.spk_closure_samples_size.argtypes = [vp, vp, ctypes.POINTER(sp), ctypes.POINTER(sp)]
        L.spk_closure_samples.argtypes = [vp, vp, vp, vp, sp, vp, sp]
        L.spk_trainer_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.spk_trainer_create_variant.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
        L.spk_closure_nparam.argtypes = [ctypes.c_int]
        L.spk_closure_rows.argtypes = [ctypes.c_int]
        L.spk_trainer_destroy.argtypes = [vp]
        L.spk_trainer_set_params.argtypes = [vp, fp]
        L.spk_trainer_get_params.argtypes = [vp, fp]
        L.spk_trainer_set_samples.argtypes = [vp, vp, sp, sp, fp]
        L.spk_trainer_loss_grad.argtypes = [vp, fp, fp]
        L.spk_trainer_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, fp]
        L.spk_spectrum.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ip, dp, dp]
        L.spk_advance_fields.argtypes = [vp, vp, ctypes.c_int]
        L.spk_compute_dt_fields.argtypes = [vp, vp, dp, dp, dp, dp]
        L.spk_rk3_fields.argtypes = [vp, vp]
        L.spk_rkl_cycle_fields.argtypes = [vp, vp, ip]
        L.spk_get_state_real.argtypes = [vp, vp, ctypes.c_int]
        L.spk_set_state_real.argtypes = [vp, vp, ctypes.c_int]
        L.spk_write_snapshot.argtypes = [vp, ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.spk_read_snapshot.argtypes = [vp, ctypes.c_char_p, dp, dp]
        L.spk_diagnostics.argtypes = [vp, ctypes.POINTER(Diagnostics)]
        L.spk_cfg_lookup_int.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip]
        L.spk_cfg_lookup_bool.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip]
        L.spk_cfg_lookup_float.argtypes = [ctypes.c_char_p, ctypes.c_char_p, dp]
        L.spk_cfg_lookup_string.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, sp]
        L.spk_cfg_setting_length.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.spk_transfer_spectra.argtypes = [vp, ctypes.c_char_p, dp, ctypes.c_int, ip, ip, dp, dp]
        L.spk_autotune.argtypes = [vp, ctypes.c_int, ip, ip, ip, dp, dp]
        L.spk_get_schedule.argtypes = [vp, ip, ip, ip, ip]
        L.spk_set_schedule.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.spk_ensemble_autotune.argtypes = [vp, ctypes.c_int]
        L.spk_last_error.restype = ctypes.c_char_p
        for name in EXPORTED:
            if name not in ("spk_params_default", "spk_last_error"):
                getattr(L, name).restype = ctypes.c_int
        _LIB = L
    return _LIB


def c_defaults():
    """spk_params_default from the library."""
    p = Params()
    lib().spk_params_default(ctypes.byref(p))
    return p


def _torch_sync():
    """Finish torch's queued work (tensors passed in may still be in flight)."""
    import sys
    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def _ptr(a):
    """(address, where) for a torch CUDA tensor (0) or numpy array (1)."""
    if hasattr(a, "data_ptr"):
        if a.is_cuda:
            return a.data_ptr(), 0
        return a.data_ptr(), 1
    return a.ctypes.data, 1


def _check_state_tensor(name, a, shape, dtype="complex128"):
    """A device array handed to an entry point: a contiguous torch CUDA
    tensor of `dtype` and `shape` (the C ABI cannot check sizes itself, and a
    wrong buffer would make the pass kernels read or write out of bounds)."""
    import sys
    torch = sys.modules.get("torch")
    if torch is None or not isinstance(a, torch.Tensor):
        raise TypeError(f"{name} must be a torch CUDA tensor")
    if not a.is_cuda:
        raise ValueError(f"{name} must be on a CUDA device")
    if a.dtype != getattr(torch, dtype):
        raise ValueError(f"{name} must be {dtype}, got {a.dtype}")
    if not a.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(a.shape)}, expected {tuple(shape)}")


def cfg_lookup(text, path, kind, default=None):
    """A key of a spooky.cfg text with libconfig's typed lookups
    (spk_cfg_lookup_*): kind is "int", "bool", "float", "string" or
    "strings" (a list or array of strings); the default when the key is
    absent or of another type."""
    L = lib()
    t, k = text.encode(), path.encode()
    if kind == "strings":
        n = L.spk_cfg_setting_length(t, k)
        if n <= 0:
            return default
        return [v for v in (cfg_lookup(text, f"{path}.[{i}]", "string") for i in range(n)) if v is not None]
    if kind == "string":
        buf = ctypes.create_string_buffer(4096)
        rc = L.spk_cfg_lookup_string(t, k, buf, len(buf))
        val = buf.value.decode() if rc == 1 else None
    else:
        box = {"int": ctypes.c_int, "bool": ctypes.c_int, "float": ctypes.c_double}[kind]()
        rc = getattr(L, f"spk_cfg_lookup_{kind}")(t, k, ctypes.byref(box))
        val = (bool(box.value) if kind == "bool" else box.value) if rc == 1 else None
    if rc < 0:
        raise SpookyError(1, L.spk_last_error(None).decode())
    return default if val is None else val


def params_from_file(path):
    """Parameters of a libconfig-format spooky.cfg (spk_params_from_file):
    the reference's keys and defaults, then its module checks.  Raises
    SpookyError (SPK_ERR_ARG for unreadable or malformed files, SPK_ERR_CONFIG
    for inconsistent modules)."""
    p = Params()
    rc = lib().spk_params_from_file(os.fsencode(path), ctypes.byref(p))
    if rc != SPK_OK:
        raise SpookyError(rc, lib().spk_last_error(None).decode())
    return p


def params_from_string(text):
    """As params_from_file, for configuration text."""
    p = Params()
    rc = lib().spk_params_from_string(text.encode(), ctypes.byref(p))
    if rc != SPK_OK:
        raise SpookyError(rc, lib().spk_last_error(None).decode())
    return p


NOALLOC_SCRATCH_BYTES = 24 << 20


def compute_dfield_noalloc(params, U, dU, stream=None):
    """dU = RHS(U) through spk_compute_dfield_noalloc: no context and no
    device allocation, for callers whose device memory belongs to another
    allocator or that must not allocate once running.  All scratch lives in
    one NOALLOC_SCRATCH_BYTES array inside the library; larger grids raise
    SpookyError(SPK_ERR_UNSUPPORTED).  U, dU: torch CUDA complex128 tensors of
    shape (F, nx, ny, nz//2+1).  stream: a CUDA stream handle (int) or None
    for the legacy default stream.  Waits for torch's queued work before the
    call and for the device after it.  Calls that overlap on the GPU race on
    the shared scratch array."""
    p = params.copy()
    shape = (num_fields(p), p.nx, p.ny, p.nz // 2 + 1)
    _check_state_tensor("U", U, shape)
    _check_state_tensor("dU", dU, shape)
    _torch_sync()
    rc = lib().spk_compute_dfield_noalloc(ctypes.byref(p), U.data_ptr(), dU.data_ptr(), stream)
    if rc != SPK_OK:
        raise SpookyError(rc, lib().spk_last_error(None).decode())
    _torch_sync()


class Context:
    """One spk_ctx: the device state and the recorded step pipelines."""

    def __init__(self, params, stream=None, _handle=None):
        self.params = params.copy()
        if _handle is None:
            h = ctypes.c_void_p()
            rc = lib().spk_ctx_create(ctypes.byref(self.params), stream, ctypes.byref(h))
            if rc != SPK_OK:
                raise SpookyError(rc, lib().spk_last_error(None).decode())
            self._owned = True
        else:   # a box of an Ensemble: the ensemble owns the context
            h = _handle
            self._owned = False
        self._h = h
        nf, ncx = ctypes.c_int(), ctypes.c_size_t()
        lib().spk_sizes(self._h, ctypes.byref(nf), ctypes.byref(ncx))
        self.F, self.nc = nf.value, ncx.value
        p = self.params
        self.shape_c = (self.F, p.nx, p.ny, p.nz // 2 + 1)
        self.shape_r = (self.F, p.nx, p.ny, p.nz)
        self.var_list = var_list(p)

    def _check(self, rc):
        if rc != SPK_OK:
            raise SpookyError(rc, lib().spk_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                lib().spk_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------------
    def set_state(self, U):
        if hasattr(U, "is_cuda") and U.is_cuda:
            _torch_sync()
        if not hasattr(U, "data_ptr"):
            U = np.ascontiguousarray(U, dtype=np.complex128)
            assert U.size == self.F * self.nc
        ptr, where = _ptr(U)
        self._check(lib().spk_set_state(self._h, ptr, where))
        if where:
            self.synchronize()

    def get_state(self, out=None):
        if out is None:
            out = np.empty(self.shape_c, dtype=np.complex128)
        ptr, where = _ptr(out)
        self._check(lib().spk_get_state(self._h, ptr, where))
        return out

    def set_time(self, t, step=0, t_lastsnap=0.0):
        self._check(lib().spk_set_time(self._h, t, step, t_lastsnap))

    def get_time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(lib().spk_get_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)))
        return t.value, dt.value, st.value

    # -- reference operations ------------------------------------------------
    def clean_divergence(self):
        self._check(lib().spk_clean_divergence(self._h))

    def compute_dt(self):
        o = [ctypes.c_double() for _ in range(4)]
        self._check(lib().spk_compute_dt(self._h, *[ctypes.byref(x) for x in o]))
        return np.array([x.value for x in o])

    def compute_dfield(self, U, dU):
        """U, dU: torch CUDA complex128 tensors of shape_c.  Waits for torch's
        current stream before and for the context stream after, so the
        tensors can be used on either side without further synchronisation."""
        _check_state_tensor("U", U, self.shape_c)
        _check_state_tensor("dU", dU, self.shape_c)
        _torch_sync()
        self._check(lib().spk_compute_dfield(self._h, U.data_ptr(), dU.data_ptr()))
        self.synchronize()

    def advance(self, nsteps=1):
        self._check(lib().spk_advance(self._h, int(nsteps)))

    # -- the same operations on a caller's state array (torch CUDA complex128, shape_c)
    def advance_fields(self, U, nsteps=1):
        """nsteps main-loop steps on U in place (spk_advance_fields; asynchronous)."""
        _check_state_tensor("U", U, self.shape_c)
        _torch_sync()
        self._check(lib().spk_advance_fields(self._h, U.data_ptr(), int(nsteps)))

    def compute_dt_fields(self, U):
        """TimeStepping::compute_dt on U: (dt_hyp, dt_par, dt_sts, dt)."""
        _check_state_tensor("U", U, self.shape_c)
        _torch_sync()
        o = [ctypes.c_double() for _ in range(4)]
        self._check(lib().spk_compute_dt_fields(self._h, U.data_ptr(), *[ctypes.byref(x) for x in o]))
        return np.array([x.value for x in o])

    def rk3_fields(self, U):
        """TimeStepping::RungeKutta3 on U with the last dt (spk_rk3_fields)."""
        _check_state_tensor("U", U, self.shape_c)
        _torch_sync()
        self._check(lib().spk_rk3_fields(self._h, U.data_ptr()))
        self.synchronize()

    def rkl_cycle_fields(self, U):
        _check_state_tensor("U", U, self.shape_c)
        _torch_sync()
        s = ctypes.c_int()
        self._check(lib().spk_rkl_cycle_fields(self._h, U.data_ptr(), ctypes.byref(s)))
        self.synchronize()
        return s.value

    def transfer_spectra(self, kind):
        """(spectra [ncomp, nbins], deltak, totals [ncomp]) of a transfer
        term (spk_transfer_spectra): "advec", "lorentz", "emfpower",
        "helicity", "th_advec", "th_aniso_diss" or "th_aniso_inj"."""
        maxb = 4096
        out = np.zeros((3, maxb))
        tot = np.zeros(3)
        nc_, nb, dk = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(lib().spk_transfer_spectra(self._h, kind.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               maxb, ctypes.byref(nc_), ctypes.byref(nb), ctypes.byref(dk),
                                               tot.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        n = min(nb.value, maxb)
        return out[: nc_.value, :n].copy(), dk.value, tot[: nc_.value].copy()

    def diagnostics(self):
        """{name: value} of the time-series quantities of spk_diagnostics
        (w2 hv j2 hm hc thetaB bz2 phiB dissgradT pv; -1 where undefined)."""
        d = Diagnostics()
        self._check(lib().spk_diagnostics(self._h, ctypes.byref(d)))
        return {n: getattr(d, n) for n in DIAGNOSTICS}

    # -- real-space state and snapshots
    def get_state_real(self):
        """Real fields [F][nx][ny][nz] (FP64, host) of the state (spk_get_state_real)."""
        R = np.empty(self.shape_r, dtype=np.float64)
        self._check(lib().spk_get_state_real(self._h, R.ctypes.data, 1))
        return R

    def set_state_real(self, R):
        """State from real fields [F][nx][ny][nz] (spk_set_state_real)."""
        R = np.ascontiguousarray(R, dtype=np.float64)
        if R.shape != self.shape_r:
            raise ValueError(f"R has shape {R.shape}, expected {self.shape_r}")
        self._check(lib().spk_set_state_real(self._h, R.ctypes.data, 1))

    def write_snapshot(self, path, t_start=0.0, t_lastsnap=0.0, t_lastvar=0.0):
        self._check(lib().spk_write_snapshot(self._h, os.fsencode(path), t_start, t_lastsnap, t_lastvar))

    def read_snapshot(self, path):
        """State, time, step and t_lastsnap from a snapshot; returns (t_lastsnap, t_lastvar)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(lib().spk_read_snapshot(self._h, os.fsencode(path), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def rkl_cycle(self):
        s = ctypes.c_int()
        self._check(lib().spk_rkl_cycle(self._h, ctypes.byref(s)))
        return s.value

    def to_real(self, R):
        """R: torch CUDA float64 tensor of shape_r (complete on return)."""
        _check_state_tensor("R", R, self.shape_r, "float64")
        _torch_sync()
        self._check(lib().spk_to_real(self._h, R.data_ptr()))
        self.synchronize()

    def synchronize(self):
        self._check(lib().spk_synchronize(self._h))

    def step_info(self):
        """(kernels launched per step, algorithmic HBM bytes per RK3 step)."""
        k, b = ctypes.c_int(), ctypes.c_double()
        self._check(lib().spk_step_info(self._h, ctypes.byref(k), ctypes.byref(b)))
        return k.value, b.value

    def profile_passes(self, reps=10):
        out = (PassStat * 8)()
        n = ctypes.c_int()
        self._check(lib().spk_profile_passes(self._h, int(reps), out, 8, ctypes.byref(n)))
        return [dict(name=out[i].name.decode(), ms=out[i].ms, bytes=out[i].bytes,
                     launches_per_step=out[i].launches_per_step) for i in range(n.value)]

    def budgets(self):
        b = Budgets()
        self._check(lib().spk_budgets(self._h, ctypes.byref(b)))
        return np.array(b.energy[: self.F]), np.array(b.dissipation[: self.F])

    def autotune(self, steps=5):
        """spk_autotune: pick the axis tile width of short axes, the z-pass
        lines per CTA, axis stages and RHS grid by timing; returns the choices
        and ms per step before/after."""
        zl, nst, rhs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        b, a = ctypes.c_double(), ctypes.c_double()
        self._check(lib().spk_autotune(self._h, int(steps), ctypes.byref(zl), ctypes.byref(nst), ctypes.byref(rhs),
                                       ctypes.byref(b), ctypes.byref(a)))
        out = dict(z_lines=zl.value, axis_stages=nst.value, rhs_ctas_per_sm=rhs.value, ms_before=b.value,
                   ms_after=a.value)
        out["axis_tile_div"] = self.get_schedule()["axis_tile_div"]
        return out

    def get_schedule(self):
        """spk_get_schedule: the launch schedule (0: the launcher's model)."""
        v = [ctypes.c_int() for _ in range(4)]
        self._check(lib().spk_get_schedule(self._h, *[ctypes.byref(x) for x in v]))
        return dict(z_lines=v[0].value, axis_stages=v[1].value, rhs_ctas_per_sm=v[2].value, axis_tile_div=v[3].value)

    def set_schedule(self, z_lines=0, axis_stages=0, rhs_ctas_per_sm=0, axis_tile_div=1):
        """spk_set_schedule: set the launch schedule (same values computed)."""
        self._check(lib().spk_set_schedule(self._h, int(z_lines), int(axis_stages), int(rhs_ctas_per_sm),
                                           int(axis_tile_div)))

    # -- diagnostics ---------------------------------------------------------
    def spectrum(self, f1, f2=None):
        """Shell spectrum of fields f1, f2 (indices or names such as "vx")
        of the state (spk_spectrum): (E[nbins], deltak, grid mean of f1 f2)."""
        f1 = self.var_list.index(f1) if isinstance(f1, str) else int(f1)
        f2 = f1 if f2 is None else (self.var_list.index(f2) if isinstance(f2, str) else int(f2))
        nb, dk, tot = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        self._check(lib().spk_spectrum(self._h, f1, f2, None, 0, ctypes.byref(nb), ctypes.byref(dk), None))
        out = np.zeros(max(nb.value, 1))
        self._check(lib().spk_spectrum(self._h, f1, f2, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       nb.value, ctypes.byref(nb), ctypes.byref(dk), ctypes.byref(tot)))
        return out[: nb.value], dk.value, tot.value

    # -- learned closure -----------------------------------------------------
    def closure_set(self, params):
        """Closure weights (closure_nparam(variant) floats) into the RHS, or
        None: off."""
        if params is None:
            self._check(lib().spk_closure_set(self._h, None))
            return
        w = np.ascontiguousarray(params, dtype=np.float32)
        if w.size != closure_nparam(self.params.closure):
            raise ValueError(f"closure variant {self.params.closure} takes {closure_nparam(self.params.closure)} "
                             f"parameters, not {w.size}")
        self._check(lib().spk_closure_set(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def products(self, U):
        """Spectral products of the torch CUDA complex128 state U (shape_c):
        a torch complex128 tensor [nprod, nx, ny, nz//2+1] (spk_products)."""
        import torch
        _check_state_tensor("U", U, self.shape_c)
        p = self.params
        P = torch.zeros((8, p.nx, p.ny, p.nz // 2 + 1), dtype=torch.complex128, device=U.device)
        n = ctypes.c_int()
        _torch_sync()
        self._check(lib().spk_products(self._h, U.data_ptr(), P.data_ptr(), ctypes.byref(n)))
        self.synchronize()
        return P[: n.value]


def closure_samples(fine, Uf, coarse):
    """Training samples of the closure from the fine context's state Uf (a
    torch CUDA complex128 tensor): a torch float32 tensor
    [closure_rows(variant of coarse), coarse nx*ny*nz] (spk_closure_samples);
    coarse's state becomes the filtered state."""
    import torch
    _check_state_tensor("Uf", Uf, fine.shape_c)
    nbytes, ns = ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib().spk_closure_samples_size(fine._h, coarse._h, ctypes.byref(nbytes), ctypes.byref(ns))
    if rc != SPK_OK:
        raise SpookyError(rc, lib().spk_last_error(None).decode())
    scratch = torch.empty(nbytes.value, dtype=torch.uint8, device=Uf.device)
    X = torch.empty((closure_rows(coarse.params.closure), ns.value), dtype=torch.float32, device=Uf.device)
    _torch_sync()
    coarse._check(lib().spk_closure_samples(fine._h, Uf.data_ptr(), coarse._h, X.data_ptr(), ns.value,
                                            scratch.data_ptr(), nbytes.value))
    coarse.synchronize()
    return X


class Trainer:
    """spk_trainer: the closure network of a variant (1, 2: the
    eddy-coefficient MLP; 3: the tensor network) trained on device samples by
    the library's own forward/backward and Adam kernels."""

    def __init__(self, params=None, stream=None, variant=1):
        h = ctypes.c_void_p()
        self.variant = variant
        self.nparam = closure_nparam(variant)
        rc = lib().spk_trainer_create_variant(stream, int(variant), ctypes.byref(h))
        if rc != SPK_OK:
            raise SpookyError(rc, lib().spk_last_error(None).decode())
        self._h = h
        self._X = None
        if params is not None:
            self.set_params(params)

    def _check(self, rc):
        if rc != SPK_OK:
            raise SpookyError(rc, lib().spk_last_error(None).decode())

    @staticmethod
    def _fp(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def set_params(self, params):
        w = np.ascontiguousarray(params, dtype=np.float32)
        if w.size != self.nparam:
            raise ValueError(f"the trainer takes {self.nparam} parameters, not {w.size}")
        self._check(lib().spk_trainer_set_params(self._h, self._fp(w)))

    def get_params(self):
        w = np.empty(self.nparam, np.float32)
        self._check(lib().spk_trainer_get_params(self._h, self._fp(w)))
        return w

    def set_samples(self, X, weights):
        """X: torch CUDA float32 [closure_rows(variant), n] (kept referenced here);
        weights: of the stress, EMF and energy-transfer errors (a third weight
        left out is 0)."""
        if X.shape[0] < closure_rows(self.variant):
            raise ValueError(f"variant {self.variant} samples have {closure_rows(self.variant)} rows")
        _torch_sync()
        self._X = X
        w = np.asarray(weights, dtype=np.float32).ravel()
        if w.size not in (2, 3):
            raise ValueError("weights: 2 or 3 values")
        w = np.ascontiguousarray(np.pad(w, (0, 3 - w.size)))
        self._check(lib().spk_trainer_set_samples(self._h, X.data_ptr(), X.shape[1], X.stride(0), self._fp(w)))

    def loss_grad(self):
        loss = np.zeros(1, np.float32)
        g = np.empty(self.nparam, np.float32)
        self._check(lib().spk_trainer_loss_grad(self._h, self._fp(loss), self._fp(g)))
        return float(loss[0]), g

    def train(self, nsteps, batch, lr):
        hist = np.empty(max(int(nsteps), 1), np.float32)
        self._check(lib().spk_trainer_train(self._h, int(nsteps), int(batch), float(lr), self._fp(hist)))
        return hist[: int(nsteps)]

    def close(self):
        if getattr(self, "_h", None):
            lib().spk_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Reference-named objects (src/supervisor, src/fields, src/timestepping, src/rkl)
# ---------------------------------------------------------------------------
class EnsembleBox:
    """Box i of an Ensemble: its state, time and budgets."""

    def __init__(self, ens, i, params):
        self._e, self.i, self.params = ens, i, params.copy()
        F = num_fields(params)
        self.shape_c = (F, params.nx, params.ny, params.nz // 2 + 1)

    def set_state(self, U):
        _torch_sync()
        if hasattr(U, "data_ptr"):
            ptr, where = _ptr(U)
            keep = U
        else:
            keep = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.shape_c)
            ptr, where = keep.ctypes.data, 1
        self._e._check(lib().spk_ensemble_set_state(self._e._h, self.i, ptr, where))
        if where == 1:
            self._e.synchronize()   # the host array may go away after this call
        del keep

    def get_state(self):
        out = np.empty(self.shape_c, np.complex128)
        self._e._check(lib().spk_ensemble_get_state(self._e._h, self.i, out.ctypes.data, 1))
        return out

    def get_time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._e._check(lib().spk_ensemble_get_time(self._e._h, self.i, ctypes.byref(t), ctypes.byref(dt),
                                                   ctypes.byref(st)))
        return t.value, dt.value, st.value

    def budgets(self):
        b = Budgets()
        self._e._check(lib().spk_ensemble_budgets(self._e._h, self.i, ctypes.byref(b)))
        F = self.shape_c[0]
        return np.array(b.energy[:F]), np.array(b.dissipation[:F])


class Ensemble:
    """Independent boxes advanced together (spk_ensemble_*): boxes that differ
    only in nu, nu_m, nu_th share one set of pass launches; one CUDA graph
    launch per step for the whole ensemble.  boxes[i] gives box i's state,
    time and budgets."""

    def __init__(self, params_list, stream=None):
        arr = (Params * len(params_list))(*[p.copy() for p in params_list])
        h = ctypes.c_void_p()
        rc = lib().spk_ensemble_create(arr, len(params_list), stream, ctypes.byref(h))
        if rc != SPK_OK:
            raise SpookyError(rc, lib().spk_last_error(None).decode())
        self._h = h
        nb, ng = ctypes.c_int(), ctypes.c_int()
        self._check(lib().spk_ensemble_size(self._h, ctypes.byref(nb), ctypes.byref(ng)))
        self.ngroups = ng.value
        self.boxes = [EnsembleBox(self, i, p) for i, p in enumerate(params_list)]

    def _check(self, rc):
        if rc != SPK_OK:
            raise SpookyError(rc, lib().spk_last_error(None).decode())

    def advance(self, nsteps=1):
        self._check(lib().spk_ensemble_advance(self._h, int(nsteps)))

    def autotune(self, steps=5):
        """spk_ensemble_autotune: tune every group's schedule by timing."""
        self._check(lib().spk_ensemble_autotune(self._h, int(steps)))

    def synchronize(self):
        self._check(lib().spk_ensemble_synchronize(self._h))

    def kernels_per_step(self):
        k = ctypes.c_int()
        self._check(lib().spk_ensemble_kernels_per_step(self._h, ctypes.byref(k)))
        return k.value

    def close(self):
        if getattr(self, "_h", None):
            lib().spk_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Parameters:
    """Parameters (src/parameters/parameters.hpp): the cfg subset the path reads."""

    def __init__(self, params=None, **kw):
        self.p = params.copy() if params is not None else default_params(**kw)
        errs = check_parameters(self.p)
        if errs:
            raise SpookyError(6, "; ".join(errs))

    def __getattr__(self, k):
        return getattr(self.__dict__["p"], k)


class Fields:
    """Fields (src/fields/fields.hpp): the state lives in the context."""

    def __init__(self, ctx):
        self._ctx = ctx

    def CleanFieldDivergence(self):
        self._ctx.clean_divergence()

    def set(self, U):
        self._ctx.set_state(U)

    def get(self):
        return self._ctx.get_state()


class RKLegendre:
    """RKLegendre (src/rkl/rkl.hpp:42): compute_cycle on the STS variables."""

    def __init__(self, ctx):
        self._ctx = ctx

    def compute_cycle(self):
        return self._ctx.rkl_cycle()


class TimeStepping:
    """TimeStepping (src/timestepping/timestepping.hpp:39-43)."""

    def __init__(self, ctx):
        self._ctx = ctx
        self.rkl = RKLegendre(ctx)

    def compute_dt(self):
        dt_hyp, dt_par, dt_sts, dt = self._ctx.compute_dt()
        self.dt_hyp, self.dt_par, self.dt_sts, self.current_dt = dt_hyp, dt_par, dt_sts, dt
        return dt

    def compute_dfield(self, U, dU):
        self._ctx.compute_dfield(U, dU)

    def HydroMHDAdvance(self, nsteps=1):
        """CleanFieldDivergence + HydroMHDAdvance, nsteps times (asynchronous)."""
        self._ctx.advance(nsteps)

    @property
    def current_time(self):
        return self._ctx.get_time()[0]

    @property
    def current_step(self):
        return self._ctx.get_time()[2]


def fileCounter(dirname):
    """Index of the most recent snapNNNN.h5 in dirname (the count of
    consecutive files from snap0000.h5, minus one; -1 when there is none),
    as src/io/hdf5_io.cu:255-276 counts them."""
    n = -1
    while os.path.exists(os.path.join(dirname, "snap%04d.h5" % (n + 1))):
        n += 1
    return n


class InputOutput:
    """InputOutput's output schedule and files (src/io/inputoutput.hpp,
    check_output.cu:14-97, hdf5_io.cu:19-276).

    After every main-loop step the supervisor calls CheckOutput.  A time
    series is due when t - t_lastvar >= toutput_time, a snapshot when
    t - t_lastsnap + 1e-8 >= toutput_flow (and both at t = 0).  As in the
    reference, each output first cleans the divergence of the state, and a
    snapshot advances t_lastsnap by toutput_flow -- which the dt rule reads,
    so that steps land on the snapshot times.

    With an output directory, snapshots go to <dir>/data/snapNNNN.h5 (the
    reference's HDF5 layout, spk_write_snapshot) and the time series to
    <dir>/timevar.spooky and <dir>/spectrum.spooky (the reference's text
    layouts).  ``on_timevar(supervisor, t)`` and ``on_snapshot(supervisor,
    num_save)`` replace those writers; with neither a directory nor a
    callable the schedule and the cleaning still run and nothing is written."""

    TIMEVAR_DEFAULT = ("t", "ev", "em")
    SPECTRA_DEFAULT = ()

    def __init__(self, sup, toutput_time=1.0, on_timevar=None, on_snapshot=None, output_dir=None,
                 timevar_vars=None, spectra_vars=None):
        self.sup = sup
        self.toutput_time = toutput_time
        self.t_lastsnap = 0.0
        self.t_lastvar = 0.0
        self.num_save = 0
        self.output_dir = output_dir
        self.timevar_vars = tuple(timevar_vars) if timevar_vars is not None else self.TIMEVAR_DEFAULT
        self.spectra_vars = tuple(spectra_vars) if spectra_vars is not None else self.SPECTRA_DEFAULT
        if output_dir is not None:
            os.makedirs(os.path.join(output_dir, "data"), exist_ok=True)
        self.on_timevar = on_timevar if on_timevar is not None else (self._write_timeseries if output_dir else None)
        self.on_snapshot = on_snapshot if on_snapshot is not None else (self.WriteDataFile if output_dir else None)

    # -- the schedule
    def CheckOutput(self):
        self.CheckTimeSeries()
        self.CheckSnapshot()

    def CheckTimeSeries(self):
        t, _, _ = self.sup.ctx.get_time()
        if t - self.t_lastvar >= self.toutput_time or t == 0.0:
            self.sup.fields.CleanFieldDivergence()
            if t != 0.0:
                self.t_lastvar += self.toutput_time
            if self.on_timevar is not None:
                self.on_timevar(self.sup, t)

    def CheckSnapshot(self):
        t, _, step = self.sup.ctx.get_time()
        if t - self.t_lastsnap + 1e-8 >= self.sup.param.toutput_flow or t == 0.0:
            self.sup.fields.CleanFieldDivergence()
            if t != 0.0:
                self.t_lastsnap += self.sup.param.toutput_flow
                self.sup.ctx.set_time(t, step, self.t_lastsnap)
            if self.on_snapshot is not None:
                self.on_snapshot(self.sup, self.num_save)
            self.num_save += 1

    # -- the files
    def snapshot_path(self, num):
        return os.path.join(self.output_dir, "data", "snap%04d.h5" % num)

    def WriteDataFile(self, sup, num):
        """InputOutput::WriteDataFile (hdf5_io.cu:19-111)."""
        sup.ctx.write_snapshot(self.snapshot_path(num), sup.param.t_initial, self.t_lastsnap, self.t_lastvar)

    def _write_timeseries(self, sup, t):
        from . import outputs
        tv = os.path.join(self.output_dir, "timevar.spooky")
        sp = os.path.join(self.output_dir, "spectrum.spooky")
        if t == 0.0:
            outputs.write_timevar_header(tv, self.timevar_vars)
            if self.spectra_vars:
                outputs.write_spectrum_header(sp, sup.ctx, self.spectra_vars)
        outputs.write_timevar(tv, sup.ctx, self.timevar_vars)
        if self.spectra_vars:
            outputs.write_spectrum(sp, sup.ctx, t, self.spectra_vars)

    def ReadDataFile(self, restart_num):
        """InputOutput::ReadDataFile (hdf5_io.cu:114-252): restart from
        snap<restart_num> (-1, or a number past the last file: the most
        recent one).  Sets the state, time, step, t_lastsnap and t_lastvar;
        num_save becomes the file's number + 1.  Returns the number read, or
        -1 when there is no snapshot (a new run, as the reference does)."""
        last = fileCounter(os.path.join(self.output_dir, "data"))
        if last < 0:
            return -1
        num = last if (restart_num == -1 or restart_num > last) else restart_num
        path = self.snapshot_path(num)
        if not os.path.exists(path):
            raise SpookyError(1, f"restart file {path} not found")
        self.t_lastsnap, self.t_lastvar = self.sup.ctx.read_snapshot(path)
        self.num_save = num + 1
        return num


class Supervisor:
    """Supervisor (src/supervisor/supervisor.hpp:24-84) for the hot path."""

    def __init__(self, params, stream=None, toutput_time=1.0, on_timevar=None, on_snapshot=None, output_dir=None,
                 timevar_vars=None, spectra_vars=None, restart_num=-2):
        """restart_num: -2 a new run; -1 restart from the most recent
        snapshot in output_dir/data; n >= 0 from snap n (main.cu's -r)."""
        self.param = Parameters(params)
        self.ctx = Context(self.param.p, stream)
        self.fields = Fields(self.ctx)
        self.timestep = TimeStepping(self.ctx)
        self.inout = InputOutput(self, toutput_time, on_timevar, on_snapshot, output_dir, timevar_vars,
                                 spectra_vars)
        self.restart_num = restart_num
        if restart_num >= -1:
            self.Restart()

    def Restart(self):
        """Supervisor::Restart (supervisor.cu:241-245); with no snapshot on
        disk the run starts anew (hdf5_io.cu:242-248)."""
        if self.inout.output_dir is None:
            raise SpookyError(1, "a restart needs an output directory")
        if self.inout.ReadDataFile(self.restart_num) < 0:
            self.restart_num = -2

    def initialDataDump(self):
        """The outputs at t = 0 (supervisor.cu:215-238): every output of a new
        run; a restart from snapshot 0 writes only the time series."""
        if self.restart_num == -2:
            self.inout.CheckOutput()
        elif self.restart_num == 0:
            self.inout.CheckTimeSeries()

    def executeMainLoop(self, max_steps=None, max_walltime_hours=None, stats_frequency=-1, log=print):
        """Advance until t_final (src/supervisor/supervisor.cu:169-213): per
        step CleanFieldDivergence + HydroMHDAdvance, then CheckOutput; the
        host reads the device time once per step.  Stops early after
        max_steps steps or max_walltime_hours of main-loop time; with
        stats_frequency > 0 prints the cell-update rate every that many steps
        (print_partial_stats, :75-80).  Returns the steps taken."""
        import time
        n = 0
        t_loop = t_part = 0.0
        nr = self.param.nx * self.param.ny * self.param.nz
        limit = None if max_walltime_hours is None else 3600.0 * max_walltime_hours
        while self.timestep.current_time < self.param.t_final and (limit is None or t_loop < limit):
            t0 = time.perf_counter()
            self.timestep.HydroMHDAdvance(1)
            n += 1
            self.inout.CheckOutput()
            dt = time.perf_counter() - t0
            t_loop += dt
            t_part += dt
            if stats_frequency > 0 and self.timestep.current_step % stats_frequency == 0:
                log("---- The avg number of cell updates / sec is %.4e [cell_updates/s]" % (nr * stats_frequency / t_part))
                t_part = 0.0
            if max_steps is not None and n >= max_steps:
                break
        if limit is not None and t_loop >= limit:
            log("The maximum wallclock elapsed time was reached. Stopping now. You can later resume from the last "
                "snapshot available.")
        self.ctx.synchronize()
        self.time_in_main_loop = t_loop
        return n
