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
            "spk_autotune", "spk_ensemble_autotune"]

# learned closure (include/spooky_b200.h, SPK_CLOSURE_*)
CLOSURE_NPARAM = 32 * 8 + 32 + 32 * 32 + 32 + 2 * 32 + 2
CLOSURE_ROWS = 33


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
        L.spk_trainer_destroy.argtypes = [vp]
        L.spk_trainer_set_params.argtypes = [vp, fp]
        L.spk_trainer_get_params.argtypes = [vp, fp]
        L.spk_trainer_set_samples.argtypes = [vp, vp, sp, sp, fp]
        L.spk_trainer_loss_grad.argtypes = [vp, fp, fp]
        L.spk_trainer_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, fp]
        L.spk_spectrum.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ip, dp, dp]
        L.spk_autotune.argtypes = [vp, ctypes.c_int, ip, ip, ip, dp, dp]
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
        """spk_autotune: pick the z-pass lines per CTA, axis stages and RHS
        grid by timing; returns the choices and ms per step before/after."""
        zl, nst, rhs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        b, a = ctypes.c_double(), ctypes.c_double()
        self._check(lib().spk_autotune(self._h, int(steps), ctypes.byref(zl), ctypes.byref(nst), ctypes.byref(rhs),
                                       ctypes.byref(b), ctypes.byref(a)))
        return dict(z_lines=zl.value, axis_stages=nst.value, rhs_ctas_per_sm=rhs.value, ms_before=b.value,
                    ms_after=a.value)

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
        """Closure weights (CLOSURE_NPARAM floats) into the RHS, or None: off."""
        if params is None:
            self._check(lib().spk_closure_set(self._h, None))
            return
        w = np.ascontiguousarray(params, dtype=np.float32)
        assert w.size == CLOSURE_NPARAM
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
    torch CUDA complex128 tensor): a torch float32 tensor [CLOSURE_ROWS,
    coarse nx*ny*nz] (spk_closure_samples); coarse's state becomes the
    filtered state."""
    import torch
    _check_state_tensor("Uf", Uf, fine.shape_c)
    nbytes, ns = ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib().spk_closure_samples_size(fine._h, coarse._h, ctypes.byref(nbytes), ctypes.byref(ns))
    if rc != SPK_OK:
        raise SpookyError(rc, lib().spk_last_error(None).decode())
    scratch = torch.empty(nbytes.value, dtype=torch.uint8, device=Uf.device)
    X = torch.empty((CLOSURE_ROWS, ns.value), dtype=torch.float32, device=Uf.device)
    _torch_sync()
    coarse._check(lib().spk_closure_samples(fine._h, Uf.data_ptr(), coarse._h, X.data_ptr(), ns.value,
                                            scratch.data_ptr(), nbytes.value))
    coarse.synchronize()
    return X


class Trainer:
    """spk_trainer: the closure MLP trained on device samples by the
    library's own forward/backward and Adam kernels."""

    def __init__(self, params=None, stream=None):
        h = ctypes.c_void_p()
        rc = lib().spk_trainer_create(stream, ctypes.byref(h))
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
        assert w.size == CLOSURE_NPARAM
        self._check(lib().spk_trainer_set_params(self._h, self._fp(w)))

    def get_params(self):
        w = np.empty(CLOSURE_NPARAM, np.float32)
        self._check(lib().spk_trainer_get_params(self._h, self._fp(w)))
        return w

    def set_samples(self, X, weights):
        """X: torch CUDA float32 [CLOSURE_ROWS, n] (kept referenced here);
        weights: of the stress, EMF and energy-transfer errors (a third weight
        left out is 0)."""
        _torch_sync()
        self._X = X
        w = np.asarray(weights, dtype=np.float32).ravel()
        if w.size not in (2, 3):
            raise ValueError("weights: 2 or 3 values")
        w = np.ascontiguousarray(np.pad(w, (0, 3 - w.size)))
        self._check(lib().spk_trainer_set_samples(self._h, X.data_ptr(), X.shape[1], X.stride(0), self._fp(w)))

    def loss_grad(self):
        loss = np.zeros(1, np.float32)
        g = np.empty(CLOSURE_NPARAM, np.float32)
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


class InputOutput:
    """InputOutput's output schedule (src/io/inputoutput.hpp, check_output.cu:14-97).

    After every main-loop step the supervisor calls CheckOutput.  A time
    series is due when t - t_lastvar >= toutput_time, a snapshot when
    t - t_lastsnap + 1e-8 >= toutput_flow (and both at t = 0).  As in the
    reference, each output first cleans the divergence of the state, and a
    snapshot advances t_lastsnap by toutput_flow -- which the dt rule reads,
    so that steps land on the snapshot times.  The writers are callables:
    ``on_timevar(supervisor, t)`` and ``on_snapshot(supervisor, num_save)``
    (None: the schedule and the cleaning still run, nothing is written)."""

    def __init__(self, sup, toutput_time=1.0, on_timevar=None, on_snapshot=None):
        self.sup = sup
        self.toutput_time = toutput_time
        self.t_lastsnap = 0.0
        self.t_lastvar = 0.0
        self.num_save = 0
        self.on_timevar = on_timevar
        self.on_snapshot = on_snapshot

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


class Supervisor:
    """Supervisor (src/supervisor/supervisor.hpp:24-84) for the hot path."""

    def __init__(self, params, stream=None, toutput_time=1.0, on_timevar=None, on_snapshot=None):
        self.param = Parameters(params)
        self.ctx = Context(self.param.p, stream)
        self.fields = Fields(self.ctx)
        self.timestep = TimeStepping(self.ctx)
        self.inout = InputOutput(self, toutput_time, on_timevar, on_snapshot)

    def initialDataDump(self):
        """The outputs at t = 0 of a run that does not restart (supervisor.cu:215-225)."""
        self.inout.CheckOutput()

    def executeMainLoop(self, max_steps=None):
        """Advance until t_final (src/supervisor/supervisor.cu:169-213): per
        step CleanFieldDivergence + HydroMHDAdvance, then CheckOutput; the
        host reads the device time once per step."""
        n = 0
        while self.timestep.current_time < self.param.t_final:
            self.timestep.HydroMHDAdvance(1)
            n += 1
            self.inout.CheckOutput()
            if max_steps is not None and n >= max_steps:
                break
        self.ctx.synchronize()
        return n
