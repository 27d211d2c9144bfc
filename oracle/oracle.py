"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product path.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run `make -C oracle`)")
        L = ctypes.CDLL(path)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_num_fields.argtypes = [vp]
        L.orc_num_fields.restype = ctypes.c_int
        L.orc_ncomplex.argtypes = [vp]
        L.orc_ncomplex.restype = ctypes.c_size_t
        for name in ("orc_set_state", "orc_get_state", "orc_compute_dt", "orc_to_real"):
            getattr(L, name).argtypes = [vp, dp]
        L.orc_set_time.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.orc_get_time.argtypes = [vp, dp, dp, ip]
        L.orc_kgrid.argtypes = [vp, dp, dp, dp]
        L.orc_clean_divergence.argtypes = [vp]
        L.orc_compute_dfield.argtypes = [vp, dp, dp]
        L.orc_step.argtypes = [vp, ctypes.c_int]
        L.orc_rkl_cycle.argtypes = [vp]
        L.orc_rkl_cycle.restype = ctypes.c_int
        L.orc_budgets.argtypes = [vp, dp, dp]
        L.orc_r2c.argtypes = [vp, dp, dp]
        L.orc_c2r.argtypes = [vp, dp, dp]
        L.orc_fft1d.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_closure_set.argtypes = [vp, dp]
        L.orc_closure_set.restype = ctypes.c_int
        L.orc_products.argtypes = [vp, dp, dp]
        L.orc_products.restype = ctypes.c_int
        L.orc_truncate.argtypes = [vp, vp, dp, ctypes.c_int, dp]
        L.orc_closure_samples.argtypes = [vp, dp, vp, dp, ctypes.c_size_t]
        L.orc_closure_features.argtypes = [dp, dp, dp, dp, dp]
        L.orc_closure_features.restype = ctypes.c_double
        L.orc_closure_mlp.argtypes = [dp, dp, dp]
        L.orc_closure_loss_grad.argtypes = [dp, ctypes.c_size_t, ctypes.c_size_t, dp, dp, dp, dp]
        L.orc_closure_adam.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_double]
        L.orc_get_tremap.argtypes = [vp]
        L.orc_get_tremap.restype = ctypes.c_double
        L.orc_closure_adam_n.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_closure3_set_rounding.argtypes = [ctypes.c_int]
        L.orc_closure3_mlp.argtypes = [dp, dp, dp]
        L.orc_closure3_terms.argtypes = [dp, ctypes.c_double, dp, dp, ctypes.c_int, dp, dp, dp, dp]
        L.orc_closure3_terms.restype = ctypes.c_double
        L.orc_closure3_loss_grad.argtypes = [dp, ctypes.c_size_t, ctypes.c_size_t, dp, dp, dp, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fft1d(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_fft1d(len(x), _dp(x), _dp(out), sign)
    return out


def set_threads(n):
    lib().orc_set_threads(int(n))


# ---- learned closure (include/spooky_b200.h, SPK_CLOSURE_*) ----------------
CLOSURE_NPARAM = 32 * 8 + 32 + 32 * 32 + 32 + 2 * 32 + 2
CLOSURE_ROWS = 33
# variant 3, the tensor network (SPK_CLOSURE3_*)
CLOSURE3_NPARAM = 64 * 18 + 64 + 2 * (64 * 64 + 64) + 12 * 64 + 12
CLOSURE3_ROWS = 51


def closure_features(A, G):
    """A, G: 3x3 gradients (A[i, j] = du_i/dx_j) -> (features[8], S[5], J[3], n)."""
    A = np.ascontiguousarray(A, dtype=np.float64).reshape(9)
    G = np.ascontiguousarray(G, dtype=np.float64).reshape(9)
    f, S, J = np.empty(8), np.empty(5), np.empty(3)
    n = lib().orc_closure_features(_dp(A), _dp(G), _dp(f), _dp(S), _dp(J))
    return f, S, J, n


def closure_mlp(params, f):
    params = np.ascontiguousarray(params, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    o = np.empty(2)
    lib().orc_closure_mlp(_dp(params), _dp(f), _dp(o))
    return o


def closure_loss_grad(samples, params, w):
    """samples: [CLOSURE_ROWS, n] rows; w: the stress, EMF and energy-transfer
    weights (a third weight left out is 0); returns (loss, grad)."""
    X = np.ascontiguousarray(samples, dtype=np.float64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    w = np.zeros(3) + np.pad(np.asarray(w, dtype=np.float64), (0, 3 - len(w)))   # w[2] defaults to 0
    g = np.empty(CLOSURE_NPARAM)
    loss = ctypes.c_double()
    lib().orc_closure_loss_grad(_dp(X), X.shape[1], X.shape[1], _dp(params), _dp(w), _dp(g), ctypes.byref(loss))
    return loss.value, g


def closure_adam(params, grad, m, v, t, lr):
    """In place on float64 arrays params, m, v (either network)."""
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    lib().orc_closure_adam_n(_dp(params), _dp(grad), _dp(m), _dp(v), int(t), float(lr), int(params.size))


def closure3_set_rounding(on):
    """Variant 3: 0 drops every BF16 rounding of the network (exact FP64)."""
    lib().orc_closure3_set_rounding(1 if on else 0)


def closure3_mlp(params, x):
    params = np.ascontiguousarray(params, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    o = np.empty(12)
    lib().orc_closure3_mlp(_dp(params), _dp(x), _dp(o))
    return o


def closure3_terms(params, delta2, A, G, mhd=True):
    """Variant 3's RHS terms at one point: (tau[5], e[3], nu_eff, eta_eff, n)."""
    params = np.ascontiguousarray(params, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64).reshape(9)
    G = np.ascontiguousarray(G, dtype=np.float64).reshape(9)
    tau, e = np.empty(5), np.empty(3)
    nu, eta = ctypes.c_double(), ctypes.c_double()
    n = lib().orc_closure3_terms(_dp(params), float(delta2), _dp(A), _dp(G), 1 if mhd else 0, _dp(tau), _dp(e),
                                 ctypes.byref(nu), ctypes.byref(eta))
    return tau, e, nu.value, eta.value, n


def closure3_loss_grad(samples, params, w):
    """samples: [CLOSURE3_ROWS, n]; returns (loss, grad[CLOSURE3_NPARAM])."""
    X = np.ascontiguousarray(samples, dtype=np.float64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    w = np.zeros(3) + np.pad(np.asarray(w, dtype=np.float64), (0, 3 - len(w)))
    g = np.empty(CLOSURE3_NPARAM)
    loss = ctypes.c_double()
    lib().orc_closure3_loss_grad(_dp(X), X.shape[1], X.shape[1], _dp(params), _dp(w), _dp(g), ctypes.byref(loss))
    return loss.value, g


class Oracle:
    """CPU restatement of the reference's Fields/TimeStepping/RKLegendre path."""

    def __init__(self, params):
        self.params = params.copy()
        self._h = lib().orc_create(ctypes.byref(self.params))
        if not self._h:
            raise RuntimeError("orc_create failed")
        self.F = lib().orc_num_fields(self._h)
        self.nc = lib().orc_ncomplex(self._h)
        p = self.params
        self.shape_c = (self.F, p.nx, p.ny, p.nz // 2 + 1)
        self.shape_r = (self.F, p.nx, p.ny, p.nz)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.shape_c)
        lib().orc_set_state(self._h, _dp(U))

    def get_state(self):
        U = np.empty(self.shape_c, dtype=np.complex128)
        lib().orc_get_state(self._h, _dp(U))
        return U

    def set_time(self, t, step=0, t_lastsnap=0.0):
        lib().orc_set_time(self._h, t, step, t_lastsnap)

    def get_time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lib().orc_get_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st))
        return t.value, dt.value, st.value

    def kgrid(self):
        p = self.params
        kvec = np.empty((3, p.nx, p.ny, p.nz // 2 + 1))
        mask = np.empty((p.nx, p.ny, p.nz // 2 + 1))
        km = np.empty(4)
        lib().orc_kgrid(self._h, _dp(kvec), _dp(mask), _dp(km))
        return kvec, mask, km

    def clean_divergence(self):
        lib().orc_clean_divergence(self._h)

    def compute_dt(self):
        out = np.empty(4)
        lib().orc_compute_dt(self._h, _dp(out))
        return out

    def compute_dfield(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.shape_c)
        dU = np.empty_like(U)
        lib().orc_compute_dfield(self._h, _dp(U), _dp(dU))
        return dU

    def step(self, n=1):
        lib().orc_step(self._h, int(n))

    def rkl_cycle(self):
        return lib().orc_rkl_cycle(self._h)

    def to_real(self):
        R = np.empty(self.shape_r)
        lib().orc_to_real(self._h, _dp(R))
        return R

    def budgets(self):
        e = np.empty(self.F)
        d = np.empty(self.F)
        lib().orc_budgets(self._h, _dp(e), _dp(d))
        return e, d

    def r2c(self, R):
        p = self.params
        R = np.ascontiguousarray(R, dtype=np.float64).reshape(p.nx, p.ny, p.nz)
        C = np.empty((p.nx, p.ny, p.nz // 2 + 1), dtype=np.complex128)
        lib().orc_r2c(self._h, _dp(R), _dp(C))
        return C

    def tremap(self):
        """The shearing box's remap clock (TimeStepping::tremap)."""
        return lib().orc_get_tremap(self._h)

    def closure_set(self, params):
        if params is None:
            return lib().orc_closure_set(self._h, None)
        self._cparams = np.ascontiguousarray(params, dtype=np.float64)
        rc = lib().orc_closure_set(self._h, _dp(self._cparams))
        if rc:
            raise ValueError("the closure needs an HD or MHD context")

    def products(self, U):
        U = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.shape_c)
        p = self.params
        P = np.zeros((8, p.nx, p.ny, p.nz // 2 + 1), dtype=np.complex128)
        n = lib().orc_products(self._h, _dp(U), _dp(P))
        return P[:n]

    def truncate_to(self, coarse, X):
        """Sharp spectral filter of this grid's spectra X[nch, ...] onto coarse."""
        X = np.ascontiguousarray(X, dtype=np.complex128)
        nch = X.shape[0]
        q = coarse.params
        out = np.empty((nch, q.nx, q.ny, q.nz // 2 + 1), dtype=np.complex128)
        lib().orc_truncate(self._h, coarse._h, _dp(X), nch, _dp(out))
        return out

    def closure_samples(self, U, coarse):
        """Samples [CLOSURE_ROWS (variant 3: CLOSURE3_ROWS), nx*ny*nz of
        coarse] from this (fine) state U."""
        U = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.shape_c)
        q = coarse.params
        n = q.nx * q.ny * q.nz
        X = np.empty((CLOSURE3_ROWS if q.closure == 3 else CLOSURE_ROWS, n))
        lib().orc_closure_samples(self._h, _dp(U), coarse._h, _dp(X), n)
        return X

    def c2r(self, C):
        p = self.params
        C = np.ascontiguousarray(C, dtype=np.complex128).reshape(p.nx, p.ny, p.nz // 2 + 1)
        R = np.empty((p.nx, p.ny, p.nz))
        lib().orc_c2r(self._h, _dp(C), _dp(R))
        return R
