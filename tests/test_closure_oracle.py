"""The learned closure's CPU oracle (oracle/spk_closure.c and the closure
parts of oracle/spk_oracle.c), pinned by properties of its definition:
rotation invariance of the features, finite differences of the loss
gradient, energy removal by the closure terms, products against numpy.fft,
and zero subgrid targets for a field that the coarse grid resolves."""
import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200.params import default_params

L = 2 * np.pi


def _rotation(rng, proper=True):
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    if not proper:
        q = -q
    return q


def _traceless(rng):
    A = rng.standard_normal((3, 3))
    return A - np.trace(A) / 3 * np.eye(3)


@pytest.mark.parametrize("proper", [True, False])
def test_features_are_rotation_invariant(proper):
    rng = np.random.default_rng(1)
    for _ in range(20):
        A, G = _traceless(rng), _traceless(rng)
        R = _rotation(rng, proper)
        f, S, J, n = O.closure_features(A, G)
        f2, S2, J2, n2 = O.closure_features(R @ A @ R.T, R @ G @ R.T)
        assert np.allclose(f, f2, atol=1e-12) and abs(n - n2) < 1e-12 * n
        # S is a tensor; J = curl B a pseudo-vector
        full = lambda s: np.array([[s[0], s[1], s[2]], [s[1], s[3], s[4]], [s[2], s[4], -s[0] - s[3]]])
        assert np.allclose(full(S2), R @ full(S) @ R.T, atol=1e-12)
        assert np.allclose(J2, np.linalg.det(R) * (R @ J), atol=1e-12)


def test_features_of_pure_strain_and_pure_rotation():
    z = np.zeros((3, 3))
    f, S, _, n = O.closure_features(np.diag([1.0, -1.0, 0.0]), z)
    assert np.allclose(f, [1, 0, 0, 0, 0, 0, 0, 0]) and abs(n - np.sqrt(2)) < 1e-14
    assert np.allclose(S, [1, 0, 0, -1, 0])
    rot = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])   # u = (-y, x, 0): w = (0, 0, 2)
    f, _, _, n = O.closure_features(rot, z)
    assert np.allclose(f, [0, 1, 0, 0, 0, 0, 0, 0]) and abs(n - np.sqrt(2)) < 1e-14
    # axisymmetric strain diag(2, -1, -1): tr(S^3)/|S|^3 = 6/6^1.5
    f, _, _, _ = O.closure_features(np.diag([2.0, -1.0, -1.0]), z)
    assert abs(f[4] - 6.0 / 6.0 ** 1.5) < 1e-14


def random_params(rng, scale=0.3):
    p = scale * rng.standard_normal(O.CLOSURE_NPARAM)
    p[-2:] = -3.0 + 0.1 * rng.standard_normal(2)   # small eddy coefficients to start
    return p


def random_samples(rng, n):
    X = np.empty((O.CLOSURE_ROWS, n))
    for s in range(n):
        f, S, J, nn = O.closure_features(_traceless(rng), _traceless(rng))
        X[0:8, s], X[8:13, s], X[13:16, s], X[16, s] = f, S, J, 0.02 * nn
    X[17:25] = 0.05 * rng.standard_normal((8, n))
    # whole-field strain and current: the model's plus other scales
    X[25:33] = X[8:16] + 0.3 * np.abs(X[8:16]).mean() * rng.standard_normal((8, n))
    return X


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    P = random_params(rng)
    P[-2:] = 0.2   # softplus away from its flat end
    X = random_samples(rng, 64)
    w = np.array([3.0, 2.0, 1.5])
    loss, g = O.closure_loss_grad(X, P, w)
    assert loss > 0
    for idx in rng.choice(O.CLOSURE_NPARAM, 40, replace=False).tolist() + [O.CLOSURE_NPARAM - 1, O.CLOSURE_NPARAM - 2]:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[idx] += h
        Pm[idx] -= h
        fd = (O.closure_loss_grad(X, Pp, w)[0] - O.closure_loss_grad(X, Pm, w)[0]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1e-3, abs(g).max()), (idx, fd, g[idx])


def test_adam_fits_a_teacher_network():
    """Targets made by a teacher network of the same form are fitted: the
    loss falls by 100x from a different starting point."""
    rng = np.random.default_rng(3)
    X = random_samples(rng, 256)
    teacher = random_params(rng)
    teacher[-2:] = [-1.0, -1.5]
    for s in range(X.shape[1]):
        o = O.closure_mlp(teacher, X[0:8, s])
        nu, eta = X[16, s] * np.log1p(np.exp(o))
        X[17:22, s] = -2 * nu * X[8:13, s]
        X[22:25, s] = -eta * X[13:16, s]
    w = np.array([1.0, 1.0, 1.0]) / np.mean(X[17:25] ** 2)
    P = random_params(rng)
    m, v = np.zeros_like(P), np.zeros_like(P)
    l0 = O.closure_loss_grad(X, P, w)[0]
    for t in range(1, 601):
        _, g = O.closure_loss_grad(X, P, w)
        O.closure_adam(P, g, m, v, t, 1e-2)
    l1 = O.closure_loss_grad(X, P, w)[0]
    assert l1 < l0 / 100, (l0, l1)


def _mhd_params(n=16, **kw):
    return default_params(incompressible=1, mhd=1, gridsize=(n, n, n), boxsize=(L, L, L), reynolds=1e3,
                          reynolds_magnetic=1e3, **kw)


def _state(p, seed):
    u = random_solenoidal(p, seed, kpeak=3.0)
    B = random_solenoidal(p, seed + 7, kpeak=3.0, rms=0.6)
    return to_spectral(np.concatenate([u, B]))


def test_closure_terms_remove_energy():
    p = _mhd_params()
    o = O.Oracle(p)
    _, mask, _ = o.kgrid()
    U = _state(p, 5) * mask            # dealiased state
    off = o.compute_dfield(U)
    rng = np.random.default_rng(4)
    o.closure_set(random_params(rng, 0.5))
    on = o.compute_dfield(U)
    d = on - off
    assert np.abs(d).max() > 1e-6 * np.abs(off).max()
    w = np.ones(p.nz // 2 + 1)
    w[1:] = 2.0
    w[-1] = 1.0 if p.nz % 2 == 0 else 2.0
    rate = np.sum(w * np.real(np.conj(U) * d))
    scale = np.sum(w * np.abs(U) * np.abs(d))
    assert rate < -1e-3 * scale


def test_products_match_numpy():
    p = _mhd_params(antialiasing=1)
    o = O.Oracle(p)
    U = _state(p, 9)
    P = o.products(U)
    o.set_state(U)
    R = o.to_real()
    u, B = R[:3], R[3:]
    T = np.stack([(2 * u[0] ** 2 - u[1] ** 2 - u[2] ** 2 - 2 * B[0] ** 2 + B[1] ** 2 + B[2] ** 2) / 3,
                  u[0] * u[1] - B[0] * B[1], u[0] * u[2] - B[0] * B[2],
                  (-u[0] ** 2 + 2 * u[1] ** 2 - u[2] ** 2 + B[0] ** 2 - 2 * B[1] ** 2 + B[2] ** 2) / 3,
                  u[1] * u[2] - B[1] * B[2],
                  -B[1] * u[2] + B[2] * u[1], B[0] * u[2] - B[2] * u[0], -B[0] * u[1] + B[1] * u[0]])
    _, mask, _ = o.kgrid()
    ref = np.fft.rfftn(T, axes=(1, 2, 3)) * mask
    assert np.abs(P - ref).max() < 1e-12 * np.abs(ref).max()


def test_resolved_field_has_no_subgrid_targets():
    """A fine state whose modes all lie inside the coarse grid's dealiased
    band is represented exactly on the coarse grid: products agree and the
    targets vanish; the features match closure_features of the gradients."""
    pf, pc = _mhd_params(32), _mhd_params(16)
    of, oc = O.Oracle(pf), O.Oracle(pc)
    Uc = _state(pc, 11)
    _, mc, _ = oc.kgrid()
    Uc = Uc * mc
    # embed into the fine grid (scaled by the point-count ratio)
    Uf = np.zeros((6, 32, 32, 17), complex)
    for ic in range(16):
        for jc in range(16):
            kx, ky = (ic if ic < 8 else ic - 16), (jc if jc < 8 else jc - 16)
            Uf[:, kx % 32, ky % 32, :9] = Uc[:, ic, jc, :] * 8.0
    X = of.closure_samples(Uf, oc)
    assert np.abs(X[17:25]).max() < 1e-12 * np.abs(Uc).max()
    assert np.allclose(oc.get_state(), Uc, atol=1e-14 * np.abs(Uc).max())
    # features row of one point from the oracle's own gradient formula
    kvec, _, _ = oc.kgrid()
    grads = np.fft.irfftn(1j * kvec[None, :] * Uc[:, None], axes=(2, 3, 4), s=(16, 16, 16))
    q = 123
    A = grads[:3].reshape(3, 3, -1)[:, :, q]
    G = grads[3:].reshape(3, 3, -1)[:, :, q]
    f, S, J, n = O.closure_features(A, G)
    assert np.allclose(X[0:8, q], f, atol=1e-12) and np.allclose(X[8:13, q], S, atol=1e-12)
    assert np.allclose(X[13:16, q], J, atol=1e-12)


def test_generic_state_has_subgrid_targets():
    pf, pc = _mhd_params(32), _mhd_params(16)
    of, oc = O.Oracle(pf), O.Oracle(pc)
    Uf = _state(pf, 13)
    X = of.closure_samples(Uf, oc)
    assert np.abs(X[17:25]).max() > 1e-3 * np.abs(oc.to_real()).max() ** 2
    assert np.all(np.isfinite(X))
