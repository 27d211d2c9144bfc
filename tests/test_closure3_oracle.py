"""The oracle of the closure's variant 3, the tensor network of the
learned-closure configuration (18 gradients -> 64 -> 64 -> 64 -> 12, BF16
operands): finite differences of its loss gradient (roundings off), the
size of the BF16 roundings, the RHS terms against their definition, the
backscatter ramp, energy removal in the RHS, the sample rows and a fit of a
teacher network."""
import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200.params import default_params
from test_closure_oracle import _traceless

L = 2 * np.pi
NI, NH, NO = 18, 64, 12
# parameter offsets: W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[12][64] b4[12]
W1, B1 = 0, 64 * 18
W2, B2 = B1 + 64, B1 + 64 + 4096
W3, B3 = B2 + 64, B2 + 64 + 4096
W4, B4 = B3 + 64, B3 + 64 + 768


def random_params3(rng, scale=1.0, out=0.05):
    p = np.zeros(O.CLOSURE3_NPARAM)
    p[W1:B1] = scale * rng.standard_normal(B1 - W1) / np.sqrt(NI)
    p[B1:W2] = 0.1 * rng.standard_normal(64)
    p[W2:B2] = scale * rng.standard_normal(4096) / np.sqrt(NH)
    p[B2:W3] = 0.1 * rng.standard_normal(64)
    p[W3:B3] = scale * rng.standard_normal(4096) / np.sqrt(NH)
    p[B3:W4] = 0.1 * rng.standard_normal(64)
    p[W4:B4] = out * rng.standard_normal(768) / np.sqrt(NH)
    p[B4:] = out * rng.standard_normal(12)
    return p


def random_samples3(rng, n, delta2=0.02):
    X = np.zeros((O.CLOSURE3_ROWS, n))
    for s in range(n):
        A, G = _traceless(rng), _traceless(rng)
        f, S, J, nn = O.closure_features(A, G)
        X[0:8, s], X[8:13, s], X[13:16, s], X[16, s] = f, S, J, delta2 * nn
        X[33:42, s], X[42:51, s] = A.ravel(), G.ravel()
    X[17:25] = 0.05 * rng.standard_normal((8, n))
    X[25:33] = X[8:16] + 0.3 * np.abs(X[8:16]).mean() * rng.standard_normal((8, n))
    return X


@pytest.fixture
def exact():
    O.closure3_set_rounding(False)
    yield
    O.closure3_set_rounding(True)


def _mlp_numpy(P, x):
    h = np.tanh(P[W1:B1].reshape(64, 18) @ x + P[B1:W2])
    h = np.tanh(P[W2:B2].reshape(64, 64) @ h + P[B2:W3])
    h = np.tanh(P[W3:B3].reshape(64, 64) @ h + P[B3:W4])
    return P[W4:B4].reshape(12, 64) @ h + P[B4:]


def test_exact_network_matches_numpy(exact):
    rng = np.random.default_rng(31)
    P = random_params3(rng, out=1.0)
    for _ in range(5):
        x = rng.standard_normal(18)
        assert np.allclose(O.closure3_mlp(P, x), _mlp_numpy(P, x), rtol=1e-13, atol=1e-13)


def test_bf16_roundings_are_at_the_bf16_level():
    rng = np.random.default_rng(32)
    P = random_params3(rng, out=1.0)
    x = rng.standard_normal((200, 18))
    a = np.stack([O.closure3_mlp(P, v) for v in x])
    b = np.stack([_mlp_numpy(P, v) for v in x])
    err = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert 1e-4 < err < 3e-2, err


def test_loss_gradient_matches_finite_differences(exact):
    rng = np.random.default_rng(33)
    P = random_params3(rng, out=0.5)
    X = random_samples3(rng, 48)
    w = np.array([3.0, 2.0, 1.5])
    loss, g = O.closure3_loss_grad(X, P, w)
    assert loss > 0
    idx = rng.choice(O.CLOSURE3_NPARAM, 60, replace=False).tolist()
    idx += [W1, B1 - 1, W2 + 5, B3 + 3, W4, B4 - 1, B4, O.CLOSURE3_NPARAM - 1]
    for i in idx:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (O.closure3_loss_grad(X, Pp, w)[0] - O.closure3_loss_grad(X, Pm, w)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g).max()), (i, fd, g[i])


def test_rounded_gradient_is_close_to_the_exact_one():
    rng = np.random.default_rng(34)
    P = random_params3(rng, out=0.5)
    X = random_samples3(rng, 256)
    w = np.array([1.0, 1.0, 1.0])
    l1, g1 = O.closure3_loss_grad(X, P, w)
    O.closure3_set_rounding(False)
    try:
        l0, g0 = O.closure3_loss_grad(X, P, w)
    finally:
        O.closure3_set_rounding(True)
    assert abs(l1 - l0) < 2e-2 * l0
    assert np.linalg.norm(g1 - g0) < 5e-2 * np.linalg.norm(g0)


def _full(s5, zz=None):
    zz = -(s5[0] + s5[3]) if zz is None else zz
    return np.array([[s5[0], s5[1], s5[2]], [s5[1], s5[3], s5[4]], [s5[2], s5[4], zz]])


@pytest.mark.parametrize("mhd", [True, False])
def test_terms_follow_their_definition(mhd):
    rng = np.random.default_rng(35)
    P = random_params3(rng, out=1.0)
    delta2 = 0.03
    hits = {"full": 0, "zero": 0, "ramp": 0}
    for _ in range(300):
        A, G = _traceless(rng), (_traceless(rng) if mhd else np.zeros((3, 3)))
        tau, e, nu, eta, n = O.closure3_terms(P, delta2, A, G, mhd)
        f, S5, J, n2 = O.closure_features(A, G)
        assert abs(n - n2) < 1e-14 * n
        x = np.concatenate([A.ravel(), G.ravel()]) / n
        s = delta2 * n * n * O.closure3_mlp(P, x)
        tr = (s[0] + s[3] + s[5]) / 3
        dT = np.array([s[0] - tr, s[1], s[2], s[3] - tr, s[4]])
        dE = 0.5 * np.array([s[9] - s[11], s[10] - s[7], s[6] - s[8]]) if mhd else np.zeros(3)
        T, Sm = _full(dT), _full(S5, A[2, 2])
        Pt = -np.sum(T * Sm) - dE @ J
        Pm = np.linalg.norm(T) * np.linalg.norm(Sm) + np.linalg.norm(dE) * np.linalg.norm(J)
        r = np.clip(Pt / (0.1 * Pm + 1e-30), 0.0, 1.0)
        hits["full" if r == 1 else ("zero" if r == 0 else "ramp")] += 1
        assert np.allclose(tau, r * dT, rtol=1e-12, atol=1e-14 * np.abs(dT).max())
        assert np.allclose(e, r * dE, rtol=1e-12, atol=1e-14 * max(np.abs(dE).max(), 1e-300))
        # the kept terms drain resolved energy at this point
        assert -np.sum(_full(tau) * Sm) - e @ J >= -1e-12 * Pm
        assert abs(nu - r * np.linalg.norm(T) / (2 * n)) < 1e-12 * max(nu, 1e-300)
        assert abs(eta - (r * np.linalg.norm(dE) / n if mhd else 0.0)) < 1e-12 * max(eta, 1e-300)
    assert min(hits.values()) > 0, hits


def _mhd_params(n=16, **kw):
    return default_params(incompressible=1, mhd=1, gridsize=(n, n, n), boxsize=(L, L, L), reynolds=1e3,
                          reynolds_magnetic=1e3, **kw)


def _state(p, seed):
    u = random_solenoidal(p, seed, kpeak=3.0)
    B = random_solenoidal(p, seed + 7, kpeak=3.0, rms=0.6)
    return to_spectral(np.concatenate([u, B]))


def test_closure_terms_remove_energy():
    p = _mhd_params(closure=3)
    o = O.Oracle(p)
    _, mask, _ = o.kgrid()
    U = _state(p, 5) * mask
    off = o.compute_dfield(U)
    o.closure_set(random_params3(np.random.default_rng(36), out=1.0))
    on = o.compute_dfield(U)
    d = on - off
    assert np.abs(d).max() > 1e-6 * np.abs(off).max()
    w = np.ones(p.nz // 2 + 1)
    w[1:] = 2.0
    w[-1] = 1.0
    rate = np.sum(w * np.real(np.conj(U) * d))
    scale = np.sum(w * np.abs(U) * np.abs(d))
    assert rate < -1e-3 * scale


def test_samples_carry_the_gradients():
    pf, pc1, pc3 = _mhd_params(32), _mhd_params(16, closure=1), _mhd_params(16, closure=3)
    Uf = _state(pf, 13)
    X1 = O.Oracle(pf).closure_samples(Uf, O.Oracle(pc1))
    oc = O.Oracle(pc3)
    X3 = O.Oracle(pf).closure_samples(Uf, oc)
    assert X1.shape[0] == O.CLOSURE_ROWS and X3.shape[0] == O.CLOSURE3_ROWS
    assert np.array_equal(X3[:33], X1)
    kvec, _, _ = oc.kgrid()
    U = oc.get_state()
    grads = np.fft.irfftn(1j * kvec[None, :] * U[:, None], axes=(2, 3, 4), s=(16, 16, 16))
    assert np.allclose(X3[33:42], grads[:3].reshape(9, -1), atol=1e-12 * np.abs(grads).max())
    assert np.allclose(X3[42:51], grads[3:].reshape(9, -1), atol=1e-12 * np.abs(grads).max())
    for q in (0, 77, 4095):
        f, S, J, n = O.closure_features(X3[33:42, q].reshape(3, 3), X3[42:51, q].reshape(3, 3))
        assert np.allclose(X3[0:8, q], f, atol=1e-12) and abs(X3[16, q] - oc_delta2(pc3) * n) < 1e-12 * n


def oc_delta2(p):
    k = lambda n, l: 2 * np.pi / l * (n // 2 - 1) * 2.0 / 3.0
    kx, ky, kz = k(p.nx, p.lx), k(p.ny, p.ly), k(p.nz, p.lz)
    return (np.pi / kx * np.pi / ky * np.pi / kz) ** (2.0 / 3.0)


def test_adam_fits_a_teacher_network():
    rng = np.random.default_rng(37)
    X = random_samples3(rng, 192)
    teacher = random_params3(rng, out=1.0)
    for s in range(X.shape[1]):
        A, G = X[33:42, s], X[42:51, s]
        n = O.closure_features(A.reshape(3, 3), G.reshape(3, 3))[3]
        sv = X[16, s] * n * O.closure3_mlp(teacher, np.concatenate([A, G]) / n)
        tr = (sv[0] + sv[3] + sv[5]) / 3
        X[17:22, s] = [sv[0] - tr, sv[1], sv[2], sv[3] - tr, sv[4]]
        X[22:25, s] = 0.5 * np.array([sv[9] - sv[11], sv[10] - sv[7], sv[6] - sv[8]])
    w = np.array([1.0, 1.0, 0.0]) / np.mean(X[17:25] ** 2)
    P = random_params3(rng, out=0.05)
    m, v = np.zeros_like(P), np.zeros_like(P)
    l0 = O.closure3_loss_grad(X, P, w)[0]
    for t in range(1, 301):
        _, g = O.closure3_loss_grad(X, P, w)
        O.closure_adam(P, g, m, v, t, 3e-3)
    l1 = O.closure3_loss_grad(X, P, w)[0]
    assert l1 < l0 / 20, (l0, l1)
