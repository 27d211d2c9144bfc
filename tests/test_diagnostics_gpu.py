"""Diagnostics on the device: shell spectra (Spectrum1d) against a numpy
restatement of the reference kernel, the Parseval totals against real-space
means, and the spectrum.spooky / timevar.spooky text formats."""
import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200 import Context
from spooky_b200 import outputs
from spooky_b200.params import SPK_FORM_FP32, default_params

pytestmark = pytest.mark.gpu


def spectrum_ref(U1, U2, p):
    """Spectrum1d (cuda_kernels_generic.cu:441-472) in numpy; shells >= nbins dropped."""
    kv = O.Oracle(p).kgrid()
    kvec, _, km = kv
    N = p.nx * p.ny * p.nz
    pw = np.real((U1 / N) * np.conj(U2 / N))
    pw[:, :, 1:] *= 2.0
    dk = 2 * np.pi / min(p.lx, p.ly, p.lz)
    nb = int(km[3] / dk + 0.5)
    m = (np.sqrt((kvec ** 2).sum(0)) / dk + 0.5).astype(int)
    E = np.bincount(m.ravel(), weights=pw.ravel(), minlength=nb + 64)[:nb]
    return E, dk


@pytest.mark.parametrize("shape,box", [((32, 32, 32), (2 * np.pi,) * 3), ((32, 16, 24), (1.0, 2.0, 1.5))])
def test_spectrum_matches_reference_kernel(shape, box):
    p = default_params(incompressible=1, mhd=1, gridsize=shape, boxsize=box, reynolds=100.0,
                       reynolds_magnetic=100.0, form=SPK_FORM_FP32)
    U = to_spectral(np.concatenate([random_solenoidal(p, 3, kpeak=8.0), random_solenoidal(p, 4, kpeak=8.0)]))
    ctx = Context(p)
    ctx.set_state(U)
    R = O.Oracle(p)
    R.set_state(U)
    R = R.to_real()
    for a, b in [("vx", "vx"), ("vx", "vy"), ("bz", "by")]:
        ia, ib = ctx.var_list.index(a), ctx.var_list.index(b)
        E, dk, tot = ctx.spectrum(a, b)
        Er, dkr = spectrum_ref(U[ia], U[ib], p)
        assert abs(dk - dkr) < 1e-15 and len(E) == len(Er)
        assert np.allclose(E, Er, rtol=1e-12, atol=1e-14 * np.abs(Er).max())
        # Parseval total: the grid mean of the product (twoFieldCorrelation)
        assert abs(tot - np.mean(R[ia] * R[ib])) < 1e-12 * max(1.0, abs(np.mean(R[ia] * R[ib])))


def test_diagnostics_files(tmp_path):
    p = default_params(incompressible=1, mhd=1, gridsize=(16, 16, 16), boxsize=(2 * np.pi,) * 3)
    U = to_spectral(np.concatenate([random_solenoidal(p, 5), random_solenoidal(p, 6)]))
    ctx = Context(p)
    ctx.set_state(U)
    sp = tmp_path / "spectrum.spooky"
    outputs.write_spectrum_header(str(sp), ctx, ["Kx", "bxby"])
    outputs.write_spectrum(str(sp), ctx, 0.0, ["Kx", "bxby"])
    lines = sp.read_text().splitlines()
    assert lines[1] == "## \tKx\tbxby\t"
    assert lines[2].startswith("wavevector \t0.00000000e+00\t1.00000000e+00\t")
    row = lines[3].split("\t")
    assert row[0] == "t" and row[2] == "Kx" and len(row) == 3 + len(ctx.spectrum(0)[0]) + 1
    tv = tmp_path / "timevar.spooky"
    names = ["t", "ev", "em", "vxvy", "w2"]
    outputs.write_timevar_header(str(tv), names)
    outputs.write_timevar(str(tv), ctx, names)
    vals = [float(x) for x in tv.read_text().splitlines()[2].split("\t")[:-1]]
    e, _ = ctx.budgets()
    # values are written with 9 significant digits (std::scientific, precision 8)
    assert vals[0] == 0.0 and abs(vals[1] - e[:3].sum()) < 1e-8 * e[:3].sum()
    assert abs(vals[2] - e[3:].sum()) < 1e-8 * e[3:].sum()
    assert abs(vals[4] - ctx.diagnostics()["w2"]) <= 1e-8 * vals[4]   # enstrophy (spk_diagnostics)
    # ev is half the Parseval total of the three components plus the Nyquist
    # plane once more: computeEnergy weights every kz > 0 plane by 2
    # (spooky_output_functions.cu:23-55)
    tot = sum(ctx.spectrum(q)[2] for q in ("vx", "vy", "vz"))
    N = p.nx * p.ny * p.nz
    nyq = 0.5 * np.sum(np.abs(U[:3, :, :, p.nz // 2]) ** 2) / N ** 2
    assert abs(e[:3].sum() - (0.5 * tot + nyq)) < 1e-12 * tot


def transfer_ref(p, U, kind):
    """The reference's transfer terms (spooky_output_spectrum.cu:186-460) in
    numpy: real fields, products, R2C, the masked contraction; returns the
    (field index, term) pairs whose spectra the library reports."""
    kvec, mask, _ = O.Oracle(p).kgrid()
    KX, KY, KZ = kvec
    shape = (p.nx, p.ny, p.nz)
    irf = lambda c: np.fft.irfftn(c, s=shape, axes=(0, 1, 2))
    rf = np.fft.rfftn
    F = U.shape[0]
    R = [irf(U[f]) for f in range(F)]
    u, B = R[0:3], R[3:6]
    th = R[-1]
    I = 1j
    if kind in ("advec", "lorentz"):
        v = u if kind == "advec" else B
        S = [rf(v[0] * v[0]), rf(v[0] * v[1]), rf(v[0] * v[2]), rf(v[1] * v[1]), rf(v[1] * v[2]), rf(v[2] * v[2])]
        T = [-I * mask * (KX * S[0] + KY * S[1] + KZ * S[2]), -I * mask * (KX * S[1] + KY * S[3] + KZ * S[4]),
             -I * mask * (KX * S[2] + KY * S[4] + KZ * S[5])]
        return [(c, T[c]) for c in range(3)]
    if kind == "emfpower":
        E = [rf(u[1] * B[2] - u[2] * B[1]), rf(u[2] * B[0] - u[0] * B[2]), rf(u[0] * B[1] - u[1] * B[0])]
        T = [I * mask * (KY * E[2] - KZ * E[1]), I * mask * (KZ * E[0] - KX * E[2]), I * mask * (KX * E[1] - KY * E[0])]
        return [(3 + c, T[c]) for c in range(3)]
    if kind == "helicity":
        K2 = KX ** 2 + KY ** 2 + KZ ** 2
        ik2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 1.0)
        b = U[3:6]
        A = [I * ik2 * (KY * b[2] - KZ * b[1]), I * ik2 * (KZ * b[0] - KX * b[2]), I * ik2 * (KX * b[1] - KY * b[0])]
        return [(3 + c, A[c]) for c in range(3)]
    if kind == "th_advec":
        Fl = [rf(u[c] * th) for c in range(3)]
        return [(F - 1, -I * mask * (KX * Fl[0] + KY * Fl[1] + KZ * Fl[2]))]
    b2 = B[0] ** 2 + B[1] ** 2 + B[2] ** 2
    bs = B[p.strat_direction]
    if kind == "th_aniso_diss":
        g = [irf(I * K * U[-1]) for K in (KX, KY, KZ)]
        bg = B[0] * g[0] + B[1] * g[1] + B[2] * g[2]
        q = [rf(B[c] * bg / b2) for c in range(3)]
    else:
        q = [rf(B[c] * bs / b2) for c in range(3)]
    return [(F - 1, I * mask * (KX * q[0] + KY * q[1] + KZ * q[2]))]


@pytest.mark.parametrize("form", [0, SPK_FORM_FP32])
@pytest.mark.parametrize("kind", ["advec", "lorentz", "emfpower", "helicity", "th_advec", "th_aniso_diss",
                                  "th_aniso_inj"])
def test_transfer_spectra_match_numpy(kind, form):
    # a box whose shells have no mode exactly half-way between two bins (where
    # the bin of |k|/dk + 0.5 would depend on the last bit of the sum)
    p = default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                       gridsize=(32, 16, 24), boxsize=(1.07, 1.31, 0.97), reynolds_ani=20.0, N2=1.0, OmegaT2=1.0,
                       form=form)
    rng = np.random.default_rng(3)
    B = random_solenoidal(p, 8, kpeak=6.0)
    B[0] += 0.5
    U = to_spectral(np.concatenate([random_solenoidal(p, 7, kpeak=6.0), B, rng.standard_normal((1, 32, 16, 24))]))
    ctx = Context(p)
    ctx.set_state(U)
    E, dk, tot = ctx.transfer_spectra(kind)
    ref = transfer_ref(p, U, kind)
    assert E.shape[0] == len(ref)
    N = p.nx * p.ny * p.nz
    tol = 1e-10 if form == 0 else 2e-4
    for c, (f, T) in enumerate(ref):
        Er, dkr = spectrum_ref(U[f], T, p)
        assert abs(dk - dkr) < 1e-15
        scale = max(np.abs(Er).max(), 1e-300)
        assert np.abs(E[c] - Er).max() <= tol * scale, (kind, c, np.abs(E[c] - Er).max() / scale)
        # the total: the Parseval sum (weight 1 at kz = 0 and at the Nyquist
        # plane), the grid mean of field x term for a real term
        w = np.full(T.shape[2], 2.0)
        w[0] = w[-1] = 1.0
        t_ref = np.sum(w * np.real(U[f] * np.conj(T))) / N ** 2
        assert abs(tot[c] - t_ref) <= tol * max(abs(t_ref), np.abs(Er).sum()) + 1e-14
    # the state is left alone
    assert np.array_equal(ctx.get_state(), U)


def test_transfer_spectra_need_their_modules():
    from spooky_b200 import SpookyError
    p = default_params(incompressible=1, gridsize=(16, 16, 16))
    ctx = Context(p)
    ctx.set_state(to_spectral(random_solenoidal(p, 1)))
    assert ctx.transfer_spectra("advec")[0].shape[0] == 3
    for kind in ("lorentz", "emfpower", "helicity", "th_advec", "th_aniso_diss"):
        with pytest.raises(SpookyError):
            ctx.transfer_spectra(kind)
