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
    assert vals[4] == -1.0    # not a quantity of this path
    # ev is half the Parseval total of the three components plus the Nyquist
    # plane once more: computeEnergy weights every kz > 0 plane by 2
    # (spooky_output_functions.cu:23-55)
    tot = sum(ctx.spectrum(q)[2] for q in ("vx", "vy", "vz"))
    N = p.nx * p.ny * p.nz
    nyq = 0.5 * np.sum(np.abs(U[:3, :, :, p.nz // 2]) ** 2) / N ** 2
    assert abs(e[:3].sum() - (0.5 * tot + nyq)) < 1e-12 * tot
