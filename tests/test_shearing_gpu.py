"""The shearing box with rotation on the GPU against its CPU oracle
(oracle/spk_oracle.c: ShiftTime, RemapField, BackgroundShear,
BackgroundRotation, GradPseudoPressureShearing, the sheared wavevector and
the dt rule), and the reference's shearing-wave test
(tests/shearing-wave/check-shearing-wave.py): 64^3 HD, S = 1.5, omega = 1,
vz = cos(ky0 y), snapshots every shear period to t = 10 through the command
line, each against the sheared, viscously decayed analytic wave (L1 < 1e-7)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200 import Context, fileCounter
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, cfg_text, default_params

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
S, OM = 1.5, 1.0


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _params(mhd, n=16, form=SPK_FORM_PLAIN, **kw):
    base = dict(incompressible=1, gridsize=(n, n, n), boxsize=(1.0, 1.5, 1.0), reynolds=2000.0, shearing=1,
                rotating=1, shear=S, omega=OM, t_final=1e9, toutput_flow=1e9, form=form)
    if mhd:
        base.update(mhd=1, reynolds_magnetic=1000.0)
    base.update(kw)
    return default_params(**base)


def _state(p, seed):
    fields = list(random_solenoidal(p, seed, kpeak=3.0))
    if p.mhd:
        fields += list(random_solenoidal(p, seed + 7, kpeak=3.0, rms=0.6))
    return to_spectral(np.stack(fields))


def _torch(U):
    import torch
    return torch.from_numpy(np.ascontiguousarray(U)).cuda()


def _aniso_params(form):
    """Boussinesq MHD with anisotropic conduction and stratification in the
    shearing box: the x-inverse pass forms d theta / dx with the sheared kx."""
    return _params(True, form=form, boussinesq=1, anisotropic_diffusion=1, stratification=1, strat_direction=2,
                   N2=0.3, OmegaT2=0.5, reynolds_ani=100.0, reynolds_thermic=1000.0)


def _bous_state(p, seed):
    U = _state(p, seed)
    th = to_spectral(np.stack(random_solenoidal(p, seed + 11, kpeak=2.0)))[:1]
    return np.concatenate([U, 0.3 * th])


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_sheared_anisotropic_conduction_rhs_matches_oracle(form):
    import torch
    p = _aniso_params(form)
    U = _bous_state(p, 9)
    o = O.Oracle(p)
    o.set_time(0.23)
    want = o.compute_dfield(U)
    ctx = Context(p)
    ctx.set_time(0.23)
    dU = torch.zeros(ctx.shape_c, dtype=torch.complex128, device="cuda")
    ctx.compute_dfield(_torch(U), dU)
    got = dU.cpu().numpy()
    assert rel_l2(got, want) < (1e-11 if form == SPK_FORM_PLAIN else 3e-5), rel_l2(got, want)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("mhd", [False, True])
def test_sheared_rhs_matches_oracle(mhd, form):
    import torch
    p = _params(mhd, form=form)
    U = _state(p, 3)
    o = O.Oracle(p)
    o.set_time(0.31)                       # a sheared wavevector
    want = o.compute_dfield(U)
    ctx = Context(p)
    ctx.set_time(0.31)
    dU = torch.zeros(ctx.shape_c, dtype=torch.complex128, device="cuda")
    ctx.compute_dfield(_torch(U), dU)
    got = dU.cpu().numpy()
    assert rel_l2(got, want) < (1e-12 if form == SPK_FORM_PLAIN else 2e-5), rel_l2(got, want)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("mhd", [False, True])
def test_steps_across_a_remap_match_oracle(mhd, form):
    """Ten steps from t = 0.45 at dt = 0.01: the remap clock passes half a
    shear period (0.5) at the fifth step and the fields are remapped."""
    p = _params(mhd, form=form, fixed_dt=0.01)
    U = _state(p, 5)
    o = O.Oracle(p)
    o.set_time(0.45)
    o.set_state(U)
    o.step(10)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.set_time(0.45)
    ctx.advance(10)
    ctx.synchronize()
    got, want = ctx.get_state(), o.get_state()
    assert abs(ctx.get_time()[0] - o.get_time()[0]) < 1e-14
    assert rel_l2(got, want) < (1e-11 if form == SPK_FORM_PLAIN else 1e-5), rel_l2(got, want)


def test_cfl_dt_matches_oracle():
    p = _params(True)
    U = _state(p, 7)
    o = O.Oracle(p)
    o.set_time(0.7)
    o.set_state(U)
    o.clean_divergence()
    want = o.compute_dt()
    ctx = Context(p)
    ctx.set_state(U)
    ctx.set_time(0.7)
    ctx.clean_divergence()
    got = ctx.compute_dt()
    for g, w in zip(got, want):
        assert g == w or abs(g - w) < 1e-12 * abs(w), (got, want)   # dt_sts: inf without STS


def test_reference_shearing_wave(tmp_path):
    import test_hdf5 as H
    n = 64
    p = default_params(incompressible=1, gridsize=(n, n, n), boxsize=(1.0, 1.5, 1.0), reynolds=2000.0, shearing=1,
                       rotating=1, shear=S, omega=OM, cfl=1.5, cfl_par=0.5, safety_source=0.2, t_final=10.0,
                       toutput_flow=1.0, antialiasing=1)
    lx, ly, lz = 1.0, 1.5, 1.0
    x = -lx / 2 + lx * np.arange(n) / n
    y = -ly / 2 + ly * np.arange(n) / n
    X, Y, _ = np.meshgrid(x, y, -lz / 2 + lz * np.arange(n) / n, indexing="ij")
    ky0 = 2 * np.pi / ly
    vz0 = np.cos(ky0 * Y)
    d = tmp_path
    (d / "data").mkdir()
    (d / "spooky.cfg").write_text(cfg_text(p, toutput_time=0.1).replace('output_dir = "./"', f'output_dir = "{d}"'))
    items = {"t_start": np.array([0.0]), "t_save": np.array([0.0]), "t_lastsnap": np.array([0.0]),
             "t_lastvar": np.array([0.0]), "step": np.array([0], dtype=np.int32),
             "vx": 0 * vz0.ravel(), "vy": 0 * vz0.ravel(), "vz": vz0.ravel()}
    H.h5_write(d / "data" / "snap0000.h5", items)
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "spooky-git_b200"))
    r = subprocess.run([sys.executable, "-m", "spooky_b200", "--input-dir", str(d), "-r", "0"], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    nsnap = fileCounter(str(d / "data"))
    assert nsnap == 10                     # t = 1, 2, ..., 10: one per shear period
    kyv = 2.0 * np.pi * np.fft.fftfreq(n, d=ly / n)
    KY = np.broadcast_to(kyv[None, :, None], X.shape)
    nu = 1.0 / 2000.0
    errs = []
    for i in range(1, nsnap + 1):
        R = H.h5_read(d / "data" / f"snap{i:04d}.h5", {k: (np.float64, n ** 3) for k in ("vx", "vy", "vz")} |
                      {"t_save": (np.float64, 1)})
        t = R["t_save"][0]
        assert abs(t - i) < 1e-12
        # check-shearing-wave.py:135-140, 166-180
        vz_an = np.real(np.fft.ifft(np.fft.fft(vz0, axis=1) * np.exp(1j * KY * X * S * t), axis=1))
        vz_an *= np.exp(-nu * (ky0 ** 2 * t + (1. / 3.) * S ** 2 * ky0 ** 2 * t ** 3))
        L1 = (np.abs(R["vx"]).sum() + np.abs(R["vy"]).sum() + np.abs(R["vz"] - vz_an.ravel()).sum()) / n ** 3
        errs.append(L1)
    assert max(errs) < 1e-7, errs


def test_reference_mri_eigenmode(tmp_path):
    """tests/mri-eigenmode/check-mri-eigenmode.py: 64^3 MHD shearing box
    (S = 1.5, omega = 1, Re = Rm = 3000) with a mean field B0z = 0.1 and the
    axisymmetric MRI eigenmode kX = 2 pi, kZ = 4 pi of amplitude 1e-4,
    through the command line to t = 1; every field against the eigenmode
    grown at its viscous-resistive rate (L1 < 1e-7)."""
    import test_hdf5 as H
    n = 64
    lx, ly, lz = 1.0, 1.5, 1.0
    p = default_params(incompressible=1, mhd=1, gridsize=(n, n, n), boxsize=(lx, ly, lz), reynolds=3000.0,
                       reynolds_magnetic=3000.0, shearing=1, rotating=1, shear=S, omega=OM, cfl=1.5, cfl_par=0.5,
                       safety_source=0.2, t_final=1.0, toutput_flow=1.0, antialiasing=1)
    # the eigenmode (check-mri-eigenmode.py:27-74)
    B0z, a = 0.1, 1e-4
    kZ, kX = 2.0 * 2.0 * np.pi / lz, 1.0 * 2.0 * np.pi / lx
    gamma2 = kZ * kZ / (kZ * kZ + kX * kX)
    kappa2 = 2 * OM * (2 * OM - S)
    omegaA2 = B0z * B0z * kZ * kZ
    omega_nu2 = omegaA2 + 0.5 * kappa2 * gamma2 * (1. - np.sqrt(1. + 16. * omegaA2 * OM * OM / (kappa2 * kappa2 * gamma2)))
    sigma_nu = np.sqrt(-omega_nu2)
    sigma = sigma_nu - (kX * kX + kZ * kZ) / 3000.0
    sigma_eta = sigma + (kX * kX + kZ * kZ) / 3000.0
    ax = [-l / 2 + l * np.arange(n) / n for l in (lx, ly, lz)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    ph = kX * X + kZ * Z
    vx0 = a * np.cos(ph)
    vy0 = vx0 * (S * omegaA2 / (sigma_eta * sigma_eta) - (2 * OM - S)) / (sigma_nu + omegaA2 / sigma_eta)
    vz0 = -(kX / kZ) * a * np.cos(ph)
    bx0 = -a * np.sin(ph) * B0z * kZ / sigma_eta
    by0 = bx0 * (-S / sigma_eta + (S * omegaA2 / (sigma_eta * sigma_eta) - (2 * OM - S)) / (sigma_nu + omegaA2 / sigma_eta))
    bz0 = B0z * (1.0 + (kX / kZ) * a * np.sin(ph) * kZ / sigma_eta)
    f0 = {"vx": vx0, "vy": vy0, "vz": vz0, "bx": bx0, "by": by0, "bz": bz0}
    d = tmp_path
    (d / "data").mkdir()
    (d / "spooky.cfg").write_text(cfg_text(p, toutput_time=0.1).replace('output_dir = "./"', f'output_dir = "{d}"'))
    items = {"t_start": np.array([0.0]), "t_save": np.array([0.0]), "t_lastsnap": np.array([0.0]),
             "t_lastvar": np.array([0.0]), "step": np.array([0], dtype=np.int32)}
    items.update({k: v.ravel() for k, v in f0.items()})
    H.h5_write(d / "data" / "snap0000.h5", items)
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "spooky-git_b200"))
    r = subprocess.run([sys.executable, "-m", "spooky_b200", "--input-dir", str(d), "-r", "0"], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    assert fileCounter(str(d / "data")) == 1
    R = H.h5_read(d / "data" / "snap0001.h5", {k: (np.float64, n ** 3) for k in f0} | {"t_save": (np.float64, 1)})
    t = R["t_save"][0]
    assert abs(t - 1.0) < 1e-12
    L1 = 0.0
    for k, v in f0.items():
        want = (v - (B0z if k == "bz" else 0.0)) * np.exp(sigma * t)   # ky = 0: shear_quantity is the identity
        got = R[k].reshape(n, n, n) - (B0z if k == "bz" else 0.0)
        L1 += np.abs(got - want).sum()
    L1 /= n ** 3
    assert L1 < 1e-7, L1
    # the mode grew: the check is not passed by a decayed field
    assert np.abs(R["vx"]).max() > 1.5 * a


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_super_time_stepped_shearing_box_matches_oracle(form):
    """MHD with RKL2 super-time-stepping of all six fields, alternating
    before and after the RK3 step, ten steps across a remap: the cycles run
    at the wavevector of the remap clock they meet."""
    p = _params(True, form=form, fixed_dt=0.01, supertimestepping=1, sts_algorithm="rkl2",
                sts_variables=["vx", "vy", "vz", "bx", "by", "bz"], safety_sts=50)
    U = _state(p, 21)
    o = O.Oracle(p)
    o.set_time(0.45)
    o.set_state(U)
    o.step(10)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.set_time(0.45)
    ctx.advance(10)
    ctx.synchronize()
    got, want = ctx.get_state(), o.get_state()
    assert rel_l2(got, want) < (1e-11 if form == SPK_FORM_PLAIN else 1e-5), rel_l2(got, want)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_anisotropic_conduction_cycle_in_the_shearing_box_matches_oracle(form):
    """Boussinesq MHD with anisotropic conduction, theta on an RKL2 cycle (the
    flux chain: sheared x derivative, staged real B, flux divergence with the
    sheared kx), ten steps across a remap."""
    p = _aniso_params(form)
    p.supertimestepping = 1
    p.sts_vars_mask = 1 << 6            # theta
    p.fixed_dt = 0.01
    p.safety_sts = 50
    U = _bous_state(p, 23)
    o = O.Oracle(p)
    o.set_time(0.45)
    o.set_state(U)
    o.step(10)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.set_time(0.45)
    ctx.advance(10)
    ctx.synchronize()
    got, want = ctx.get_state(), o.get_state()
    assert rel_l2(got, want) < (1e-10 if form == SPK_FORM_PLAIN else 2e-5), rel_l2(got, want)
