"""The oracle's shearing box with rotation (TimeStepping::ShiftTime /
RemapField, Physics::BackgroundShear / BackgroundRotation,
GradPseudoPressureShearing, the sheared wavevector and the dt rule's
shearing terms), pinned by analytic solutions: the viscous shearing wave of
the reference's shearing-wave test across remaps, the epicyclic oscillation
of a mean flow, the projection's invariant, the remap rule and the dt rule."""
import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200.params import default_params

S, OM = 1.5, 1.0


def _params(n=16, **kw):
    base = dict(incompressible=1, gridsize=(n, n, n), boxsize=(1.0, 1.5, 1.0), reynolds=2000.0, shearing=1,
                rotating=1, shear=S, omega=OM, t_final=1e9, toutput_flow=1e9, safety_source=0.2, cfl=1.5)
    base.update(kw)
    return default_params(**base)


def test_remap_clock_follows_shift_time():
    p = _params()
    o = O.Oracle(p)
    assert o.tremap() == 0.0
    h = p.ly / (2 * S * p.lx)
    for t in (0.3, 0.7, 1.9, 5.25):
        o.set_time(t)
        assert abs(o.tremap() - ((t + h) % (2 * h) - h)) < 1e-15


def test_shearing_wave_decays_as_the_analytic_solution():
    """vz = cos(ky0 y): the mode stays a single shearing wave whose physical
    kx(t) = S t ky0 grows; it decays by exp(-nu (ky0^2 t + S^2 ky0^2 t^3/3))
    (check-shearing-wave.py:166-171) and hops one x index per remap."""
    p = _params(fixed_dt=0.004)
    o = O.Oracle(p)
    nzh = p.nz // 2 + 1
    U = np.zeros((3, p.nx, p.ny, nzh), complex)
    N = p.nx * p.ny * p.nz
    U[2, 0, 1, 0] = U[2, 0, -1, 0] = 0.5 * N          # cos(ky0 y)
    o.set_state(U)
    ky0, nu = 2 * np.pi / p.ly, p.nu
    h = p.ly / (2 * S * p.lx)
    t = 0.0
    for target in (0.4, 0.6, 1.4, 1.6, 2.0):
        nsteps = int(round((target - t) / 0.004))
        o.step(nsteps)
        t = o.get_time()[0]
        V = o.get_state()
        m = int(np.floor((t + h) / (2 * h)))            # remaps so far
        amp = 0.5 * N * np.exp(-nu * (ky0 ** 2 * t + S ** 2 * ky0 ** 2 * t ** 3 / 3))
        assert abs(V[2, m % p.nx, 1, 0] - amp) < 1e-7 * amp, (t, V[2, m % p.nx, 1, 0], amp)
        assert abs(V[2, (-m) % p.nx, -1, 0] - amp) < 1e-7 * amp
        rest = np.abs(V).copy()
        rest[2, m % p.nx, 1, 0] = rest[2, (-m) % p.nx, -1, 0] = 0
        assert rest.max() < 1e-12 * amp
        assert abs(o.tremap() - ((t + h) % (2 * h) - h)) < 1e-9


def test_mean_flow_oscillates_at_the_epicyclic_frequency():
    """A mean (k = 0) flow feels only the shear and the Coriolis force:
    vx'' = -kappa^2 vx, kappa^2 = 2 omega (2 omega - S)."""
    p = _params(n=8, fixed_dt=1e-3)
    o = O.Oracle(p)
    N = p.nx * p.ny * p.nz
    U = np.zeros((3, p.nx, p.ny, p.nz // 2 + 1), complex)
    U[0, 0, 0, 0] = 1e-3 * N
    o.set_state(U)
    kappa = np.sqrt(2 * OM * (2 * OM - S))
    o.step(1500)
    t = o.get_time()[0]
    V = o.get_state()
    assert abs(V[0, 0, 0, 0].real / N - 1e-3 * np.cos(kappa * t)) < 1e-10
    assert abs(V[1, 0, 0, 0].real / N - (-1e-3 * kappa / (2 * OM) * np.sin(kappa * t))) < 1e-10


def test_projection_keeps_the_sheared_divergence_free():
    """With kx(t) = kx0 + S t ky, d/dt (k.v) = S ky vx + k.dv: the shearing
    pressure makes it vanish at every mode."""
    p = _params(n=16)
    o = O.Oracle(p)
    o.set_time(0.31)
    U = to_spectral(np.stack(random_solenoidal(p, 3, kpeak=3.0)))
    o.set_state(U)
    o.clean_divergence()
    U = o.get_state()
    dU = o.compute_dfield(U)
    kvec, _, _ = o.kgrid()
    div = kvec[0] * dU[0] + kvec[1] * dU[1] + kvec[2] * dU[2] + S * kvec[1] * U[0]
    assert np.abs(div).max() < 1e-10 * np.abs(kvec[1] * U[0]).max()
    # the sheared wavevector
    k0 = 2 * np.pi / p.lx * np.fft.fftfreq(p.nx, 1.0 / p.nx)
    ky = 2 * np.pi / p.ly * np.fft.fftfreq(p.ny, 1.0 / p.ny)
    assert np.allclose(kvec[0], (k0[:, None] + S * o.tremap() * ky[None, :])[:, :, None], atol=1e-12)


def test_remap_moves_modes_by_ny():
    """A step of 1e-12 that crosses half a shear period: the state comes back
    remapped, mode (nx, ny) at nx + ny when that lies strictly inside
    (-NX/2, NX/2), then masked (RemapComplexVec, MaskVector)."""
    p = _params(n=16, fixed_dt=1e-12)
    o = O.Oracle(p)
    h = p.ly / (2 * S * p.lx)
    o.set_time(h - 5e-13)
    U = to_spectral(np.stack(random_solenoidal(p, 4, kpeak=2.0)))
    _, mask, _ = o.kgrid()
    o.set_state(U * mask)
    o.clean_divergence()                               # divergence-free for the sheared wavevector
    U = o.get_state()
    o.step(1)
    assert o.tremap() < 0                              # the clock restarted at -h
    nx = p.nx
    ix = np.fft.fftfreq(nx, 1.0 / nx).astype(int)
    iy = np.fft.fftfreq(p.ny, 1.0 / p.ny).astype(int)
    R = np.zeros_like(U)
    for i in range(nx):
        for j in range(p.ny):
            nt = ix[i] + iy[j]
            if -nx // 2 < nt < nx // 2:
                R[:, nt % nx, j] = U[:, i, j]
    R = R * mask
    V = o.get_state()
    assert np.abs(V - R).max() < 1e-9 * np.abs(R).max()
    assert np.abs(R - U).max() > 0.1 * np.abs(U).max()


def test_dt_counts_the_shear_and_rotation_rates():
    p = _params(n=16)
    o = O.Oracle(p)
    o.set_time(0.3)
    U = to_spectral(np.stack(random_solenoidal(p, 6, kpeak=3.0)))
    o.set_state(U)
    dt_hyp, dt_par, _, _ = o.compute_dt()
    R = np.fft.irfftn(U, axes=(1, 2, 3), s=(p.nx, p.ny, p.nz))
    kx, ky, kz = [2 * np.pi / l * (n // 2 - 1) * 2 / 3 for n, l in ((p.nx, p.lx), (p.ny, p.ly), (p.nz, p.lz))]
    kxs = kx + abs(o.tremap()) * ky
    m = np.abs(R).reshape(3, -1).max(1)
    gv = kxs * m[0] + ky * m[1] + kz * m[2] + abs(OM) / p.safety_source + abs(S) / p.safety_source
    assert abs(dt_hyp - p.cfl / gv) < 1e-12 * dt_hyp
    assert abs(dt_par - p.cfl_par / ((kxs ** 2 + ky ** 2 + kz ** 2) * p.nu)) < 1e-12 * dt_par


@pytest.mark.parametrize("every", [0, 1])
def test_shearing_wave_with_super_time_stepped_viscosity(every):
    """The shearing wave with its viscosity on an RKL2 cycle (alternating
    before / after the RK3 step, or after every step): the same analytic
    decay across two remaps.  The alternating cycle keeps second order
    (1e-6); a cycle after every step sees the wavevector of the step's end,
    a first-order lag of (dt/2) nu k^2 in the exponent (about 1.6e-4 at
    t = 2)."""
    p = _params(fixed_dt=0.004, supertimestepping=1, sts_algorithm="rkl2", sts_variables=["vx", "vy", "vz"],
                safety_sts=50, sts_every_step=every)
    assert p.supertimestepping == 1
    o = O.Oracle(p)
    nzh = p.nz // 2 + 1
    U = np.zeros((3, p.nx, p.ny, nzh), complex)
    N = p.nx * p.ny * p.nz
    U[2, 0, 1, 0] = U[2, 0, -1, 0] = 0.5 * N
    o.set_state(U)
    ky0, nu = 2 * np.pi / p.ly, p.nu
    h = p.ly / (2 * S * p.lx)
    o.step(500)
    t = o.get_time()[0]
    V = o.get_state()
    m = int(np.floor((t + h) / (2 * h)))
    amp = 0.5 * N * np.exp(-nu * (ky0 ** 2 * t + S ** 2 * ky0 ** 2 * t ** 3 / 3))
    tol = 1e-6 if every == 0 else 3e-4
    assert abs(V[2, m % p.nx, 1, 0] - amp) < tol * amp, (V[2, m % p.nx, 1, 0], amp)
