"""Pins the CPU FP64 oracle against numpy.fft, the reference's analytic
tests and the golden vectors generated from the reference's own Python.

Every check here runs on CPU (no GPU marker).  The reference checks restated:
  taylor-green-vortex  tests/taylor-green-vortex/check-taylor-green.py:129-155 (L1 < 1e-7)
  heat-diffusion       tests/heat-diffusion/check-heat-diffusion.py:157-166  (L1 < 1e-15)
  alfven-wave          tests/alfven-wave/check-alfven-wave.py:152-176        (L1 < 1e-7)
  mti-eigenmode        tests/mti-eigenmode/check-mti-eigenmode.py:171-200    (L1 < 1e-7)
  heat-diffusion-sts   tests/heat-diffusion-sts/check-heat-diffusion-sts.py: the L1 error at
                       t = 0.5 for sts, rkl1 and rkl2, tabulated against nx (first order in
                       dt for sts and rkl1, second order for rkl2)
  fft-forward-inverse  src/tests/tests.cu:18-137 (round trip)
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from fields import grid, kvectors, random_solenoidal, to_spectral
from spooky_b200.params import default_params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 8, 12, 16, 24, 32, 48, 64, 100, 128, 256, 7])
def test_fft1d_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    scale = max(np.abs(ref).max(), 1.0)
    assert np.abs(O.fft1d(x, -1) - ref).max() / scale < 1e-14
    assert np.abs(O.fft1d(x, +1) - np.fft.ifft(x) * n).max() / scale < 1e-14


@pytest.mark.parametrize("shape", [(16, 12, 8), (8, 8, 2), (32, 4, 4), (12, 10, 6)])
def test_r2c_c2r_match_numpy(shape):
    p = default_params(incompressible=1, gridsize=shape, boxsize=(1.0, 2.0, 3.0))
    o = O.Oracle(p)
    rng = np.random.default_rng(1)
    R = rng.standard_normal(shape)
    C = o.r2c(R)
    ref = np.fft.rfftn(R)
    assert np.abs(C - ref).max() / np.abs(ref).max() < 1e-14
    # c2r pre-scales by 1/N (cufft_routines.cu:30) -> round trip is identity
    assert np.abs(o.c2r(C) - R).max() < 1e-13


def test_fft_forward_inverse_round_trip_index_data():
    """src/tests/tests.cu:18-137 fills the real array with its index and
    checks D2Z then (scaled) Z2D returns it; restated at 64x32x16."""
    shape = (64, 32, 16)
    p = default_params(incompressible=1, gridsize=shape)
    o = O.Oracle(p)
    R = np.arange(np.prod(shape), dtype=np.float64).reshape(shape)
    R2 = o.c2r(o.r2c(R))
    assert np.abs(R2 - R).max() / R.max() < 1e-14


def test_wavevector_and_mask_reference_expressions():
    """Wavevector::Wavevector (src/fields/wavevector.cu:50-112), including the
    N=32 case where 2/3 kmax falls on an integer mode (|n| = 10)."""
    for n, L in ((32, 2 * np.pi), (32, 1.0), (128, 2 * np.pi), (24, 1.0)):
        p = default_params(incompressible=1, gridsize=(n, n, n), boxsize=(L, L, L))
        kvec, mask, km = O.Oracle(p).kgrid()
        i = np.arange(n)
        kx = (2.0 * np.pi) / L * (np.fmod(i + n / 2, n) - n / 2)
        assert np.array_equal(kvec[0][:, 0, 0], kx)
        kxmax = 2.0 * np.pi / L * (n // 2 - 1)
        keep = ~(np.abs(kx) > 2.0 / 3.0 * kxmax)
        assert np.array_equal(mask[:, 0, 0] == 1.0, keep)
        assert km[0] == (2.0 / 3.0) * kxmax
    # The boundary mode |n| = 2(N/2-1)/3 is decided by FP64 rounding of
    # fabs(kx) > 2.0/3.0*kxmax: at N=32 it is dropped for L=1 and kept for
    # L=2*pi; at N=128 (|n|=42) it is kept for both.
    for L, n, nb, kept in ((1.0, 32, 10, 0.0), (2 * np.pi, 32, 10, 1.0), (1.0, 128, 42, 1.0), (2 * np.pi, 128, 42, 1.0)):
        p = default_params(incompressible=1, gridsize=(n, n, n), boxsize=(L, L, L))
        _, mask, _ = O.Oracle(p).kgrid()
        assert mask[nb, 0, 0] == kept and mask[0, nb, 0] == kept and mask[0, 0, nb] == kept
        assert mask[nb + 1, 0, 0] == 0.0 and mask[nb - 1, 0, 0] == 1.0


def test_clean_divergence_projects():
    p = default_params(incompressible=1, mhd=1, gridsize=(16, 16, 16))
    o = O.Oracle(p)
    rng = np.random.default_rng(3)
    R = rng.standard_normal((6, 16, 16, 16))
    o.set_state(to_spectral(R))
    o.clean_divergence()
    U = o.get_state()
    KX, KY, KZ = kvectors(p)
    for v in (0, 3):
        div = KX * U[v] + KY * U[v + 1] + KZ * U[v + 2]
        assert np.abs(div).max() < 1e-10 * np.abs(U[v]).max() * 16


def test_dfield_leray_projected_and_antialiased():
    p = default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, gridsize=(16, 16, 16),
                       reynolds=100.0, reynolds_magnetic=100.0, reynolds_thermic=100.0, N2=0.3)
    o = O.Oracle(p)
    rng = np.random.default_rng(4)
    U = to_spectral(rng.standard_normal((7, 16, 16, 16)))
    dU = o.compute_dfield(U)
    KX, KY, KZ = kvectors(p)
    div = KX * dU[0] + KY * dU[1] + KZ * dU[2]
    assert np.abs(div).max() < 1e-9 * np.abs(dU[0]).max()


def test_taylor_green_decay():
    n = 16
    p = default_params(incompressible=1, gridsize=(n, n, n), reynolds=200.0, t_final=1.0, toutput_flow=1.0)
    X, Y, Z = grid(p)
    u0 = np.stack([0 * X, np.sin(2 * np.pi * Y) * np.cos(2 * np.pi * Z), -np.cos(2 * np.pi * Y) * np.sin(2 * np.pi * Z)])
    o = O.Oracle(p)
    o.set_state(to_spectral(u0))
    while o.get_time()[0] < p.t_final:
        o.step(1)
    t = o.get_time()[0]
    ua = u0 * np.exp(-2 * p.nu * t * (2 * np.pi) ** 2)
    assert abs(t - 1.0) < 1e-15
    assert np.abs(o.to_real() - ua).sum() / n ** 3 < 1e-7


def _run_with_snapshots(o, p):
    """Main loop with the reference's snapshot bookkeeping: t_lastsnap
    advances by toutput_flow when a snapshot is due (check_output.cu:63-93)."""
    while o.get_time()[0] < p.t_final:
        o.step(1)
        t, _, st = o.get_time()
        _, _, _ = t, _, st
        if t - o._lastsnap + 1e-8 >= p.toutput_flow:
            o._lastsnap += p.toutput_flow
            o.set_time(t, st, o._lastsnap)


def test_heat_diffusion_rk3_golden():
    """Matches the reference's own numpy RK3 (golden) at t=10 to L1 < 1e-15."""
    g = np.load(os.path.join(GOLDEN, "heat_diffusion_rk3.npz"))
    nx = int(g["nx"])
    p = default_params(heat_equation=1, gridsize=(nx, 2, 2), reynolds_thermic=1000.0, cfl=1.5, cfl_par=1.5,
                       antialiasing=0, t_final=10.0, toutput_flow=5.0)
    X, _, _ = grid(p)
    a = 0.01
    T0 = 1.0 + 0.5 * (np.tanh((X + 0.375) / a) - np.tanh((X + 0.125) / a)) + 0.5 * (
        np.tanh((X - 0.125) / a) - np.tanh((X - 0.375) / a))
    assert np.abs(T0[:, 0, 0] - g["T"][0]).max() == 0.0
    o = O.Oracle(p)
    o.set_state(to_spectral(T0[None]))
    o._lastsnap = 0.0
    _run_with_snapshots(o, p)
    assert o.get_time()[0] == 10.0
    T = o.to_real()[0]
    assert np.all(T == T[:, :1, :1])
    L1 = np.abs(g["T"][-1] - T[:, 0, 0]).sum() / (nx * 4)
    assert L1 < 1e-15, L1


def test_advected_mhd_vortex_first_snapshot():
    """tests/advected-mhd-vortex (512x512x2, box 1, nu = eta = 1e-4, CFL 1.5):
    the vortex and its field loop advected by (0.05, 0.05); L1 over the six
    fields / N against the advected profile < 1e-4 (check-advected-mhd-vortex.py:
    11-66, 181-197), here at the first snapshot, t = 0.2."""
    p = default_params(incompressible=1, mhd=1, gridsize=(512, 512, 2), boxsize=(1.0, 1.0, 1.0), reynolds=1e4,
                       reynolds_magnetic=1e4, cfl=1.5, t_final=1.1, toutput_flow=0.2)
    X, Y, _ = grid(p)

    def profile(t):
        Xt, Yt = X - 0.05 * t, Y - 0.05 * t
        e = np.exp((1.0 - 200.0 * (Xt ** 2 + Yt ** 2)) / 2.0) / (2.0 * np.pi)
        return np.stack([0.05 - e * Yt, 0.05 + e * Xt, 0 * X, -e * Yt, e * Xt, 0 * X])

    o = O.Oracle(p)
    o.set_state(to_spectral(profile(0.0)))
    o.clean_divergence()
    while True:
        o.step(1)
        t = o.get_time()[0]
        if t + 1e-8 >= p.toutput_flow:
            break
    assert abs(t - 0.2) < 1e-14
    L1 = np.abs(o.to_real() - profile(t)).sum() / (512 * 512 * 2)
    assert L1 < 1e-4, L1


def test_alfven_wave():
    n = 32
    p = default_params(incompressible=1, mhd=1, gridsize=(n, n, n), reynolds=1e4, reynolds_magnetic=1e4,
                       t_final=1.0, toutput_flow=0.1)
    X, Y, Z = grid(p)
    vx0 = np.real(1e-5 * np.exp(1j * 2 * np.pi * Z - 1j * np.pi / 2))
    f0 = np.stack([vx0, 0 * X, 0 * X, -vx0, 0 * X, np.ones_like(X)])
    o = O.Oracle(p)
    o.set_state(to_spectral(f0))
    o._lastsnap = 0.0
    _run_with_snapshots(o, p)
    t = o.get_time()[0]
    fa = f0.copy()
    fa[0] *= np.cos(2 * np.pi * t)
    fa[3] *= np.cos(2 * np.pi * t)
    assert np.abs(o.to_real() - fa).sum() / n ** 3 < 1e-7


def _mti_setup(t_final):
    g = json.load(open(os.path.join(GOLDEN, "mti_eigenmode.json")))
    nx, ny, nz = g["grid"]
    sigma = g["sigma_check_script"]
    kpar = 2 * np.pi * g["n_mode"]
    B0, N2, Pe, Reeta = g["B0"], g["N2"], g["Pe"], g["ReEta"]
    p = default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                       gridsize=(nx, ny, nz), reynolds=g["ReNu"], reynolds_magnetic=Reeta,
                       reynolds_thermic=g["reynolds_thermic"], reynolds_ani=Pe, N2=N2, OmegaT2=g["OmegaT2"],
                       t_final=t_final, toutput_flow=100.0)
    X, _, _ = grid(p)
    vz0 = -1e-5 * np.sin(kpar * X)
    bz0 = -1e-5 * np.cos(kpar * X) * B0 * kpar / (sigma + kpar ** 2 / Reeta)
    th0 = 1.0 / (sigma + kpar ** 2 / Pe) * (N2 - kpar ** 2 / Pe / (sigma + kpar ** 2 / Reeta)) * vz0
    f0 = np.stack([0 * X, 0 * X, vz0, B0 * np.ones_like(X), 0 * X, bz0, th0])
    return p, f0, sigma, g


def test_mti_dispersion_cubic_matches_golden():
    """Own restatement of the MTI dispersion cubic (mti_disp_rel.py:44-70)."""
    g = json.load(open(os.path.join(GOLDEN, "mti_eigenmode.json")))
    Pe, ReNu, ReEta, B0, N2 = g["Pe"], g["ReNu"], g["ReEta"], g["B0"], g["N2"]
    Pr, q, Lam = Pe / ReNu, Pe / ReEta, B0 ** 2 * Pe
    k2 = (2 * np.pi * g["n_mode"]) ** 2 / Pe
    roots = np.roots([1.0, k2 * (1 + q + Pr), N2 + k2 * Lam + (q + Pr) * k2 ** 2 + q * Pr * k2 ** 2,
                      q * Pr * k2 ** 3 + N2 * q * k2 + Lam * k2 ** 2 - k2])
    sigma = np.max(np.real(roots[np.imag(roots) == 0]))
    assert abs(sigma - g["sigma_dispersion_cubic"]) < 1e-12
    assert abs(sigma - g["sigma_check_script"]) < 1e-12


def test_mti_eigenmode_growth():
    p, f0, sigma, g = _mti_setup(t_final=0.04)
    o = O.Oracle(p)
    o.set_state(to_spectral(f0))
    while o.get_time()[0] < p.t_final:
        o.step(1)
    t = o.get_time()[0]
    fa = f0.copy()
    for f in (2, 5, 6):
        fa[f] *= np.exp(sigma * t)
    R = o.to_real()
    assert np.abs(R - fa).sum() / np.prod(g["grid"]) < g["tolerance_L1"]
    amp = np.abs(np.fft.rfftn(R[2])).max() / np.abs(np.fft.rfftn(f0[2])).max()
    assert abs(np.log(amp) / t - sigma) < 1e-4


def _heat_sts_l1(alg, nx):
    """heat-diffusion-sts: forward Euler at dt = 0.002 lx/nx plus one
    super-time-stepping cycle every step (the reference's test build,
    tests/heat-diffusion-sts/hydro_mhd_advance.cu and compute_dt.cu:57-62);
    L1 distance to the analytic decay at t = 0.5."""
    lx = 4.0
    p = default_params(heat_equation=1, gridsize=(nx, 2, 2), boxsize=(lx, 1.0, 1.0), reynolds_thermic=1.0,
                       cfl_par=0.5, safety_sts=1, t_final=0.5, toutput_flow=0.1, antialiasing=0,
                       supertimestepping=1, sts_algorithm=alg, sts_variables=["th"], integrator=1,
                       sts_every_step=1, fixed_dt=0.002 * lx / nx)
    X, _, _ = grid(p)
    T0 = 1.0 / np.sqrt(2 * np.pi * 0.01) * np.exp(-0.5 * X ** 2 / 0.01)
    o = O.Oracle(p)
    o.set_state(to_spectral(T0[None]))
    o._lastsnap = 0.0
    _run_with_snapshots(o, p)
    t = o.get_time()[0]
    assert abs(t - 0.5) < 1e-12
    KX, _, _ = kvectors(p)
    Ta = np.fft.irfftn(np.fft.rfftn(T0) * np.exp(-KX ** 2 * t), s=T0.shape, axes=(0, 1, 2))
    return np.abs(o.to_real()[0] - Ta).sum() / (nx * 4)


# L1 bound at nx = 256 and the error ratio from nx = 128 to 256 (order 1: ~2, order 2: ~4)
HEAT_STS = {"sts": (4e-6, (1.8, 2.2)), "rkl1": (3.5e-6, (1.8, 2.2)), "rkl2": (1.5e-10, (3.6, 4.4))}


@pytest.mark.parametrize("alg", sorted(HEAT_STS))
def test_heat_diffusion_sts_convergence(alg):
    bound, (lo, hi) = HEAT_STS[alg]
    e128, e256 = _heat_sts_l1(alg, 128), _heat_sts_l1(alg, 256)
    assert e256 < bound, e256
    assert lo < e128 / e256 < hi, (e128, e256)


def _single_mode_cycle(alg, ratio, m=11, nx=64, lx=4.0):
    """One super-time-stepping cycle of dt = ratio * dt_sts applied to the
    single mode kx = 2 pi m / lx of the heat equation: returns the stage
    count, dt and the amplification of the mode."""
    kw = dict(heat_equation=1, gridsize=(nx, 2, 2), boxsize=(lx, 1.0, 1.0), reynolds_thermic=1.0, cfl_par=0.5,
              t_final=1e9, toutput_flow=1e9, antialiasing=0, supertimestepping=1, sts_algorithm=alg,
              sts_variables=["th"], integrator=1, sts_every_step=1)
    dt_sts = O.Oracle(default_params(fixed_dt=1e-3, **kw)).compute_dt()[2]
    o = O.Oracle(default_params(fixed_dt=ratio * dt_sts, **kw))
    U = np.zeros((1, nx, 2, 2), complex)
    U[0, m, 0, 0] = 1.0
    o.set_state(U)
    dt = o.compute_dt()[3]
    s = o.rkl_cycle()
    return s, dt, o.get_state()[0, m, 0, 0], -(2 * np.pi / lx * m) ** 2 * dt


@pytest.mark.parametrize("ratio", [1.0, 3.7, 20.0, 100.0])
@pytest.mark.parametrize("alg", ["sts", "rkl1", "rkl2"])
def test_sts_cycle_matches_stability_polynomial(alg, ratio):
    """A cycle multiplies the mode exp(i k x) by the scheme's stability
    polynomial R(z), z = -nu k^2 dt:
      rkl1  P_s(1 + w1 z), w1 = 2/(s^2+s)             (Meyer, Balsara & Aslam 2014, RKL1)
      rkl2  a_s + b_s P_s(1 + w1 z), w1 = 4/(s^2+s-2),
            b_s = (s^2+s-2)/(2s(s+1)), a_s = 1 - b_s    (the same paper, RKL2)
      sts   prod_i (1 + tau_i z / dt) over the sub-steps tau_i of
            Alexiades, Amiez & Gremaud 1996, whose sum is dt."""
    from numpy.polynomial import legendre
    s, dt, got, z = _single_mode_cycle(alg, ratio)
    if alg == "rkl1":
        assert s == 1 + int(4 * ratio / (1 + np.sqrt(1 + 8 * ratio)) + 1e-12)
        want = legendre.legval(1 + 2 / (s * s + s) * z, [0] * s + [1])
    elif alg == "rkl2":
        assert s == 1 + int(4 * (1 + 2 * ratio) / (1 + np.sqrt(9 + 16 * ratio)) + 1e-12)
        b = (s * s + s - 2) / (2 * s * (s + 1))
        want = 1 - b + b * legendre.legval(1 + 4 / (s * s + s - 2) * z, [0] * s + [1])
    else:
        nu = 1e-3
        a = (1 - np.sqrt(nu)) / (1 + np.sqrt(nu))
        c = (1 - a ** (2 * s)) / (1 + a ** (2 * s))
        if s > 1:
            tau = dt * 2 * np.sqrt(nu) / (s * c) / ((nu - 1) * np.cos((2 * np.arange(s) + 1) * np.pi / (2 * s)) + 1 + nu)
        else:
            tau = np.array([dt])
        assert abs(tau.sum() / dt - 1) < 1e-13
        # the sub-step count grows like sqrt(dt/dt_sts) at first
        assert s >= 2 and s <= 2 + 2 * np.sqrt(ratio)
        want = np.prod(1 + tau * z / dt)
    assert abs(got - want) < 1e-13, (s, got, want)


def test_energy_budget_matches_real_space():
    p = default_params(incompressible=1, gridsize=(16, 16, 16))
    o = O.Oracle(p)
    R = random_solenoidal(p, seed=5)
    o.set_state(to_spectral(R))
    e, _ = o.budgets()
    assert np.allclose(e, 0.5 * np.mean(R ** 2, axis=(1, 2, 3)), rtol=1e-12)
