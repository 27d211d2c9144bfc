"""GPU parity: the CUDA path (through the C ABI) against the CPU FP64 oracle.

Tolerances (relative L2 over the whole state):
  plain form (FP64 passes): 1e-12 for one RHS, 1e-10 after many steps
  FP32 form (FP32 passes, FP64 state): 2e-5 for one RHS, 1e-4 after tens of steps
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from fields import grid, kvectors, random_solenoidal, to_spectral
from spooky_b200 import Context, SpookyError, Supervisor
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, default_params

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TOL_RHS = {SPK_FORM_PLAIN: 1e-12, SPK_FORM_FP32: 2e-5}
TOL_RUN = {SPK_FORM_PLAIN: 1e-10, SPK_FORM_FP32: 1e-4}


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def torch_dev(arr):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
    torch.cuda.synchronize()
    return t


CASES = {
    "hd": dict(incompressible=1, reynolds=100.0),
    "mhd": dict(incompressible=1, mhd=1, reynolds=100.0, reynolds_magnetic=50.0),
    "bous": dict(incompressible=1, boussinesq=1, stratification=1, reynolds=100.0, reynolds_thermic=80.0,
                 N2=0.5, strat_direction=2),
    "bous_mhd_aniso": dict(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                           reynolds=100.0, reynolds_magnetic=100.0, reynolds_thermic=100.0, reynolds_ani=20.0,
                           N2=1.0, OmegaT2=1.0, strat_direction=2),
    "bous_mhd_x": dict(incompressible=1, mhd=1, boussinesq=1, stratification=1, reynolds=300.0,
                       reynolds_magnetic=200.0, reynolds_thermic=100.0, N2=-0.3, strat_direction=0),
}


def make_state(p, seed):
    """Random solenoidal u, B (+ B0) and a random theta, in spectral layout."""
    fields = []
    if p.incompressible:
        fields += list(random_solenoidal(p, seed, kpeak=3.0))
    if p.mhd:
        B = random_solenoidal(p, seed + 100, kpeak=3.0, rms=0.7)
        B[0] += 0.3
        fields += list(B)
    if p.boussinesq:
        rng = np.random.default_rng(seed + 200)
        fields.append(0.3 * rng.standard_normal((p.nx, p.ny, p.nz)))
    return to_spectral(np.stack(fields))


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 16, 8)])
def test_compute_dfield_matches_oracle(case, shape, form):
    p = default_params(gridsize=shape, boxsize=(1.0, 1.5, 2.0), form=form, **CASES[case])
    U = make_state(p, seed=11)
    ref = O.Oracle(p).compute_dfield(U)
    ctx = Context(p)
    Ud = torch_dev(U)
    dUd = torch_dev(np.zeros_like(U))
    ctx.compute_dfield(Ud, dUd)
    ctx.synchronize()
    assert rel_l2(dUd.cpu().numpy(), ref) < TOL_RHS[form]


# Long axes: every transform length from 2 to 1024 and every stage layout of
# the register FFT (one stage, full stages, full stages + a radix-2/4/8 tail,
# and the 3*2^k lengths) along x, y and z, in both precisions.
LONG_SHAPES = [(256, 32, 16), (32, 256, 8), (1024, 8, 4), (8, 512, 16), (128, 64, 2), (16, 8, 512),
               (64, 16, 1024), (4, 2, 256),
               # 3*2^k lengths: a radix-3 stage, radix-4 stages, a radix-2 tail
               (24, 48, 12), (96, 6, 24), (12, 192, 48), (6, 12, 384), (768, 6, 6), (48, 384, 6)]


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("shape", LONG_SHAPES)
def test_compute_dfield_long_axes_matches_oracle(shape, form):
    case = "bous_mhd_aniso" if shape[0] * shape[1] * shape[2] <= 65536 else "mhd"
    p = default_params(gridsize=shape, boxsize=(1.0, 1.5, 2.0), form=form, **CASES[case])
    U = make_state(p, seed=17)
    ref = O.Oracle(p).compute_dfield(U)
    ctx = Context(p)
    Ud = torch_dev(U)
    dUd = torch_dev(np.zeros_like(U))
    ctx.compute_dfield(Ud, dUd)
    ctx.synchronize()
    assert rel_l2(dUd.cpu().numpy(), ref) < TOL_RHS[form]


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 8, 16), (8, 8, 2)])
def test_to_real_matches_oracle(shape, form):
    p = default_params(incompressible=1, mhd=1, gridsize=shape, form=form)
    U = make_state(p, seed=3)
    o = O.Oracle(p)
    o.set_state(U)
    ctx = Context(p)
    ctx.set_state(U)
    import torch
    R = torch.zeros(ctx.shape_r, dtype=torch.float64, device="cuda")
    ctx.to_real(R)
    ctx.synchronize()
    assert rel_l2(R.cpu().numpy(), o.to_real()) < (1e-13 if form == SPK_FORM_PLAIN else 1e-6)


@pytest.mark.parametrize("case", ["hd", "mhd", "bous_mhd_aniso"])
def test_compute_dt_matches_oracle(case):
    p = default_params(gridsize=(16, 16, 16), **CASES[case])
    U = make_state(p, seed=5)
    o = O.Oracle(p)
    o.set_state(U)
    ref = o.compute_dt()
    ctx = Context(p)
    ctx.set_state(U)
    got = ctx.compute_dt()
    assert np.allclose(got, ref, rtol=1e-13, atol=0)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("case", sorted(CASES))
def test_rk3_steps_match_oracle(case, form):
    p = default_params(gridsize=(16, 16, 16), form=form, t_final=100.0, toutput_flow=100.0, **CASES[case])
    U = make_state(p, seed=21)
    o = O.Oracle(p)
    o.set_state(U)
    o.step(10)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(10)
    ctx.synchronize()
    t, dt, step = ctx.get_time()
    to, dto, _ = o.get_time()
    assert step == 10
    assert abs(t - to) / to < (1e-12 if form == SPK_FORM_PLAIN else 1e-5)
    assert rel_l2(ctx.get_state(), o.get_state()) < TOL_RUN[form]


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("case", ["hd", "mhd"])
def test_rk3_with_dealiased_out_content_matches_oracle(case, form):
    """A state with O(1) content outside the 2/3 mask: those modes only
    diffuse, and the RK3 step handles them apart from the kept ones (kept
    modes only in stages 0 and 1, the whole step's amplification in stage 2,
    the stage values in the x-inverse passes); the result follows the oracle's
    staged update."""
    L = 2 * np.pi
    p = default_params(gridsize=(16, 16, 16), boxsize=(L, L, L), form=form, t_final=100.0, toutput_flow=100.0,
                       **CASES[case])
    fields = list(random_solenoidal(p, 31, kpeak=7.0))
    if p.mhd:
        fields += list(random_solenoidal(p, 32, kpeak=7.0, rms=0.5))
    U = to_spectral(np.stack(fields))
    _, mask, _ = O.Oracle(p).kgrid()
    outside = np.linalg.norm((U * (1 - mask)).ravel()) / np.linalg.norm(U.ravel())
    assert outside > 0.3
    o = O.Oracle(p)
    o.set_state(U)
    o.step(10)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(10)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < TOL_RUN[form]
    Ug, Uo = ctx.get_state(), o.get_state()
    assert rel_l2(Ug * (1 - mask), Uo * (1 - mask)) < TOL_RUN[form]


def test_config1_taylor_green_32_fixed_dt_100_steps():
    """32^3 HD, box 2pi, nu=0.01, u0 = (sin x cos y cos z, -cos x sin y cos z, 0),
    RK3 at dt=1e-3 for 100 steps: rel L2 of u vs the FP64 oracle <= 1e-10 and the
    kinetic-energy decay matches."""
    L = 2 * np.pi
    p = default_params(incompressible=1, gridsize=(32, 32, 32), boxsize=(L, L, L), reynolds=100.0,
                       fixed_dt=1e-3, t_final=1.0, toutput_flow=10.0)
    X, Y, Z = grid(p)
    u0 = np.stack([np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), 0 * X])
    U = to_spectral(u0)
    o = O.Oracle(p)
    o.set_state(U)
    o.step(100)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(100)
    ctx.synchronize()
    assert abs(ctx.get_time()[0] - 0.1) < 1e-12
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-10
    e_gpu, _ = ctx.budgets()
    e_orc, _ = o.budgets()
    assert np.allclose(e_gpu, e_orc, rtol=1e-10)


def test_config2_mhd128_fp32_form_within_1e5_of_fp64_after_1000_steps():
    """128^3 MHD, box 2pi, nu=eta=1e-3, B0=0.1z, CFL 1.5, random solenoidal u, B
    with E(k) ~ k^4 exp(-2(k/4)^2), rms 1 (seeds 1, 2).  The plain form follows
    the FP64 oracle (3 steps, rel L2 <= 1e-10); after 1000 steps the FP32 form is
    within rel L2 1e-5 of the plain form and its total energy within 1e-6."""
    from spooky_b200.initial import mhd_random_state
    L = 2 * np.pi
    kw = dict(incompressible=1, mhd=1, gridsize=(128, 128, 128), boxsize=(L, L, L), reynolds=1e3,
              reynolds_magnetic=1e3, cfl=1.5, t_final=1e30, toutput_flow=1e30)
    p64 = default_params(form=SPK_FORM_PLAIN, **kw)
    p32 = default_params(form=SPK_FORM_FP32, **kw)
    U0 = mhd_random_state(p64)
    o = O.Oracle(p64)
    o.set_state(U0)
    o.step(3)
    c64, c32 = Context(p64), Context(p32)
    c64.set_state(U0)
    c32.set_state(U0)
    c64.advance(3)
    assert rel_l2(c64.get_state(), o.get_state()) < 1e-10
    c64.advance(997)
    c32.advance(1000)
    c64.synchronize()
    c32.synchronize()
    assert rel_l2(c32.get_state(), c64.get_state()) < 1e-5
    e32, _ = c32.budgets()
    e64, _ = c64.budgets()
    assert abs(np.sum(e32) - np.sum(e64)) / np.sum(e64) < 1e-6


def test_taylor_green_reference_check():
    """tests/taylor-green-vortex/check-taylor-green.py:129-155 at 32^3 (L1 < 1e-7)."""
    n = 32
    p = default_params(incompressible=1, gridsize=(n, n, n), reynolds=200.0, t_final=1.0, toutput_flow=1.0)
    X, Y, Z = grid(p)
    u0 = np.stack([0 * X, np.sin(2 * np.pi * Y) * np.cos(2 * np.pi * Z), -np.cos(2 * np.pi * Y) * np.sin(2 * np.pi * Z)])
    sup = Supervisor(p)
    sup.fields.set(to_spectral(u0))
    sup.executeMainLoop()
    t = sup.timestep.current_time
    import torch
    R = torch.zeros(sup.ctx.shape_r, dtype=torch.float64, device="cuda")
    sup.ctx.to_real(R)
    ua = u0 * np.exp(-2 * p.nu * t * (2 * np.pi) ** 2)
    assert abs(t - 1.0) < 1e-14
    assert np.abs(R.cpu().numpy() - ua).sum() / n ** 3 < 1e-7


def test_mti_eigenmode_growth_rate():
    """tests/mti-eigenmode: 512x4x4 Boussinesq-MHD with anisotropic conduction;
    the GPU run follows exp(sigma t) (L1 < 1e-7) and the oracle to 1e-10."""
    g = json.load(open(os.path.join(GOLDEN, "mti_eigenmode.json")))
    nx, ny, nz = g["grid"]
    sigma = g["sigma_check_script"]
    kpar = 2 * np.pi * g["n_mode"]
    B0, N2, Pe, Reeta = g["B0"], g["N2"], g["Pe"], g["ReEta"]
    p = default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                       gridsize=(nx, ny, nz), reynolds=g["ReNu"], reynolds_magnetic=Reeta,
                       reynolds_thermic=g["reynolds_thermic"], reynolds_ani=Pe, N2=N2, OmegaT2=g["OmegaT2"],
                       t_final=0.5, toutput_flow=100.0)
    X, _, _ = grid(p)
    vz0 = -1e-5 * np.sin(kpar * X)
    bz0 = -1e-5 * np.cos(kpar * X) * B0 * kpar / (sigma + kpar ** 2 / Reeta)
    th0 = 1.0 / (sigma + kpar ** 2 / Pe) * (N2 - kpar ** 2 / Pe / (sigma + kpar ** 2 / Reeta)) * vz0
    f0 = np.stack([0 * X, 0 * X, vz0, B0 * np.ones_like(X), 0 * X, bz0, th0])
    sup = Supervisor(p)
    sup.fields.set(to_spectral(f0))
    sup.executeMainLoop()
    t = sup.timestep.current_time
    import torch
    R = torch.zeros(sup.ctx.shape_r, dtype=torch.float64, device="cuda")
    sup.ctx.to_real(R)
    R = R.cpu().numpy()
    fa = f0.copy()
    for f in (2, 5, 6):
        fa[f] *= np.exp(sigma * t)
    assert np.abs(R - fa).sum() / (nx * ny * nz) < g["tolerance_L1"]
    amp = np.abs(np.fft.rfftn(R[2])).max() / np.abs(np.fft.rfftn(f0[2])).max()
    assert abs(np.log(amp) / t - sigma) < 1e-4


def _heat_sts_params(nx, alg="rkl2", **kw):
    lx = 4.0
    kw.setdefault("fixed_dt", 0.002 * lx / nx)
    return default_params(heat_equation=1, gridsize=(nx, 2, 2), boxsize=(lx, 1.0, 1.0), reynolds_thermic=1.0,
                          cfl_par=0.5, safety_sts=1, t_final=0.5, toutput_flow=100.0, antialiasing=0,
                          supertimestepping=1, sts_algorithm=alg, sts_variables=["th"], integrator=1,
                          sts_every_step=1, **kw)


# analytic L1 bound at t = 0.5 (the oracle's own errors at nx = 256 are
# 3.5e-6, 3.1e-6 and 1.1e-10: first order for sts and rkl1, second for rkl2)
HEAT_STS_L1 = {"sts": 4e-6, "rkl1": 3.5e-6, "rkl2": 1e-7}


@pytest.mark.parametrize("alg", ["sts", "rkl1", "rkl2"])
def test_sts_heat_diffusion_matches_oracle_and_analytic(alg):
    nx = 256
    p = _heat_sts_params(nx, alg)
    X, _, _ = grid(p)
    T0 = 1.0 / np.sqrt(2 * np.pi * 0.01) * np.exp(-0.5 * X ** 2 / 0.01)
    U = to_spectral(T0[None])
    o = O.Oracle(p)
    o.set_state(U)
    o.step(200)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(200)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-12
    # run to t_final and compare with the analytic decay
    sup = Supervisor(p)
    sup.fields.set(U)
    sup.executeMainLoop()
    t = sup.timestep.current_time
    assert abs(t - 0.5) < 1e-12
    KX, _, _ = kvectors(p)
    Ta = np.fft.irfftn(np.fft.rfftn(T0) * np.exp(-KX ** 2 * t), s=T0.shape, axes=(0, 1, 2))
    Tg = np.fft.irfftn(sup.ctx.get_state()[0], s=T0.shape, axes=(0, 1, 2))
    assert np.abs(Tg - Ta).sum() / (nx * 4) < HEAT_STS_L1[alg]


@pytest.mark.parametrize("alg", ["sts", "rkl1", "rkl2"])
def test_sts_cycle_stage_count_matches_oracle(alg):
    """spk_rkl_cycle reports the stage count the device computed; it equals
    the oracle's for the same dt / dt_sts."""
    p = _heat_sts_params(64, alg, fixed_dt=0.05)
    U = to_spectral(np.random.default_rng(3).standard_normal((1, 64, 2, 2)))
    o = O.Oracle(p)
    o.set_state(U)
    o.compute_dt()
    s_or = o.rkl_cycle()
    ctx = Context(p)
    ctx.set_state(U)
    ctx.compute_dt()
    s_gpu = ctx.rkl_cycle()
    ctx.synchronize()
    assert s_gpu == s_or and s_or > 3
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-12


@pytest.mark.parametrize("alg", ["sts", "rkl1", "rkl2"])
@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_sts_anisotropic_matches_oracle(form, alg):
    """Boussinesq-MHD with anisotropic conduction super-time-stepped,
    alternating before/after RK3 (hydro_mhd_advance.cu:43-64)."""
    p = default_params(gridsize=(16, 16, 16), form=form, t_final=100.0, toutput_flow=100.0,
                       supertimestepping=1, sts_algorithm=alg, sts_variables=["th"], safety_sts=10, cfl_par=1.0,
                       **CASES["bous_mhd_aniso"])
    U = make_state(p, seed=31)
    o = O.Oracle(p)
    o.set_state(U)
    o.step(6)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(6)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < TOL_RUN[form]


@pytest.mark.parametrize("alg", ["sts", "rkl1", "rkl2"])
def test_isotropic_sts_velocity_matches_oracle(alg):
    p = default_params(gridsize=(16, 16, 16), t_final=100.0, toutput_flow=100.0, supertimestepping=1,
                       sts_algorithm=alg, sts_variables=["vx", "vy", "vz", "th"], safety_sts=5, **CASES["bous"])
    U = make_state(p, seed=41)
    o = O.Oracle(p)
    o.set_state(U)
    o.step(4)
    ctx = Context(p)
    ctx.set_state(U)
    ctx.advance(4)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-10


def test_nonfinite_state_is_reported():
    p = default_params(gridsize=(16, 16, 16), **CASES["hd"])
    U = make_state(p, seed=1)
    U[0, 1, 2, 3] = np.nan
    ctx = Context(p)
    ctx.set_state(U)
    with pytest.raises(SpookyError) as e:
        ctx.compute_dt()
    assert e.value.code == 5
