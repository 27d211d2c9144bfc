"""Ensembles of independent boxes (spk_ensemble_*): every box advanced inside
the ensemble's single graph must follow the same box advanced alone."""
import numpy as np
import pytest

import spooky_b200 as S
from fields import random_solenoidal, to_spectral
from spooky_b200 import Context, Ensemble
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, default_params

L = 2 * np.pi


def box_params():
    out = []
    # three boxes of one group (same geometry, different viscosities) ...
    for nu in (1e-2, 1e-3, 3e-4):
        out.append(default_params(incompressible=1, gridsize=(16, 16, 16), boxsize=(L, L, L), reynolds=1.0 / nu,
                                   form=SPK_FORM_FP32, t_final=1e30, toutput_flow=1e30))
    # ... two of another (different resistivities), and single-box groups
    out.append(default_params(incompressible=1, gridsize=(16, 16, 16), boxsize=(L, L, L), reynolds=100.0,
                               form=SPK_FORM_FP32, t_final=1e30, toutput_flow=1e30))
    for eta in (2e-3, 2e-4):
        out.append(default_params(incompressible=1, mhd=1, gridsize=(32, 32, 32), boxsize=(L, L, L), reynolds=1e3,
                                   reynolds_magnetic=1.0 / eta, form=SPK_FORM_FP32, t_final=1e30, toutput_flow=1e30))
    out.append(default_params(incompressible=1, gridsize=(32, 16, 64), boxsize=(1.0, 0.5, 2.0), reynolds=300.0,
                               form=SPK_FORM_PLAIN, t_final=1e30, toutput_flow=1e30))
    out.append(default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                               gridsize=(16, 16, 32), boxsize=(1.0, 1.0, 1.0), reynolds=100.0, reynolds_magnetic=100.0,
                               reynolds_thermic=100.0, reynolds_ani=20.0, N2=1.0, OmegaT2=1.0, form=SPK_FORM_PLAIN,
                               t_final=1e30, toutput_flow=1e30))
    out.append(default_params(heat_equation=1, gridsize=(16, 8, 8), reynolds_thermic=10.0, form=SPK_FORM_PLAIN,
                               t_final=1e30, toutput_flow=1e30))
    for nu in (5e-3, 5e-4):   # a 3*2^k group
        out.append(default_params(incompressible=1, mhd=1, gridsize=(24, 24, 24), boxsize=(L, L, L),
                                   reynolds=1.0 / nu, reynolds_magnetic=300.0, form=SPK_FORM_FP32, t_final=1e30,
                                   toutput_flow=1e30))
    return out


def initial_state(p, seed):
    fields = []
    if p.incompressible:
        fields += list(random_solenoidal(p, seed, kpeak=3.0))
    if p.mhd:
        B = random_solenoidal(p, seed + 50, kpeak=3.0, rms=0.5)
        B[0] += 0.2
        fields += list(B)
    if p.boussinesq or p.heat_equation:
        rng = np.random.default_rng(seed + 99)
        fields.append(0.2 * rng.standard_normal((p.nx, p.ny, p.nz)))
    return to_spectral(np.stack(fields))


@pytest.mark.gpu
def test_ensemble_boxes_follow_the_same_boxes_alone():
    params = box_params()
    states = [initial_state(p, 10 + i) for i, p in enumerate(params)]
    ens = Ensemble(params)
    for b, U in zip(ens.boxes, states):
        b.set_state(U)
    ens.advance(4)
    ens.advance(3)
    ens.synchronize()
    assert ens.ngroups == 6 and ens.kernels_per_step() > 0
    for i, (p, U) in enumerate(zip(params, states)):
        ctx = Context(p)
        ctx.set_state(U)
        ctx.advance(7)
        ctx.synchronize()
        got, want = ens.boxes[i].get_state(), ctx.get_state()
        assert np.array_equal(got, want), i
        assert ens.boxes[i].get_time() == ctx.get_time(), i
        e_ens, _ = ens.boxes[i].budgets()
        e_one, _ = ctx.budgets()
        # the budget reductions sum with atomics: equal up to summation order
        assert np.allclose(e_ens, e_one, rtol=1e-12, atol=0), i
    ens.close()


def test_ensemble_rejects_alternating_sts_and_empty_lists():
    p = default_params(incompressible=1, boussinesq=1, supertimestepping=1, sts_variables=["th"])
    with pytest.raises(S.SpookyError) as e:
        Ensemble([p])
    assert e.value.code == 2 and "alternates" in str(e.value)
    with pytest.raises(S.SpookyError) as e:
        Ensemble([])
    assert e.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("form", [SPK_FORM_FP32, SPK_FORM_PLAIN])
@pytest.mark.parametrize("n", [24, 32])
def test_autotuned_short_hd_boxes_compute_the_same_bits(n, form):
    """Short HD lines at one line per CTA (an autotuner candidate) share the
    z pass's exchange slots with its input area, and the CFL block maxima
    then use the real-field area: it must hold them.  Tuned and untuned
    contexts give the same state."""
    p = default_params(incompressible=1, gridsize=(n, n, n), boxsize=(L, L, L), reynolds=300.0, form=form,
                       t_final=1e30, toutput_flow=1e30)
    U = initial_state(p, 11)
    a, b = Context(p), Context(p)
    a.set_state(U)
    b.set_state(U)
    r = a.autotune(steps=2)
    assert r["ms_after"] <= r["ms_before"]
    a.advance(4)
    b.advance(4)
    a.synchronize()
    b.synchronize()
    assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.gpu
def test_autotuned_runs_compute_the_same_bits():
    """spk_autotune changes launch choices only: a tuned context and an
    untuned one give the same state, and the ensemble likewise."""
    p = default_params(incompressible=1, mhd=1, gridsize=(32, 32, 32), boxsize=(L, L, L), reynolds=300.0,
                       reynolds_magnetic=300.0, form=SPK_FORM_FP32, t_final=1e30, toutput_flow=1e30)
    U = initial_state(p, 7)
    a, b = Context(p), Context(p)
    a.set_state(U)
    b.set_state(U)
    r = a.autotune(steps=2)
    assert r["ms_after"] <= r["ms_before"] and a.get_time()[2] == 0
    a.advance(5)
    b.advance(5)
    a.synchronize()
    b.synchronize()
    assert np.array_equal(a.get_state(), b.get_state())
    params = box_params()[:4]
    ens = Ensemble(params)
    ref = Ensemble(params)
    for i, q in enumerate(params):
        ens.boxes[i].set_state(initial_state(q, 40 + i))
        ref.boxes[i].set_state(initial_state(q, 40 + i))
    ens.autotune(steps=2)
    ens.advance(3)
    ref.advance(3)
    ens.synchronize()
    ref.synchronize()
    for i in range(len(params)):
        assert np.array_equal(ens.boxes[i].get_state(), ref.boxes[i].get_state()), i
    ens.close()
    ref.close()


def _short_params(n, form, kind):
    base = dict(gridsize=(n, n, n), boxsize=(L, L, L), form=form, t_final=1e30, toutput_flow=1e30)
    if kind == "hd":
        return default_params(incompressible=1, reynolds=300.0, **base)
    if kind == "mhd":
        return default_params(incompressible=1, mhd=1, reynolds=300.0, reynolds_magnetic=300.0, **base)
    return default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                          reynolds=100.0, reynolds_magnetic=100.0, reynolds_thermic=100.0, reynolds_ani=20.0,
                          N2=1.0, OmegaT2=1.0, supertimestepping=1, sts_variables=["th"], safety_sts=20,
                          **base)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [SPK_FORM_FP32, SPK_FORM_PLAIN])
@pytest.mark.parametrize("n", [16, 24, 32, 48, 64])
@pytest.mark.parametrize("kind", ["hd", "mhd", "aniso"])
def test_half_width_axis_tiles_compute_the_same_bits(kind, n, form):
    """The autotuner's half-width axis tiles of short axes (spk_set_schedule
    axis_tile_div 2) transform the same columns as the full tiles: the
    same state after steps that use every axis pass (inverse passes with
    derivatives, forward passes, the RKL2 flux chain of anisotropic
    conduction)."""
    p = _short_params(n, form, kind)
    U = initial_state(p, 13)
    a, b = Context(p), Context(p)
    a.set_schedule(axis_tile_div=2)
    assert a.get_schedule()["axis_tile_div"] == 2 and b.get_schedule()["axis_tile_div"] == 1
    a.set_state(U)
    b.set_state(U)
    a.advance(4)
    b.advance(4)
    a.synchronize()
    b.synchronize()
    assert np.array_equal(a.get_state(), b.get_state())
