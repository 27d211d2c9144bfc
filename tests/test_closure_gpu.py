"""GPU parity of the learned closure against its CPU FP64 oracle: the
training kernels' loss and gradient, one Adam step, the spectral products,
the closure terms in the RHS, steps and dt, and the training samples.

The MLP runs in FP32 on the GPU in both forms, so closure results carry
FP32 rounding (tolerances below); everything else follows the forms'
usual tolerances."""
import numpy as np
import pytest

import oracle as O
from fields import random_solenoidal, to_spectral
from spooky_b200 import Context, Trainer, closure_samples, CLOSURE_NPARAM
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, default_params
from test_closure_oracle import random_params, random_samples

pytestmark = pytest.mark.gpu
L = 2 * np.pi


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def torch_dev(arr, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr if dtype is None else arr.astype(dtype))).cuda()
    torch.cuda.synchronize()
    return t


def _params(mhd=True, n=16, form=SPK_FORM_PLAIN, variant=1, **kw):
    base = dict(incompressible=1, gridsize=(n, n, n), boxsize=(L, L, L), reynolds=1e3, form=form, closure=variant,
                t_final=1e9, toutput_flow=1e9)
    if mhd:
        base.update(mhd=1, reynolds_magnetic=1e3)
    base.update(kw)
    return default_params(**base)


def _state(p, seed):
    fields = list(random_solenoidal(p, seed, kpeak=3.0))
    if p.mhd:
        fields += list(random_solenoidal(p, seed + 7, kpeak=3.0, rms=0.6))
    return to_spectral(np.stack(fields))


def test_trainer_loss_and_gradient_match_oracle():
    rng = np.random.default_rng(21)
    X = random_samples(rng, 3000)
    P = random_params(rng)
    P[-2:] = 0.1
    P32 = P.astype(np.float32)
    w = np.array([2.0, 3.0, 1.5])
    loss_o, g_o = O.closure_loss_grad(X.astype(np.float32).astype(np.float64), P32.astype(np.float64), w)
    tr = Trainer(P32)
    tr.set_samples(torch_dev(X, np.float32), w)
    loss_g, g_g = tr.loss_grad()
    assert abs(loss_g - loss_o) < 1e-5 * loss_o
    assert rel_l2(g_g, g_o) < 1e-4
    # the same evaluation twice gives the same bits (fixed-order sums)
    loss_2, g_2 = tr.loss_grad()
    assert loss_2 == loss_g and np.array_equal(g_2, g_g)


def test_first_adam_step_is_signed_lr():
    """From zero moments, bias-corrected Adam moves every parameter by
    -lr * sign(g) (up to eps): the oracle's gradient signs fix the step."""
    rng = np.random.default_rng(22)
    X = random_samples(rng, 2048)
    P = random_params(rng).astype(np.float32)
    w = np.array([1.0, 1.0, 1.0])
    tr = Trainer(P)
    tr.set_samples(torch_dev(X, np.float32), w)
    _, g_o = O.closure_loss_grad(X.astype(np.float32).astype(np.float64), P.astype(np.float64), w)
    lr = 1e-3
    tr.train(1, 2048, lr)
    d = tr.get_params().astype(np.float64) - P
    big = np.abs(g_o) > 1e-3 * np.abs(g_o).max()
    assert big.sum() > 0.5 * CLOSURE_NPARAM
    assert np.allclose(d[big], -lr * np.sign(g_o[big]), rtol=1e-3, atol=1e-7)


def test_trainer_fits_a_teacher_network():
    rng = np.random.default_rng(23)
    X = random_samples(rng, 16384)
    teacher = random_params(rng)
    teacher[-2:] = [-1.0, -1.5]
    for s in range(X.shape[1]):
        o = O.closure_mlp(teacher, X[0:8, s])
        nu, eta = X[16, s] * np.log1p(np.exp(o))
        X[17:22, s] = -2 * nu * X[8:13, s]
        X[22:25, s] = -eta * X[13:16, s]
    w = np.array([1.0, 1.0, 1.0]) / np.mean(X[17:25] ** 2)
    tr = Trainer(random_params(rng).astype(np.float32))
    tr.set_samples(torch_dev(X, np.float32), w)
    l0, _ = tr.loss_grad()
    hist = tr.train(1500, 1024, 1e-2)
    l1, _ = tr.loss_grad()
    assert np.all(np.isfinite(hist)) and l1 < l0 / 100, (l0, l1)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("mhd", [False, True])
def test_products_match_oracle(mhd, form):
    p = _params(mhd, form=form)
    U = _state(p, 3)
    o = O.Oracle(p)
    want = o.products(U)
    ctx = Context(p)
    got = ctx.products(torch_dev(U)).cpu().numpy()
    assert rel_l2(got, want) < (1e-12 if form == SPK_FORM_PLAIN else 2e-5)


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("mhd", [False, True])
def test_closure_rhs_matches_oracle(mhd, form, variant):
    import torch
    p = _params(mhd, form=form, variant=variant)
    U = _state(p, 5)
    cp = random_params(np.random.default_rng(6), 0.5).astype(np.float32)
    o = O.Oracle(p)
    o.closure_set(cp.astype(np.float64))
    want = o.compute_dfield(U)
    off = O.Oracle(p).compute_dfield(U)
    ctx = Context(p)
    ctx.closure_set(cp)
    dU = torch.zeros(ctx.shape_c, dtype=torch.complex128, device="cuda")
    ctx.compute_dfield(torch_dev(U), dU)
    got = dU.cpu().numpy()
    # the closure's own contribution is resolved, not lost in the rest
    assert rel_l2(got - off, want - off) < (1e-5 if form == SPK_FORM_PLAIN else 1e-3)
    assert rel_l2(got, want) < (1e-6 if form == SPK_FORM_PLAIN else 3e-5)


@pytest.mark.parametrize("variant", [1, 2])
def test_closure_dt_and_steps_match_oracle(variant):
    p = _params(True, n=16, variant=variant)
    U = _state(p, 7)
    cp = random_params(np.random.default_rng(8), 0.5).astype(np.float32)
    cp[-2:] = 0.5   # eddy coefficients large enough to set dt
    o = O.Oracle(p)
    o.closure_set(cp.astype(np.float64))
    o.set_state(U)
    o.clean_divergence()
    dto = o.compute_dt()
    ctx = Context(p)
    ctx.closure_set(cp)
    ctx.set_state(U)
    ctx.clean_divergence()
    dtg = ctx.compute_dt()
    assert abs(dtg[1] - dto[1]) < 1e-5 * dto[1]           # dt_par carries the closure's rate
    off = Context(_params(True, n=16))
    off.set_state(U)
    off.clean_divergence()
    assert off.compute_dt()[1] > (1.5 if variant == 1 else 1.05) * dtg[1]
    # steps at a fixed dt
    pf = _params(True, n=16, fixed_dt=2e-3, variant=variant)
    o = O.Oracle(pf)
    o.closure_set(cp.astype(np.float64))
    o.set_state(U)
    o.step(5)
    ctx = Context(pf)
    ctx.closure_set(cp)
    ctx.set_state(U)
    ctx.advance(5)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-6
    # switching the closure off re-records the plain step
    ctx.closure_set(None)
    o.closure_set(None)
    ctx.advance(2)
    o.step(2)
    ctx.synchronize()
    assert rel_l2(ctx.get_state(), o.get_state()) < 1e-6


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("mhd", [False, True])
def test_samples_match_oracle(mhd, variant):
    pf, pc = _params(mhd, n=32, variant=variant), _params(mhd, n=16, variant=variant)
    Uf = _state(pf, 13)
    of, oc = O.Oracle(pf), O.Oracle(pc)
    want = of.closure_samples(Uf, oc)
    fine, coarse = Context(pf), Context(pc)
    got = closure_samples(fine, torch_dev(Uf), coarse).cpu().numpy().astype(np.float64)
    assert rel_l2(coarse.get_state(), oc.get_state()) < 1e-14
    groups = [(0, 8), (8, 13), (13, 16), (16, 17), (17, 22), (22, 25), (25, 30), (30, 33)]
    for a, b in groups:
        if not mhd and a in (13, 22, 30):
            assert np.abs(got[a:b]).max() == 0.0
            continue
        assert rel_l2(got[a:b], want[a:b]) < 1e-5, (a, b)
    # the whole field's strain and current: the model's own in variant 1
    if variant == 1:
        assert np.array_equal(got[25:33], got[8:16])
    else:
        assert rel_l2(got[25:30], got[8:13]) > 1e-2


def test_trained_closure_beats_the_plain_coarse_run():
    """The closure workflow at reduced size: a 128^3 MHD truth (nu = eta =
    2e-4), samples from it, GPU training, and 32^3 runs with and without
    the closure to the truth's final time.  The closure run's shell spectrum
    is closer to the filtered truth than the plain coarse run's, and it is
    cheaper than the truth."""
    from spooky_b200 import closure as C
    r = C.run(n_fine=128, n_coarse=32, steps=600, snap_every=100, train_steps=1200, batch=8192, lr=3e-3)
    assert np.isfinite(r["loss_history"]).all() and r["loss_final"] < r["loss_initial"]
    assert np.isfinite(r["error_closure"]) and np.isfinite(r["error_plain"])
    assert r["error_closure"] < 0.8 * r["error_plain"], (r["error_closure"], r["error_plain"])
    assert r["cost_advantage"] > 1.0
