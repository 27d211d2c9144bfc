"""GPU parity of the closure's variant 3, the tensor network on the tensor
cores (mma.sync BF16, FP32 accumulation), against its CPU oracle, which
rounds to BF16 at the same places and sums in FP64: the trainer's loss and
gradient, one Adam step, a teacher fit, the fused inference in the RHS (both
forms, HD and MHD), the products, the dt rule, steps at a fixed dt and the
sample rows.

Tolerances: the GPU sums in FP32 and takes its inputs from FP32 gradients,
so a few BF16 roundings land on the other side of a tie; each moves one
operand by a BF16 step (2^-8 relative)."""
import numpy as np
import pytest

import oracle as O
from spooky_b200 import CLOSURE3_NPARAM, CLOSURE3_ROWS, Context, Trainer, closure_samples
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN
from test_closure3_oracle import random_params3, random_samples3
from test_closure_gpu import _params, _state, rel_l2, torch_dev

pytestmark = pytest.mark.gpu


def test_trainer_loss_and_gradient_match_oracle():
    rng = np.random.default_rng(41)
    X = random_samples3(rng, 3000)
    P = random_params3(rng, out=0.5).astype(np.float32)
    w = np.array([2.0, 3.0, 1.5])
    Xf = X.astype(np.float32)
    loss_o, g_o = O.closure3_loss_grad(Xf.astype(np.float64), P.astype(np.float64), w)
    tr = Trainer(P, variant=3)
    tr.set_samples(torch_dev(Xf), w)
    loss_g, g_g = tr.loss_grad()
    assert abs(loss_g - loss_o) < 1e-3 * loss_o, (loss_g, loss_o)
    assert rel_l2(g_g, g_o) < 5e-3, rel_l2(g_g, g_o)
    # every layer's gradient block is resolved, not only the large ones
    for a, b in [(0, 1152), (1152, 1216), (1216, 5312), (5312, 5376), (5376, 9472), (9472, 9536), (9536, 10304),
                 (10304, 10316)]:
        assert rel_l2(g_g[a:b], g_o[a:b]) < 2e-2, (a, b, rel_l2(g_g[a:b], g_o[a:b]))
    loss_2, g_2 = tr.loss_grad()
    assert loss_2 == loss_g and np.array_equal(g_2, g_g)


def test_first_adam_step_is_signed_lr():
    rng = np.random.default_rng(42)
    X = random_samples3(rng, 2048).astype(np.float32)
    P = random_params3(rng, out=0.5).astype(np.float32)
    w = np.array([1.0, 1.0, 1.0])
    tr = Trainer(P, variant=3)
    tr.set_samples(torch_dev(X), w)
    _, g_o = O.closure3_loss_grad(X.astype(np.float64), P.astype(np.float64), w)
    lr = 1e-3
    tr.train(1, 2048, lr)
    d = tr.get_params().astype(np.float64) - P
    big = np.abs(g_o) > 1e-3 * np.abs(g_o).max()
    assert big.sum() > 0.3 * CLOSURE3_NPARAM, big.sum()
    agree = np.isclose(d[big], -lr * np.sign(g_o[big]), rtol=1e-3, atol=1e-7)
    assert agree.mean() > 0.99, agree.mean()


def test_trainer_fits_a_teacher_network():
    rng = np.random.default_rng(43)
    X = random_samples3(rng, 8192)
    teacher = random_params3(rng, out=1.0)
    for s in range(X.shape[1]):
        A, G = X[33:42, s], X[42:51, s]
        n = O.closure_features(A.reshape(3, 3), G.reshape(3, 3))[3]
        sv = X[16, s] * n * O.closure3_mlp(teacher, np.concatenate([A, G]) / n)
        tr_ = (sv[0] + sv[3] + sv[5]) / 3
        X[17:22, s] = [sv[0] - tr_, sv[1], sv[2], sv[3] - tr_, sv[4]]
        X[22:25, s] = 0.5 * np.array([sv[9] - sv[11], sv[10] - sv[7], sv[6] - sv[8]])
    w = np.array([1.0, 1.0, 0.0]) / np.mean(X[17:25] ** 2)
    tr = Trainer(random_params3(rng, out=0.05).astype(np.float32), variant=3)
    tr.set_samples(torch_dev(X, np.float32), w)
    l0, _ = tr.loss_grad()
    hist = tr.train(1500, 1024, 3e-3)
    l1, _ = tr.loss_grad()
    assert np.all(np.isfinite(hist)) and l1 < l0 / 20, (l0, l1)


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("mhd", [False, True])
def test_closure3_rhs_matches_oracle(mhd, form):
    import torch
    p = _params(mhd, form=form, variant=3)
    U = _state(p, 5)
    cp = random_params3(np.random.default_rng(46), out=1.0).astype(np.float32)
    o = O.Oracle(p)
    o.closure_set(cp.astype(np.float64))
    want = o.compute_dfield(U)
    off = O.Oracle(p).compute_dfield(U)
    ctx = Context(p)
    ctx.closure_set(cp)
    dU = torch.zeros(ctx.shape_c, dtype=torch.complex128, device="cuda")
    ctx.compute_dfield(torch_dev(U), dU)
    got = dU.cpu().numpy()
    assert rel_l2(want - off, off) > 1e-3          # the closure term is not negligible
    assert rel_l2(got - off, want - off) < 1e-2, rel_l2(got - off, want - off)
    assert rel_l2(got, want) < 1e-3
    # products: the closure terms enter the stress and EMF before their transforms
    Pg = ctx.products(torch_dev(U)).cpu().numpy()
    Po = o.products(U)
    Poff = O.Oracle(p).products(U)
    assert rel_l2(Pg - Poff, Po - Poff) < 1e-2


def test_closure3_dt_and_steps_match_oracle():
    p = _params(True, n=16, variant=3)
    U = _state(p, 7)
    cp = random_params3(np.random.default_rng(48), out=3.0).astype(np.float32)
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
    assert abs(dtg[1] - dto[1]) < 1e-2 * dto[1], (dtg, dto)
    pf = _params(True, n=16, fixed_dt=2e-3, variant=3)
    o = O.Oracle(pf)
    o.closure_set(cp.astype(np.float64))
    o.set_state(U)
    o.step(5)
    ctx = Context(pf)
    ctx.closure_set(cp)
    ctx.set_state(U)
    ctx.advance(5)
    ctx.synchronize()
    off = O.Oracle(pf)
    off.set_state(U)
    off.step(5)
    # the closure's share of the five steps is reproduced to the RHS test's accuracy
    got, want, base = ctx.get_state(), o.get_state(), off.get_state()
    assert rel_l2(want - base, base) > 1e-3
    assert rel_l2(got - base, want - base) < 2e-2, rel_l2(got - base, want - base)


@pytest.mark.parametrize("mhd", [False, True])
def test_closure3_samples_match_oracle(mhd):
    pf, pc = _params(mhd, n=32, variant=3), _params(mhd, n=16, variant=3)
    Uf = _state(pf, 13)
    want = O.Oracle(pf).closure_samples(Uf, O.Oracle(pc))
    fine, coarse = Context(pf), Context(pc)
    got = closure_samples(fine, torch_dev(Uf), coarse).cpu().numpy().astype(np.float64)
    assert got.shape[0] == CLOSURE3_ROWS
    for a, b in [(0, 8), (8, 13), (16, 17), (17, 22), (25, 30), (33, 42)] + ([(13, 16), (22, 25), (42, 51)] if mhd else []):
        assert rel_l2(got[a:b], want[a:b]) < 1e-5, (a, b)
    if not mhd:
        assert np.abs(got[42:51]).max() == 0.0


def test_trained_tensor_network_beats_the_plain_coarse_run():
    """The closure workflow with the tensor network at reduced size: a 128^3
    MHD truth (nu = eta = 2e-4), samples, GPU training of the network on the
    tensor cores, and 32^3 runs with and without it to the truth's final
    time; the eddy-coefficient network is trained on the same samples and
    run beside it.  The tensor network's shell spectrum is closer to the
    filtered truth than the plain coarse run's, and its run is cheaper than
    the truth."""
    from spooky_b200 import closure as C
    r = C.run(n_fine=128, n_coarse=32, steps=600, snap_every=100, train_steps=1200, batch=8192, lr=3e-3, variant=3,
              extra_variants=(1,), train_steps3=6000)
    assert np.isfinite(r["loss_history"]).all() and r["loss_final"] < r["loss_initial"]
    assert np.isfinite(r["error_closure"]) and np.isfinite(r["error_plain"])
    assert r["error_closure"] < 0.5 * r["error_plain"], (r["error_closure"], r["error_plain"])
    assert r["v1"]["finite"] and r["v1"]["error"] < 0.5 * r["error_plain"]
    assert r["cost_advantage"] > 1.0
