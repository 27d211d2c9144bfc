"""Workflow of the learned subgrid closure: a fine-grid truth run of this
solver, training samples from it, training on the GPU, and coarse runs with
and without the closure judged by their shell energy spectra against the
filtered truth (the 64^3-closure-vs-filtered-256^3 configuration, or any
smaller pair of grids).

All GPU work goes through libspooky_b200.so: the truth and coarse runs
(spk_advance), the samples (spk_closure_samples), the training
(spk_trainer_*).  torch only holds device memory; numpy does the host-side
bookkeeping (initial fields, spectral filter of the initial state, spectra).
"""
import time

import numpy as np

from . import CLOSURE3_NPARAM, CLOSURE_NPARAM, Context, Trainer, closure_samples
from .initial import mhd_random_state
from .params import SPK_FORM_PLAIN, default_params

# parameter offsets (include/spooky_b200.h): W1[32][8] b1[32] W2[32][32] b2[32] W3[2][32] b3[2]
_W1, _B1, _W2, _B2, _W3, _B3 = 0, 256, 288, 1312, 1344, 1408


def init_params(seed=0, c0=0.02):
    """Scaled-normal weights; the output biases start the eddy coefficients
    at softplus(b3) = c0."""
    rng = np.random.default_rng(seed)
    p = np.zeros(CLOSURE_NPARAM, np.float32)
    p[_W1:_B1] = rng.standard_normal(_B1 - _W1) / np.sqrt(8.0)
    p[_W2:_B2] = rng.standard_normal(_B2 - _W2) / np.sqrt(32.0)
    p[_W3:_B3] = 0.1 * rng.standard_normal(_B3 - _W3) / np.sqrt(32.0)
    p[_B3:] = np.log(np.expm1(c0))
    return p


# variant 3 (the tensor network): W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[12][64] b4[12]
_V1, _VB1 = 0, 1152
_V2, _VB2 = 1216, 5312
_V3, _VB3 = 5376, 9472
_V4, _VB4 = 9536, 10304


def init_params3(seed=0, out=0.05):
    """Scaled-normal hidden weights, small output weights: the network starts
    near zero stress and EMF."""
    rng = np.random.default_rng(seed)
    p = np.zeros(CLOSURE3_NPARAM, np.float32)
    p[_V1:_VB1] = rng.standard_normal(_VB1 - _V1) / np.sqrt(18.0)
    p[_V2:_VB2] = rng.standard_normal(_VB2 - _V2) / np.sqrt(64.0)
    p[_V3:_VB3] = rng.standard_normal(_VB3 - _V3) / np.sqrt(64.0)
    p[_V4:_VB4] = out * rng.standard_normal(_VB4 - _V4) / np.sqrt(64.0)
    return p


def _k_index(n):
    return np.fft.fftfreq(n, 1.0 / n)


def kept_mask(p):
    """The 2/3 mask of the reference (wavevector.cu:82-95) on an index grid."""
    def axis(n, length, half):
        k = 2 * np.pi / length * (_k_index(n) if not half else np.arange(n // 2 + 1))
        kmax = 2 * np.pi / length * (n // 2 - 1)
        return np.abs(k) <= 2.0 / 3.0 * kmax
    mx, my, mz = axis(p.nx, p.lx, False), axis(p.ny, p.ly, False), axis(p.nz, p.lz, True)
    return mx[:, None, None] & my[None, :, None] & mz[None, None, :]


def filter_to(U, pf, pc):
    """Sharp spectral filter of the fine spectra U [F, ...] onto the coarse
    grid's kept modes (scaled by the point-count ratio)."""
    scale = (pc.nx * pc.ny * pc.nz) / (pf.nx * pf.ny * pf.nz)
    ix = _k_index(pc.nx).astype(int) % pf.nx
    iy = _k_index(pc.ny).astype(int) % pf.ny
    out = U[:, ix][:, :, iy][:, :, :, : pc.nz // 2 + 1] * scale
    return out * kept_mask(pc)[None]


def shell_spectrum(U, p):
    """Energy per integer shell |k| L / 2 pi in [s - 1/2, s + 1/2), per field
    group: returns (E_u, E_B) (E_B zero without B); E sums to the mean of
    u^2 / 2 over the box."""
    N = p.nx * p.ny * p.nz
    kx, ky = _k_index(p.nx), _k_index(p.ny)
    kz = np.arange(p.nz // 2 + 1)
    K = np.sqrt(kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2)
    w = np.full(p.nz // 2 + 1, 2.0)
    w[0] = 1.0
    w[-1] = 1.0
    shell = np.rint(K).astype(int)
    ns = shell.max() + 1
    e = 0.5 * w[None, None, None, :] * np.abs(U) ** 2 / N ** 2
    Eu = np.bincount(shell.ravel(), weights=e[:3].sum(0).ravel(), minlength=ns)
    Eb = np.bincount(shell.ravel(), weights=e[3:6].sum(0).ravel(), minlength=ns) if U.shape[0] >= 6 else 0 * Eu
    return Eu, Eb


def spectral_error(E, Eref, kmin, kmax):
    """RMS over shells kmin..kmax of the relative deviation of E from Eref."""
    r = (E[kmin:kmax + 1] - Eref[kmin:kmax + 1]) / Eref[kmin:kmax + 1]
    return float(np.sqrt(np.mean(r ** 2)))


def _run_to(ctx, t_end, chunk=50):
    """Advance with the CFL dt until t_end (dt is clamped to land on it);
    returns (steps, seconds)."""
    steps = 0
    t0 = time.perf_counter()
    while ctx.get_time()[0] < t_end - 1e-12:
        ctx.advance(chunk)
        ctx.synchronize()
        steps += chunk
    return steps, time.perf_counter() - t0


def subgrid_weights(X, transfer=1.0):
    """Loss weights 1/<|T|_F^2>, 1/<|E|^2> and transfer/<P^2> of the targets
    in samples X, P = -T:Sf - E.Jf the true energy transfer into the subgrid
    scales."""
    t = X[17:22].double()
    fro = t[0] ** 2 + t[3] ** 2 + (t[0] + t[3]) ** 2 + 2 * (t[1] ** 2 + t[2] ** 2 + t[4] ** 2)
    e = X[22:25].double()
    e2 = (e ** 2).sum(0)
    sf, jf = X[25:30].double(), X[30:33].double()
    tsf = t[0] * sf[0] + t[3] * sf[3] + (t[0] + t[3]) * (sf[0] + sf[3]) + 2 * (t[1] * sf[1] + t[2] * sf[2] + t[4] * sf[4])
    P = -tsf - (e * jf).sum(0)
    wt = 1.0 / float(fro.mean())
    we = 1.0 / float(e2.mean()) if float(e2.mean()) > 0 else 0.0
    p2 = float((P ** 2).mean())
    wp = transfer / p2 if p2 > 0 else 0.0
    return np.array([wt, we, wp])


# loss weight of the energy-transfer error per variant: for variants 1 and 2
# the better of 0, 1 and 4, for variant 3 of 0, 1, 4 and 10, in the
# 64^3-vs-256^3 workload
TRANSFER_DEFAULT = {1: 0.0, 2: 4.0, 3: 0.0}


def run(n_fine=256, n_coarse=64, nu=2e-4, steps=2000, snap_every=250, train_steps=3000, batch=16384, lr=2e-3,
        seed=0, form=SPK_FORM_PLAIN, variant=1, transfer=None, kc_frac=0.0, log=None, extra_variants=(),
        lr3=1e-3, train_steps3=20000):
    """Truth, samples, training and the two coarse runs; returns a dict of
    the measured quantities (spectral errors with and without the closure,
    run costs, losses).  variant: 1 the full-field model, 2 the small-scale
    model (gradients of the modes above half the cut-off), 3 the tensor
    network; transfer: the relative weight of the energy-transfer error in
    the loss (0: stress and EMF errors only; None: TRANSFER_DEFAULT, for
    variants 1 and 2 the better of 0, 1 and 4 in the 64^3-vs-256^3
    workload); kc_frac: variant 2's small scales are |k| > kc_frac * k_c
    (0: 1/2).  extra_variants: more networks (of 1 and 3) trained on the
    same truth and run on the same coarse grid, their results under
    "v<variant>" (a variant-3 sampler's rows hold every row variant 1
    reads); lr3, train_steps3: the tensor network's learning rate and Adam
    steps (its training is cheap: 20000 steps of 16384 samples take about a
    second)."""
    if transfer is None:
        transfer = TRANSFER_DEFAULT[variant]
    variants = [variant] + [v for v in extra_variants if v != variant]
    if 2 in variants and len(variants) > 1:
        raise ValueError("variant 2 samples differ from the others: run it alone")
    sample_variant = 3 if 3 in variants else variant
    import torch
    say = log or (lambda *a: None)
    L = 2 * np.pi
    common = dict(incompressible=1, mhd=1, boxsize=(L, L, L), reynolds=1.0 / nu, reynolds_magnetic=1.0 / nu,
                  cfl=1.5, form=form, toutput_flow=1e30)
    pf = default_params(gridsize=(n_fine,) * 3, t_final=1e30, **common)
    U0 = mhd_random_state(pf, 1, 2)
    fine = Context(pf)
    fine.set_state(U0)
    pc0 = default_params(gridsize=(n_coarse,) * 3, t_final=1e30, closure=sample_variant, closure_kc_frac=kc_frac,
                         **common)
    sampler = Context(pc0)
    Uf = torch.empty(fine.shape_c, dtype=torch.complex128, device="cuda")
    samples, truth_s, done = [], 0.0, 0
    while done < steps:
        k = min(snap_every, steps - done)
        t0 = time.perf_counter()
        fine.advance(k)
        fine.synchronize()
        truth_s += time.perf_counter() - t0
        done += k
        fine.get_state(Uf)
        torch.cuda.synchronize()
        samples.append(closure_samples(fine, Uf, sampler))
    T = fine.get_time()[0]
    truth_filtered = sampler.get_state()          # the filtered truth at T
    say(f"truth {n_fine}^3: {steps} steps to t = {T:.4f} in {truth_s:.2f} s")
    del fine, Uf
    X = torch.cat(samples, dim=1).contiguous()
    del samples
    trained = {}
    for v in variants:
        wv = subgrid_weights(X, transfer if v == variant else TRANSFER_DEFAULT[v])
        tr = Trainer(init_params3(seed) if v == 3 else init_params(seed), variant=v)
        tr.set_samples(X, wv)
        l0, _ = tr.loss_grad()
        lv, nt = (lr3, train_steps3) if v == 3 else (lr, train_steps)
        t0 = time.perf_counter()
        h1 = tr.train(int(nt * 2 // 3), batch, lv)
        h2 = tr.train(nt - int(nt * 2 // 3), batch, lv / 4)
        torch.cuda.synchronize()
        ts = time.perf_counter() - t0
        l1, _ = tr.loss_grad()
        trained[v] = dict(params=tr.get_params(), loss_initial=l0, loss_final=l1, train_seconds=ts,
                          loss_history=np.concatenate([h1, h2]))
        say(f"training variant {v}: {X.shape[1]} samples, loss {l0:.4f} -> {l1:.4f} in {ts:.2f} s")
        del tr
    del X
    params, loss0, loss1 = trained[variant]["params"], trained[variant]["loss_initial"], trained[variant]["loss_final"]
    train_s = trained[variant]["train_seconds"]
    # coarse runs from the filtered initial state to the truth's final time
    U0c = filter_to(U0, pf, pc0)
    res = {}
    runs = [("closure", variant, params), ("plain", variant, None)]
    runs += [(f"v{v}", v, trained[v]["params"]) for v in variants[1:]]
    for name, v, cp in runs:
        pc = default_params(gridsize=(n_coarse,) * 3, t_final=T, closure=v, closure_kc_frac=kc_frac, **common)
        ctx = Context(pc)
        if cp is not None:
            ctx.closure_set(cp)
        ctx.set_state(U0c)
        nst, secs = _run_to(ctx, T)
        res[name] = (ctx.get_state(), nst, secs)
        say(f"coarse {n_coarse}^3 {name}: {nst} step launches in {secs:.3f} s")
    kc = int(np.floor(2.0 / 3.0 * (n_coarse // 2 - 1)))
    Eu_t, Eb_t = shell_spectrum(truth_filtered, pc0)
    out = dict(t_end=T, truth_steps=steps, truth_seconds=truth_s, train_seconds=train_s,
               loss_initial=loss0, loss_final=loss1, loss_history=trained[variant]["loss_history"], k_cut=kc,
               spectrum_truth=Eu_t + Eb_t, params=params)
    for name, (U, nst, secs) in res.items():
        Eu, Eb = shell_spectrum(U, pc0)
        d = {"error": spectral_error(Eu + Eb, Eu_t + Eb_t, 1, kc), "error_u": spectral_error(Eu, Eu_t, 1, kc),
             "error_b": spectral_error(Eb, Eb_t, 1, kc), "energy": float((Eu + Eb).sum()), "seconds": secs,
             "spectrum": Eu + Eb, "steps": nst}
        if name.startswith("v"):
            v = int(name[1:])
            d.update({k: trained[v][k] for k in ("loss_initial", "loss_final", "train_seconds")})
            d["cost_advantage"] = truth_s / max(secs, 1e-9)
            d["finite"] = bool(np.isfinite(U).all())
            out[name] = d
            continue
        for k, val in d.items():
            if k != "steps":
                out[f"{k}_{name}"] = val
    out["energy_truth"] = float((Eu_t + Eb_t).sum())
    out["cost_advantage"] = truth_s / max(out["seconds_closure"], 1e-9)
    return out
