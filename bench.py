"""Benchmark: 256^3 incompressible MHD, low-storage RK3 steps per second on B200.

Workload (the headline metric: 256^3 MHD RK3 steps/s, FP32 form beside the
plain FP64 form): 256^3 box [0, 2 pi)^3, u and B independent random
solenoidal Gaussian fields with shell spectrum E(k) ~ k^4 exp(-2 (k/4)^2),
rms 1 per component, B0 = 0.1 z added to the k=0 mode of B, nu = eta = 1e-3,
CFL 1.5, 2/3 dealiasing, dt from the reference's CFL rule every step.

A step = one main-loop iteration (CleanFieldDivergence + HydroMHDAdvance:
compute_dt, three RK3 stages), run through the C ABI on a CUDA graph.

Arms:
  default            this library (value = FP32 form; the plain FP64 form,
                     the FP32-vs-FP64 error, the per-pass roofline, the
                     end-to-end host-buffer run and a CPU baseline are reported
                     in the same JSON line)
  --impl reference   the CPU FP64 oracle (restatement of the reference's
                     algorithm; the reference itself has no CPU path) on all
                     host cores, same workload

Multi-GPU: one independent box per rank (the single-box path does not shard
without a distributed FFT); value = box-steps/s summed over ranks, timed as
the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "spooky-git_b200"))

from spooky_b200.initial import masked_noise_state, mhd_random_state  # noqa: E402
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, cfg_text, default_params  # noqa: E402

METRIC = "256^3 MHD RK3 steps/s, FP32 form vs plain, 1xB200, at <=1e-5 rel L2 vs FP64"
HBM_FALLBACK = 6650.0


def workload_params(n, form):
    L = 2 * np.pi
    return default_params(incompressible=1, mhd=1, gridsize=(n, n, n), boxsize=(L, L, L),
                          reynolds=1e3, reynolds_magnetic=1e3, cfl=1.5, form=form,
                          t_final=1e30, toutput_flow=1e30)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def config_dict(n, world):
    return {"workload": f"incompressible MHD {n}^3, box 2pi, nu=eta=1e-3, B0=0.1z, CFL 1.5, random solenoidal "
                        f"E(k)~k^4 exp(-2(k/4)^2) u,B (seeds 1,2)",
            "grid": [n, n, n], "fields": 6, "integrator": "low-storage RK3 (3 stages/step)",
            "parallelism": f"replicas x{world}" if world > 1 else "single box",
            "l2_flush": "not needed: working set (state 0.8 GB + pass buffers) >> 126 MB L2"}


class ClockSampler:
    def __init__(self, gpu_index, path):
        self.path = path
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args):
    """CPU FP64 oracle on all host cores (the reference arm)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    p = workload_params(args.n, SPK_FORM_PLAIN)
    U0 = mhd_random_state(p)
    o = O.Oracle(p)
    o.set_state(U0)
    t0 = time.perf_counter()
    o.step(args.warmup)            # warm-up steps (about a second each at 256^3 on 16 cores)
    t_step = (time.perf_counter() - t0) / args.warmup
    budget = 150.0
    k = max(1, min(args.steps, int(budget / max(t_step, 1e-3))))
    t0 = time.perf_counter()
    o.step(k)
    el = time.perf_counter() - t0
    v = k / el
    sample = (f"{k} of the requested {args.steps} RK3 steps at {args.n}^3 MHD after {args.warmup} warm-up steps "
              f"(steps capped so the run stays within ~{int(budget)} s)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * el / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args.n, 1),
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU path; this arm is the project's FP64 C restatement of its "
                    "algorithm (oracle/), OpenMP over pencils"}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(n):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    p = workload_params(n, SPK_FORM_PLAIN)
    o = O.Oracle(p)
    o.set_state(mhd_random_state(p))
    steps, el = 0, 0.0
    while el < 10.0 and steps < 20:
        t0 = time.perf_counter()
        o.step(1)
        el += time.perf_counter() - t0
        steps += 1
    return {"value": steps / el, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} RK3 step(s) of {n}^3 MHD from the same initial state (FP64 C oracle, OpenMP)"}


def reference_cufft_leg(p, U0, warmup, steps, U_plain, timeout=900):
    """The reference's own CUDA build (cuFFT + cuBLAS, FP64; oracle/refbuild)
    on the same workload and GPU: its main-loop body for `warmup` + `steps`
    steps from U0, the timed steps between CUDA events.  Returns its rate and
    the rel L2 of its final state against this library's plain form after
    the same number of steps (U_plain)."""
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "spooky_ref")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/spooky_ref is not built (make -C oracle/refbuild REF=<reference checkout>)"}
    with tempfile.TemporaryDirectory(prefix="spk_ref_") as d:
        with open(os.path.join(d, "spooky.cfg"), "w") as f:
            f.write(cfg_text(p, configname="reference timing run"))
        u0, u1 = os.path.join(d, "u0.bin"), os.path.join(d, "u1.bin")
        np.ascontiguousarray(U0, dtype=np.complex128).tofile(u0)
        try:
            r = subprocess.run([exe, d, u0, str(warmup), str(steps), u1], capture_output=True, text=True,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"reference build did not finish within {timeout} s"}
        if r.returncode != 0:
            return {"unavailable": f"reference build exited {r.returncode}: " + (r.stderr or r.stdout)[-300:]}
        js = [l for l in r.stdout.splitlines() if l.startswith("{")]
        if not js:
            return {"unavailable": "reference build printed no result line"}
        j = json.loads(js[-1])
        U1 = np.fromfile(u1, dtype=np.complex128).reshape(U0.shape)
    rel = float(np.linalg.norm((U1 - U_plain).ravel()) / np.linalg.norm(U_plain.ravel()))
    return {"value": j["steps_per_s"], "unit": "steps/s", "ms_per_step": j["ms_per_step"], "steps": j["steps"],
            "warmup": j["warmup"], "ffts_per_step": j["ffts_per_step"], "rel_l2_vs_plain_fp64": rel,
            "after_steps": j["warmup"] + j["steps"],
            "what": "the reference's own sources (cuFFT + cuBLAS, FP64) built for sm_100a by oracle/refbuild; "
                    "main-loop body CleanFieldDivergence + HydroMHDAdvance, CUDA events on the legacy stream"}


ENSEMBLE_SIZES = (16, 24, 32, 48, 64)


def ensemble_boxes(nbox, seed=2024):
    """Config 4: box sizes uniform over ENSEMBLE_SIZES, HD or MHD with equal
    odds, nu and eta log-uniform in [1e-4, 1e-2], FP32 form; ICs drawn per box
    like config 2 (random solenoidal u and B, E(k) ~ k^4 exp(-2(k/4)^2), rms 1,
    B0 = 0.1 z), seeds from the box index."""
    rng = np.random.default_rng(seed)
    L = 2 * np.pi
    boxes = []
    for i in range(nbox):
        n = int(rng.choice(ENSEMBLE_SIZES))
        mhd = int(rng.integers(0, 2))
        nu, eta = 10 ** rng.uniform(-4, -2), 10 ** rng.uniform(-4, -2)
        p = default_params(incompressible=1, mhd=mhd, gridsize=(n, n, n), boxsize=(L, L, L), reynolds=1.0 / nu,
                           reynolds_magnetic=1.0 / eta, cfl=1.5, form=SPK_FORM_FP32, t_final=1e30,
                           toutput_flow=1e30)
        boxes.append((i, p))
    return boxes


def box_state(i, p):
    from spooky_b200.initial import random_solenoidal, to_spectral
    u = random_solenoidal(p, 1000 + 2 * i)
    if not p.mhd:
        return to_spectral(u)
    B = random_solenoidal(p, 1001 + 2 * i)
    B[2] += 0.1
    return to_spectral(np.concatenate([u, B]))


def partition_boxes(costs, world):
    """Greedy longest-processing-time assignment of boxes to ranks by cost
    (N^3 log N per box): returns one list of box indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: load[k])
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def ensemble_timing(params, states, steps, warmup, stream, barrier=None):
    """Advance one ensemble of the given boxes: `steps` timed steps with the
    launchers' own schedule, then spk_ensemble_autotune and `steps` timed
    steps again.  Returns (ms untuned, ms tuned, autotune seconds, kernels
    per ensemble step, all budgets finite)."""
    import torch
    import spooky_b200 as S
    ens = S.Ensemble(params, stream=stream.cuda_stream)
    for b, U in zip(ens.boxes, states):
        b.set_state(U)
    ens.advance(warmup)
    ens.synchronize()

    def timed():
        if barrier is not None:
            barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.advance(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    ms_untuned = timed()
    # the schedule autotuner (spk_ensemble_autotune), then the timed steps
    t_tune = time.perf_counter()
    ens.autotune(steps=3)
    ens.advance(warmup)
    ens.synchronize()
    t_tune = time.perf_counter() - t_tune
    ms = timed()
    kps = ens.kernels_per_step()
    ens.synchronize()
    finite = all(np.isfinite(b.budgets()[0]).all() for b in ens.boxes)
    ens.close()
    return ms_untuned, ms, t_tune, kps, finite


def run_ensemble(args, world, rank, local_rank):
    import torch
    import torch.distributed as dist
    import spooky_b200 as S
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    boxes = ensemble_boxes(args.boxes)
    costs = [p.nx * p.ny * p.nz * np.log2(p.nx * p.ny * p.nz) for _, p in boxes]
    mine = partition_boxes(costs, world)[rank]
    params = [boxes[i][1] for i in mine]
    states = [box_state(*boxes[i]) for i in mine]
    stream = torch.cuda.Stream()
    ms_untuned, ms, t_tune, kps, finite = ensemble_timing(params, states, args.steps, args.warmup, stream,
                                                          dist.barrier if world > 1 else None)
    # one box at a time: each box alone through its own graph, on a sample
    nsample = min(len(mine), 64)
    one_ms = 0.0
    for k in range(nsample):
        ctx = S.Context(params[k], stream=stream.cuda_stream)
        ctx.set_state(states[k])
        ctx.advance(args.warmup)
        ctx.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        ctx.advance(args.steps)
        a1.record(stream)
        torch.cuda.synchronize()
        one_ms += a0.elapsed_time(a1)
        ctx.close()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if rank == 0:
        value = args.boxes * args.steps / (ms * 1e-3)
        sizes = {str(n): sum(1 for _, p in boxes if p.nx == n) for n in ENSEMBLE_SIZES}
        line = {
            "metric": "ensemble box-steps/s (config 4: independent HD/MHD boxes, FP32 form, one graph per step)",
            "value": value, "unit": "box-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak" if world == 1 else "strong",
            "vs_baseline": None, "dtype": "fp32 passes, fp64 state", "data": "synthetic (seeded random fields)",
            "config": {"workload": f"{args.boxes} boxes, sizes {list(ENSEMBLE_SIZES)}^3 uniform, HD/MHD 50/50, "
                                   f"nu, eta log-uniform [1e-4, 1e-2], CFL 1.5", "boxes_per_size": sizes,
                       "parallelism": f"boxes partitioned over {world} rank(s) by N^3 log N"},
            "one_box_at_a_time": {"value": nsample * args.steps / (one_ms * 1e-3), "unit": "box-steps/s",
                                  "sample_boxes": nsample, "rank": 0},
            "untuned": {"value": args.boxes * args.steps / (ms_untuned * 1e-3), "unit": "box-steps/s",
                        "what": "the launchers' own schedule, before spk_ensemble_autotune (rank 0)"},
            "autotune_seconds": t_tune,
            "kernels_per_ensemble_step_rank0": kps,
            "gpu_launches": kps * args.steps,
            "all_finite": finite,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def mti_params(n, safety_sts=95):
    """Config 3: Boussinesq MHD with field-aligned anisotropic conduction in a
    2 pi box; gravity along z, N^2 = omega_T^2 = 1, chi_par = 1/20, chi_perp = 0,
    nu = eta = 1e-4, theta conducted by RKL2 super-time-stepping with dt capped
    at 95 dt_sts (s <= 20 stages), FP32 form."""
    L = 2 * np.pi
    return default_params(incompressible=1, mhd=1, boussinesq=1, stratification=1, strat_direction=2,
                          anisotropic_diffusion=1, supertimestepping=1, sts_variables=["th"], safety_sts=safety_sts,
                          gridsize=(n, n, n), boxsize=(L, L, L), reynolds=1e4, reynolds_magnetic=1e4,
                          reynolds_ani=20.0, N2=1.0, OmegaT2=1.0, cfl=1.5, form=SPK_FORM_FP32,
                          t_final=1e30, toutput_flow=1e30)


def mti_state(p):
    """Seeded white noise of amplitude 1e-4 in u (seed 3) and theta (seed 4),
    B0 = 1e-3 x; spectral layout (the first step's cleaning projects u)."""
    from spooky_b200.initial import to_spectral
    shape = (p.nx, p.ny, p.nz)
    u = 1e-4 * np.random.default_rng(3).standard_normal((3,) + shape)
    th = 1e-4 * np.random.default_rng(4).standard_normal(shape)
    B = np.zeros((3,) + shape)
    B[0] += 1e-3
    return to_spectral(np.concatenate([u, B, th[None]]))


def mti_timing(n, steps, warmup, stream):
    """Config 3 at n^3: `warmup` steps, then `steps` steps between CUDA events.
    Returns (ms per step, RKL2 stages per cycle, kernels per recorded step,
    simulated time, (dt_hyp, dt_par, dt_sts, dt), energies)."""
    import torch
    import spooky_b200 as S
    p = mti_params(n)
    ctx = S.Context(p, stream=stream.cuda_stream)
    ctx.set_state(mti_state(p))
    ctx.advance(warmup)
    ctx.synchronize()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ctx.synchronize()
    t, _, _ = ctx.get_time()
    hyp, par, sts, cur = ctx.compute_dt()
    s_rkl = int(1 + 4.0 * (1.0 + 2.0 * cur / sts) / (1.0 + np.sqrt(9.0 + 16.0 * cur / sts)))
    kps = ctx.step_info()[0]
    e, _ = ctx.budgets()
    ctx.close()
    return ms, s_rkl, kps, t, (hyp, par, sts, cur), e


def mti_sigma(k, chi, nu, eta, vA2, N2, OmegaT2):
    """Growth rate of the magnetothermal instability for k along B0: the
    largest real root of the dispersion cubic of the reference's MTI test
    (tests/mti-eigenmode/mti_disp_rel.py:44-70) with omega_T^2 kept general,
    x = chi k^2, Pr = nu/chi, q = eta/chi:
    s^3 + x(1+q+Pr) s^2 + (N2 + k^2 vA^2 + (q+Pr+qPr) x^2) s
    + qPr x^3 + N2 q x + k^2 vA^2 x - OmegaT2 x = 0."""
    x, Pr, q = chi * k * k, nu / chi, eta / chi
    c = [1.0, x * (1 + q + Pr), N2 + k * k * vA2 + (q + Pr + q * Pr) * x * x,
         q * Pr * x ** 3 + N2 * q * x + k * k * vA2 * x - OmegaT2 * x]
    r = np.roots(c)
    return float(np.max(r[np.abs(r.imag) < 1e-12].real))


def mti_growth_rates(n, ns=(8, 10, 12, 16), t_end=7.0, t_fit=5.0, safety_sts=95):
    """Config 3 from its white-noise start to t_end: the slope of
    log|theta(k = m x)| over [t_fit, t_end] for each m in ns, against the
    dispersion relation.  safety_sts caps dt at that many dt_sts."""
    import torch
    import spooky_b200 as S
    p = mti_params(n, safety_sts)
    ctx = S.Context(p)
    ctx.set_state(mti_state(p))
    buf = torch.empty(ctx.shape_c, dtype=torch.complex128, device="cuda")
    ts, amps = [], []
    while True:
        ctx.advance(1)
        t = ctx.get_time()[0]
        ctx.get_state(buf)
        torch.cuda.synchronize()
        amps.append(buf[ctx.F - 1, list(ns), 0, 0].abs().cpu().numpy())
        ts.append(t)
        if t > t_end:
            break
    ctx.close()
    ts, amps = np.array(ts), np.array(amps)
    sel = ts >= t_fit
    out = []
    for i, m in enumerate(ns):
        fit = float(np.polyfit(ts[sel], np.log(amps[sel, i]), 1)[0])
        ana = mti_sigma(float(m), 1.0 / p.reynolds_ani, p.nu, p.nu_m, 1e-6, p.N2, p.OmegaT2)
        out.append({"k": m, "sigma_fit": fit, "sigma_dispersion": ana, "rel_err": abs(fit - ana) / ana})
    return {"modes": out, "fit_window": [t_fit, float(ts[-1])], "steps": int(len(ts)), "dt_cap_dt_sts": safety_sts,
            "dt_last": float(ts[-1] - ts[-2])}


def run_mti(args, world, rank, local_rank):
    import torch
    import spooky_b200 as S
    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream()
    ms, s_rkl, kps, t, (hyp, par, sts, cur), e = mti_timing(args.n, args.steps, args.warmup, stream)
    if rank == 0:
        print(json.dumps({
            "metric": f"{args.n}^3 Boussinesq-MHD + anisotropic conduction, RK3 + RKL2 steps/s (config 3)",
            "value": 1000.0 / ms, "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 passes, fp64 state", "data": "synthetic (seeded white noise)",
            "config": {"workload": f"{args.n}^3 box 2pi, N2 = omega_T^2 = 1, chi_par = 0.05, nu = eta = 1e-4, "
                                   f"B0 = 1e-3 x, RKL2 on theta, dt <= 95 dt_sts",
                       "rkl2_stages_per_cycle": s_rkl, "dt": cur, "dt_sts": sts, "dt_hyp": hyp},
            "mmode_steps_per_s": (1000.0 / ms) * args.n ** 3 / 1e6,
            "kernels_per_step_recorded": kps, "sim_time": t, "energies_finite": bool(np.isfinite(e).all()),
            "growth_rates": mti_growth_rates(args.n),
            "growth_rates_dt_over_4": mti_growth_rates(args.n, safety_sts=24),
        }), flush=True)


def run_closure(args, world, rank, local_rank):
    """The learned-closure configuration: a 256^3 MHD truth run (nu = eta =
    2e-4, config-2 fields) in the plain form, closure samples every 250
    steps, GPU training, and 64^3 runs with and without the closure to the
    truth's final time; one JSON line with the spectral errors against the
    filtered truth and the costs.  The default trains both networks on the
    same samples: the line's value is the tensor network's (variant 3, the
    configuration's 18 -> 64 -> 64 -> 64 -> 12 BF16 network), the
    eddy-coefficient network (variant 1) is reported beside it under
    "models"."""
    import torch
    from spooky_b200 import closure as C
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return
    nf, ncs = args.n, args.n // 4
    # weight of the energy-transfer error in the loss (None: the workflow's
    # per-variant default)
    transfer = (args.closure_transfer if args.closure_transfer is not None
                else C.TRANSFER_DEFAULT[args.closure_variant])
    extra = (1,) if args.closure_variant == 3 else ()
    r = C.run(n_fine=nf, n_coarse=ncs, steps=args.closure_steps, snap_every=max(args.closure_steps // 8, 1),
              train_steps=3000, batch=16384, lr=2e-3, variant=args.closure_variant, transfer=transfer,
              extra_variants=extra, log=lambda m: print(m, file=sys.stderr, flush=True))
    names = {1: "eddy-coefficient network, full field (8 invariants -> 32 -> 32 -> 2, FP32)",
             2: "eddy-coefficient network, small scales (8 invariants -> 32 -> 32 -> 2, FP32)",
             3: "tensor network (18 gradients -> 64 -> 64 -> 64 -> 12, BF16 tensor cores)"}
    models = {names[args.closure_variant]: {
        "error": r["error_closure"], "error_u": r["error_u_closure"], "error_b": r["error_b_closure"],
        "energy": r["energy_closure"], "run_seconds": r["seconds_closure"], "cost_advantage": r["cost_advantage"],
        "train_seconds": r["train_seconds"], "loss": {"initial": r["loss_initial"], "final": r["loss_final"]}}}
    for v in extra:
        d = r[f"v{v}"]
        models[names[v]] = {"error": d["error"], "error_u": d["error_u"], "error_b": d["error_b"],
                            "energy": d["energy"], "run_seconds": d["seconds"], "cost_advantage": d["cost_advantage"],
                            "train_seconds": d["train_seconds"], "finite": d["finite"],
                            "loss": {"initial": d["loss_initial"], "final": d["loss_final"]}}
    print(json.dumps({
        "metric": f"{ncs}^3 learned-closure run vs filtered {nf}^3 truth: RMS relative shell-spectrum error",
        "value": r["error_closure"], "unit": "relative error (shells 1..k_c)", "higher_is_better": False,
        "n_gpus": 1, "vs_baseline": None,
        "dtype": "fp64 state, " + ("bf16 MLP operands, fp32 accumulation" if args.closure_variant == 3 else "fp32 MLP"),
        "data": "synthetic (seeded config-2 fields)",
        "config": {"workload": f"MHD {nf}^3 truth (plain form, {args.closure_steps} steps, nu = eta = 2e-4) -> "
                               f"{ncs}^3 closure run, sharp filter k_c = {r['k_cut']}",
                   "train_steps": {"variant 1/2": 3000, "variant 3": 20000}, "batch": 16384,
                   "closure_variant": names[args.closure_variant],
                   "loss_transfer_weight": transfer},
        "models": models,
        "error_without_closure": r["error_plain"],
        "error_u": {"closure": r["error_u_closure"], "plain": r["error_u_plain"]},
        "error_b": {"closure": r["error_b_closure"], "plain": r["error_b_plain"]},
        "energy": {"truth": r["energy_truth"], "closure": r["energy_closure"], "plain": r["energy_plain"]},
        "t_end": r["t_end"], "truth_seconds": r["truth_seconds"], "closure_run_seconds": r["seconds_closure"],
        "plain_coarse_run_seconds": r["seconds_plain"], "cost_advantage": r["cost_advantage"],
        "train_seconds": r["train_seconds"], "loss": {"initial": r["loss_initial"], "final": r["loss_final"]},
        "shell_spectra": dict({k: [float("%.5g" % v) for v in r["spectrum_" + k][: r["k_cut"] + 1]]
                               for k in ("truth", "closure", "plain")},
                              **{f"variant{v}": [float("%.5g" % x) for x in r[f"v{v}"]["spectrum"][: r["k_cut"] + 1]]
                                 for v in extra}),
    }), flush=True)


def run_closure_probe(args, world, rank, local_rank):
    """The closure's fused inference alone, the small case for ncu captures
    of its z pass: a --n^3 MHD context in the plain form (closure variant
    --closure-variant, 0: none; fixed dt 1e-3; config-2 fields) with the
    workflow's initial network (tensor network: output weights at scale 1),
    W warm-up + K steps timed with CUDA events; one short JSON line with the
    ms per step and the per-pass times."""
    import torch
    import spooky_b200 as S
    from spooky_b200 import closure as C
    from spooky_b200.initial import mhd_random_state
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return
    v, n = args.closure_variant, args.n
    L = 2 * np.pi
    p = default_params(gridsize=(n,) * 3, boxsize=(L, L, L), incompressible=1, mhd=1, reynolds=5000.0,
                       reynolds_magnetic=5000.0, cfl=1.5, form=SPK_FORM_PLAIN, closure=v, t_final=1e30,
                       toutput_flow=1e30, fixed_dt=1e-3)
    stream = torch.cuda.Stream()
    ctx = S.Context(p, stream=stream.cuda_stream)
    ctx.set_state(mhd_random_state(p, 1, 2))
    if v == 3:
        ctx.closure_set(C.init_params3(0, out=1.0))
    elif v in (1, 2):
        ctx.closure_set(C.init_params(0))
    ctx.advance(args.warmup)
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"closure_probe": True, "n": n, "closure_variant": v, "form": "plain",
                      "ms_per_step": e0.elapsed_time(e1) / args.steps, "steps": args.steps, "warmup": args.warmup,
                      "passes": ctx.profile_passes(5)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the reference-build, config-3 and config-4 legs of the default line")
    ap.add_argument("--ensemble", action="store_true",
                    help="batched-ensemble workload instead: --boxes independent HD/MHD boxes (config 4)")
    ap.add_argument("--boxes", type=int, default=512)
    ap.add_argument("--mti", action="store_true",
                    help="config 3 instead: Boussinesq MHD + anisotropic conduction with RKL2 super-time-stepping")
    ap.add_argument("--closure", action="store_true",
                    help="learned-closure workload instead: --n truth, --n/4 closure run (config 5)")
    ap.add_argument("--closure-steps", type=int, default=2000)
    ap.add_argument("--closure-variant", type=int, default=3, choices=[1, 2, 3],
                    help="3 (default): the tensor network, with variant 1 trained and run beside it")
    ap.add_argument("--closure-transfer", type=float, default=None,
                    help="weight of the energy-transfer error in the closure loss (default: 0 variant 1, "
                         "4 variant 2, 0 variant 3)")
    ap.add_argument("--closure-probe", action="store_true",
                    help="the closure's fused inference alone: --n^3 MHD, plain form, --closure-variant network "
                         "(the small case for ncu captures of its z pass)")
    ap.add_argument("--profile-form", default="fp32", choices=["fp32", "plain"],
                    help="the form of --profile-run")
    ap.add_argument("--profile-run", action="store_true",
                    help="one form only (--profile-form), W warm-up + K timed steps, one short JSON line "
                         "(the small case for ncu captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if args.ensemble:
        run_ensemble(args, world, rank, local_rank)
        return
    if args.mti:
        run_mti(args, world, rank, local_rank)
        return
    if args.closure_probe:
        run_closure_probe(args, world, rank, local_rank)
        return
    if args.closure:
        run_closure(args, world, rank, local_rank)
        return

    import torch
    import torch.distributed as dist
    import spooky_b200 as S

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.n
    U0 = mhd_random_state(workload_params(n, SPK_FORM_PLAIN))
    stream = torch.cuda.Stream()

    def timed_run(form, sampler_path=None):
        ctx = S.Context(workload_params(n, form), stream=stream.cuda_stream)
        ctx.set_state(U0)
        ctx.advance(args.warmup)
        ctx.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local_rank, sampler_path) if sampler_path else None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.advance(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        ctx.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        return ctx, max_over_ranks(ms), clocks

    if args.profile_run:
        ctxp, msp, _ = timed_run(SPK_FORM_PLAIN if args.profile_form == "plain" else SPK_FORM_FP32)
        kps, bytes_step = ctxp.step_info()
        if rank == 0:
            print(json.dumps({"profile_run": True, "form": args.profile_form, "n": n, "ms_per_step": msp,
                              "steps": args.steps,
                              "warmup": args.warmup, "kernels_per_step": kps, "step_bytes": bytes_step}),
                  flush=True)
        del ctxp
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    import tempfile
    clk_fd, clk_path = tempfile.mkstemp(prefix=f"spk_bench_clocks_rank{rank}_", suffix=".csv")
    os.close(clk_fd)
    ctx32, ms32, clocks = timed_run(SPK_FORM_FP32, clk_path)
    kps, bytes_step = ctx32.step_info()
    ctx64, ms64, _ = timed_run(SPK_FORM_PLAIN)
    _, bytes_step64 = ctx64.step_info()

    # FP32 form vs the FP64 plain form after the same steps from the same state
    U32 = ctx32.get_state()
    U64 = ctx64.get_state()
    rel = float(np.linalg.norm((U32 - U64).ravel()) / np.linalg.norm(U64.ravel()))
    t32 = ctx32.get_time()
    prof64 = ctx64.profile_passes(reps=5)   # after the comparison: profiling rewrites the state
    del ctx64
    torch.cuda.empty_cache()

    # end to end through the public API with host buffers: initial state H2D
    # from pinned memory, per step an energy-budget read-back (D2H), final
    # state D2H into pinned memory
    hostU = torch.from_numpy(U0.view(np.float64).copy()).pin_memory()
    hostOut = torch.empty_like(hostU).pin_memory()
    state_bytes = hostU.numel() * 8
    ctxe = S.Context(workload_params(n, SPK_FORM_FP32), stream=stream.cuda_stream)
    ctxe.set_state(hostU)
    ctxe.advance(args.warmup)
    ctxe.budgets()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctxe.set_state(hostU)
    for _ in range(args.steps):
        ctxe.advance(1)
        ctxe.budgets()
    ctxe.get_state(hostOut)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    del ctxe

    # per-pass roofline on the FP32 context (its state is no longer needed)
    prof = ctx32.profile_passes(reps=5)
    peak, peak_kind = peaks()
    for pz in prof:
        pz["gbs"] = pz["bytes"] / (pz["ms"] * 1e-3) / 1e9
        pz["frac_of_peak"] = pz["gbs"] / peak
        pz["share_of_step"] = pz["ms"] * pz["launches_per_step"] / ms32
    for pz in prof64:
        pz["gbs"] = pz["bytes"] / (pz["ms"] * 1e-3) / 1e9
        pz["frac_of_peak"] = pz["gbs"] / peak
        pz["share_of_step"] = pz["ms"] * pz["launches_per_step"] / ms64
    dom = max(prof, key=lambda d: d["ms"] * d["launches_per_step"])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(dom["name"], {}).get("dram_bytes_per_launch_256")
        except Exception:
            traffic = None

    # the same FP32 step on a state with content outside the 2/3 mask (1e-3 of
    # the norm): the path that carries the dealiased-out modes through every
    # stage, which a band-limited state lets the step skip
    Um = masked_noise_state(workload_params(n, SPK_FORM_PLAIN), U0)
    ctxm = S.Context(workload_params(n, SPK_FORM_FP32), stream=stream.cuda_stream)
    ctxm.set_state(Um)
    ctxm.advance(args.warmup)
    ctxm.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctxm.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_masked = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    _, bytes_masked = ctxm.step_info()
    ctxm.close()
    del ctxm
    torch.cuda.empty_cache()
    untrimmed = {"value": world * 1000.0 / ms_masked, "unit": "steps/s", "ms_per_step": ms_masked,
                 "bytes_per_step": bytes_masked,
                 "step_hbm_frac": bytes_masked / (ms_masked * 1e-3) / 1e9 / peaks()[0],
                 "what": "FP32 form, same workload plus solenoidal noise of 1e-3 of the state's norm on the "
                         "modes outside the 2/3 mask: the dealiased-out modes are carried through every stage"}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        del ctx32
        torch.cuda.empty_cache()
        try:
            extras["reference_cufft"] = reference_cufft_leg(workload_params(n, SPK_FORM_PLAIN), U0, args.warmup,
                                                            args.steps, U64)
            rc = extras["reference_cufft"]
            if "value" in rc:
                rc["plain_fp64_over_reference"] = (1000.0 / ms64) / rc["value"]
                rc["fp32_over_reference"] = (1000.0 / ms32) / rc["value"]
        except Exception as ex:   # the extra legs never stop the headline line
            extras["reference_cufft"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
        try:
            ms3, s3, k3, t3, dts3, _ = mti_timing(256, 10, 3, stream)
            extras["config3_sample"] = {
                "value": 1000.0 / ms3, "unit": "steps/s", "ms_per_step": ms3, "steps": 10, "warmup": 3,
                "rkl2_stages_per_cycle": s3, "dt": dts3[3], "kernels_per_step": k3,
                "workload": "256^3 Boussinesq MHD + anisotropic conduction, RKL2 on theta (bench.py --mti)"}
        except Exception as ex:
            extras["config3_sample"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
        try:
            boxes = ensemble_boxes(512)
            params = [p for _, p in boxes]
            states = [box_state(i, p) for i, p in boxes]
            msu, ms4, tt4, k4, fin4 = ensemble_timing(params, states, 20, 3, stream)
            extras["config4_sample"] = {
                "value": 512 * 20 / (ms4 * 1e-3), "unit": "box-steps/s", "steps": 20, "warmup": 3,
                "untuned_value": 512 * 20 / (msu * 1e-3), "autotune_seconds": tt4, "kernels_per_step": k4,
                "all_finite": fin4,
                "workload": "512 independent boxes, sizes {16,24,32,48,64}^3, HD/MHD, FP32 (bench.py --ensemble)"}
        except Exception as ex:
            extras["config4_sample"] = {"unavailable": f"{type(ex).__name__}: {ex}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(n)

    if rank == 0:
        value = world * 1000.0 / ms32
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 passes, fp64 state", "data": "synthetic (seeded random fields)",
            "config": config_dict(n, world),
            "plain_fp64": {"value": world * 1000.0 / ms64, "unit": "steps/s", "ms_per_step": ms64,
                           "bytes_per_step": bytes_step64,
                           "step_hbm_frac": bytes_step64 / (ms64 * 1e-3) / 1e9 / peak,
                           "passes": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in pz.items()}
                                      for pz in prof64]},
            "fp32_vs_fp64_rel_l2": rel, "fp32_vs_fp64_after_steps": args.warmup + args.steps,
            "sim_time": t32[0], "last_dt": t32[1],
            "mmode_steps_per_s": value * n ** 3 / 1e6,
            "step_bytes": bytes_step, "step_hbm_frac": bytes_step / (ms32 * 1e-3) / 1e9 / peak,
            "roofline": {"bound": "hbm", "kernel": dom["name"], "achieved": dom["gbs"], "peak": peak,
                         "unit": "GB/s", "frac": dom["gbs"] / peak, "traffic": traffic,
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                         "algorithmic_bytes_per_launch": dom["bytes"], "ms_per_launch": dom["ms"]},
            "passes": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in pz.items()} for pz in prof],
            "clocks": clocks,
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "steps/s",
                    "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps + 128,
                    "what": "C ABI with host pinned buffers: state H2D at start, per-step spk_advance + "
                            "spk_budgets read-back (128 B), state D2H at end"},
            "gpu_launches": kps * args.steps,
            "kernels_per_step": kps,
            "cpu_baseline": cpu,
            "untrimmed": untrimmed,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
