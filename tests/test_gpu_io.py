"""GPU checks of the real-space state, snapshots and restarts, the
time-series diagnostics and the entry points that act on a caller's state
array -- all through the C ABI, against the oracle or a numpy restatement.

  real fields      spk_get_state_real / spk_set_state_real vs numpy's irfftn / rfftn
  snapshots        spk_write_snapshot / spk_read_snapshot: the reference's layout
                   (src/io/hdf5_io.cu:19-111), restart selection (:114-276)
  restart          a run continued from a snapshot equals the uninterrupted run
  diagnostics      spk_diagnostics vs a numpy restatement of spooky_output_functions.cu
  caller memory    spk_advance_fields / spk_rk3_fields / spk_compute_dt_fields /
                   spk_rkl_cycle_fields vs the context forms and the oracle
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from fields import grid, kvectors, random_solenoidal, to_spectral
from spooky_b200 import Context, Supervisor, fileCounter
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, cfg_text, default_params

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def mhd_state(p, seed):
    u = random_solenoidal(p, seed, kpeak=3.0)
    B = random_solenoidal(p, seed + 1, kpeak=3.0, rms=0.6)
    B[0] += 0.2
    fields = [u, B]
    if p.boussinesq:
        fields.append(0.3 * np.random.default_rng(seed + 2).standard_normal((1, p.nx, p.ny, p.nz)))
    return to_spectral(np.concatenate(fields))


def torch_dev(arr):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 8, 12), (8, 24, 2)])
def test_real_fields_round_trip(shape):
    p = default_params(incompressible=1, mhd=1, boussinesq=1, gridsize=shape, boxsize=(1.0, 2.0, 1.5))
    U = mhd_state(p, 3)
    ctx = Context(p)
    ctx.set_state(U)
    R = ctx.get_state_real()
    Rn = np.stack([np.fft.irfftn(u, s=shape, axes=(0, 1, 2)) for u in U])
    assert rel_l2(R, Rn) < 1e-13
    # back to spectral: the unnormalised R2C of the same real fields
    ctx.set_state_real(Rn)
    assert rel_l2(ctx.get_state(), np.stack([np.fft.rfftn(r) for r in Rn])) < 1e-13


def test_heat_equation_real_fields():
    p = default_params(heat_equation=1, gridsize=(64, 4, 2), antialiasing=0)
    T = np.random.default_rng(1).standard_normal((1, 64, 4, 2))
    ctx = Context(p)
    ctx.set_state_real(T)
    assert rel_l2(ctx.get_state(), to_spectral(T)) < 1e-13
    assert rel_l2(ctx.get_state_real(), T) < 1e-13


def test_snapshot_file_round_trip(tmp_path):
    p = default_params(incompressible=1, mhd=1, gridsize=(16, 12, 8), t_final=10.0, toutput_flow=0.5)
    U = mhd_state(p, 4)
    a = Context(p)
    a.set_state(U)
    a.advance(3)
    a.synchronize()
    path = str(tmp_path / "snap0002.h5")
    a.write_snapshot(path, t_start=0.0, t_lastsnap=0.5, t_lastvar=0.25)
    import test_hdf5 as H
    names = ["vx", "vy", "vz", "bx", "by", "bz"]
    nr = 16 * 12 * 8
    spec = {"t_start": (np.float64, 1), "t_save": (np.float64, 1), "t_lastsnap": (np.float64, 1),
            "t_lastvar": (np.float64, 1), "step": (np.int32, 1)}
    spec.update({n: (np.float64, nr) for n in names})
    d = H.h5_read(path, spec)
    t, _, step = a.get_time()
    assert d["t_save"][0] == t and d["step"][0] == step == 3
    assert d["t_lastsnap"][0] == 0.5 and d["t_lastvar"][0] == 0.25 and d["t_start"][0] == 0.0
    R = a.get_state_real()
    for f, n in enumerate(names):
        assert np.array_equal(d[n], R[f].ravel())
    w = H.SpecWalk(open(path, "rb").read())
    assert sorted(w.walk()) == sorted(spec)
    b = Context(p)
    tls, tlv = b.read_snapshot(path)
    assert (tls, tlv) == (0.5, 0.25)
    assert b.get_time()[0] == t and b.get_time()[2] == 3
    assert rel_l2(b.get_state(), a.get_state()) < 1e-13


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_restart_continues_the_run(tmp_path, form):
    """Snapshots every 0.05 to t = 0.2 through the Supervisor; a second
    Supervisor restarted from snapshot 2 (-r 2) reaches the same state at
    t = 0.2 as the uninterrupted run, up to the real-space round trip of the
    snapshot; -r -1 picks the most recent file and num_save continues."""
    L = 2 * np.pi
    p = default_params(incompressible=1, mhd=1, gridsize=(32, 32, 32), boxsize=(L, L, L), reynolds=300.0,
                       reynolds_magnetic=300.0, t_final=0.2, toutput_flow=0.05, form=form)
    U0 = mhd_state(p, 7)
    out = str(tmp_path / "run")
    a = Supervisor(p, output_dir=out, toutput_time=0.05, timevar_vars=["t", "ev", "em", "w2", "j2", "hc"])
    a.fields.set(U0)
    a.initialDataDump()
    a.executeMainLoop()
    assert fileCounter(os.path.join(out, "data")) == 4
    Ua = a.fields.get()
    ta = a.timestep.current_time
    b = Supervisor(p, output_dir=out, restart_num=2)
    assert b.inout.num_save == 3 and abs(b.timestep.current_time - 0.1) < 1e-12
    assert b.inout.t_lastsnap == pytest.approx(0.1)
    b.executeMainLoop()
    assert b.timestep.current_time == pytest.approx(ta, abs=1e-13)
    assert b.timestep.current_step == a.timestep.current_step
    assert rel_l2(b.fields.get(), Ua) < (1e-12 if form == SPK_FORM_PLAIN else 1e-5)
    c = Supervisor(p, output_dir=out, restart_num=-1)
    assert c.inout.num_save == 5 and c.timestep.current_time == pytest.approx(ta, abs=1e-13)
    # the time series: header, one line per output time, the reference's
    # format.  Its schedule has no tolerance (check_output.cu:31): at t = 0.2
    # the accumulated t_lastvar (0.15000000000000002) leaves t - t_lastvar a
    # hair under 0.05, so run a writes t = 0, 0.05, 0.1, 0.15, as the
    # reference would, and the restarted run appends its own lines.
    lines = open(os.path.join(out, "timevar.spooky")).read().splitlines()
    assert lines[0].startswith("## This file contains") and lines[1].split() == ["##", "t", "ev", "em", "w2", "j2", "hc"]
    rows = [list(map(float, l.split())) for l in lines[2:]]
    assert [r[0] for r in rows[:4]] == pytest.approx([0.0, 0.05, 0.1, 0.15])
    assert all(r[3] > 0 and r[4] > 0 for r in rows)


def numpy_diagnostics(p, U):
    """spooky_output_functions.cu restated with numpy on the same state."""
    KX, KY, KZ = kvectors(p)
    n = p.nx * p.ny * p.nz
    shape = (p.nx, p.ny, p.nz)
    irf = lambda c: np.fft.irfftn(c, s=shape, axes=(0, 1, 2))
    kk = np.arange(p.nz // 2 + 1)
    we = np.where(kk > 0, 2.0, 1.0)[None, None, :]

    def energy(q):   # computeEnergy: Nyquist plane counted twice
        return 0.5 * np.sum(we * np.abs(q) ** 2) / n ** 2

    def curl(v):
        return np.stack([1j * (KY * v[2] - KZ * v[1]), 1j * (KZ * v[0] - KX * v[2]), 1j * (KX * v[1] - KY * v[0])])

    def helicity(v):
        K2 = KX ** 2 + KY ** 2 + KZ ** 2
        ik2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 1.0)
        A = -ik2 * (-curl(v))       # Helicity kernel: -ik2 * (-i k x V)
        return sum(np.mean(irf(A[c]) * irf(v[c])) for c in range(3))

    out = {}
    u = U[0:3]
    out["w2"] = sum(energy(c) for c in curl(u))
    out["hv"] = helicity(u)
    if p.mhd:
        B = U[3:6]
        out["j2"] = sum(energy(c) for c in curl(B))
        out["hm"] = helicity(B)
        out["hc"] = sum(np.mean(irf(u[c]) * irf(B[c])) for c in range(3))
        Br = np.stack([irf(B[c]) for c in range(3)])
        nb = 1e-16 + np.sqrt((Br ** 2).sum(0))
        out["thetaB"] = np.mean(np.abs(Br[2] / nb))
        out["bz2"] = np.mean((Br[2] / nb) ** 2)
        nh = 1e-16 + np.sqrt(Br[0] ** 2 + Br[1] ** 2)
        out["phiB"] = np.mean(np.arccos((np.abs(Br[0]) / nh).astype(np.float32)).astype(np.float64))
    if p.boussinesq:
        th = U[-1]
        out["dissgradT"] = energy(1j * KX * th) + energy(1j * KY * th) + energy(1j * KZ * th)
        w = curl(u)
        out["pv"] = sum(np.mean(irf(w[c]) * irf(g)) for c, g in enumerate((1j * KX * th, 1j * KY * th, 1j * KZ * th)))
    return out


def test_diagnostics_match_numpy():
    p = default_params(incompressible=1, mhd=1, boussinesq=1, gridsize=(16, 16, 12), boxsize=(1.0, 1.3, 0.9))
    U = mhd_state(p, 9)
    ctx = Context(p)
    ctx.set_state(U)
    got = ctx.diagnostics()
    want = numpy_diagnostics(p, U)
    for k, v in want.items():
        scale = max(abs(v), 1e-12 * max(abs(want["w2"]), 1.0))
        tol = 1e-6 if k == "phiB" else 1e-10
        assert abs(got[k] - v) <= tol * scale + 1e-14, (k, got[k], v)
    h = default_params(incompressible=1, gridsize=(16, 16, 16))
    c = Context(h)
    c.set_state(to_spectral(random_solenoidal(h, 2)))
    d = c.diagnostics()
    assert d["j2"] == -1.0 and d["hc"] == -1.0 and d["dissgradT"] == -1.0 and d["w2"] > 0


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
def test_entry_points_on_caller_memory(form):
    """The *_fields forms on a torch array give the context forms' results:
    advance_fields == set_state + advance (each call also cleans the array
    first, as every iteration of the reference's main loop does, so the two
    agree to rounding), compute_dt_fields == compute_dt (bitwise),
    rk3_fields == one RungeKutta3 of the oracle at the same dt, and the
    context's own state is left alone."""
    L = 2 * np.pi
    p = default_params(incompressible=1, mhd=1, gridsize=(32, 16, 16), boxsize=(L, L, L), reynolds=200.0,
                       reynolds_magnetic=200.0, form=form, t_final=100.0, toutput_flow=100.0)
    # a divergence-free state on the grid (numpy's round trip leaves the Nyquist planes of
    # the random fields with some divergence, which the first cleaning would remove)
    c0 = Context(p)
    c0.set_state(mhd_state(p, 11))
    c0.clean_divergence()
    U = c0.get_state()
    ref = Context(p)
    ref.set_state(U)
    ref.advance(4)
    ctx = Context(p)
    own = mhd_state(p, 12)
    ctx.set_state(own)
    Ud = torch_dev(U)
    ctx.advance_fields(Ud, 2)
    ctx.advance_fields(Ud, 2)          # the recorded graph is replayed for the same array
    ctx.synchronize()
    assert rel_l2(Ud.cpu().numpy(), ref.get_state()) < (1e-13 if form == SPK_FORM_PLAIN else 1e-6)
    assert ctx.get_time()[2] == 4
    # the context's own state is untouched and still advances correctly
    assert np.array_equal(ctx.get_state(), own)
    # compute_dt on caller memory
    Vd = torch_dev(U)
    c2 = Context(p)
    c2.set_state(U)
    assert np.array_equal(c2.compute_dt_fields(Vd), c2.compute_dt())
    # RungeKutta3 alone on caller memory, at the dt of the last compute_dt
    if form == SPK_FORM_PLAIN:
        o = O.Oracle(p)
        o.set_state(U)
        o.clean_divergence()
        o.step(1)
        dt = o.get_time()[1]
        c3 = Context(p)
        Wd = torch_dev(U)
        dts = c3.compute_dt_fields(Wd)
        assert abs(dts[3] - dt) <= 1e-13 * dt
        c3.rk3_fields(Wd)
        # the oracle's step cleans the state first and after; a clean field is unchanged by it
        assert rel_l2(Wd.cpu().numpy(), o.get_state()) < 1e-10


def test_rkl_cycle_on_caller_memory():
    p = default_params(heat_equation=1, gridsize=(128, 2, 2), boxsize=(4.0, 1.0, 1.0), reynolds_thermic=1.0,
                       cfl_par=0.5, safety_sts=1, t_final=0.5, toutput_flow=100.0, antialiasing=0,
                       supertimestepping=1, sts_algorithm="rkl2", sts_variables=["th"], integrator=1,
                       sts_every_step=1, fixed_dt=0.002 * 4.0 / 128)
    X, _, _ = grid(p)
    T0 = np.exp(-0.5 * X ** 2 / 0.01)[None]
    a = Context(p)
    a.set_state(to_spectral(T0))
    a.compute_dt()
    s_a = a.rkl_cycle()
    b = Context(p)
    b.set_state(to_spectral(T0))
    b.compute_dt()
    Td = torch_dev(to_spectral(T0))
    s_b = b.rkl_cycle_fields(Td)
    assert s_a == s_b > 1
    assert np.array_equal(Td.cpu().numpy(), a.get_state())


def test_command_line_run_with_restart_from_snapshot_zero(tmp_path):
    """The reference's test flow: initial fields written as snap0000.h5,
    then `spooky --input-dir D --output-dir D -r 0` (here python -m
    spooky_b200); Taylor-Green at 32^3 to t = 1 against its analytic decay
    (L1 < 1e-7, check-taylor-green.py:129-155)."""
    import test_hdf5 as H
    n = 32
    p = default_params(incompressible=1, gridsize=(n, n, n), reynolds=200.0, t_final=1.0, toutput_flow=0.5)
    X, Y, Z = grid(p)
    u0 = np.stack([0 * X, np.sin(2 * np.pi * Y) * np.cos(2 * np.pi * Z), -np.cos(2 * np.pi * Y) * np.sin(2 * np.pi * Z)])
    d = tmp_path
    (d / "data").mkdir()
    (d / "spooky.cfg").write_text(cfg_text(p, toutput_time=0.5).replace('output_dir = "./"', f'output_dir = "{d}"')
                                  .replace("output:\n{", 'output:\n{\n  timevar_vars = ("t", "ev", "w2");'))
    items = {"t_start": np.array([0.0]), "t_save": np.array([0.0]), "t_lastsnap": np.array([0.0]),
             "t_lastvar": np.array([0.0]), "step": np.array([0], dtype=np.int32)}
    for c, name in enumerate(("vx", "vy", "vz")):
        items[name] = u0[c].ravel()
    H.h5_write(d / "data" / "snap0000.h5", items)
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "spooky-git_b200"))
    r = subprocess.run([sys.executable, "-m", "spooky_b200", "--input-dir", str(d), "-r", "0"], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "cell_updates/s" in r.stdout
    assert fileCounter(str(d / "data")) == 2          # snapshots at t = 0.5 and 1
    R = H.h5_read(d / "data" / "snap0002.h5", {"vx": (np.float64, n ** 3), "vy": (np.float64, n ** 3),
                                               "vz": (np.float64, n ** 3), "t_save": (np.float64, 1)})
    t = R["t_save"][0]
    assert abs(t - 1.0) < 1e-14
    ua = u0 * np.exp(-2 * p.nu * t * (2 * np.pi) ** 2)
    got = np.stack([R[k].reshape(n, n, n) for k in ("vx", "vy", "vz")])
    assert np.abs(got - ua).sum() / n ** 3 < 1e-7
    rows = [l.split() for l in (d / "timevar.spooky").read_text().splitlines()[2:]]
    assert [float(r[0]) for r in rows] == pytest.approx([0.0, 0.5, 1.0])
