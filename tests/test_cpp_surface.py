"""The C++ surface (include/spooky_b200.hpp): a small program built with g++
against libspooky_b200.so reads a configuration through
spooky_b200::Parameters (CPU) and, on a GPU, runs Supervisor::executeMainLoop;
its output is compared with the Python binding of the same C ABI."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import spooky_b200 as S
from spooky_b200 import Context

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "spooky-git_b200", "lib")

CFG = """
modules: { incompressible = true; mhd = true; };
physics: { boxsize = (1.0, 1.0, 2.0); gridsize = (16, 8, 4); reynolds = 50.0; reynolds_magnetic = 20.0; };
code: { cfl = 1.2; t_final = 0.75; };
"""


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cpp") / "params_main")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "params_main.cpp"), "-L", LIBDIR, "-lspooky_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", out], check=True)
    return out


def run(program, cfg_text, tmp_path, *extra):
    path = tmp_path / "spooky.cfg"
    path.write_text(cfg_text)
    res = subprocess.run([program, str(path), *extra], check=True, capture_output=True, text=True)
    vals = {}
    for line in res.stdout.splitlines():
        k, _, v = line.partition(" ")
        vals[k] = v
    return vals


def test_cpp_parameters_match_the_python_reader(program, tmp_path):
    vals = run(program, CFG, tmp_path)
    p = S.params_from_string(CFG)
    for k in ("nx", "ny", "nz", "incompressible", "mhd", "boussinesq"):
        assert int(vals[k]) == getattr(p, k), k
    for k in ("lx", "ly", "lz", "nu", "nu_m", "cfl", "t_final"):
        assert float(vals[k]) == getattr(p, k), k


def test_cpp_errors_become_exceptions(program, tmp_path):
    vals = run(program, "modules: { incompressible = true; heat_equation = true; };", tmp_path)
    assert vals["error"].startswith("6 ")
    vals = run(program, "modules:\n{ incompressible = ; };", tmp_path)
    assert vals["error"].startswith("1 ") and "line 2" in vals["error"]


@pytest.mark.gpu
def test_cpp_supervisor_main_loop_matches_python(program, tmp_path):
    vals = run(program, CFG, tmp_path, "--run", "5")
    p = S.params_from_string(CFG)
    ctx = Context(p)
    U = np.zeros(ctx.shape_c, np.complex128)
    U[0, 0, 1, 0] = 0.25 * p.nx * p.ny * p.nz
    ctx.set_state(U)
    ctx.advance(5)
    ctx.synchronize()
    t, _, step = ctx.get_time()
    e, _ = ctx.budgets()
    assert int(vals["steps"]) == 5 and int(vals["step"]) == step == 5
    assert float(vals["time"]) == pytest.approx(t, rel=1e-14)
    assert float(vals["energy0"]) == pytest.approx(e[0], rel=1e-12)


@pytest.mark.gpu
def test_cpp_snapshots_and_restart(program, tmp_path):
    """Supervisor with an output directory: snapshots every toutput_flow in the
    reference's HDF5 layout, then Supervisor(p, 0, dir, -1) restarts from the
    most recent one (its time, step, t_lastsnap and state)."""
    cfg = CFG.replace("code: { cfl = 1.2; t_final = 0.75; };",
                      "code: { cfl = 1.2; t_final = 0.75; };\noutput: { snapshot_step = 0.25; };")
    out = tmp_path / "run"
    (out / "data").mkdir(parents=True)
    vals = run(program, cfg, tmp_path, "--snap", str(out))
    assert int(vals["last"]) == 3 and int(vals["num_save"]) == 4      # t = 0, 0.25, 0.5, 0.75
    assert float(vals["time"]) == pytest.approx(0.75, abs=1e-14)
    assert int(vals["restart_num_save"]) == 4
    assert float(vals["restart_time"]) == pytest.approx(0.75, abs=1e-14)
    assert float(vals["restart_lastsnap"]) == pytest.approx(0.75, abs=1e-12)
    assert int(vals["restart_step"]) > 0
    assert float(vals["restart_energy0"]) > 0
