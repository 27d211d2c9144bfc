"""CPU tests of the libconfig-format reader behind spk_params_from_file /
spk_params_from_string: the reference's keys and defaults
(Parameters::Parameters, src/parameters/parameters.cu:59-505), libconfig's
typed lookups (no automatic int -> float conversion), the STS variable list
and Parameters::checkParameters (:511-566).  No GPU call is made."""
import os

import numpy as np
import pytest

import spooky_b200 as S
from spooky_b200.params import Params, default_params, SPK_STS_RKL2

FULL = """
# a configuration in the reference's layout
configname = "MTI-like" "test";   // adjacent strings concatenate

modules:
{
    debug = 0;
    incompressible = true;
    heat_equation = false;
    boussinesq = TRUE;
    stratification = true;
    strat_direction = 0x2;
    mhd = true;
    anisotropic_diffusion = true;
    supertimestepping = true;
    sts_algorithm = "rkl2";
    sts_variables = ("th");
};

physics:
{
    boxsize = (1.0, 2.0, 3.5);
    gridsize = (64, 32, 16);
    reynolds = 100000.0;
    reynolds_thermic = 1e6;
    reynolds_magnetic = 2.5e4;
    reynolds_anisotropic = 100.0;
    brunt_vaissala_squared = 0.1;
    mti_frequency_squared = 1.0;
};

/* code parameters
   over several lines */
code:
{
    cfl = 1.2;
    cfl_par = 0.9;
    safety_sts = 100;
    safety_source = 0.25;
    t_initial = 0.5;
    t_final = 2.0;
    antialiasing = false;
    restart = false;
};

output: { timevar_step = 0.1; snapshot_step = 0.5; timevar_vars = ["ev", "em"]; };
"""


def test_full_configuration_matches_the_reference_defaults_and_keys():
    p = S.params_from_string(FULL)
    want = default_params(incompressible=1, boussinesq=1, stratification=1, strat_direction=2, mhd=1,
                          anisotropic_diffusion=1, supertimestepping=1, sts_variables=["th"],
                          boxsize=(1.0, 2.0, 3.5), gridsize=(64, 32, 16), reynolds=1e5, reynolds_thermic=1e6,
                          reynolds_magnetic=2.5e4, reynolds_ani=100.0, N2=0.1, OmegaT2=1.0, cfl=1.2, cfl_par=0.9,
                          safety_sts=100, safety_source=0.25, t_initial=0.5, t_final=2.0, antialiasing=0,
                          toutput_flow=0.5)
    for name, _ in Params._fields_:
        assert getattr(p, name) == getattr(want, name), name
    assert p.sts_algorithm == SPK_STS_RKL2
    assert p.sts_vars_mask == 1 << 6   # th is the seventh field of vx vy vz bx by bz th


def test_empty_configuration_gives_the_reference_defaults_and_fails_the_module_check():
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string("")
    assert e.value.code == 6   # neither incompressible nor heat_equation


def test_integer_written_for_a_float_key_keeps_the_default():
    # libconfig's lookup_float does not accept an integer setting (no automatic
    # conversion), so the reference keeps reynolds = 1.0
    p = S.params_from_string("modules: { incompressible = true; }; physics: { reynolds = 100; };")
    assert p.nu == 1.0
    p = S.params_from_string("modules: { incompressible = true; }; physics: { reynolds = 100.0; };")
    assert p.nu == 1.0 / 100.0
    # and a float written for an integer key, or a number for a bool key, keeps the default
    p = S.params_from_string("modules: { incompressible = true; mhd = 1; }; physics: { gridsize = (16.0, 8, 8); };")
    assert p.mhd == 0 and (p.nx, p.ny, p.nz) == (32, 8, 8)


def test_sts_variable_list():
    base = "modules: { incompressible = true; mhd = true; supertimestepping = true; sts_algorithm = \"rkl2\"; %s };"
    p = S.params_from_string(base % 'sts_variables = ("bx", "vz", "nope");')
    assert p.supertimestepping == 1 and p.sts_vars_mask == (1 << 3) | (1 << 2)
    p = S.params_from_string(base % 'sts_variables = ["by"];')
    assert p.sts_vars_mask == 1 << 4
    # an empty or missing list switches super-time-stepping off (parameters.cu:123-147)
    assert S.params_from_string(base % "sts_variables = ();").supertimestepping == 0
    assert S.params_from_string(base % "").supertimestepping == 0
    # without supertimestepping the list is not read
    p = S.params_from_string('modules: { incompressible = true; sts_variables = ("vx"); };')
    assert p.supertimestepping == 0 and p.sts_vars_mask == 0


def test_heat_equation_sts_variable_and_unknown_algorithm():
    p = S.params_from_string('modules: { heat_equation = true; supertimestepping = true; sts_algorithm = "rkl1";'
                             ' sts_variables = ("th"); };')
    assert p.sts_vars_mask == 1 and p.sts_algorithm == 2
    # the three names of RKLegendre::compute_cycle (rkl.cu:185-199); any other is a configuration error
    text = 'modules: { heat_equation = true; supertimestepping = true; sts_algorithm = "%s"; sts_variables = ("th"); };'
    for name, code in (("sts", 1), ("rkl1", 2), ("rkl2", 3)):
        assert S.params_from_string(text % name).sts_algorithm == code, name
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string(text % "rkl3")
    assert "sts_algorithm" in str(e.value)


@pytest.mark.parametrize("text", [
    "a : 1; b = 2, c = 3",                          # ':' assignment, ',' terminator, last terminator optional
    "g = { h = { i = [1, 2, 0x10]; }; };",
    "l = (1, \"two\", 3.0, (4, 5), { x = 1; });",   # lists mix types and nest
    "s = \"esc \\\" \\\\ \\t \\x41\";",
    "f = (1e3, -2.5E-2, .5, 7.);",
    "big = 5000000000; lng = 12L;",
])
def test_syntax_accepted(text):
    # parse errors raise; module errors (no module chosen) give code 6
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string(text)
    assert e.value.code == 6


@pytest.mark.parametrize("text,line", [
    ("modules:\n{\n  incompressible true;\n};", 3),
    ("a = [1, 2.0];", 1),
    ("a = (1, 2,);", 1),
    ("\n\na = \"unterminated;\n", 3),
    ("x = {\n y = 1;\n", 3),
    ("a = 1; a = 2;", 1),
    ("@include \"other.cfg\"", 1),
])
def test_syntax_errors_name_the_line(text, line):
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string(text)
    assert e.value.code == 1
    assert f"line {line}:" in str(e.value)


def test_module_consistency_checks():
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string("modules: { incompressible = true; heat_equation = true; };")
    assert e.value.code == 6 and "mutually exclusive" in str(e.value)
    with pytest.raises(S.SpookyError) as e:
        S.params_from_string("modules: { incompressible = true; anisotropic_diffusion = true; boussinesq = true; };")
    assert e.value.code == 6


def test_read_from_file(tmp_path):
    path = tmp_path / "spooky.cfg"
    path.write_text(FULL)
    p = S.params_from_file(str(path))
    q = S.params_from_string(FULL)
    for name, _ in Params._fields_:
        assert getattr(p, name) == getattr(q, name), name
    with pytest.raises(S.SpookyError) as e:
        S.params_from_file(os.path.join(str(tmp_path), "missing.cfg"))
    assert e.value.code == 1 and "cannot open" in str(e.value)


@pytest.mark.parametrize("kw", [
    dict(incompressible=1, mhd=1, gridsize=(256, 256, 256), boxsize=(2 * np.pi,) * 3, reynolds=1e3,
         reynolds_magnetic=1e3, cfl=1.5, t_final=1e30, toutput_flow=1e30),
    dict(incompressible=1, mhd=1, boussinesq=1, stratification=1, strat_direction=2, anisotropic_diffusion=1,
         supertimestepping=1, sts_variables=["th"], safety_sts=95, gridsize=(64, 32, 16), boxsize=(1.0, 2.0, 0.5),
         reynolds=1e4, reynolds_magnetic=1e4, reynolds_ani=20.0, N2=1.0, OmegaT2=1.0, cfl=1.5),
    dict(heat_equation=1, gridsize=(1024, 2, 2), reynolds_thermic=1000.0, cfl_par=1.5, antialiasing=0,
         t_final=10.0, toutput_flow=5.0),
])
def test_cfg_text_round_trip(kw):
    """params.cfg_text writes a spooky.cfg (the reference's keys) that reads
    back to the same parameters: the file given to the reference's own build
    when it is timed on the same workload."""
    from spooky_b200.params import cfg_text
    p = default_params(**kw)
    q = S.params_from_string(cfg_text(p))
    for name, _ in p._fields_:
        assert getattr(q, name) == getattr(p, name), name


CFG_EXTRA = """
configname = "extras";
modules: { incompressible = true; mhd = true; };
physics: { boxsize = (1.0, 1.0, 1.0); gridsize = (16, 16, 8); reynolds = 100.0; };
code: { t_final = 2.0; max_walltime_elapsed = 1.5; symmetries_step = 7; };
output: {
    timevar_step = 0.25;
    snapshot_step = 0.5;
    output_dir = "/tmp/run";
    timevar_vars = ("t", "ev", "em", "w2", "hc");
    spectra_vars = ["Kx", "Mx"];
    vorticity = true;
};
"""


def test_cfg_lookup_reads_any_key_with_libconfig_typing():
    t = CFG_EXTRA
    assert S.cfg_lookup(t, "output.timevar_step", "float") == 0.25
    assert S.cfg_lookup(t, "output.output_dir", "string") == "/tmp/run"
    assert S.cfg_lookup(t, "output.timevar_vars", "strings") == ["t", "ev", "em", "w2", "hc"]
    assert S.cfg_lookup(t, "output.spectra_vars", "strings") == ["Kx", "Mx"]
    assert S.cfg_lookup(t, "code.symmetries_step", "int") == 7
    assert S.cfg_lookup(t, "output.vorticity", "bool") is True
    # typed: an int key does not satisfy a float lookup, absent keys give the default
    assert S.cfg_lookup(t, "code.symmetries_step", "float", -1.0) == -1.0
    assert S.cfg_lookup(t, "output.nothing", "string", "dflt") == "dflt"
    with pytest.raises(S.SpookyError):
        S.cfg_lookup("physics: { a = ; }", "physics.a", "float")


def test_command_line_overrides_follow_main_cu():
    """src/main.cu:28-134: -n overrides the grid, --with-2d forces 2D,
    --output-dir the cfg's output_dir, -t the wall-clock limit (x 0.95),
    -r the restart number (absent: a new run)."""
    from spooky_b200 import __main__ as M
    a = M.parse_args(["--input-dir", "/x", "--output-dir", "/y", "-r", "3", "-t", "1", "30", "0",
                      "-n", "32", "16", "8", "--with-2d", "--stats", "5"])
    assert a.input_dir == "/x" and a.restart == 3 and a.ngrid == [32, 16, 8] and a.with_2d and a.stats == 5
    rc = M.run_config(CFG_EXTRA, a)
    assert rc["output_dir"] == "/y"
    assert abs(rc["max_walltime_hours"] - 0.95 * 1.5) < 1e-15
    assert rc["toutput_time"] == 0.25 and rc["timevar_vars"][3] == "w2"
    b = M.parse_args([])
    assert b.restart is None and b.ngrid is None and not b.with_2d
    rc = M.run_config(CFG_EXTRA, b)
    assert rc["output_dir"] == "/tmp/run" and rc["max_walltime_hours"] == 1.5


def test_mti_dispersion_cubic_of_the_bench_matches_the_reference_golden():
    """bench.mti_sigma (the growth rate config 3's check uses) reproduces the
    reference's own dispersion cubic (tests/golden/mti_eigenmode.json, from
    tests/mti-eigenmode/mti_disp_rel.py) at its parameters."""
    import json
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import mti_sigma
    g = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mti_eigenmode.json")))
    s = mti_sigma(2 * np.pi * g["n_mode"], 1.0 / g["Pe"], 1.0 / g["ReNu"], 1.0 / g["ReEta"], g["B0"] ** 2, g["N2"],
                  g["OmegaT2"])
    assert abs(s - g["sigma_dispersion_cubic"]) < 1e-13
    assert abs(s - g["sigma_check_script"]) < 1e-13


SHEARING = """
modules: { incompressible = true; mhd = true; shearing = true; rotating = true; };
physics: { boxsize = (1.0, 3.0, 1.0); gridsize = (16, 16, 16); omega = 1.0; shear = 1.5; };
output: { snapshot_step = %s; };
"""


# shear period ly / (S lx) = 2
@pytest.mark.parametrize("step, want", [(0.5, 2.0), (2.0, 1.0), (7.5, 3.0)])
def test_shearing_keys_and_snapshot_step(step, want):
    """modules.shearing / rotating and physics.shear / omega; with shearing
    the snapshot step becomes the shear period ly / (S lx) when shorter, else
    int(step / period) -- the reference's arithmetic (parameters.cu:551-562),
    kept as written: a count of periods, not their length."""
    p = S.params_from_string(SHEARING % step)
    assert (p.shearing, p.rotating, p.shear, p.omega) == (1, 1, 1.5, 1.0)
    assert p.toutput_flow == want
    q = S.params_from_string((SHEARING % step).replace("shearing = true", "shearing = false"))
    assert q.shearing == 0 and q.toutput_flow == step
