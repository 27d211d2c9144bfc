"""spk_params_t as a ctypes structure, plus the reference's cfg defaults.

Field order and types mirror ``include/spooky_b200.h``.  Defaults follow
``Parameters::Parameters`` (src/parameters/parameters.cu:77-505 in
LorenzoLMP/spooky-git): every key has the default the reference uses when the
cfg omits it, and the diffusivities are the inverses of the ``reynolds*``
keys (:205-219).
"""
import ctypes

SPK_FORM_PLAIN = 0
SPK_FORM_FP32 = 1
SPK_STS_STS = 1
SPK_STS_RKL1 = 2
SPK_STS_RKL2 = 3
STS_ALGORITHMS = {"sts": SPK_STS_STS, "rkl1": SPK_STS_RKL1, "rkl2": SPK_STS_RKL2}
SPK_INT_RK3 = 0
SPK_INT_EULER = 1


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("incompressible", ctypes.c_int), ("heat_equation", ctypes.c_int),
        ("mhd", ctypes.c_int), ("boussinesq", ctypes.c_int),
        ("stratification", ctypes.c_int), ("strat_direction", ctypes.c_int),
        ("anisotropic_diffusion", ctypes.c_int),
        ("supertimestepping", ctypes.c_int), ("sts_algorithm", ctypes.c_int),
        ("sts_vars_mask", ctypes.c_uint),
        ("with2d", ctypes.c_int), ("antialiasing", ctypes.c_int),
        ("nu", ctypes.c_double), ("nu_m", ctypes.c_double), ("nu_th", ctypes.c_double),
        ("reynolds_ani", ctypes.c_double),
        ("N2", ctypes.c_double), ("OmegaT2", ctypes.c_double),
        ("cfl", ctypes.c_double), ("cfl_par", ctypes.c_double),
        ("cfl_sts", ctypes.c_double), ("safety_source", ctypes.c_double),
        ("safety_sts", ctypes.c_int),
        ("t_initial", ctypes.c_double), ("t_final", ctypes.c_double),
        ("toutput_flow", ctypes.c_double),
        ("fixed_dt", ctypes.c_double), ("integrator", ctypes.c_int),
        ("sts_every_step", ctypes.c_int), ("form", ctypes.c_int),
        ("closure", ctypes.c_int),
        ("closure_kc_frac", ctypes.c_double),
        ("shearing", ctypes.c_int), ("rotating", ctypes.c_int),
        ("shear", ctypes.c_double), ("omega", ctypes.c_double),
    ]

    def copy(self):
        out = Params()
        ctypes.pointer(out)[0] = self
        return out

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_params(**overrides):
    """Reference defaults (parameters.cu:77-505) with keyword overrides.

    ``reynolds``/``reynolds_magnetic``/``reynolds_thermic`` may be given
    instead of ``nu``/``nu_m``/``nu_th`` and are inverted as the reference
    does.  ``sts_variables`` (a list of field names) sets ``sts_vars_mask``;
    ``sts_algorithm`` may be given by its cfg name ("sts", "rkl1", "rkl2").
    """
    p = Params()
    p.nx = p.ny = p.nz = 32
    p.lx = p.ly = p.lz = 1.0
    p.incompressible = 0
    p.heat_equation = 0
    p.mhd = 0
    p.boussinesq = 0
    p.stratification = 0
    p.strat_direction = 2
    p.anisotropic_diffusion = 0
    p.supertimestepping = 0
    p.sts_algorithm = SPK_STS_RKL2
    p.sts_vars_mask = 0
    p.with2d = 0
    p.antialiasing = 1
    p.nu = 1.0 / 1.0
    p.nu_m = 1.0 / 1.0
    p.nu_th = 1.0 / 1.0
    p.reynolds_ani = 1.0
    p.N2 = 0.0
    p.OmegaT2 = 0.0
    p.cfl = 1.5
    p.cfl_par = 1.0
    p.cfl_sts = 1.0
    p.safety_source = 0.2
    p.safety_sts = 1
    p.t_initial = 0.0
    p.t_final = 1.0
    p.toutput_flow = 1.0
    p.fixed_dt = 0.0
    p.integrator = SPK_INT_RK3
    p.sts_every_step = 0
    p.form = SPK_FORM_PLAIN
    p.closure = 0
    p.shearing = 0
    p.rotating = 0
    p.shear = 0.0
    p.omega = 0.0
    sts_vars = overrides.pop("sts_variables", None)
    if isinstance(overrides.get("sts_algorithm"), str):
        overrides["sts_algorithm"] = STS_ALGORITHMS[overrides["sts_algorithm"]]
    for key, inv in (("reynolds", "nu"), ("reynolds_magnetic", "nu_m"), ("reynolds_thermic", "nu_th")):
        if key in overrides:
            setattr(p, inv, 1.0 / overrides.pop(key))
    if "gridsize" in overrides:
        p.nx, p.ny, p.nz = overrides.pop("gridsize")
    if "boxsize" in overrides:
        p.lx, p.ly, p.lz = overrides.pop("boxsize")
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k!r}")
        setattr(p, k, v)
    if sts_vars is not None:
        names = var_list(p)
        mask = 0
        for name in sts_vars:
            if name in names:
                mask |= 1 << names.index(name)
        p.sts_vars_mask = mask
        if mask == 0:
            # parameters.cu:114-148: an empty sts list switches STS off
            p.supertimestepping = 0
    return p


def var_list(p):
    """Parameters::popVariablesGrid field order (parameters.cu:617-638)."""
    if p.heat_equation:
        return ["th"]
    if not p.incompressible:
        return []
    names = ["vx", "vy", "vz"]
    if p.mhd:
        names += ["bx", "by", "bz"]
    if p.boussinesq:
        names += ["th"]
    return names


def num_fields(p):
    return len(var_list(p))


def check_parameters(p):
    """Parameters::checkParameters (parameters.cu:511-566); returns a list of errors."""
    errs = []
    if p.incompressible and p.heat_equation:
        errs.append("incompressible and heat_equation modules are mutually exclusive")
    if not p.incompressible and not p.heat_equation:
        errs.append("you have to chose either incompressible or heat_equation module")
    if p.boussinesq and not p.incompressible:
        errs.append("Boussinesq requires incompressible module")
    if p.stratification and not p.boussinesq:
        errs.append("stratification requires Boussinesq module")
    if p.mhd and not p.incompressible:
        errs.append("mhd requires incompressible module")
    if p.anisotropic_diffusion and not (p.mhd and p.boussinesq):
        errs.append("anisotropic_diffusion requires mhd and boussinesq module")
    return errs


def _cfg_float(x):
    """A float literal libconfig reads as a float (a '.' or an exponent)."""
    s = repr(float(x))
    if s in ("inf", "-inf", "nan"):
        raise ValueError(f"{x} has no libconfig float form")
    return s if ("." in s or "e" in s or "E" in s) else s + ".0"


def cfg_text(p, configname="spooky_b200", toutput_time=None, output_dir="./"):
    """A libconfig-format spooky.cfg that gives Parameters::Parameters
    (src/parameters/parameters.cu:59-505) the physics, modules and time
    controls of ``p``; keys the path does not use keep the reference's
    defaults.  Extensions of spk_params_t without a cfg key (form, fixed_dt,
    integrator, sts_every_step, closure) are not written.  With shearing on,
    the reader moves snapshot_step to a multiple of the shear period as the
    reference does (parameters.cu:551-562)."""
    b = lambda v: "true" if v else "false"
    names = var_list(p)
    sts = [n for i, n in enumerate(names) if p.sts_vars_mask >> i & 1]
    alg = {v: k for k, v in STS_ALGORITHMS.items()}[p.sts_algorithm]
    lines = [
        f'configname = "{configname}";',
        "modules:", "{",
        f"  with2d = {b(p.with2d)};",
        f"  incompressible = {b(p.incompressible)};",
        f"  heat_equation = {b(p.heat_equation)};",
        f"  boussinesq = {b(p.boussinesq)};",
        f"  stratification = {b(p.stratification)};",
        f"  strat_direction = {int(p.strat_direction)};",
        f"  mhd = {b(p.mhd)};",
        f"  anisotropic_diffusion = {b(p.anisotropic_diffusion)};",
        f"  supertimestepping = {b(p.supertimestepping)};",
        f"  shearing = {b(p.shearing)};",
        f"  rotating = {b(p.rotating)};",
        f'  sts_algorithm = "{alg}";',
        "  sts_variables = (" + ", ".join(f'"{n}"' for n in sts) + ");" if sts else "",
        "};",
        "physics:", "{",
        f"  boxsize = ({_cfg_float(p.lx)}, {_cfg_float(p.ly)}, {_cfg_float(p.lz)});",
        f"  gridsize = ({int(p.nx)}, {int(p.ny)}, {int(p.nz)});",
        f"  reynolds = {_cfg_float(1.0 / p.nu)};",
        f"  reynolds_magnetic = {_cfg_float(1.0 / p.nu_m)};",
        f"  reynolds_thermic = {_cfg_float(1.0 / p.nu_th)};",
        f"  reynolds_anisotropic = {_cfg_float(p.reynolds_ani)};",
        f"  brunt_vaissala_squared = {_cfg_float(p.N2)};",
        f"  mti_frequency_squared = {_cfg_float(p.OmegaT2)};",
        f"  shear = {_cfg_float(p.shear)};",
        f"  omega = {_cfg_float(p.omega)};",
        "};",
        "code:", "{",
        f"  cfl = {_cfg_float(p.cfl)};",
        f"  cfl_par = {_cfg_float(p.cfl_par)};",
        f"  cfl_sts = {_cfg_float(p.cfl_sts)};",
        f"  safety_sts = {int(p.safety_sts)};",
        f"  safety_source = {_cfg_float(p.safety_source)};",
        f"  t_initial = {_cfg_float(p.t_initial)};",
        f"  t_final = {_cfg_float(p.t_final)};",
        "  max_walltime_elapsed = 1e30;",
        f"  antialiasing = {b(p.antialiasing)};",
        "  restart = false;",
        "};",
        "output:", "{",
        f"  snapshot_step = {_cfg_float(p.toutput_flow)};",
        f"  timevar_step = {_cfg_float(p.toutput_flow if toutput_time is None else toutput_time)};",
        f'  output_dir = "{output_dir}";',
        "};",
        "init:", "{",
        "  spatial_structure = false;",
        "};",
    ]
    return "\n".join(l for l in lines if l) + "\n"
