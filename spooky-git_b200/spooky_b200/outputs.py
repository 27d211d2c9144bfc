"""The reference's text diagnostics, written from the library's device
reductions: spectrum.spooky (InputOutput::WriteSpectrumOutputHeader /
WriteSpectrumOutput, src/io/spooky_output_spectrum.cu:22-460) and
timevar.spooky (InputOutput::WriteTimevarOutput,
src/io/spooky_output_timevar.cu:18-213) for the quantities of this path:
t, the energies (ev, Kx, Ky, Kz, em, Mx, My, Mz, et -- computeEnergy through
spk_budgets) and the two-field correlations (vxvy ... thvz --
twoFieldCorrelation through the Parseval sum of spk_spectrum), and the
enstrophies, helicities, field-direction means, thermal dissipation and
potential vorticity of spk_diagnostics, the field-aligned conduction terms
(dissgradT with anisotropic conduction and MHD, fluxbbgradT) and the
transfer spectra of spk_transfer_spectra.  A name the modules do not define
is written as -1 (time series) or skipped (spectra), as the reference
does."""

# spectrum names -> field pairs (spooky_output_spectrum.cu:53-186)
SPECTRA = {"Kx": ("vx", "vx"), "Ky": ("vy", "vy"), "Kz": ("vz", "vz"),
           "Mx": ("bx", "bx"), "My": ("by", "by"), "Mz": ("bz", "bz"), "Eth": ("th", "th"),
           "vxvy": ("vx", "vy"), "vyvz": ("vy", "vz"), "vxvz": ("vx", "vz"),
           "bxby": ("bx", "by"), "bybz": ("by", "bz"), "bxbz": ("bx", "bz"),
           "thvx": ("th", "vx"), "thvy": ("th", "vy"), "thvz": ("th", "vz")}
ENERGIES = {"ev": ("vx", "vy", "vz"), "Kx": ("vx",), "Ky": ("vy",), "Kz": ("vz",),
            "em": ("bx", "by", "bz"), "Mx": ("bx",), "My": ("by",), "Mz": ("bz",), "et": ("th",)}
CORRELATIONS = {"vxvy": ("vx", "vy"), "vxvz": ("vx", "vz"), "vyvz": ("vy", "vz"),
                "bxby": ("bx", "by"), "bxbz": ("bx", "bz"), "bybz": ("by", "bz"),
                "thvx": ("th", "vx"), "thvy": ("th", "vy"), "thvz": ("th", "vz")}


# enstrophy, helicities, field-direction means, thermal dissipation and
# potential vorticity (spk_diagnostics)
DIAGNOSTIC_NAMES = ("w2", "hv", "j2", "hm", "hc", "thetaB", "bz2", "phiB", "dissgradT", "pv")


def _fmt(x):
    return "%.8e" % x


def write_spectrum_header(path, ctx, names):
    """Header of spectrum.spooky: the quantity names and the bin wavevectors."""
    E, dk, _ = ctx.spectrum(0)
    with open(path, "a") as f:
        f.write("## This file contains the 1d (shell-integrated) energy spectral densities of the following "
                "quantities: \n")
        f.write("## \t" + "".join(n + "\t" for n in names) + "\n")
        f.write("wavevector \t" + "".join(_fmt(i * dk) + "\t" for i in range(len(E))) + "\n")


# transfer spectra: name -> (kind of spk_transfer_spectra, component)
TRANSFER = {f"{k}_{c}": (k, i) for k in ("advec", "emfpower", "lorentz", "helicity") for i, c in enumerate("xyz")}
TRANSFER.update({"th_advec": ("th_advec", 0), "th_aniso_diss": ("th_aniso_diss", 0),
                 "th_aniso_inj": ("th_aniso_inj", 0)})


def write_spectrum(path, ctx, t, names):
    """One line per name: t, the name, the shell values (writeSpectrumHelper).
    Names the modules do not define are skipped, as the reference skips them."""
    from . import SpookyError
    cache = {}
    with open(path, "a") as f:
        for name in names:
            pair = SPECTRA.get(name)
            if pair is not None:
                if pair[0] not in ctx.var_list or pair[1] not in ctx.var_list:
                    continue
                E, _, _ = ctx.spectrum(pair[0], pair[1])
            elif name in TRANSFER:
                kind, comp = TRANSFER[name]
                if kind not in cache:
                    try:
                        cache[kind] = ctx.transfer_spectra(kind)[0]
                    except SpookyError:
                        cache[kind] = None
                if cache[kind] is None:
                    continue
                E = cache[kind][comp]
            else:
                continue
            f.write("t\t" + _fmt(t) + "\t" + name + "\t" + "".join(_fmt(v) + "\t" for v in E) + "\n")


def write_timevar_header(path, names):
    with open(path, "a") as f:
        f.write("## This file contains the time evolution of the following quantities: \n")
        f.write("## \t" + "".join(n + "\t" for n in names) + "\n")


def timevar_values(ctx, names):
    t = ctx.get_time()[0]
    e, _ = ctx.budgets()
    diag = None
    out = []
    for name in names:
        v = -1.0
        if name == "t":
            v = t
        elif name in ENERGIES and all(q in ctx.var_list for q in ENERGIES[name]):
            v = float(sum(e[ctx.var_list.index(q)] for q in ENERGIES[name]))
        elif name in CORRELATIONS and all(q in ctx.var_list for q in CORRELATIONS[name]):
            v = ctx.spectrum(*CORRELATIONS[name])[2]
        elif name in DIAGNOSTIC_NAMES:
            if diag is None:
                diag = ctx.diagnostics()
            v = diag[name]
            if name == "dissgradT" and v == -1.0 and ctx.params.anisotropic_diffusion and ctx.params.mhd:
                # computeAnisoDissipation, with the reference's sign (spooky_output_timevar.cu:171-180)
                v = -float(ctx.transfer_spectra("th_aniso_diss")[2][0])
        elif name == "fluxbbgradT" and ctx.params.anisotropic_diffusion and ctx.params.boussinesq and ctx.params.mhd:
            v = float(ctx.transfer_spectra("th_aniso_inj")[2][0])
        out.append(v)
    return out


def write_timevar(path, ctx, names):
    with open(path, "a") as f:
        f.write("".join(_fmt(v) + "\t" for v in timevar_values(ctx, names)) + "\n")
