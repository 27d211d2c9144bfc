"""The reference's command line (src/main.cu:26-172) over this library:

    python -m spooky_b200 --input-dir DIR [--output-dir DIR] [-r N] [--stats N]
                          [-t HH MM SS] [-n NX NY NZ] [--with-2d] [--form plain|fp32]

reads DIR/spooky.cfg, applies the overrides (grid, 2D, output directory,
wall-clock limit x 0.95, restart number), restarts from
<output_dir>/data/snapNNNN.h5 when -r is given (-1: the most recent), writes
the initial outputs of a new run, runs the main loop to t_final with the
reference's snapshot and time-series outputs, and prints the final
statistics.  --form chooses the arithmetic form (plain FP64 by default, the
reference's precision).  A run without -r starts from zero fields: the
reference's initial conditions are user code compiled into its binary, so
initial fields are given as snapshot 0 and read with -r 0, as the
reference's tests do."""
import argparse
import os
import sys
import time

from . import SPK_FORM_FP32, SPK_FORM_PLAIN, Supervisor, cfg_lookup, params_from_string


def parse_args(argv):
    ap = argparse.ArgumentParser(prog="spooky_b200", description="SPOOKY main loop on the B200 library")
    ap.add_argument("--input-dir", default="./", help="input directory for cfg file")
    ap.add_argument("--output-dir", help="output directory for data files")
    ap.add_argument("-r", "--restart", type=int, default=None, help="restart from data file (-1: the most recent)")
    ap.add_argument("--stats", type=int, default=-1, help="print stats every n steps (-1: none)")
    ap.add_argument("-t", "--time", type=int, nargs=3, metavar=("HH", "MM", "SS"),
                    help="override the maximum wallclock elapsed time")
    ap.add_argument("-n", "--ngrid", type=int, nargs=3, metavar=("NX", "NY", "NZ"),
                    help="override the number of grid points")
    ap.add_argument("--with-2d", action="store_true", help="force problem to be 2d (x,y)")
    ap.add_argument("--form", choices=["plain", "fp32"], default="plain", help="arithmetic form of the passes")
    ap.add_argument("--max-steps", type=int, default=None, help="stop after this many steps")
    return ap.parse_args(argv)


def run_config(text, args):
    """The cfg keys of the run that spk_params_t does not carry, with the
    reference's defaults (parameters.cu:300-440) and the command-line
    overrides of main.cu:79-134."""
    out = {
        "output_dir": cfg_lookup(text, "output.output_dir", "string", "./"),
        "toutput_time": cfg_lookup(text, "output.timevar_step", "float", 1.0),
        "timevar_vars": cfg_lookup(text, "output.timevar_vars", "strings", []),
        "spectra_vars": cfg_lookup(text, "output.spectra_vars", "strings", []),
        "max_walltime_hours": cfg_lookup(text, "code.max_walltime_elapsed", "float", 1e30),
    }
    if args.output_dir is not None:
        out["output_dir"] = args.output_dir
    if args.time is not None:
        hh, mm, ss = args.time
        out["max_walltime_hours"] = 0.95 * (hh + mm / 60.0 + ss / 3600.0)
    return out


def main(argv=None):
    args = parse_args(sys.argv[1:] if argv is None else argv)
    cfg_path = os.path.join(args.input_dir, "spooky.cfg")
    with open(cfg_path) as f:
        text = f.read()
    p = params_from_string(text)
    if args.ngrid is not None:
        p.nx, p.ny, p.nz = args.ngrid
    if args.with_2d:
        p.with2d = 1
    p.form = SPK_FORM_FP32 if args.form == "fp32" else SPK_FORM_PLAIN
    rc = run_config(text, args)
    restart = -2 if args.restart is None else args.restart
    t_start = time.perf_counter()
    sup = Supervisor(p, toutput_time=rc["toutput_time"], output_dir=rc["output_dir"],
                     timevar_vars=rc["timevar_vars"] or None, spectra_vars=rc["spectra_vars"] or None,
                     restart_num=restart)
    print(f"Input directory: {args.input_dir}\nOutput directory: {rc['output_dir']}")
    print(f"grid size: {p.nx} {p.ny} {p.nz}   fields: {' '.join(sup.ctx.var_list)}")
    if sup.restart_num >= -1:
        t, _, step = sup.ctx.get_time()
        print(f"restarted from snapshot {sup.inout.num_save - 1} at t = {t:.6e}, step {step}")
    sup.initialDataDump()
    steps = sup.executeMainLoop(max_steps=args.max_steps, max_walltime_hours=rc["max_walltime_hours"],
                                stats_frequency=args.stats)
    t, _, step = sup.ctx.get_time()
    loop = max(sup.time_in_main_loop, 1e-30)
    print("@@ FINAL STATISTICS REPORT")
    print(f"@@\tThe total execution time was: {time.perf_counter() - t_start:.2e} [s]")
    print(f"@@\tThe time spent in the mainloop was: {loop:.2e} [s]")
    print(f"@@\tThe mainloop took {steps} steps to reach t = {t:.6e} (step {step})")
    print(f"@@\tThe average performance is: {p.nx * p.ny * p.nz * steps / loop:.4e} [cell_updates/s]")
    return 0


if __name__ == "__main__":
    sys.exit(main())
