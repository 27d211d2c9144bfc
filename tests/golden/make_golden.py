"""Regenerate the golden fixtures in this directory from the reference's own
Python code (LorenzoLMP/spooky-git, read from a local checkout).

    python tests/golden/make_golden.py /path/to/spooky-git

Fixtures written:
  heat_diffusion_rk3.npz  -- the reference's numpy RK3 restatement of the
      heat-diffusion test (tests/heat-diffusion/test_rk3_heatdiff.py:32-83,
      main() :104-190): 1024x2x2, chi=1e-3, cfl=1.5, snapshots at t=0,5,10.
      The reference's CUDA build must match these to L1 < 1e-15
      (tests/heat-diffusion/check-heat-diffusion.py:29,157-166).
  mti_eigenmode.json      -- the MTI growth rate from the reference's
      dispersion cubic (tests/mti-eigenmode/mti_disp_rel.py:44-70) and the
      value its check script hard-codes (check-mti-eigenmode.py:21).

Only this script reads the reference checkout; tests read the fixtures.
matplotlib is absent in this image, so a stub module stands in for the
plotting imports (the computations never call it).
"""
import glob
import importlib.util
import json
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class _Anything(types.ModuleType):
    """Stands in for any plotting object: attributes, calls and item
    assignment all succeed and return another stand-in."""

    def __getattr__(self, name):
        return _Anything(name)

    def __call__(self, *a, **k):
        return _Anything("call")

    def __setitem__(self, key, value):
        pass

    def __getitem__(self, key):
        return _Anything("item")


def _stub_plotting():
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.ticker", "pylab",
                 "matplotlib.legend_handler"):
        sys.modules.setdefault(name, _Anything(name))


def _load(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def heat_diffusion(ref):
    mod = _load(os.path.join(ref, "tests/heat-diffusion/test_rk3_heatdiff.py"), "ref_rk3_heatdiff")
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "data"))
        argv = sys.argv
        sys.argv = ["test_rk3_heatdiff.py", "--output-dir", tmp]
        try:
            mod.main()
        finally:
            sys.argv = argv
        files = sorted(glob.glob(os.path.join(tmp, "data", "py_snap.*.npz")))
        Ts, ts = [], []
        for f in files:
            d = np.load(f)
            Ts.append(d["T"].copy())
            ts.append(float(d["t"]))
            x = d["x"].copy()
    out = os.path.join(HERE, "heat_diffusion_rk3.npz")
    np.savez(out, x=x, T=np.array(Ts), t=np.array(ts), nx=mod.nx, chi=mod.chi0, cfl=mod.cfl,
             tend=mod.tend, dt=mod.get_dt())
    print("wrote", out, "times", ts)


def mti(ref):
    mod = _load(os.path.join(ref, "tests/mti-eigenmode/mti_disp_rel.py"), "ref_mti_disp_rel")
    sigma_cubic = float(mod.mti_root_sim[0])
    src = open(os.path.join(ref, "tests/mti-eigenmode/check-mti-eigenmode.py")).read()
    sigma_check = None
    for line in src.splitlines():
        s = line.strip()
        if s.startswith("sigma") and "=" in s:
            sigma_check = float(s.split("=")[1].split("#")[0])
            break
    out = os.path.join(HERE, "mti_eigenmode.json")
    data = {
        "sigma_dispersion_cubic": sigma_cubic,
        "sigma_check_script": sigma_check,
        "Pe": mod.Pe, "ReNu": mod.ReNu, "ReEta": mod.ReEta, "B0": mod.B0, "N2": mod.N2,
        "n_mode": 12, "grid": [512, 4, 4], "box": [1.0, 1.0, 1.0], "OmegaT2": 1.0,
        "reynolds_thermic": 1e6, "tolerance_L1": 1e-7,
    }
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", out, data["sigma_dispersion_cubic"], data["sigma_check_script"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of a LorenzoLMP/spooky-git checkout>")
    ref = sys.argv[1]
    _stub_plotting()
    heat_diffusion(ref)
    mti(ref)
