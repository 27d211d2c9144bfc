"""GPU checks of spk_compute_dfield_noalloc, the RHS entry point for callers
that cannot allocate device memory (their memory belongs to another
allocator, or they must not allocate once running).  It keeps all scratch in
one array inside the library, so its results must equal those of
spk_compute_dfield on a normal context, call after call, whatever the
previous call left in that array.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import numpy as np
import pytest

import spooky_b200 as S
from fields import random_solenoidal, to_spectral
from spooky_b200 import Context, SpookyError, compute_dfield_noalloc
from spooky_b200.params import SPK_FORM_FP32, SPK_FORM_PLAIN, default_params

pytestmark = pytest.mark.gpu

# same tolerances as the RHS parity tests against the oracle
TOL_RHS = {SPK_FORM_PLAIN: 1e-12, SPK_FORM_FP32: 2e-5}

CASES = {
    "hd": dict(incompressible=1, reynolds=100.0),
    "mhd": dict(incompressible=1, mhd=1, reynolds=100.0, reynolds_magnetic=50.0),
    "bous": dict(incompressible=1, boussinesq=1, stratification=1, reynolds=100.0, reynolds_thermic=80.0,
                 N2=0.5, strat_direction=2),
    "bous_mhd_aniso": dict(incompressible=1, mhd=1, boussinesq=1, stratification=1, anisotropic_diffusion=1,
                           reynolds=100.0, reynolds_magnetic=100.0, reynolds_thermic=100.0, reynolds_ani=20.0,
                           N2=1.0, OmegaT2=1.0, strat_direction=2),
    "heat": dict(heat_equation=1, reynolds_thermic=50.0),
}


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def make_state(p, seed):
    fields = []
    if p.incompressible:
        fields += list(random_solenoidal(p, seed, kpeak=3.0))
    if p.mhd:
        B = random_solenoidal(p, seed + 100, kpeak=3.0, rms=0.7)
        B[0] += 0.3
        fields += list(B)
    if p.boussinesq or p.heat_equation:
        rng = np.random.default_rng(seed + 200)
        fields.append(0.3 * rng.standard_normal((p.nx, p.ny, p.nz)))
    return to_spectral(np.stack(fields))


def on_device(arr):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
    torch.cuda.synchronize()
    return t


def dfield_with_context(p, U):
    ctx = Context(p)
    Ud = on_device(U)
    dUd = on_device(np.zeros_like(U))
    ctx.compute_dfield(Ud, dUd)
    ctx.synchronize()
    return dUd.cpu().numpy()


def dfield_noalloc(p, U):
    Ud = on_device(U)
    dUd = on_device(np.zeros_like(U))
    compute_dfield_noalloc(p, Ud, dUd)
    return dUd.cpu().numpy()


@pytest.mark.parametrize("form", [SPK_FORM_PLAIN, SPK_FORM_FP32])
@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_context_on_two_calls_in_a_row(case, form):
    p = default_params(gridsize=(32, 32, 32), boxsize=(1.0, 1.5, 2.0), form=form, **CASES[case])
    for seed in (5, 6):
        U = make_state(p, seed)
        ref = dfield_with_context(p, U)
        got = dfield_noalloc(p, U)
        assert np.all(np.isfinite(got))
        assert rel_l2(got, ref) < TOL_RHS[form], (case, form, seed)


def test_noalloc_after_a_larger_configuration():
    """The scratch keeps the previous call's contents: a small HD call after a
    large MHD + Boussinesq call must not see any of it."""
    big = default_params(gridsize=(32, 32, 32), form=SPK_FORM_PLAIN, **CASES["bous_mhd_aniso"])
    small = default_params(gridsize=(16, 8, 32), boxsize=(2.0, 1.0, 1.0), form=SPK_FORM_PLAIN, **CASES["hd"])
    dfield_noalloc(big, make_state(big, 1))
    U = make_state(small, 2)
    assert rel_l2(dfield_noalloc(small, U), dfield_with_context(small, U)) < TOL_RHS[SPK_FORM_PLAIN]


def test_noalloc_rejects_grids_beyond_the_scratch():
    p = default_params(gridsize=(128, 128, 128), form=SPK_FORM_PLAIN, **CASES["mhd"])
    U = on_device(np.zeros((6, 128, 128, 65), np.complex128))
    dU = on_device(np.zeros((6, 128, 128, 65), np.complex128))
    with pytest.raises(SpookyError) as e:
        compute_dfield_noalloc(p, U, dU)
    assert e.value.code == 2
    assert "MiB" in str(e.value) and str(S.NOALLOC_SCRATCH_BYTES >> 20) in str(e.value)


def test_noalloc_allocates_no_device_memory():
    """The entry point's promise: after one warm-up call (which loads the
    library's device code and its scratch array), further calls leave the
    device's free memory unchanged.  A context of the same 32^3 MHD case
    allocates several MiB, so the check tells the two apart."""
    import torch
    p = default_params(gridsize=(32, 32, 32), form=SPK_FORM_PLAIN, **CASES["mhd"])
    U = on_device(make_state(p, 7))
    dU = on_device(np.zeros(tuple(U.shape), np.complex128))
    compute_dfield_noalloc(p, U, dU)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        compute_dfield_noalloc(p, U, dU)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, (free0, free1)
    ctx = Context(p)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free1 - free2 >= 4 << 20, "a context should allocate its buffers (sanity check of the measurement)"
    ctx.close()


def test_noalloc_rejects_bad_tensors_and_closure():
    import torch
    p = default_params(gridsize=(16, 16, 16), form=SPK_FORM_PLAIN, **CASES["hd"])
    good = on_device(np.zeros((3, 16, 16, 9), np.complex128))
    with pytest.raises(ValueError):
        compute_dfield_noalloc(p, good[:2], good)
    with pytest.raises(ValueError):
        compute_dfield_noalloc(p, good.to(torch.complex64), good)
    with pytest.raises(ValueError):
        compute_dfield_noalloc(p, good.cpu(), good)
    pc = default_params(gridsize=(16, 16, 16), form=SPK_FORM_PLAIN, closure=1, **CASES["hd"])
    with pytest.raises(SpookyError) as e:
        compute_dfield_noalloc(pc, good, torch.zeros_like(good))
    assert e.value.code == 2


def test_noalloc_refuses_a_capturing_stream():
    """A call on a stream under capture is refused before anything is queued
    (its host tables would be recorded as copies from freed memory)."""
    import ctypes
    import torch
    p = default_params(gridsize=(16, 16, 16), form=SPK_FORM_PLAIN, **CASES["hd"])
    U = on_device(make_state(p, 3))
    dU = torch.zeros_like(U)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    rc = None
    with torch.cuda.graph(g, stream=s):
        rc = S.lib().spk_compute_dfield_noalloc(ctypes.byref(p.copy()), U.data_ptr(), dU.data_ptr(),
                                                 s.cuda_stream)
        dU.add_(0)   # keep the captured graph non-empty
    assert rc == 2
    assert "captur" in S.lib().spk_last_error(None).decode()
    del g
    # the entry point still works after the refused call
    ref = dfield_with_context(p, U.cpu().numpy())
    assert rel_l2(dfield_noalloc(p, U.cpu().numpy()), ref) < TOL_RHS[SPK_FORM_PLAIN]
