"""CPU checks of the C ABI: the library loads without a GPU, exports every
symbol include/spooky_b200.h declares, and its defaults equal the Python
mirror of the reference's cfg defaults.  No compute call is made here."""
import ctypes
import re

import pytest

import spooky_b200 as S
from spooky_b200.params import Params, check_parameters, default_params


def declared_symbols():
    src = open(S.HEADER_PATH).read()
    return sorted(set(re.findall(r"\b(spk_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_exactly_the_exported_list():
    assert declared_symbols() == sorted(S.EXPORTED)


def test_library_loads_and_exports_every_declared_symbol():
    L = S.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_c_defaults_equal_python_defaults():
    c = S.c_defaults()
    py = default_params()
    for name, _ in Params._fields_:
        assert getattr(c, name) == getattr(py, name), name


def test_params_struct_size_matches_c_layout():
    # 3 int + 3 double + 14 ints/unsigned + 6 doubles + 4 doubles + int + 3 doubles + double + 3 ints (+ padding)
    assert ctypes.sizeof(Params) % 8 == 0
    assert Params.fixed_dt.offset % 8 == 0


def test_check_parameters_mirrors_reference_rules():
    assert check_parameters(default_params(incompressible=1)) == []
    assert check_parameters(default_params()) != []
    assert check_parameters(default_params(incompressible=1, heat_equation=1)) != []
    assert check_parameters(default_params(incompressible=1, anisotropic_diffusion=1, mhd=1)) != []
    assert check_parameters(default_params(heat_equation=1, boussinesq=1)) != []


def test_sts_variables_mask_and_empty_list_disables_sts():
    p = default_params(incompressible=1, mhd=1, boussinesq=1, supertimestepping=1, sts_variables=["th", "bx"])
    assert p.sts_vars_mask == (1 << 6) | (1 << 3)
    q = default_params(incompressible=1, supertimestepping=1, sts_variables=[])
    assert q.supertimestepping == 0


def test_context_creation_rejects_bad_config_without_gpu():
    """Config validation happens before any CUDA call."""
    p = default_params()  # neither incompressible nor heat_equation
    with pytest.raises(S.SpookyError) as e:
        S.Context(p)
    assert e.value.code == 6


def test_closure_threshold_outside_unit_interval_is_rejected_without_gpu():
    """closure_kc_frac (variant 2's small-scale threshold, a fraction of the
    cut-off) must lie in [0, 1); the check runs before any CUDA call."""
    L = 6.283185307179586
    p = default_params(incompressible=1, mhd=1, gridsize=(16, 16, 16), boxsize=(L, L, L), closure=2,
                       closure_kc_frac=1.2)
    with pytest.raises(S.SpookyError) as e:
        S.Context(p)
    assert e.value.code == 1   # SPK_ERR_ARG
    assert "closure_kc_frac" in str(e.value)
