"""The C-ABI library loads without a GPU and exports every function that
include/symmetry.h declares; parameter validation is host-only logic."""
import ctypes
import math

import pytest

from symmetry_b200 import lib as symlib
from symmetry_b200.params import SymParams, SymParticles, config_params, reference_params


def test_library_exports_every_declared_symbol():
    L = symlib.lib()
    names = symlib.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_header_layout():
    # sym_params: 10 int32 + 21 doubles; sym_particles: 10*(3*32) + 32 doubles
    assert ctypes.sizeof(SymParams) == 10 * 4 + 21 * 8
    assert ctypes.sizeof(SymParticles) == (10 * 96 + 32) * 8


def test_reference_params_match_library():
    p = SymParams()
    assert symlib.lib().sym_params_reference(ctypes.byref(p), 152, 152, 152) == 0
    q = reference_params(152, 152, 152)
    for f, _ in SymParams._fields_:
        a, b = getattr(p, f), getattr(q, f)
        if f == "body":
            assert list(a) == list(b)
        else:
            assert a == b, (f, a, b)
    # tau_R = 3 nu_R + 1/2 = 2.1432, tau_B = 0.6643 (Source1.f90:71-72)
    assert abs(3 * p.nu_r + 0.5 - 2.1432) < 1e-4 and abs(3 * p.nu_b + 0.5 - 0.6643) < 1e-4


@pytest.mark.parametrize("bad", [
    dict(tau_r=0.5), dict(tau_r=0.4), dict(tau_r=float("nan")), dict(sigma=float("inf")),
    dict(s_e=2.5), dict(par=1, rad=0.0), dict(par=SymParams and 64, rad=2.0),
])
def test_params_check_rejects(bad):
    kw = dict(tau_r=1.0)
    kw.update(bad)
    p = config_params(16, 16, 16, **kw)
    msg = symlib.params_check(p)
    assert msg is not None


def test_params_check_accepts_configs():
    from symmetry_b200 import configs
    for w in [configs.c1_thread(), configs.c2_wall_particle(), configs.c3_thread()]:
        assert symlib.params_check(w.params) is None
    for w in configs.c4_manifest()[:8]:
        assert symlib.params_check(w.params) is None
    assert symlib.params_check(reference_params()) is None


def test_footprint_scales_with_storage():
    a = symlib.footprint(config_params(64, 64, 64, storage="fp64"))
    b = symlib.footprint(config_params(64, 64, 64, storage="fp16"))
    assert a > b > 64 ** 3 * 19 * 8
