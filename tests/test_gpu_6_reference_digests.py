"""The library against the reference's own arrays, on the GPU.

tests/golden/reference_pin.json holds digests of the reference's arrays
(Source1.f90 executed through its mechanical translation) along the pinning
cases of tests/pin_cases.py.  Here the drop-in per-subroutine path takes the
state of each case after main's set-up and runs calmacros (Source1.f90:770-831,
the first call of the time loop): every array and particle variable has the
reference's digest, that is, equals the reference's bit for bit.

The calls after it (Lagrange_points onwards) agree with the oracle to rounding
only -- CUDA's double sin, cos and acos are not the C library's, and the
force sums are added as a tree -- and are bounded by the parity tests of
test_gpu_1_canonical.py instead.
"""
import json
import os

import numpy as np
import pytest

from symmetry_b200.lib import Lattice
from tests.common import copy_oracle_to_lattice
from tests.pin_cases import CASES, FIELDS, MASKS, PARTICLE_MATS, PARTICLE_VECS, OracleCase, digest, hexes

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pin.json")
LAGRANGE = {"Lax", "Lay", "Laz", "La_rhoN", "La_nx", "La_ny", "La_nz", "La_flag", "ds"}


def snapshot(L, par):
    lag = L.lagrange()
    arrays = {f: digest(lag[on] if on in LAGRANGE else L.get(on), f in MASKS) for f, on in FIELDS.items()}
    s = L.particles()
    parts = {f: hexes(np.array(getattr(s, on)[:3 * par])) for f, on in PARTICLE_MATS.items()}
    parts.update({on: hexes(np.array(getattr(s, on)[:3 * par])) for on in PARTICLE_VECS})
    parts["shb"] = hexes(np.array(s.shb[:par]))
    return {"arrays": arrays, "particles": parts}


def mismatches(want, got):
    return [k for k, v in want["arrays"].items() if got["arrays"][k] != v] + \
           [k for k, v in want["particles"].items() if got["particles"][k] != v]


@pytest.mark.parametrize("name", list(CASES))
def test_calmacros_reproduces_reference_bit_for_bit(name):
    with open(GOLD) as f:
        snaps = json.load(f)[name]["snapshots"]
    oc = OracleCase(name)
    L = Lattice(oc.o.p)
    copy_oracle_to_lattice(oc.o, L)
    assert snaps[0]["after"] == "setup"
    assert mismatches(snaps[0], snapshot(L, oc.par)) == []
    L.call("calmacros")
    assert snaps[1]["after"] == "0:0:calmacros"
    assert mismatches(snaps[1], snapshot(L, oc.par)) == []
