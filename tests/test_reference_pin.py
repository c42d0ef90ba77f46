"""The oracle pinned to the reference itself, routine by routine.

No Fortran compiler exists here, so the reference cannot be built.  Instead
oracle/f90py.py translates its source statement by statement into Python
(the reference's own subroutines and its main program up to the time loop,
as written) and these tests run that translation beside the oracle's C++
restatement on the same state, in REFERENCE mode, along the cases of
tests/pin_cases.py:

  * main's set-up -- parameters, the moment matrix M from its DATA statement
    and M_inv, the velocity tables, tables / initia_center / set_walls /
    initialization / derivatives -- against setup_reference();
  * then every call of the time loop's body (Source1.f90:216-251) in order,
    each followed by a comparison of every array and particle variable.

Every array and particle variable must be equal bit for bit.  The reference
leaves one order of additions to its threads -- momentum's OpenMP REDUCTION
of the force and torque (Source1.f90:1192-1193) -- and the translation runs
it as one thread does, in loop order; the oracle adds in that order too.
The same pass checks that the translated reference still produces the
digests committed in tests/golden/reference_pin.json, which
tests/test_reference_golden.py holds the oracle to where the source is
absent.  About four minutes (the translation runs as Python).  Skipped where
the reference source is absent.
"""
import json
import os
import warnings

import numpy as np
import pytest

from oracle import f90py
from oracle.oracle import setup_reference
from symmetry_b200.params import reference_params
from tests.pin_cases import (CASES, FIELDS, FULL, LOOP_CALLS, PARTICLE_MATS, PARTICLE_VECS, OracleCase,
                             ReferenceCase)

REF = f90py.load_reference()
pytestmark = pytest.mark.skipif(REF is None, reason="reference source not on this machine")
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pin.json")


def _diff(a, b) -> float:
    """0 when equal (NaN where the other is NaN), else the largest difference
    relative to max(1, |b|); inf for differing integers or flags."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind in "biu" or b.dtype.kind in "biu":
        if a.dtype == bool or b.dtype == bool:
            a, b = a.astype(np.int64) != 0, b.astype(np.int64) != 0
        return 0.0 if np.array_equal(a, b) else np.inf
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return np.inf
    m = ~na
    if np.array_equal(a[m], b[m]):
        return 0.0
    return float((np.abs(a[m] - b[m]) / np.maximum(np.abs(b[m]), 1.0)).max())


def compare(rc: ReferenceCase, oc: OracleCase) -> dict:
    V, o, par = rc.V, oc.o, rc.par
    out = {}
    for f, on in FIELDS.items():
        a = V[f]
        out[f] = _diff(a, o.arr(on).reshape(-1).reshape(a.shape, order="F"))
    s = o.particles
    for f, on in PARTICLE_MATS.items():
        out[f] = _diff(V[f], np.array(getattr(s, on)[:3 * par]).reshape((par, 3), order="F"))
    for on, names in PARTICLE_VECS.items():
        b = np.array(getattr(s, on)[:3 * par]).reshape((par, 3), order="F")
        out[on] = _diff(np.stack([V[n] for n in names], 1), b)
    out["shb"] = _diff(V["shb"], np.array(s.shb[:par]))
    return {k: v for k, v in out.items() if v != 0.0}


class Run:
    """A case on both sides, compared after set-up and after every call."""

    def __init__(self, name):
        self.rc = ReferenceCase(f90py.load_reference(), name)   # a fresh module: its own constants
        self.oc = OracleCase(name)
        self.log = [("setup", compare(self.rc, self.oc))]
        self.snaps = [dict(after="setup", **self.rc.snapshot())]
        for (step, k, name_r), (_, _, name_o) in zip(self.rc.steps(), self.oc.steps()):
            assert name_r == name_o
            where = f"{step}:{k}:{name_r}"
            self.log.append((where, compare(self.rc, self.oc)))
            self.snaps.append(dict(after=where, **self.rc.snapshot()))


@pytest.fixture(scope="module", params=list(CASES))
def run(request):
    return request.param, Run(request.param)


def test_loop_calls_are_mains(run):
    _, r = run
    assert [c[0] for c in r.rc.R.MAIN_LOOP_CALLS] == LOOP_CALLS


def test_every_call_matches_oracle_bit_for_bit(run):
    _, r = run
    for where, bad in r.log:
        assert bad == {}, (where, bad)


def test_committed_digests_are_the_references(run):
    name, r = run
    with open(GOLD) as f:
        gold = json.load(f)[name]["snapshots"]
    assert gold == r.snaps


def test_particles_stay_in_the_domain(run):
    """The comparison is not vacuous: every particle is still solid in the
    domain after the steps, next to an interface."""
    name, r = run
    V = r.rc.V
    for k in range(1, r.rc.par + 1):          # whole spheres, or halves cut by mirror planes
        assert int((V["walls"] == k).sum()) > 500
    assert int(V["flag"].sum()) > 1000
    assert np.all(np.isfinite(V["center"]))
    if CASES[name]["velocity"] is not None:
        shift = np.abs(V["center"] - np.array(CASES[name]["centers"])).max()
        assert 0.0 < shift < 2.0
        # nodes the pair left were refilled: the last set_walls made fluid
        # nodes that were solid before it
        assert int(((V["walls_old"] >= 1) & (V["walls_all"] == 0)).sum()) > 0


@pytest.mark.skipif(not os.environ.get("SYM_PIN_152"), reason="about 45 minutes as Python; set SYM_PIN_152=1")
def test_reference_grid_152_one_step():
    """The reference as written: its 152^3 grid and 12 particles, main's
    set-up and one step, every call equal to the oracle bit for bit."""
    r = Run(FULL)
    for where, bad in r.log:
        assert bad == {}, (where, bad)


def test_reference_constants_reproduced():
    """main's own parameters, moment matrix and tables equal the ones the
    oracle and the library use."""
    R = f90py.load_reference()
    R.C.xl, R.C.yl, R.C.zl, R.C.par = 36, 42, 36, 2
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        V = R.main_setup()
    p = reference_params(36, 42, 36, 2)
    C = R.C
    assert (C.sigma, C.rho0, C.nu_r, C.nu_b, C.rad, C.beta, C.cita, C.alpha, C.evap_lim) == \
        (p.sigma, p.rho0, p.nu_r, p.nu_b, p.rad, p.beta, p.cita, p.alpha, p.evap_lim)
    assert (V["mass"], V["inertia_moment"], V["fg"]) == (p.mass, p.inertia, p.fg)
    o = setup_reference(p)
    M, Mi = o.matrices()
    assert np.array_equal(V["m"], M) and np.array_equal(V["m_inv"], Mi)
    assert o.la_num == C.la_num


def test_output3_stop_rule_matches_oracle(run):
    """output3's neck reading (Source1.f90:1673-1717), from the values its
    WRITE statement puts out: hmin / Rad_c and y0 / lamda_d."""
    name, r = run
    V, R, o = r.rc.V, r.rc.R, r.oc.o
    r.rc.call("calmacros")
    o.call("calmacros")
    R.OUT_LOG.clear()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        # main: call output3(rho_N,t,tr,walls_all,pout,lamda_d)
        R.output3(V["rho_n"], 0, V["tr"], V["walls_all"], V["pout"], V["lamda_d"])
    unit, (t, tt, h_over_rc, y_over_lamda) = R.OUT_LOG[-1]
    hmin, y0 = o.output3()
    assert h_over_rc == hmin / R.C.rad_c
    assert y_over_lamda == y0 / V["lamda_d"]
    assert 0.0 < hmin < CASES[name]["domain"][2]
