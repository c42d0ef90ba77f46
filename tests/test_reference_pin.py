"""The oracle pinned to the reference itself, routine by routine.

No Fortran compiler exists here, so the reference cannot be built.  Instead
oracle/f90py.py translates its source statement by statement into Python
(the reference's own subroutines and its main program up to the time loop,
as written) and these tests run that translation beside the oracle's C++
restatement on the same state, in REFERENCE mode:

  * main's set-up -- parameters, the moment matrix M from its DATA statement
    and M_inv, the velocity tables, tables / initia_center / set_walls /
    initialization / derivatives -- against setup_reference();
  * then every call of the time loop's body (Source1.f90:216-251) in order,
    each followed by a comparison of every array and particle variable.

Every array and particle variable must be equal bit for bit.  The reference
leaves one order of additions to its threads -- momentum's OpenMP REDUCTION
of the force and torque (Source1.f90:1192-1193) -- and the translation runs
it as one thread does, in loop order; the oracle adds in that order too.

The domains are small (the translation runs as Python): the reference's own
12-particle layout on the 48 x 88 x 48 grid of the GPU parity tests (the
smallest it fits: below that its particles overlap and reach past x = 1,
where the Fortran reads outside its arrays), and 36 x 42 x 36 with two
particles placed across the thread's interface and launched so that nodes
are refilled, with either bounce-back.  About four minutes in all.  The
tests are skipped where the reference source is absent.
"""
import warnings

import numpy as np
import pytest

from oracle import f90py
from oracle.oracle import setup_reference
from symmetry_b200.params import particles_set, reference_params

REF = f90py.load_reference()
pytestmark = pytest.mark.skipif(REF is None, reason="reference source not on this machine")

FIELDS = {"rho": "rho", "ux": "ux", "uy": "uy", "uz": "uz", "rho_n": "rho_N", "rho_r": "rho_R", "rho_b": "rho_B",
          "n_x": "n_x", "n_y": "n_y", "n_z": "n_z", "gradx": "gradx", "grady": "grady", "gradz": "gradz",
          "fi": "fi", "ffi": "ffi", "ri": "ri", "bi": "bi", "walls": "walls", "walls_old": "walls_old",
          "walls_all": "walls_all", "pin": "pin", "pout": "pout", "flag": "flag",
          "lax": "Lax", "lay": "Lay", "laz": "Laz", "la_rhon": "La_rhoN", "la_nx": "La_nx", "la_ny": "La_ny",
          "la_nz": "La_nz", "ds": "ds", "la_flag": "La_flag"}
PARTICLE_MATS = {"center": "center", "center_old": "center_old", "center0": "center0", "tension": "tension",
                 "tension_t": "tension_t"}
PARTICLE_VECS = {"fp": ("fpx", "fpy", "fpz"), "tp": ("tpx", "tpy", "tpz"), "up": ("upx", "upy", "upz"),
                 "rp": ("rpx", "rpy", "rpz"), "fre": ("frex", "frey", "frez")}


def _diff(a, b) -> float:
    """0 when equal bit for bit (NaN where the other is NaN), else the largest
    difference relative to max(1, |b|); inf for differing integers or flags."""
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


class Pair:
    """The translated reference (main's variables V) and the oracle side by side."""

    def __init__(self, nx, ny, nz, centers, velocity=None, bounce=False):
        self.R = R = f90py.load_reference()          # a fresh module: its own constants
        self.par = par = len(centers)
        self.bounce = bounce                        # curve2 in place of curve
        R.C.xl, R.C.yl, R.C.zl, R.C.par = nx, ny, nz, par
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            self.V = R.main_setup()
        prm = reference_params(nx, ny, nz, par)
        prm.bounce = 1 if bounce else 0
        self.o = setup_reference(prm)
        self.setup_diffs = self.compare()
        # the same particles on both sides, then their masks and the derivatives
        V, s = self.V, self.o.particles
        for k, c in enumerate(centers):
            V["center"][k, :] = c
            V["center0"][k, :] = c
        particles_set(s, "center", par, centers)
        particles_set(s, "center0", par, centers)
        if velocity is not None:
            for k in range(par):
                for j, n in enumerate(("upx", "upy", "upz")):
                    V[n][k] = velocity[k][j]
            particles_set(s, "up", par, velocity)
        for name in ("set_walls", "derivatives"):
            self.ref_call(name)
            self.o.call(name)
        self.placed_diffs = self.compare()

    def ref_call(self, name, acts=None):
        if acts is None:
            acts = next(c[1] for c in self.R.MAIN_LOOP_CALLS if c[0] == name)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            getattr(self.R, name)(*[self.V[self.R.pyname(a)] for a in acts])

    def compare(self):
        V, o, par = self.V, self.o, self.par
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
        return out

    def run_steps(self, steps):
        """main's time-loop body, call by call on both sides; the comparison
        after each call, keyed (step, call index, subroutine)."""
        log = []
        for step in range(steps):
            n_stream = 0
            for k, (name, acts, line) in enumerate(self.R.MAIN_LOOP_CALLS):
                # curve2 takes curve's arguments (Source1.f90:1036); the
                # oracle's curve runs curve2 when the bounce switch is on
                self.ref_call("curve2" if name == "curve" and self.bounce else name, acts)
                if name == "streaming":
                    self.o.streaming(n_stream)
                    n_stream += 1
                else:
                    self.o.call(name)
                log.append(((step, k, name, line), self.compare()))
        return log


def _check(diffs, where):
    for key, d in diffs.items():
        assert d == 0.0, (where, key, d)


# 36 x 42 x 36: the thread of radius 30 about the corner line x = z = 35.5
# (initialization) crosses x = z = 14.3; two particles of radius 7.5 sit on
# that interface, outside the 3-node wall repulsion range of every face
# (repulsive, Source1.f90:1606-1649) and 2.6 nodes apart, inside each other's
DOMAIN = (36, 42, 36)
CENTERS = [[14.3, 12.2, 14.3], [15.0, 29.8, 13.6]]


@pytest.fixture(scope="module")
def moving():
    # the same pair launched across the interface fast enough that nodes it
    # leaves are refilled within the steps
    p = Pair(*DOMAIN, CENTERS, velocity=[[0.3, 0.25, -0.2], [-0.25, -0.3, 0.25]])
    return p, p.run_steps(2)


def test_reference_layout_one_step():
    """The reference's own 12-particle layout (initia_center, unplaced) on the
    48 x 88 x 48 grid of the GPU parity tests: main's set-up and one step of
    the time loop, every array equal bit for bit after every call."""
    R = f90py.load_reference()
    R.C.xl, R.C.yl, R.C.zl, R.C.par = 48, 88, 48, 12
    p = Pair.__new__(Pair)
    p.R, p.par, p.bounce = R, 12, False
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p.V = R.main_setup()
    p.o = setup_reference(reference_params(48, 88, 48, 12))
    _check(p.compare(), "main set-up")
    for k in range(1, 13):      # whole spheres, or halves cut by the mirror planes
        assert int((p.V["walls"] == k).sum()) > 500
    for where, diffs in p.run_steps(1):
        _check(diffs, where)


def test_reference_constants_reproduced():
    """main's own parameters, moment matrix and tables equal the ones the
    oracle and the library use."""
    R = f90py.load_reference()
    R.C.xl, R.C.yl, R.C.zl, R.C.par = DOMAIN[0], DOMAIN[1], DOMAIN[2], 2
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        V = R.main_setup()
    p = reference_params(*DOMAIN, 2)
    C = R.C
    assert (C.sigma, C.rho0, C.nu_r, C.nu_b, C.rad, C.beta, C.cita, C.alpha, C.evap_lim) == \
        (p.sigma, p.rho0, p.nu_r, p.nu_b, p.rad, p.beta, p.cita, p.alpha, p.evap_lim)
    assert (V["mass"], V["inertia_moment"], V["fg"]) == (p.mass, p.inertia, p.fg)
    o = setup_reference(p)
    M, Mi = o.matrices()
    assert np.array_equal(V["m"], M) and np.array_equal(V["m_inv"], Mi)
    assert o.la_num == C.la_num


def test_main_setup_matches_oracle(moving):
    p, _ = moving
    _check(p.setup_diffs, "main set-up")
    _check(p.placed_diffs, "placed particles")


@pytest.fixture(scope="module")
def bouncing():
    # the moving pair with the interpolated bounce-back (curve2), which the
    # reference keeps beside curve without calling it
    p = Pair(*DOMAIN, CENTERS, velocity=[[0.3, 0.25, -0.2], [-0.25, -0.3, 0.25]], bounce=True)
    return p, p.run_steps(1)


@pytest.mark.parametrize("case", ["moving", "bouncing"])
def test_time_loop_routines_match_oracle(case, request):
    p, log = request.getfixturevalue(case)
    assert [c[0] for c in p.R.MAIN_LOOP_CALLS] == [
        "calmacros", "lagrange_points", "capillary_force2", "momentum", "repulsive", "movement", "set_walls",
        "refilling", "derivatives", "collision", "recolor", "boundary", "streaming", "streaming", "curve"]
    for where, diffs in log:
        _check(diffs, where)


@pytest.mark.parametrize("case", ["moving", "bouncing"])
def test_particles_stay_in_the_domain(case, request):
    """The comparison is not vacuous: both particles are still solid in the
    domain after the steps, next to an interface, and moved."""
    p, _ = request.getfixturevalue(case)
    V = p.V
    for k in (1, 2):
        assert int((V["walls"] == k).sum()) > 1500
    assert int(V["flag"].sum()) > 1000
    assert np.all(np.isfinite(V["center"]))
    shift = np.abs(V["center"] - np.array(CENTERS)).max()
    assert 0.0 < shift < 2.0


def test_moving_case_refills_nodes(moving):
    """The moving pair uncovers nodes, so refilling ran on real work: the
    last set_walls left fluid nodes that were solid before it."""
    p, _ = moving
    assert int(((p.V["walls_old"] >= 1) & (p.V["walls_all"] == 0)).sum()) > 0


def test_output3_stop_rule_matches_oracle(moving):
    """output3's neck reading (Source1.f90:1673-1717), from the values its
    WRITE statement puts out: hmin / Rad_c and y0 / lamda_d."""
    p, _ = moving
    V, R = p.V, p.R
    p.ref_call("calmacros")
    p.o.call("calmacros")
    R.OUT_LOG.clear()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        # main: call output3(rho_N,t,tr,walls_all,pout,lamda_d)
        R.output3(V["rho_n"], 0, V["tr"], V["walls_all"], V["pout"], V["lamda_d"])
    unit, (t, tt, h_over_rc, y_over_lamda) = R.OUT_LOG[-1]
    hmin, y0 = p.o.output3()
    assert h_over_rc == hmin / R.C.rad_c
    assert y_over_lamda == y0 / V["lamda_d"]
    assert 0.0 < hmin < DOMAIN[2]
