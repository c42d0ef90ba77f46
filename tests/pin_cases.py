"""The cases that pin the oracle to the reference, shared by
tests/test_reference_pin.py (the translated reference beside the oracle),
tests/golden/make_reference_pin.py (digests of the translated reference's
arrays, committed as tests/golden/reference_pin.json) and
tests/test_reference_golden.py (the oracle against those digests, where the
reference source is absent).

A case is main's set-up on a grid (Source1.f90:28-214), optionally with
particles placed and launched identically on both sides, then calls of the
time-loop body (Source1.f90:216-251) for a number of steps.
"""
from __future__ import annotations

import hashlib
import warnings

import numpy as np

from oracle.oracle import setup_reference
from symmetry_b200.params import particles_set, reference_params

# translated reference (main's variable) -> oracle array
FIELDS = {"rho": "rho", "ux": "ux", "uy": "uy", "uz": "uz", "rho_n": "rho_N", "rho_r": "rho_R", "rho_b": "rho_B",
          "n_x": "n_x", "n_y": "n_y", "n_z": "n_z", "gradx": "gradx", "grady": "grady", "gradz": "gradz",
          "fi": "fi", "ffi": "ffi", "ri": "ri", "bi": "bi", "walls": "walls", "walls_old": "walls_old",
          "walls_all": "walls_all", "pin": "pin", "pout": "pout", "flag": "flag",
          "lax": "Lax", "lay": "Lay", "laz": "Laz", "la_rhon": "La_rhoN", "la_nx": "La_nx", "la_ny": "La_ny",
          "la_nz": "La_nz", "ds": "ds", "la_flag": "La_flag"}
MASKS = {"walls", "walls_old", "walls_all", "pin", "pout", "flag", "la_flag"}
PARTICLE_MATS = {"center": "center", "center_old": "center_old", "center0": "center0", "tension": "tension",
                 "tension_t": "tension_t"}
PARTICLE_VECS = {"fp": ("fpx", "fpy", "fpz"), "tp": ("tpx", "tpy", "tpz"), "up": ("upx", "upy", "upz"),
                 "rp": ("rpx", "rpy", "rpz"), "fre": ("frex", "frey", "frez")}

# the calls of main's time-loop body, in order (Source1.f90:216-251)
LOOP_CALLS = ["calmacros", "lagrange_points", "capillary_force2", "momentum", "repulsive", "movement", "set_walls",
              "refilling", "derivatives", "collision", "recolor", "boundary", "streaming", "streaming", "curve"]

# 36 x 42 x 36: the thread of radius 30 about the corner line x = z = 35.5
# (initialization) crosses x = z = 14.3; two particles of radius 7.5 sit on
# that interface, outside the 3-node wall repulsion range of every face
# (repulsive, Source1.f90:1606-1649) and 2.6 nodes apart, inside each
# other's, launched fast enough that nodes they leave are refilled
PLACED = [[14.3, 12.2, 14.3], [15.0, 29.8, 13.6]]
LAUNCH = [[0.3, 0.25, -0.2], [-0.25, -0.3, 0.25]]
# the reference's own grid and layout as written (xl = yl = zl = 152, par = 12):
# too slow for the default suite as Python, run on request
FULL = dict(domain=(152, 152, 152), par=12, centers=None, velocity=None, bounce=False, steps=1)
CASES = {
    # the reference's own 12 particles (initia_center) on the smallest grid
    # they fit: below it they overlap and reach past x = 1
    "layout": dict(domain=(48, 88, 48), par=12, centers=None, velocity=None, bounce=False, steps=1),
    "moving": dict(domain=(36, 42, 36), par=2, centers=PLACED, velocity=LAUNCH, bounce=False, steps=2),
    # curve2 (Source1.f90:1036-1101) in place of curve: the oracle's bounce switch
    "bouncing": dict(domain=(36, 42, 36), par=2, centers=PLACED, velocity=LAUNCH, bounce=True, steps=1),
}


def _canon(a: np.ndarray) -> np.ndarray:
    """Values as compared: +0 for -0 and one NaN for every NaN."""
    a = np.asarray(a, dtype=np.float64) + 0.0
    return np.where(np.isnan(a), np.nan, a)


def digest(a: np.ndarray, mask: bool) -> str:
    """Digest of an array's values in Fortran element order (given flat)."""
    a = np.asarray(a).reshape(-1)
    b = (a != 0).astype(np.int32) if a.dtype == bool else a.astype(np.int32) if mask else _canon(a)
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()[:16]


def hexes(a) -> str:
    """Digest of a short float array's exact values."""
    return digest(np.asarray(a, dtype=np.float64), False)


class OracleCase:
    """One case on the oracle alone."""

    def __init__(self, name):
        c = CASES[name] if isinstance(name, str) else name
        self.c = c
        nx, ny, nz = c["domain"]
        prm = reference_params(nx, ny, nz, c["par"])
        prm.bounce = 1 if c["bounce"] else 0
        self.o = o = setup_reference(prm)
        self.par = c["par"]
        if c["centers"] is not None:
            s = o.particles
            particles_set(s, "center", self.par, c["centers"])
            particles_set(s, "center0", self.par, c["centers"])
            if c["velocity"] is not None:
                particles_set(s, "up", self.par, c["velocity"])
            o.call("set_walls")
            o.call("derivatives")

    def steps(self):
        """Run the case's steps, yielding (step, call index, subroutine) after each call."""
        for step in range(self.c["steps"]):
            n_stream = 0
            for k, name in enumerate(LOOP_CALLS):
                if name == "streaming":
                    self.o.streaming(n_stream)
                    n_stream += 1
                else:
                    self.o.call(name)
                yield step, k, name

    def snapshot(self) -> dict:
        o, par = self.o, self.par
        arrays = {f: digest(o.arr(on), f in MASKS) for f, on in FIELDS.items()}
        s = o.particles
        parts = {f: hexes(np.array(getattr(s, on)[:3 * par])) for f, on in PARTICLE_MATS.items()}
        parts.update({on: hexes(np.array(getattr(s, on)[:3 * par])) for on in PARTICLE_VECS})
        parts["shb"] = hexes(np.array(s.shb[:par]))
        return {"arrays": arrays, "particles": parts}


class ReferenceCase:
    """One case on the translated reference (main's variables by name)."""

    def __init__(self, R, name):
        c = CASES[name] if isinstance(name, str) else name
        self.c, self.R, self.par = c, R, c["par"]
        R.C.xl, R.C.yl, R.C.zl = c["domain"]
        R.C.par = c["par"]
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            self.V = V = R.main_setup()
        if c["centers"] is not None:
            for k, ctr in enumerate(c["centers"]):
                V["center"][k, :] = ctr
                V["center0"][k, :] = ctr
            if c["velocity"] is not None:
                for k in range(self.par):
                    for j, n in enumerate(("upx", "upy", "upz")):
                        V[n][k] = c["velocity"][k][j]
            self.call("set_walls")
            self.call("derivatives")

    def call(self, name, acts=None):
        if acts is None:
            acts = next(a for n, a, _ in self.R.MAIN_LOOP_CALLS if n == name)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            getattr(self.R, name)(*[self.V[self.R.pyname(a)] for a in acts])

    def steps(self):
        for step in range(self.c["steps"]):
            for k, (name, acts, _line) in enumerate(self.R.MAIN_LOOP_CALLS):
                # curve2 takes curve's arguments (Source1.f90:1036)
                self.call("curve2" if name == "curve" and self.c["bounce"] else name, acts)
                yield step, k, name

    def snapshot(self) -> dict:
        V, par = self.V, self.par
        arrays = {f: digest(np.asarray(V[f]).ravel(order="F"), f in MASKS) for f in FIELDS}
        parts = {f: hexes(np.asarray(V[f]).ravel(order="F")) for f in PARTICLE_MATS}
        parts.update({on: hexes(np.stack([V[n] for n in names], 1).ravel(order="F"))
                      for on, names in PARTICLE_VECS.items()})
        parts["shb"] = hexes(V["shb"])
        return {"arrays": arrays, "particles": parts}
