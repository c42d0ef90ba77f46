"""Shared helpers for the parity tests: move state between the oracle and the
library and compare fields."""
from __future__ import annotations

import numpy as np

from symmetry_b200.params import FIELDS, SymParticles, particles_get

STATE_FIELDS = [f for f in FIELDS]
SCALARS = ["rho", "ux", "uy", "uz", "rho_N", "rho_R", "rho_B", "n_x", "n_y", "n_z", "gradx", "grady", "gradz"]
MASKS = ["flag", "walls", "walls_old", "walls_all", "pin", "pout"]
PART_ARRAYS = ["center", "center_old", "center0", "up", "rp", "fp", "tp", "fre", "tension", "tension_t"]


def copy_oracle_to_lattice(o, L):
    for f in STATE_FIELDS:
        L.set(f, o.arr(f))
    s = SymParticles()
    src = o.particles
    import ctypes
    ctypes.memmove(ctypes.byref(s), ctypes.byref(src), ctypes.sizeof(SymParticles))
    L.set_particles(s)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def max_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


VEL = ("ux", "uy", "uz")


def compare_fields(o, L, fields, tol, mask=None):
    """Max abs difference / scale for each field.  Scale: the field's max
    magnitude; for a velocity component the max over all three components
    (a component that is rounding noise in a symmetric flow is compared
    against the flow speed, not against its own noise)."""
    errs = {}
    vscale = max(np.abs(o.arr(k)).max() for k in VEL) if any(f in VEL for f in fields) else 0.0
    for f in fields:
        a, b = L.get(f), o.arr(f)
        if mask is not None:
            m = mask if a.ndim == mask.ndim else mask[..., None]
            a, b = np.where(m, a, 0), np.where(m, b, 0)
        if f in VEL:
            errs[f] = float(np.abs(a - b).max() / max(vscale, 1e-300))
        else:
            errs[f] = max_rel(a, b)
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"fields beyond {tol}: {bad}"
    return errs


def compare_masks(o, L, fields=MASKS):
    for f in fields:
        a, b = L.get(f), o.arr(f)
        n = int((a != b).sum())
        assert n == 0, f"mask {f}: {n} nodes differ"


def compare_particles(o, L, par, tol, arrays=PART_ARRAYS, floor=1e-3):
    """Max |a-b| / max(|b|max, floor): forces on a sphere in symmetric flow cancel
    to rounding level, so a purely relative comparison would be meaningless."""
    s = L.particles()
    so = o.particles
    errs = {}
    for name in arrays:
        a = np.array(particles_get(s, name, par))
        b = np.array(particles_get(so, name, par))
        scale = max(np.abs(b).max(), floor)
        errs[name] = float(np.abs(a - b).max() / scale)
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"particle arrays beyond {tol}: {bad}"
    return errs
