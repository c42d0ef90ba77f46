"""Precision study of the population storage modes on one large domain.

The 256x256x512 Rayleigh-Plateau thread (R=24, 2% perturbation over one
512-node wavelength, tau=0.7, sigma=8e-3, beta=0.7, seed 1003) runs in FP64,
FP32 and FP16 shifted storage side by side, in lockstep, until breakup (the
minimum over z of r_eq(z) = sqrt(sum_xy (1+phi)/2 / pi) falls below one
lattice unit, read every 10 steps and linearly interpolated) or the step cap.
Every `snap_every` steps each reduced mode's density, velocity and phase
fields are compared with FP64 (relative L2 over the domain; velocity as one
vector field) and every mode's total mass is compared with its initial value
(mass drift).  The breakup step of each mode is compared with FP64's.

  python -m symmetry_b200.study [--max-steps 40000] [--size 256x256x512] [--out study.json]

A snapshot exports the fused state to the canonical arrays, which re-encodes
the 16-bit populations once: one extra rounding per snapshot interval.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import configs
from .lib import setup_workload


def rel_l2(a, b):
    d = np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel())
    n = np.linalg.norm(np.asarray(b).ravel())
    return float(d / n) if n > 0 else float(d)


def snapshot(L):
    L.call("calmacros")
    return {k: L.get(k) for k in ("rho", "ux", "uy", "uz", "rho_N")}


def run(size=None, modes=("fp64", "fp32", "fp16"), max_steps=40000, check=10, snap_every=5000,
        threshold=1.0, log=sys.stderr):
    if size:
        nx, ny, nz = (int(v) for v in size.lower().split("x"))
        mk = lambda m: configs.c3_thread(nx=nx, ny=ny, nz=nz, storage=m, radius=24.0 * nx / 256.0)  # noqa: E731
    else:
        mk = lambda m: configs.c3_thread(storage=m)  # noqa: E731
    lat = {m: setup_workload(mk(m)) for m in modes}
    mass0 = {}
    for m, L in lat.items():
        mm = L.mass_momentum()
        mass0[m] = mm[0] + mm[1]
    prev = {m: (0, L.neck_radius()) for m, L in lat.items()}
    breakup = {m: None for m in modes}
    snaps, t, t0 = [], 0, time.time()
    while t < max_steps and any(breakup[m] is None for m in modes):
        for m, L in lat.items():
            if breakup[m] is not None:
                continue
            L.step(check)
            r = L.neck_radius()          # phase field of the state after t+check-1 steps
            s = t + check - 1
            if not math.isfinite(r):
                breakup[m] = float("nan")
            elif r < threshold:
                s0, r0 = prev[m]
                f = (r0 - threshold) / (r0 - r) if r0 > r else 1.0
                breakup[m] = s0 + min(1.0, max(0.0, f)) * (s - s0)
            prev[m] = (s, r)
        t += check
        if t % snap_every == 0 and all(breakup[m] is None for m in modes):
            ref = snapshot(lat[modes[0]])
            row = {"step": t, "rmin": {m: prev[m][1] for m in modes}}
            for m in modes:
                mm = lat[m].mass_momentum()
                row.setdefault("mass_drift", {})[m] = (mm[0] + mm[1] - mass0[m]) / mass0[m]
                if m == modes[0]:
                    continue
                sn = snapshot(lat[m])
                u = np.stack([sn[k] for k in ("ux", "uy", "uz")])
                uref = np.stack([ref[k] for k in ("ux", "uy", "uz")])
                row.setdefault("l2", {})[m] = {"u": rel_l2(u, uref), "rho": rel_l2(sn["rho"], ref["rho"]),
                                                "phi": rel_l2(sn["rho_N"], ref["rho_N"])}
            snaps.append(row)
            print(json.dumps(row), file=log, flush=True)
    base = breakup[modes[0]]
    out = {
        "workload": f"c3_thread {mk('fp64').params.nx}x{mk('fp64').params.ny}x{mk('fp64').params.nz}",
        "modes": list(modes), "check_every": check, "threshold": threshold, "max_steps": max_steps,
        "steps_run": t, "wall_s": time.time() - t0, "breakup_step": breakup,
        "breakup_rel_err": {m: (abs(breakup[m] - base) / base if (breakup[m] is not None and base) else None)
                            for m in modes},
        "snapshots": snaps,
    }
    for L in lat.values():
        L.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default=None)
    ap.add_argument("--max-steps", type=int, default=40000)
    ap.add_argument("--snap-every", type=int, default=5000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    res = run(size=a.size, max_steps=a.max_steps, snap_every=a.snap_every)
    s = json.dumps(res)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")
    print(s)


if __name__ == "__main__":
    main()
