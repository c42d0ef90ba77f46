"""Precision study of the population storage modes.

Each case runs in FP64, FP32 and 16-bit shifted storage side by side, in
lockstep, until breakup (the minimum over z of r_eq(z) = sqrt(sum_xy
(1+phi)/2 / pi) falls below one lattice unit, read every `check` steps and
linearly interpolated) or the step cap.  Every `snap_every` steps each reduced
mode's density, velocity and phase fields are compared with FP64 (relative L2
over the domain; velocity as one vector field) and every mode's total mass is
compared with its initial value (mass drift).  The breakup step of each mode
is compared with FP64's.  Snapshots read the macroscopic fields through
sym_get_macros, which leaves the stepping state untouched (no re-encoding).

Cases:
  c3       the 256x256x512 Rayleigh-Plateau thread (R=24, 2% perturbation
           over one 512-node wavelength, tau=0.7, sigma=8e-3, beta=0.7,
           seed 1003), 40,000-step cap (--size scales it down)
  mix:K    the first K sphere-free domains of the batched-mix manifest whose
           wavelength is unstable (lambda > 2 pi R): threads that break within
           the cap, for the breakup-time error

  python -m symmetry_b200.study [--case c3|mix:K] [--max-steps N] [--size NXxNYxNZ] [--out study.json]
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

MODES = ("fp64", "fp32", "fp16")


def rel_l2(a, b):
    d = np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel())
    n = np.linalg.norm(np.asarray(b).ravel())
    return float(d / n) if n > 0 else float(d)


def with_storage(w, mode):
    p = w.params.copy()
    p.storage = {"fp64": 0, "fp32": 1, "fp16": 2}[mode]
    return configs.Workload(w.name, p, w.kind, dict(w.gen), w.steps, list(w.particles))


def run_case(w, modes=MODES, max_steps=40000, check=10, snap_every=5000, threshold=1.0, log=sys.stderr):
    lat = {m: setup_workload(with_storage(w, m)) for m in modes}
    # total mass = the sum of rho over the domain (sphere-free cases: every
    # node is fluid), read through sym_get_macros so that the fused state of
    # the reduced modes is never exported and re-encoded mid-run
    mass0 = {m: float(L.macros()["rho"].sum()) for m, L in lat.items()}
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
            ref = lat[modes[0]].macros()
            row = {"step": t, "rmin": {m: prev[m][1] for m in modes}}
            for m in modes:
                sn = ref if m == modes[0] else lat[m].macros()
                row.setdefault("mass_drift", {})[m] = (float(sn["rho"].sum()) - mass0[m]) / mass0[m]
                if m == modes[0]:
                    continue
                u = np.stack([sn[k] for k in ("ux", "uy", "uz")])
                uref = np.stack([ref[k] for k in ("ux", "uy", "uz")])
                row.setdefault("l2", {})[m] = {"u": rel_l2(u, uref), "rho": rel_l2(sn["rho"], ref["rho"]),
                                                "phi": rel_l2(sn["rho_N"], ref["rho_N"])}
            snaps.append(row)
            print(json.dumps({"case": w.name, **row}), file=log, flush=True)
    base = breakup[modes[0]]
    out = {
        "case": w.name, "size": [w.params.nx, w.params.ny, w.params.nz], "gen": w.gen,
        "tau": 3.0 * w.params.nu_r + 0.5, "sigma": w.params.sigma,
        "modes": list(modes), "check_every": check, "threshold": threshold, "max_steps": max_steps,
        "steps_run": t, "wall_s": time.time() - t0, "breakup_step": breakup,
        "breakup_rel_err": {m: (abs(breakup[m] - base) / base if (breakup[m] is not None and base) else None)
                            for m in modes},
        "max_l2_u": {m: max((r["l2"][m]["u"] for r in snaps), default=None) for m in modes[1:]},
        "last_l2": snaps[-1]["l2"] if snaps else None,
        "snapshots": snaps,
    }
    for L in lat.values():
        L.close()
    return out


def mix_cases(k):
    """The first k sphere-free manifest domains with an unstable wavelength."""
    out = []
    for w in configs.c4_manifest(storage="fp64"):
        if w.params.par:
            continue
        if w.gen["wavelength"] > 2.0 * math.pi * w.gen["radius"]:
            out.append(w)
        if len(out) == k:
            break
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c3")
    ap.add_argument("--size", default=None)
    ap.add_argument("--max-steps", type=int, default=40000)
    ap.add_argument("--snap-every", type=int, default=5000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.case == "c3":
        if a.size:
            nx, ny, nz = (int(v) for v in a.size.lower().split("x"))
            ws = [configs.c3_thread(nx=nx, ny=ny, nz=nz, radius=24.0 * nx / 256.0)]
        else:
            ws = [configs.c3_thread()]
    elif a.case.startswith("mix:"):
        ws = mix_cases(int(a.case.split(":")[1]))
    else:
        raise SystemExit(f"unknown case {a.case}")
    res = []
    for w in ws:
        res.append(run_case(w, max_steps=a.max_steps, snap_every=a.snap_every))
        if a.out:   # keep what finished if a later case is cut short
            with open(a.out, "w") as f:
                f.write(json.dumps(res) + "\n")
    print(json.dumps(res))


if __name__ == "__main__":
    main()
