"""Digests of the reference's arrays along the pinning cases, from the
reference source itself run through its mechanical translation
(oracle/f90py.py), into reference_pin.json beside this script.  Run where the
reference source is present; the JSON is committed and
tests/test_reference_golden.py checks the oracle against it anywhere.

  python tests/golden/make_reference_pin.py           # the cases -> reference_pin.json
  python tests/golden/make_reference_pin.py --full    # the 152^3 grid -> reference_pin_152.json (~45 min)

For each case of tests/pin_cases.py: a digest of every array and particle
variable after main's set-up (and the particles' placement), then after each
call of the time-loop body.  Digests are SHA-256 of the values in Fortran
element order, with -0 as +0 and one NaN.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import f90py  # noqa: E402
from tests.pin_cases import CASES, FULL, ReferenceCase  # noqa: E402


def case_record(case):
    R = f90py.load_reference()
    if R is None:
        raise SystemExit("the reference source is not on this machine")
    rc = ReferenceCase(R, case)
    snaps = [dict(after="setup", **rc.snapshot())]
    for step, k, call in rc.steps():
        snaps.append(dict(after=f"{step}:{k}:{call}", **rc.snapshot()))
    return {"case": rc.c, "snapshots": snaps}


def main():
    if "--full" in sys.argv[1:]:
        out, name = {"full": case_record(FULL)}, "reference_pin_152.json"
    else:
        out, name = {n: case_record(n) for n in CASES}, "reference_pin.json"
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), name)
    with open(path, "w") as f:
        json.dump(out, f, sort_keys=True, separators=(",", ":"))
        f.write("\n")
    print(path)


if __name__ == "__main__":
    main()
