"""The oracle against digests of the reference's own arrays
(tests/golden/reference_pin.json, made by tests/golden/make_reference_pin.py
from the reference source run through its mechanical translation).

This needs no reference source: it runs the pinning cases of
tests/pin_cases.py on the oracle alone -- main's set-up and the calls of the
time-loop body, on the reference's own 12-particle layout and on a placed,
moving pair with either bounce-back -- and requires every array and particle
variable to have the reference's digest after every call, that is, to be
equal to the reference's bit for bit.
"""
import json
import os

import pytest

from tests.pin_cases import CASES, OracleCase

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pin.json")


def _gold():
    with open(GOLD) as f:
        return json.load(f)


def _mismatch(want: dict, got: dict) -> list:
    bad = [k for k, v in want["arrays"].items() if got["arrays"].get(k) != v]
    bad += [k for k, v in want["particles"].items() if got["particles"].get(k) != v]
    return bad


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_reference_digests(name):
    g = _gold()[name]
    case = json.loads(json.dumps(CASES[name]))          # as stored (tuples as lists)
    assert g["case"] == case
    snaps = g["snapshots"]
    oc = OracleCase(name)
    assert snaps[0]["after"] == "setup"
    assert _mismatch(snaps[0], oc.snapshot()) == [], "setup"
    i = 0
    for step, k, call in oc.steps():
        i += 1
        assert snaps[i]["after"] == f"{step}:{k}:{call}"
        assert _mismatch(snaps[i], oc.snapshot()) == [], snaps[i]["after"]
    assert i == len(snaps) - 1


def test_digests_cover_every_call():
    g = _gold()
    for name, c in CASES.items():
        assert len(g[name]["snapshots"]) == 1 + 15 * c["steps"]
