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

from tests.pin_cases import CASES, FULL, OracleCase

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pin.json")
GOLD152 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_pin_152.json")


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


@pytest.mark.skipif(not os.path.exists(GOLD152), reason="no digests of the 152^3 run")
def test_oracle_reproduces_reference_on_its_own_grid():
    """The reference as written -- 152^3, the 12 particles of initia_center --
    main's set-up and one step: the oracle's arrays have the reference's
    digests after the set-up and after the step (after every call with
    SYM_PIN_EVERY_CALL=1; hashing 2.4 GB per comparison takes a few seconds)."""
    with open(GOLD152) as f:
        g = json.load(f)["full"]
    assert g["case"] == json.loads(json.dumps(FULL))
    snaps = g["snapshots"]
    every = bool(os.environ.get("SYM_PIN_EVERY_CALL"))
    oc = OracleCase(FULL)
    assert _mismatch(snaps[0], oc.snapshot()) == [], "setup"
    i = 0
    for step, k, call in oc.steps():
        i += 1
        assert snaps[i]["after"] == f"{step}:{k}:{call}"
        if every or i == len(snaps) - 1:
            assert _mismatch(snaps[i], oc.snapshot()) == [], snaps[i]["after"]
    assert i == len(snaps) - 1
