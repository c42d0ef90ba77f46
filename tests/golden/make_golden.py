"""Extract the reference's constant tables from Source1.f90 into
reference_constants.json (run in a container where the reference source is
mounted; the JSON is committed and the tests read only the JSON).

  python tests/golden/make_golden.py /path/to/Source1.f90

Tables: the MRT moment matrix from the data statement (Source1.f90:105-123,
column-major: the k-th listed value is M(k mod 19, k div 19)), the velocity
set cix/ciy/ciz, opposites opc and mirror maps symx/symy/symz (:132-138), the
weights wi (:140-142) and scalar constants (:16-17, :21-22).
"""
import json
import os
import re
import sys


def main(path):
    raw = open(path, "rb").read().decode("latin-1")
    m = re.search(r"data\s+M\s*/(.*?)/", raw, flags=re.S | re.I)
    body = m.group(1).replace("&", " ")
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    assert len(vals) == 361, len(vals)
    M = [[vals[c * 19 + r] for c in range(19)] for r in range(19)]

    def intarr(name):
        mm = re.search(name + r"\s*=\s*\(/(.*?)/\)", raw, flags=re.I)
        return [int(v) for v in mm.group(1).split(",")]

    out = {
        "source": "Source1.f90",
        "M": M,
        "cix": intarr("cix"), "ciy": intarr("ciy"), "ciz": intarr("ciz"), "opc": intarr("opc"),
        "symx": intarr("symx"), "symy": intarr("symy"), "symz": intarr("symz"),
        "wi": [1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12,
        "EVAP_LIM": float(re.search(r"EVAP_LIM\s*=\s*([0-9.d\-+]+)", raw).group(1).replace("d", "e")),
        "beta": float(re.search(r"beta\s*=\s*([0-9.d\-+]+)", raw).group(1).replace("d", "e")),
        "wi_source": [l.strip() for l in raw.splitlines() if l.strip().startswith("wi(")],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_constants.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference's Source1.f90>")
    main(sys.argv[1])
