"""The Fortran binding module (symmetry_b200/fortran/symmetry_gpu.f90) held to
the C ABI it binds.  No Fortran compiler exists here, so the module is
shipped uncompiled; this test reads it as text instead: every bind(C)
interface names a function that include/symmetry.h declares and the library
exports, with as many arguments as the C prototype; the derived types
sym_params and sym_particles have the C structs' members in the same order
and of the same kinds; and the named constants have the header's values."""
import ctypes
import os
import re

import pytest

from symmetry_b200 import lib as symlib
from symmetry_b200.params import SymParams, SymParticles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "symmetry_b200", "fortran", "symmetry_gpu.f90")
HDR = os.path.join(ROOT, "include", "symmetry.h")


def _fortran_statements():
    out, buf = [], ""
    for raw in open(F90).read().split("\n"):
        s = raw.split("!")[0].rstrip()
        if not s.strip():
            continue
        t = s.strip()
        if buf and t.startswith("&"):
            t = t[1:]
        if t.endswith("&"):
            buf += t[:-1] + " "
            continue
        out.append((buf + t).strip())
        buf = ""
    return out


def _interfaces():
    """C name -> number of dummy arguments, for every bind(C) function."""
    out = {}
    for s in _fortran_statements():
        m = re.match(r"^.*\bfunction\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*c\s*,\s*name\s*=\s*\"(\w+)\"\s*\)",
                     s, re.I)
        if m:
            args = [a for a in m.group(2).split(",") if a.strip()]
            out[m.group(3)] = len(args)
    return out


def _split_params(p: str):
    p = p.strip()
    if p in ("", "void"):
        return []
    depth, cur, out = 0, "", []
    for ch in p:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return out


def _prototypes():
    """C name -> number of parameters, for every sym_* prototype of the header."""
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(sym_\w+)\s*\(([^;{]*?)\)\s*;", text):
        out[m.group(1)] = len(_split_params(m.group(2)))
    return out


def _header_constants():
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    vals = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(SYM_\w+)\s+(-?\d+)\b", text)}
    enum = re.search(r"enum\s*\w*\s*\{([^}]*SYM_F_RI[^}]*)\}", text).group(1)
    v = -1
    for item in enum.split(","):
        item = item.strip()
        if not item:
            continue
        if "=" in item:
            name, val = (x.strip() for x in item.split("="))
            v = int(val)
        else:
            name, v = item, v + 1
        vals[name] = v
    return vals


def test_every_interface_binds_a_declared_exported_function_with_its_arity():
    ifs, protos = _interfaces(), _prototypes()
    assert len(ifs) >= 30
    L = symlib.lib()
    for cname, nargs in ifs.items():
        assert cname in protos, f"{cname}: not declared in include/symmetry.h"
        assert nargs == protos[cname], f"{cname}: {nargs} dummies, C prototype has {protos[cname]}"
        assert hasattr(L, cname), f"{cname}: not exported by the library"


def test_every_per_subroutine_entry_point_has_a_fortran_interface():
    ifs = _interfaces()
    for name in ("sym_set_walls", "sym_calmacros", "sym_derivatives", "sym_collision", "sym_recolor",
                 "sym_boundary", "sym_streaming", "sym_curve", "sym_lagrange_points", "sym_capillary_force2",
                 "sym_momentum", "sym_repulsive", "sym_movement", "sym_refilling", "sym_initialization",
                 "sym_initia_center", "sym_step"):
        assert name in ifs, name


def _fortran_type(name):
    """Member names and kinds ('i' 32-bit integer, 'd' double) of a derived type, in order."""
    out, inside = [], False
    for s in _fortran_statements():
        if re.match(rf"^type\s*,\s*bind\s*\(\s*c\s*\)\s*::\s*{name}$", s, re.I):
            inside = True
            continue
        if inside and re.match(r"^end\s*type", s, re.I):
            return out
        if inside:
            kind = "i" if "c_int32_t" in s else "d"
            for m in re.finditer(r"(\w+)\s*(?:\(([^)]*)\))?\s*(?:,|$)", s.split("::")[1]):
                n = 1
                for f in (m.group(2) or "1").split("*"):    # a product of literals and SYM_MAX_PAR
                    f = f.strip()
                    n *= 32 if f == "SYM_MAX_PAR" else int(f)
                out.append((m.group(1), kind, n))
    raise AssertionError(f"type {name} not found")


@pytest.mark.parametrize("fname,ctype", [("sym_params", SymParams), ("sym_particles", SymParticles)])
def test_derived_types_match_the_c_structs(fname, ctype):
    got = _fortran_type(fname)
    want = []
    for n, t in ctype._fields_:
        if issubclass(t, ctypes.Array):
            kind = "i" if t._type_ in (ctypes.c_int32,) else "d"
            want.append((n, kind, t._length_))
        else:
            want.append((n, "i" if t is ctypes.c_int32 else "d", 1))
    assert got == want


def test_named_constants_have_the_header_values():
    hdr = _header_constants()
    seen = 0
    for s in _fortran_statements():
        if "parameter" not in s.lower():
            continue
        for m in re.finditer(r"\b(SYM_\w+)\s*=\s*(-?\d+)", s):
            assert hdr[m.group(1)] == int(m.group(2)), m.group(1)
            seen += 1
    assert seen >= 25
