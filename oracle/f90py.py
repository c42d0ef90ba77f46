"""Mechanical Fortran-to-Python translation of the reference solver -- TEST
INFRASTRUCTURE ONLY (it pins the oracle; nothing in the library uses it).

No Fortran compiler exists on this image, so the reference (Source1.f90, one
free-form Fortran 90 file) cannot be built and run.  This module translates
the subset of Fortran that file is written in -- a module of constants,
subroutines with explicit-shape array dummies, DO / IF blocks, array
sections and constructors, MATMUL / SUM / DOT_PRODUCT / MAXVAL and the
scalar intrinsics -- statement by statement into Python over numpy arrays,
so that the reference's own subroutines, exactly as written, can be executed
on small domains beside the oracle's restatement (tests/test_reference_pin.py).

What the translation fixes that the Fortran source leaves to the compiler,
chosen as gfortran -O3 without -ffast-math on x86-64 does it:
  * every operation is IEEE double (or single, for default-REAL literals and
    REAL()) in source order, no contraction into fused multiply-add;
  * x**n with an integer n is square-and-multiply (libgcc's __powidf2);
  * MATMUL(A, v) accumulates each row over the columns in ascending order,
    SUM and DOT_PRODUCT accumulate in array-element order;
  * sqrt, acos, sin, cos, ... are the C library's (Python's math module).
Integer division truncates toward zero and MOD takes the sign of its first
argument, as in Fortran.  OPEN and CLOSE are dropped; a WRITE appends its
unit and the values of its output items to the module's OUT_LOG.
The module's compile-time constants (grid extents, particle count) become
attributes of the generated module's `C` namespace, so a test can size the
domain; every other line keeps the source's arithmetic.

Usage:  python -m oracle.f90py <Source1.f90> <out.py>
"""
from __future__ import annotations

import re
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

# ---- source handling ------------------------------------------------------------


def _strip_comment(line: str) -> str:
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def logical_lines(text: str) -> List[Tuple[int, str]]:
    """(first physical line number, statement) with comments removed,
    continuations joined and everything outside strings lower-cased."""
    out: List[Tuple[int, str]] = []
    buf, start = "", 0
    for n, raw in enumerate(text.split("\n"), 1):
        s = _strip_comment(raw).rstrip()
        if not s.strip():
            if buf:
                continue
            continue
        t = s.strip()
        if buf and t.startswith("&"):
            t = t[1:]
        if not buf:
            start = n
        if t.endswith("&"):
            buf += t[:-1] + " "
            continue
        buf += t
        for stmt in _split_semicolons(buf):
            if stmt.strip():
                out.append((start, _lower_outside_strings(stmt.strip())))
        buf = ""
    return out


def _split_semicolons(s: str) -> List[str]:
    parts, cur, q = [], [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == ";":
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return parts


def _lower_outside_strings(s: str) -> str:
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


def split_top(s: str, sep: str = ",") -> List[str]:
    """Split at `sep` outside parentheses, array constructors and strings."""
    parts, cur, depth, q = [], [], 0, None
    i = 0
    while i < len(s):
        ch = s[i]
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch == "(":
            depth += 1
            cur.append(ch)
        elif ch == ")":
            depth -= 1
            cur.append(ch)
        elif ch == sep and depth == 0:
            parts.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
        i += 1
    if "".join(cur).strip():
        parts.append("".join(cur).strip())
    return parts


# ---- program units and declarations -------------------------------------------


@dataclass
class Var:
    name: str
    typ: str                      # 'i' integer, 'r' double, 's' default real, 'l' logical, 'c' character
    dims: Optional[List[Tuple[str, str]]] = None   # (lower, upper) source expressions; None: scalar
    param: bool = False
    init: Optional[str] = None

    @property
    def rank(self) -> int:
        return len(self.dims) if self.dims else 0


@dataclass
class Unit:
    kind: str                     # 'module', 'program', 'subroutine'
    name: str
    args: List[str]
    line: int
    decls: List[Tuple[int, str]] = field(default_factory=list)
    body: List[Tuple[int, str]] = field(default_factory=list)
    uses: List[str] = field(default_factory=list)
    vars: Dict[str, Var] = field(default_factory=dict)
    data: List[Tuple[int, str]] = field(default_factory=list)   # DATA statements, wherever they stand


_TYPE_RE = re.compile(r"^(integer|double\s+precision|real\s*\*\s*8|real\s*\(\s*8\s*\)|real\s*\(\s*kind\s*=\s*8\s*\)|"
                      r"real|logical|character(?:\s*\*\s*\d+|\s*\([^)]*\))?)\b(.*)$")


def _type_code(t: str) -> str:
    t = re.sub(r"\s+", "", t)
    if t == "integer":
        return "i"
    if t in ("doubleprecision", "real*8", "real(8)", "real(kind=8)"):
        return "r"
    if t == "real":
        return "s"
    if t == "logical":
        return "l"
    return "c"


def parse_units(text: str) -> Dict[str, Unit]:
    units: Dict[str, Unit] = {}
    cur: Optional[Unit] = None
    in_decls = False
    for n, s in logical_lines(text):
        m = re.match(r"^module\s+(\w+)$", s)
        if m and cur is None:
            cur = Unit("module", m.group(1), [], n)
            in_decls = True
            continue
        m = re.match(r"^program\s+(\w+)$", s)
        if m and cur is None:
            cur = Unit("program", m.group(1), [], n)
            in_decls = True
            continue
        m = re.match(r"^subroutine\s+(\w+)\s*(?:\((.*)\))?$", s)
        if m and cur is None:
            args = [a.strip() for a in (m.group(2) or "").split(",") if a.strip()]
            cur = Unit("subroutine", m.group(1), args, n)
            in_decls = True
            continue
        if re.match(r"^end\s*(module|program|subroutine)\b", s) or (s == "end" and cur is not None):
            units[cur.name] = cur
            cur = None
            continue
        if cur is None:
            continue
        if s.startswith("use "):
            cur.uses.append(s[4:].split(",")[0].strip())
            continue
        if s.startswith("implicit"):
            continue
        if in_decls and (_TYPE_RE.match(s) and ("::" in s or not re.match(r"^real\s*\(", s))) and \
                not re.match(r"^(integer|real|logical)\s*=", s):
            cur.decls.append((n, s))
            continue
        if re.match(r"^data\s", s):
            cur.data.append((n, s))
            continue
        in_decls = False
        cur.body.append((n, s))
    for u in units.values():
        for n, s in u.decls:
            _parse_decl(u, s)
    return units


def _parse_decl(u: Unit, s: str) -> None:
    m = _TYPE_RE.match(s)
    typ = _type_code(m.group(1))
    rest = m.group(2)
    if "::" in rest:
        attrs_s, ents_s = rest.split("::", 1)
    else:
        attrs_s, ents_s = "", rest
    attrs = split_top(attrs_s.lstrip(","))
    dims = None
    param = False
    for a in attrs:
        a = a.strip()
        if a.startswith("dimension"):
            dims = _parse_dims(a[a.index("(") + 1:a.rindex(")")])
        elif a == "parameter":
            param = True
    for e in split_top(ents_s):
        init = None
        if "=" in e and not e.strip().startswith("("):
            k = _top_eq(e)
            if k >= 0:
                e, init = e[:k].strip(), e[k + 1:].strip()
        mm = re.match(r"^(\w+)\s*(?:\((.*)\))?$", e.strip())
        name = mm.group(1)
        d = _parse_dims(mm.group(2)) if mm.group(2) else dims
        u.vars[name] = Var(name, typ, d, param, init)


def _top_eq(e: str) -> int:
    depth = 0
    for i, ch in enumerate(e):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0 and e[i + 1:i + 2] != "=" and e[i - 1:i] not in "<>/=":
            return i
    return -1


def _parse_dims(s: str) -> List[Tuple[str, str]]:
    out = []
    for d in split_top(s):
        if d == ":":
            out.append(("1", ""))
        elif ":" in d:
            lo, hi = d.split(":", 1)
            out.append((lo.strip() or "1", hi.strip()))
        else:
            out.append(("1", d.strip()))
    return out


# ---- expressions ------------------------------------------------------------------

_TOK = re.compile(r"""
   (?P<ws>\s+)
 | (?P<real>\d+\.\d*[ed][+-]?\d+|\d*\.\d+(?:[ed][+-]?\d+)?|\d+\.(?![a-z])|\d+[ed][+-]?\d+)
 | (?P<int>\d+)
 | (?P<dot>\.(?:and|or|not|eqv|neqv|eq|ne|lt|le|gt|ge|true|false)\.)
 | (?P<acon>\(/|/\))
 | (?P<op>\*\*|==|/=|<=|>=|<|>|\+|-|\*|/|\(|\)|,|:|=)
 | (?P<name>[a-z_]\w*)
 | (?P<str>'[^']*'|"[^"]*")
""", re.X)


def tokenize(s: str) -> List[Tuple[str, str]]:
    out, i = [], 0
    while i < len(s):
        m = _TOK.match(s, i)
        if not m:
            raise SyntaxError(f"cannot tokenize at {s[i:i + 20]!r} in {s!r}")
        i = m.end()
        k = m.lastgroup
        if k != "ws":
            out.append((k, m.group(k)))
    return out


@dataclass
class Ex:
    code: str
    typ: str        # 'i', 'r', 's', 'l', 'c'
    arr: bool = False


_REL = {"==": "==", ".eq.": "==", "/=": "!=", ".ne.": "!=", "<": "<", ".lt.": "<", "<=": "<=", ".le.": "<=",
        ">": ">", ".gt.": ">", ">=": ">=", ".ge.": ">="}


def _num_type(a: str, b: str) -> str:
    if "r" in (a, b):
        return "r"
    if "s" in (a, b):
        return "s"
    return "i"


import builtins as _builtins
import keyword as _keyword

_RESERVED = set(_keyword.kwlist) | set(dir(_builtins)) | {"np", "math", "C"}


def pyname(name: str) -> str:
    """Python name of a Fortran variable (renamed where it would shadow a
    Python keyword, builtin or a name of the generated module)."""
    return name + "_v" if name in _RESERVED or name.startswith("_") else name


class Ctx:
    """Name resolution for one program unit: its own variables, then those of
    the modules it uses (as C.<name>)."""

    def __init__(self, unit: Unit, modules: Dict[str, Unit]):
        self.unit = unit
        self.modvars: Dict[str, Var] = {}
        for m in unit.uses:
            if m in modules:
                self.modvars.update(modules[m].vars)

    def lookup(self, name: str) -> Tuple[Optional[Var], str]:
        if name in self.unit.vars:
            return self.unit.vars[name], pyname(name)
        if name in self.modvars:
            return self.modvars[name], "C." + name
        return None, name


class Parser:
    def __init__(self, s: str, ctx: Ctx):
        self.t = tokenize(s)
        self.i = 0
        self.ctx = ctx
        self.src = s

    def peek(self, k: int = 0) -> Tuple[str, str]:
        j = self.i + k
        return self.t[j] if j < len(self.t) else ("eof", "")

    def take(self, val: Optional[str] = None) -> Tuple[str, str]:
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError(f"expected {val!r}, got {tok[1]!r} in {self.src!r}")
        self.i += 1
        return tok

    def done(self) -> bool:
        return self.i >= len(self.t)

    # precedence climbing, lowest first
    def expr(self) -> Ex:
        a = self.and_()
        while self.peek()[1] == ".or.":
            self.take()
            b = self.and_()
            a = Ex(f"np.logical_or({a.code}, {b.code})" if (a.arr or b.arr) else f"({a.code} or {b.code})", "l",
                   a.arr or b.arr)
        return a

    def and_(self) -> Ex:
        a = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            b = self.not_()
            a = Ex(f"np.logical_and({a.code}, {b.code})" if (a.arr or b.arr) else f"({a.code} and {b.code})", "l",
                   a.arr or b.arr)
        return a

    def not_(self) -> Ex:
        if self.peek()[1] == ".not.":
            self.take()
            a = self.not_()
            return Ex(f"np.logical_not({a.code})" if a.arr else f"(not {a.code})", "l", a.arr)
        return self.rel()

    def rel(self) -> Ex:
        a = self.add()
        op = self.peek()[1]
        if op in _REL:
            self.take()
            b = self.add()
            return Ex(f"({a.code} {_REL[op]} {b.code})", "l", a.arr or b.arr)
        return a

    def add(self) -> Ex:
        if self.peek()[1] in ("+", "-"):
            sign = self.take()[1]
            a = self.mul()
            if sign == "-":
                a = Ex(f"(-{a.code})", a.typ, a.arr)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            b = self.mul()
            a = self.arith(a, op, b)
        return a

    def mul(self) -> Ex:
        a = self.pow_()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            b = self.pow_()
            a = self.arith(a, op, b)
        return a

    def pow_(self) -> Ex:
        a = self.unary()
        if self.peek()[1] == "**":
            self.take()
            b = self.pow_()
            if b.typ == "i":
                if a.typ == "i":
                    return Ex(f"({a.code} ** {b.code})", "i", a.arr)
                code = f"_powi({a.code}, {b.code})"
                return Ex(f"_s({code})" if a.typ == "s" else code, a.typ, a.arr)
            t = _num_type(a.typ, b.typ)
            code = f"_powr({a.code}, {b.code})"
            return Ex(f"_s({code})" if t == "s" else code, t, a.arr or b.arr)
        return a

    def unary(self) -> Ex:
        if self.peek()[1] in ("+", "-"):          # a*-b (an extension gfortran accepts)
            sign = self.take()[1]
            a = self.pow_()
            return Ex(f"(-{a.code})" if sign == "-" else a.code, a.typ, a.arr)
        return self.primary()

    def arith(self, a: Ex, op: str, b: Ex) -> Ex:
        t = _num_type(a.typ, b.typ)
        arr = a.arr or b.arr
        if t == "i" and op == "/":
            return Ex(f"_idiv({a.code}, {b.code})", "i", arr)
        code = f"({a.code} {op} {b.code})"
        if t == "s":
            code = f"_s{code}"
        return Ex(code, t, arr)

    def primary(self) -> Ex:
        k, v = self.peek()
        if k == "real":
            self.take()
            if "d" in v:
                return Ex(repr(float(v.replace("d", "e"))), "r")
            return Ex(f"_s({float(v)!r})", "s")           # default REAL literal: single precision
        if k == "int":
            self.take()
            return Ex(v, "i")
        if k == "dot" and v in (".true.", ".false."):
            self.take()
            return Ex("True" if v == ".true." else "False", "l")
        if k == "str":
            self.take()
            return Ex(repr(v[1:-1]), "c")          # the literal's characters, as a Python string
        if v == "(/":
            self.take()
            items = []
            while self.peek()[1] != "/)":
                items.append(self.expr())
                if self.peek()[1] == ",":
                    self.take()
            self.take("/)")
            t = "i"
            for it in items:
                t = _num_type(t, it.typ) if it.typ in "irs" else it.typ
            dt = {"i": "np.int32", "r": "np.float64", "s": "np.float64", "l": "np.bool_"}[t]
            return Ex(f"np.array([{', '.join(it.code for it in items)}], dtype={dt})", t, True)
        if v == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return Ex(f"({e.code})", e.typ, e.arr)
        if k == "name":
            self.take()
            var, py = self.ctx.lookup(v)
            if self.peek()[1] == "(":
                if var is not None and var.dims:
                    return self.array_ref(var, py)
                return self.intrinsic(v)
            if var is None:
                raise SyntaxError(f"unknown name {v!r} in {self.src!r}")
            return Ex(py, var.typ, bool(var.dims))
        raise SyntaxError(f"unexpected {v!r} in {self.src!r}")

    def subscripts(self) -> List[object]:
        """Items of a parenthesised subscript list: Ex, or ('sec', lo, hi) for a triplet."""
        self.take("(")
        out: List[object] = []
        while True:
            if self.peek()[1] == ":":
                self.take()
                hi = None if self.peek()[1] in (",", ")") else self.expr()
                out.append(("sec", None, hi))
            else:
                e = self.expr()
                if self.peek()[1] == ":":
                    self.take()
                    hi = None if self.peek()[1] in (",", ")") else self.expr()
                    out.append(("sec", e, hi))
                else:
                    out.append(e)
            if self.peek()[1] == ",":
                self.take()
                continue
            self.take(")")
            return out

    def array_ref(self, var: Var, py: str) -> Ex:
        subs = self.subscripts()
        if len(subs) != var.rank:
            raise SyntaxError(f"rank mismatch for {var.name} in {self.src!r}")
        parts, arr = [], False
        for (lo, _hi), s in zip(var.dims, subs):
            off = _offset(lo)
            if isinstance(s, tuple):
                arr = True
                a = "" if s[1] is None else f"{s[1].code}{off}"
                b = "" if s[2] is None else f"{s[2].code}{off}+1"
                parts.append(f"{a}:{b}")
            else:
                parts.append(f"{s.code}{off}")
        return Ex(f"{py}[{', '.join(parts)}]", var.typ, arr)

    def args(self) -> List[Ex]:
        self.take("(")
        out = []
        if self.peek()[1] != ")":
            while True:
                out.append(self.expr())
                if self.peek()[1] == ",":
                    self.take()
                    continue
                break
        self.take(")")
        return out

    def intrinsic(self, name: str) -> Ex:
        a = self.args()
        c = [x.code for x in a]
        arr = any(x.arr for x in a)
        if name in ("dble", "dfloat"):
            return Ex(f"_dble({c[0]})", "r", arr)
        if name in ("real", "float", "sngl"):
            return Ex(f"_s(_dble({c[0]}))", "s", arr)
        if name == "int":
            return Ex(f"_int({c[0]})", "i", arr)
        if name == "nint":
            return Ex(f"_nint({c[0]})", "i", arr)
        if name == "floor":
            return Ex(f"_floor({c[0]})", "i", arr)
        if name in ("abs", "dabs", "iabs"):
            return Ex(f"np.abs({c[0]})" if arr else f"abs({c[0]})", a[0].typ, arr)
        if name in ("sqrt", "dsqrt", "acos", "dacos", "asin", "dasin", "atan", "datan", "sin", "dsin", "cos", "dcos",
                    "tan", "dtan", "tanh", "dtanh", "exp", "dexp", "log", "dlog"):
            base = name[1:] if name[0] == "d" and name not in ("dble",) else name
            if arr:
                raise SyntaxError(f"elemental {name} on an array is not supported: {self.src!r}")
            code = f"_m_{base}({c[0]})"
            return Ex(f"_s({code})" if a[0].typ == "s" else code, "s" if a[0].typ == "s" else "r")
        if name in ("atan2", "datan2"):
            return Ex(f"_m_atan2({c[0]}, {c[1]})", "r")
        if name in ("max", "min", "dmax1", "dmin1", "max0", "min0", "amax1", "amin1"):
            t = "i"
            for x in a:
                t = _num_type(t, x.typ)
            f = "max" if "max" in name else "min"
            conv = "float" if t in "rs" else "int"
            return Ex(f"_{f}({', '.join(f'{conv}({x})' for x in c)})", t)
        if name in ("mod", "dmod"):
            t = _num_type(a[0].typ, a[1].typ)
            return Ex(f"_imod({c[0]}, {c[1]})" if t == "i" else f"_rmod({c[0]}, {c[1]})", t)
        if name in ("sign", "dsign", "isign"):
            t = _num_type(a[0].typ, a[1].typ)
            return Ex(f"_sign({c[0]}, {c[1]})", t)
        if name == "sum":
            return Ex(f"_sum({c[0]})", a[0].typ)
        if name == "maxval":
            return Ex(f"_maxval({c[0]})", a[0].typ)
        if name == "minval":
            return Ex(f"_minval({c[0]})", a[0].typ)
        if name == "dot_product":
            return Ex(f"_dot({c[0]}, {c[1]})", _num_type(a[0].typ, a[1].typ))
        if name == "matmul":
            return Ex(f"_matmul({c[0]}, {c[1]})", _num_type(a[0].typ, a[1].typ), True)
        if name == "isnan":
            return Ex(f"np.isnan({c[0]})", "l", arr)
        if name == "size":
            return Ex(f"_size({', '.join(c)})", "i")
        raise SyntaxError(f"unsupported intrinsic {name!r} in {self.src!r}")


def _offset(lo: str) -> str:
    """Index offset for a lower bound; only integer literals are supported
    (a unit with another form is reported untranslated)."""
    lo = lo.strip()
    if lo == "0":
        return ""
    if re.fullmatch(r"-?\d+", lo):
        v = int(lo)
        return f"-{v}" if v > 0 else f"+{-v}"
    raise SyntaxError(f"lower bound {lo!r} is not an integer literal")


def parse_expr(s: str, ctx: Ctx) -> Ex:
    p = Parser(s, ctx)
    e = p.expr()
    if not p.done():
        raise SyntaxError(f"trailing tokens in {s!r}")
    return e


# ---- statements -------------------------------------------------------------------

_IO = re.compile(r"^(write|open|close|print|read|format|flush|rewind|inquire)\b")


def _paren_end(s: str, start: int) -> int:
    """Index just past the parenthesis that closes the one at s[start]."""
    depth = 0
    for i in range(start, len(s)):
        if s[i] == "(":
            depth += 1
        elif s[i] == ")":
            depth -= 1
            if depth == 0:
                return i + 1
    raise SyntaxError(f"unbalanced parentheses in {s!r}")


class Emitter:
    def __init__(self, units: Dict[str, Unit]):
        self.units = units
        self.modules = {n: u for n, u in units.items() if u.kind == "module"}
        self.out: List[str] = []
        self.outs: Dict[str, List[str]] = {}
        for n, u in units.items():
            if u.kind == "subroutine":
                self.outs[n] = self._scalar_outs(u)

    @staticmethod
    def _scalar_outs(u: Unit) -> List[str]:
        outs = []
        for a in u.args:
            v = u.vars.get(a)
            if v is None or v.dims:
                continue
            pat = re.compile(rf"^{a}\s*=[^=]|^do\s+{a}\s*=")
            if any(pat.match(s) for _, s in u.body):
                outs.append(a)
        return outs

    def w(self, ind: int, s: str) -> None:
        self.out.append("    " * ind + s)

    # -- one subroutine
    def subroutine(self, u: Unit) -> None:
        ctx = Ctx(u, self.modules)
        self.w(0, f"def {u.name}({', '.join(pyname(a) for a in u.args)}):")
        self.w(1, f"# Source1.f90:{u.line}")
        for name, v in u.vars.items():
            if name in u.args:
                continue
            self._init_var(1, v, ctx, pyname(name))
        self.stack: List[list] = [["sub", 0]]
        self.ctx, self.unit, self.ind = ctx, u, 1
        for n, s in u.data + u.body:          # DATA initialises before the first statement
            try:
                self.stmt(n, s)
            except SyntaxError as e:
                raise SyntaxError(f"Source1.f90:{n}: {e}") from None
        self._ret(1, u)
        self.w(0, "")

    def _ret(self, ind: int, u: Unit) -> None:
        outs = [pyname(o) for o in self.outs[u.name]]
        self.w(ind, f"return ({', '.join(outs)},)" if outs else "return")

    def _init_var(self, ind: int, v: Var, ctx: Ctx, target: str) -> None:
        if v.dims:
            shape = []
            for lo, hi in v.dims:
                if not hi:
                    raise SyntaxError(f"deferred shape of local {v.name}")
                shape.append(f"({parse_expr(hi, ctx).code}) - ({parse_expr(lo, ctx).code}) + 1")
            dt = {"i": "np.int32", "r": "np.float64", "s": "np.float64", "l": "np.bool_", "c": "object"}[v.typ]
            self.w(ind, f"{target} = np.zeros(({', '.join(shape)},), dtype={dt}, order='F')")
            if v.init:
                self.w(ind, f"{target}[...] = {parse_expr(v.init, ctx).code}")
        else:
            if v.init is not None:
                e = parse_expr(v.init, ctx)
                self.w(ind, f"{target} = {self._conv(v.typ, e)}")
            else:
                self.w(ind, f"{target} = {dict(i='0', r='0.0', s='0.0', l='False', c=repr(''))[v.typ]}")

    @staticmethod
    def _conv(typ: str, e: Ex) -> str:
        if typ == "i" and e.typ in "rs":
            return f"_int({e.code})"
        if typ == "r" and e.typ == "i":
            return f"float({e.code})"
        if typ == "s" and e.typ in "ir":
            return f"_s({e.code})"
        return e.code

    def open_block(self, kind: str) -> None:
        self.stack.append([kind, 0])
        self.ind += 1

    def close_block(self) -> None:
        kind, cnt = self.stack.pop()
        if cnt == 0:
            self.w(self.ind, "pass")
        self.ind -= 1

    def emit(self, s: str) -> None:
        self.stack[-1][1] += 1
        self.w(self.ind, s)

    def stmt(self, n: int, s: str) -> None:
        ctx = self.ctx
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", s)
        if m:
            var = m.group(1)
            bounds = split_top(m.group(2))
            a, b = parse_expr(bounds[0], ctx), parse_expr(bounds[1], ctx)
            _, py = ctx.lookup(var)
            if len(bounds) == 3:
                st = parse_expr(bounds[2], ctx)
                self.emit(f"for {py} in _drange({a.code}, {b.code}, {st.code}):")
            else:
                self.emit(f"for {py} in range({a.code}, {b.code} + 1):")
            self.open_block("do")
            return
        m = re.match(r"^do\s+while\s*(\(.*\))$", s)
        if m:
            self.emit(f"while {parse_expr(m.group(1), ctx).code}:")
            self.open_block("do")
            return
        if re.match(r"^end\s*do$", s):
            self.close_block()
            return
        if re.match(r"^if\s*\(", s):
            k = s.index("(")
            e = _paren_end(s, k)
            cond = parse_expr(s[k:e], ctx).code
            rest = s[e:].strip()
            if rest == "then":
                self.emit(f"if {cond}:")
                self.open_block("if")
            else:
                self.emit(f"if {cond}:")
                self.open_block("if1")
                self.stmt(n, rest)
                self.close_block()
            return
        m = re.match(r"^else\s*if\s*(\(.*)$", s)
        if m:
            t = m.group(1)
            e = _paren_end(t, 0)
            cond = parse_expr(t[:e], ctx).code
            self.close_block()
            self.emit(f"elif {cond}:")
            self.open_block("if")
            return
        if s == "else":
            self.close_block()
            self.emit("else:")
            self.open_block("if")
            return
        if re.match(r"^end\s*if$", s):
            self.close_block()
            return
        if s == "cycle":
            self.emit("continue")
            return
        if s == "exit":
            self.emit("break")
            return
        if s == "return":
            outs = [pyname(o) for o in self.outs[self.unit.name]]
            self.emit(f"return ({', '.join(outs)},)" if outs else "return")
            return
        if s == "continue":
            self.emit("pass")
            return
        if s == "stop" or s.startswith("stop "):
            self.emit("raise RuntimeError('STOP')")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", s)
        if m:
            for item in split_top(m.group(1)):
                mm = re.match(r"^(\w+)\s*\((.*)\)$", item)
                var, py = ctx.lookup(mm.group(1))
                var.dims = _parse_dims(mm.group(2))       # the bounds indexing uses from here on
                self._init_var(self.ind, var, ctx, py)
                self.stack[-1][1] += 1
            return
        m = re.match(r"^write\s*\(", s)
        if m:
            e = _paren_end(s, s.index("("))
            ctl = split_top(s[s.index("(") + 1:e - 1])
            items = split_top(s[e:].strip()) if s[e:].strip() else []
            try:
                codes = [parse_expr(it, ctx).code for it in items]
                unit = repr(ctl[0].strip()) if ctl else "'*'"
                # items that index outside their arrays (undefined in Fortran)
                # record None instead of values
                self.emit("try:")
                self.open_block("try")
                self.emit(f"_out({unit}, [{', '.join(codes)}])")
                self.close_block()
                self.emit("except IndexError:")
                self.open_block("except")
                self.emit(f"_out({unit}, None)")
                self.close_block()
            except SyntaxError:
                self.emit("pass  # write")
            return
        if _IO.match(s) or s.startswith("deallocate"):
            self.emit("pass  # " + s.split("(")[0])
            return
        m = re.match(r"^call\s+(\w+)\s*(\(.*\))?$", s)
        if m:
            self.call(m.group(1), m.group(2) or "()")
            return
        m = re.match(r"^data\s+(\w+)\s*/(.*)/$", s)
        if m:
            var, py = ctx.lookup(m.group(1))
            vals = [parse_expr(v, ctx).code for v in split_top(m.group(2))]
            self.emit(f"_data({py}, [{', '.join(vals)}])")
            return
        k = _top_eq(s)
        if k > 0:
            self.assign(s[:k].strip(), s[k + 1:].strip())
            return
        raise SyntaxError(f"unsupported statement {s!r}")

    def lhs(self, s: str) -> Tuple[Ex, Optional[Var]]:
        p = Parser(s, self.ctx)
        k, v = p.peek()
        var, py = self.ctx.lookup(v)
        if var is None:
            raise SyntaxError(f"assignment to undeclared {v!r}")
        e = p.primary()
        if not p.done():
            raise SyntaxError(f"bad assignment target {s!r}")
        if var.dims and "[" not in e.code:
            e = Ex(f"{py}[...]", var.typ, True)
        return e, var

    def assign(self, lhs: str, rhs: str) -> None:
        t, var = self.lhs(lhs)
        e = parse_expr(rhs, self.ctx)
        if t.arr or "[" in t.code:
            code = e.code
            if var.typ == "s" and e.typ in "ir":
                code = f"_s({code})"
            self.emit(f"{t.code} = {code}")
        else:
            self.emit(f"{t.code} = {self._conv(var.typ, e)}")

    def call(self, name: str, argstr: str) -> None:
        callee = self.units.get(name)
        if callee is None or callee.kind != "subroutine":
            raise SyntaxError(f"call of unknown subroutine {name!r}")
        acts = split_top(argstr.strip()[1:-1]) if argstr.strip() != "()" else []
        if len(acts) != len(callee.args):
            raise SyntaxError(f"{name}: {len(acts)} actual arguments for {len(callee.args)} dummies")
        codes = []
        for a, d in zip(acts, callee.args):
            dv = callee.vars.get(d)
            e = parse_expr(a, self.ctx)
            if dv is not None and dv.dims and not e.arr:
                raise SyntaxError(f"{name}: scalar {a!r} passed to array dummy {d}")
            codes.append(e.code)
        outs = self.outs[name]
        if not outs:
            self.emit(f"{name}({', '.join(codes)})")
            return
        self.emit(f"_r = {name}({', '.join(codes)})")
        for j, d in enumerate(outs):
            a = acts[callee.args.index(d)]
            t, var = self.lhs(a)
            self.emit(f"{t.code} = _r[{j}]")

    # -- the main program up to its time loop: parameters, the moment matrix
    # and its inverse, the velocity tables, the allocations and the initial
    # calls (tables, initia_center, set_walls, initialization, derivatives);
    # returns main's variables by name
    def main_setup(self, u: Unit) -> None:
        ctx = Ctx(u, self.modules)
        self.w(0, "def main_setup():")
        self.w(1, f"# Source1.f90:{u.line}")
        for name, v in u.vars.items():
            if v.dims and any(not hi for _, hi in v.dims):
                self.w(1, f"{pyname(name)} = None")
            else:
                self._init_var(1, v, ctx, pyname(name))
        self.stack = [["sub", 0]]
        self.ctx, self.unit, self.ind = ctx, u, 1
        self.outs.setdefault(u.name, [])
        for n, s in u.data + u.body:          # DATA initialises before the first statement
            if re.match(r"^do\s+t\s*=", s):
                break
            try:
                self.stmt(n, s)
            except SyntaxError as e:
                raise SyntaxError(f"Source1.f90:{n}: {e}") from None
        self.w(1, "return dict(locals())")
        self.w(0, "")

    # -- the module of constants
    def module(self, u: Unit) -> None:
        class _ModCtx(Ctx):
            def lookup(self_, name):
                if name in u.vars:
                    return u.vars[name], "C." + name
                return None, name
        ctx = _ModCtx(u, {})
        self.w(0, f"def init_{u.name}():")
        self.w(1, f"# Source1.f90:{u.line}")
        for name, v in u.vars.items():
            self._init_var(1, v, ctx, "C." + name)
        self.w(0, "")


PRELUDE = '''"""Generated by oracle/f90py.py from Source1.f90 -- do not edit, do not commit.
Test infrastructure only: the reference's subroutines as written, for pinning
the oracle."""
import builtins as _builtins
import keyword as _keyword
import math
import numpy as np

_RESERVED = set(_keyword.kwlist) | set(dir(_builtins)) | {"np", "math", "C"}


def pyname(name):
    """Python name of a Fortran variable of the source."""
    return name + "_v" if name in _RESERVED or name.startswith("_") else name


class C:
    """The module of constants (use const)."""


def _s(x):
    if isinstance(x, np.ndarray):
        return x.astype(np.float32).astype(np.float64)
    return float(np.float32(x))


def _dble(x):
    if isinstance(x, np.ndarray):
        return x.astype(np.float64)
    return float(x)


def _int(x):
    if isinstance(x, np.ndarray):
        return np.trunc(x).astype(np.int32)
    return int(x)


def _nint(x):
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _floor(x):
    return int(math.floor(x))


def _idiv(a, b):
    a, b = int(a), int(b)
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _imod(a, b):
    return int(a) - _idiv(a, b) * int(b)


def _rmod(a, b):
    return math.fmod(a, b)


def _sign(a, b):
    return abs(a) if b >= 0 else -abs(a)


def _powi(x, m):
    """x**m for an integer m: libgcc's __powidf2 (square and multiply)."""
    m = int(m)
    n = -m if m < 0 else m
    y = x if n % 2 else 1.0
    n >>= 1
    while n:
        x = x * x
        if n % 2:
            y = y * x
        n >>= 1
    return 1.0 / y if m < 0 else y


def _powr(x, y):
    try:
        return math.pow(x, y)
    except ValueError:
        return math.nan


def _max(*a):
    return max(a)


def _min(*a):
    return min(a)


def _seq(v):
    """Sum of a 1-D array added one element after the other (np.add.accumulate
    is sequential, so its last entry is that sum)."""
    return np.add.accumulate(v)[-1] if v.size else v.dtype.type(0)


def _sum(a):
    return _seq(np.asarray(a).ravel(order="F"))


def _maxval(a):
    return np.max(a)


def _minval(a):
    return np.min(a)


def _dot(a, b):
    return _seq(np.asarray(a).ravel(order="F") * np.asarray(b).ravel(order="F"))


def _matmul(A, v):
    """MATMUL of a matrix and a vector: each row's products added over
    ascending columns."""
    A = np.asarray(A, dtype=np.float64)
    return np.add.accumulate(A * np.asarray(v, dtype=np.float64)[None, :], axis=1)[:, -1]


OUT_LOG = []


def _out(unit, values):
    """A WRITE statement: its unit and the values of its output items."""
    OUT_LOG.append((unit, values))


def _data(a, vals):
    a[...] = np.array(vals, dtype=a.dtype).reshape(a.shape, order="F")


def _size(a, d=None):
    return a.size if d is None else a.shape[int(d) - 1]


def _drange(a, b, s):
    return range(a, b + (1 if s > 0 else -1), s)


def _m_sqrt(x):
    return math.sqrt(x) if x >= 0 else math.nan


def _m_acos(x):
    return math.acos(x) if -1.0 <= x <= 1.0 else math.nan


def _m_asin(x):
    return math.asin(x) if -1.0 <= x <= 1.0 else math.nan


def _m_log(x):
    return math.log(x) if x > 0 else (-math.inf if x == 0 else math.nan)


_m_atan, _m_sin, _m_cos, _m_tan, _m_tanh, _m_exp = math.atan, math.sin, math.cos, math.tan, math.tanh, math.exp
_m_atan2 = math.atan2

'''


def translate(text: str) -> str:
    units = parse_units(text)
    em = Emitter(units)
    em.out.append(PRELUDE)
    for u in units.values():
        if u.kind == "module":
            em.module(u)
    done, failed = [], {}
    for name, u in units.items():
        if u.kind != "subroutine":
            continue
        mark = len(em.out)
        try:
            em.subroutine(u)
            done.append(name)
        except SyntaxError as e:
            del em.out[mark:]
            failed[name] = str(e)
            em.w(0, f"def {name}(*args):")
            em.w(1, f"raise NotImplementedError({str(e)!r})")
            em.w(0, "")
    for u in units.values():
        if u.kind == "program":
            em.main_setup(u)
    em.w(0, f"TRANSLATED = {done!r}")
    em.w(0, f"UNTRANSLATED = {failed!r}")
    em.w(0, f"ARGS = {({n: u.args for n, u in units.items() if u.kind == 'subroutine'})!r}")
    em.w(0, f"SCALAR_OUTS = {em.outs!r}")
    # the calls of the time loop's body, in order, outside its IF blocks (the
    # periodic output): (subroutine, actual argument names, source line)
    calls = []
    for u in units.values():
        if u.kind != "program":
            continue
        depth, inloop = 0, False
        for n, s in u.body:
            if re.match(r"^do\s+t\s*=", s):
                inloop = True
                continue
            if not inloop:
                continue
            if re.match(r"^if\s*\(.*\)\s*then$", s):
                depth += 1
            elif re.match(r"^end\s*if$", s):
                depth -= 1
            elif re.match(r"^end\s*do$", s) and depth == 0:
                break
            m = re.match(r"^call\s+(\w+)\s*\((.*)\)$", s)
            if m and depth == 0:
                calls.append((m.group(1), [a.strip() for a in split_top(m.group(2))], n))
    em.w(0, f"MAIN_LOOP_CALLS = {calls!r}")
    for u in units.values():
        if u.kind == "module":
            em.w(0, f"init_{u.name}()")
    return "\n".join(em.out) + "\n"


# ---- building the translation for the tests ----------------------------------------

REFERENCE_SOURCE = "/root/reference/Source1.f90"
_HERE = __import__("os").path.dirname(__import__("os").path.abspath(__file__))
TRANSLATION = __import__("os").path.join(_HERE, "_ref", "source1_ref.py")


def load_reference(source: str = REFERENCE_SOURCE):
    """A fresh instance of the translated reference module (its own `C`
    namespace), translating the source into oracle/_ref/ first when the
    translation is missing or older than the source or this translator.
    None when the source is not on this machine."""
    import importlib.util
    import os
    if not os.path.exists(source):
        return None
    stale = not os.path.exists(TRANSLATION) or any(
        os.path.getmtime(TRANSLATION) < os.path.getmtime(f) for f in (source, __file__))
    if stale:
        os.makedirs(os.path.dirname(TRANSLATION), exist_ok=True)
        with open(source, encoding="latin-1") as f:
            code = translate(f.read())
        tmp = TRANSLATION + ".tmp"
        with open(tmp, "w") as f:
            f.write(code)
        os.replace(tmp, TRANSLATION)
    spec = importlib.util.spec_from_file_location("source1_ref", TRANSLATION)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(argv: List[str]) -> int:
    src, out = argv[1], argv[2]
    with open(src, encoding="latin-1") as f:
        text = f.read()
    code = translate(text)
    with open(out, "w") as f:
        f.write(code)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
