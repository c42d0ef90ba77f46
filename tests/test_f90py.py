"""The Fortran-to-Python translator that pins the oracle (oracle/f90py.py),
on small Fortran programs written here: each construct the reference's
source uses, with the semantics the translation fixes (integer division,
MOD, integer powers, default-REAL literals, array bounds and sections,
array constructors, MATMUL and SUM order, scalar arguments by reference,
WRITE capture).  Needs no reference source."""
import importlib.util
import math
import sys
import types

import numpy as np
import pytest

from oracle import f90py

SRC = """
  module const
implicit none
integer, parameter:: n=4
double precision, dimension(0:3):: w
real*8, parameter:: PI=4.0d0*datan(1.0d0)
integer:: k_mod
end module const

program main
use const
implicit none
integer i
double precision, dimension(0:3,0:3):: a
double precision:: v(0:3), r(0:3), s
data a /1,2,3,4, 5,6,7,8, 9,10,11,12, 13,14,15,16/
w(0) = 1.0d0/3.0d0
w(1:3) = 0.25d0
v = (/1.0d0, 2.0d0, 3.0d0, 4.0d0/)
r = MATMUL(a, v)
s = sum(r*w)
call scale(v, s, 2)
k_mod = mod(-7, 3)
write(*,*) s, k_mod
do i = 1, 10
end do
end program main

subroutine scale(x, total, m)
use const
implicit none
double precision :: x(0:3), total
integer :: m, j
do j = 0, 3
    x(j) = x(j)*m
end do
total = total + x(3)
return
end subroutine scale

subroutine arith(out, iout)
use const
implicit none
double precision :: out(8)
integer :: iout(6)
double precision :: t
integer :: p, q
p = -7
q = 2
iout(1) = p/q
iout(2) = mod(p, q)
iout(3) = 7/(-2)
iout(4) = int(-2.7d0)
iout(5) = nint(-2.5d0)
iout(6) = 2**5
t = 1.1d0
out(1) = t**3
out(2) = t**(-2)
out(3) = 0.1
out(4) = 0.1d0
out(5) = real(7)/3.0
out(6) = dble(7)/3.0d0
out(7) = -t**2
if (t > 1.0d0 .and. .not. (p >= 0)) then
    out(8) = 1.0d0
elseif (t < 0.0d0) then
    out(8) = 2.0d0
else
    out(8) = 3.0d0
endif
return
end subroutine arith

subroutine bounds(f, col)
use const
implicit none
double precision :: f(0:2, 3, 2)
double precision :: col(0:2)
integer :: y, z
do z = 1, 2
  do y = 1, 3
    f(:, y, z) = dble(y) + 10.0d0*dble(z)
    if (y == 2) cycle
    f(0, y, z) = -1.0d0
  end do
end do
f(:, 3, :) = f(:, 1, :)
col = f(:, 2, 2)
return
end subroutine bounds
"""


@pytest.fixture(scope="module")
def R():
    code = f90py.translate(SRC)
    mod = types.ModuleType("f90py_case")
    exec(compile(code, "f90py_case", "exec"), mod.__dict__)
    return mod


def test_everything_translates(R):
    assert set(R.TRANSLATED) == {"scale", "arith", "bounds"}
    assert R.UNTRANSLATED == {}
    assert R.SCALAR_OUTS["scale"] == ["total"]


def test_main_setup_data_matmul_sum_and_by_reference_scalars(R):
    V = R.main_setup()
    a = np.arange(1, 17, dtype=float).reshape((4, 4), order="F")     # DATA fills in element order
    assert np.array_equal(V["a"], a)
    v0 = np.array([1.0, 2.0, 3.0, 4.0])
    r = np.zeros(4)
    for i in range(4):                 # MATMUL: each row over ascending columns
        acc = 0.0
        for j in range(4):
            acc = acc + a[i, j] * v0[j]
        r[i] = acc
    assert np.array_equal(V["r"], r)
    w = np.array([1.0 / 3.0, 0.25, 0.25, 0.25])
    s = 0.0
    for i in range(4):                 # SUM in element order
        s = s + r[i] * w[i]
    # scale doubled v and added v(3) to s through its scalar argument
    assert np.array_equal(V["v"], 2 * v0)
    assert V["s"] == s + 8.0
    assert R.C.k_mod == -1             # MOD takes the sign of its first argument
    assert R.OUT_LOG[-1] == ("*", [s + 8.0, -1])
    assert R.C.pi == 4.0 * math.atan(1.0)


def test_integer_and_real_arithmetic(R):
    out = np.zeros(8)
    iout = np.zeros(6, dtype=np.int32)
    R.arith(out, iout)
    assert list(iout) == [-3, -1, -3, -2, -3, 32]    # truncating division, MOD, INT, NINT, **
    t = 1.1
    assert out[0] == (t * t) * t                      # x**3 by multiplication, not pow()
    assert out[1] == 1.0 / (t * t)
    assert out[2] == float(np.float32(0.1))           # a default-REAL literal is single precision
    assert out[3] == 0.1
    assert out[4] == float(np.float32(np.float32(7.0) / np.float32(3.0)))
    assert out[5] == 7.0 / 3.0
    assert out[6] == -(t * t)                         # -t**2 is -(t**2)
    assert out[7] == 1.0


def test_lower_bounds_sections_and_cycle(R):
    f = np.zeros((3, 3, 2), order="F")
    col = np.zeros(3)
    R.bounds(f, col)
    for z in (1, 2):
        for y in (1, 2, 3):
            yy = 1 if y == 3 else y                   # plane 3 copied from plane 1
            want = [yy + 10.0 * z] * 3
            if yy != 2:
                want[0] = -1.0
            assert list(f[:, y - 1, z - 1]) == want
    assert list(col) == [22.0, 22.0, 22.0]


def test_python_names_do_not_shadow_builtins():
    code = f90py.translate("""
subroutine r(range, x)
implicit none
double precision :: range, x(2)
integer :: i
do i = 1, 2
  x(i) = range*i
end do
range = 0.0d0
return
end subroutine r
""")
    mod = types.ModuleType("f90py_names")
    exec(compile(code, "f90py_names", "exec"), mod.__dict__)
    x = np.zeros(2)
    assert mod.r(1.5, x) == (0.0,)
    assert list(x) == [1.5, 3.0]


def test_unsupported_constructs_are_reported_not_guessed():
    code = f90py.translate("""
subroutine odd(x)
implicit none
double precision :: x(2)
x = cshift(x, 1)
return
end subroutine odd
""")
    mod = types.ModuleType("f90py_odd")
    exec(compile(code, "f90py_odd", "exec"), mod.__dict__)
    assert "odd" in mod.UNTRANSLATED
    with pytest.raises(NotImplementedError):
        mod.odd(np.zeros(2))
