"""ctypes wrapper of the CPU oracle (liborc.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm may import this module, and only as the checker or the timed CPU
baseline.  The oracle restates Source1.f90 (see sym_oracle.cpp); with no
Fortran compiler here, it is pinned bit for bit against the reference's own
source run through a mechanical translation (oracle/f90py.py,
tests/test_reference_pin.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from symmetry_b200.params import SymParams, SymParticles, POP_FIELDS

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(SymParams)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_array.restype = ctypes.c_void_p
        L.orc_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_int32)]
        L.orc_particles.restype = ctypes.POINTER(SymParticles)
        L.orc_particles.argtypes = [ctypes.c_void_p]
        L.orc_matrices.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_la_num.restype = ctypes.c_int
        L.orc_la_num.argtypes = [ctypes.c_void_p]
        for n in ["set_walls", "calmacros", "derivatives", "collision", "recolor", "boundary",
                  "curve", "lagrange_points", "capillary_force2", "momentum", "repulsive",
                  "movement", "refilling", "initialization", "initia_center"]:
            getattr(L, "orc_" + n).argtypes = [ctypes.c_void_p]
        L.orc_streaming.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_init_phase.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_output3.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_int32)]
        L.orc_neck_radius.restype = ctypes.c_double
        L.orc_neck_radius.argtypes = [ctypes.c_void_p]
        L.orc_energy.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_threads.restype = ctypes.c_int
        _lib = L
    return _lib


class Oracle:
    SUBROUTINES = ["set_walls", "calmacros", "derivatives", "collision", "recolor", "boundary",
                   "curve", "lagrange_points", "capillary_force2", "momentum", "repulsive",
                   "movement", "refilling", "initialization", "initia_center"]

    def __init__(self, params: SymParams):
        self.p = params.copy()
        self.h = lib().orc_create(ctypes.byref(self.p))
        self.shape = (params.nx, params.ny, params.nz)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def arr(self, name: str) -> np.ndarray:
        """Live numpy view of an oracle array (Fortran layout)."""
        cnt, isint = ctypes.c_int64(), ctypes.c_int32()
        ptr = lib().orc_array(self.h, name.encode(), ctypes.byref(cnt), ctypes.byref(isint))
        if not ptr:
            raise KeyError(name)
        ct = ctypes.c_int32 if isint.value else ctypes.c_double
        a = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(cnt.value,))
        if name in POP_FIELDS:
            return a.reshape(self.shape + (19,))
        if cnt.value == self.p.n_nodes:
            return a.reshape(self.shape)
        return a

    @property
    def particles(self) -> SymParticles:
        return lib().orc_particles(self.h).contents

    def matrices(self):
        M = np.zeros((19, 19)); Mi = np.zeros((19, 19))
        lib().orc_matrices(self.h, M.ctypes.data, Mi.ctypes.data)
        return M, Mi

    @property
    def la_num(self) -> int:
        return lib().orc_la_num(self.h)

    def call(self, name: str, *args):
        getattr(lib(), "orc_" + name)(self.h, *args)

    def streaming(self, which: int):
        lib().orc_streaming(self.h, which)

    def step(self, n: int = 1):
        lib().orc_step(self.h, n)

    def init_phase(self, phi: np.ndarray, rho: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        lib().orc_init_phase(self.h, phi.ctypes.data, rho.ctypes.data)

    def output3(self):
        h, y = ctypes.c_double(), ctypes.c_int32()
        lib().orc_output3(self.h, ctypes.byref(h), ctypes.byref(y))
        return h.value, y.value

    def neck_radius(self) -> float:
        return lib().orc_neck_radius(self.h)

    def energy(self) -> np.ndarray:
        """output4's field sums on the arrays of the last calmacros."""
        out = np.zeros(3)
        lib().orc_energy(self.h, out.ctypes.data)
        return out


def threads() -> int:
    return lib().orc_threads()


def setup_workload(w) -> Oracle:
    """Oracle initialised like main (Source1.f90:208-214) for a CONFIG workload."""
    from symmetry_b200.params import particles_set
    o = Oracle(w.params)
    if w.params.par:
        s = o.particles
        particles_set(s, "center", w.params.par, [q["center"] for q in w.particles])
        particles_set(s, "center0", w.params.par, [q["center"] for q in w.particles])
        particles_set(s, "up", w.params.par, [q.get("up", [0, 0, 0]) for q in w.particles])
    o.call("set_walls")
    phi, rho = w.phase()
    o.init_phase(phi, rho)
    o.call("derivatives")
    return o


def setup_reference(params: SymParams) -> Oracle:
    """Oracle initialised exactly like main (Source1.f90:208-214), REFERENCE mode."""
    o = Oracle(params)
    o.call("initia_center")
    o.call("set_walls")
    o.call("initialization")
    o.call("derivatives")
    return o
