"""Python binding of libsymmetry_b200.so (the C ABI in include/symmetry.h).

The Fortran reference calls its subroutines directly (Source1.f90:215-252);
:class:`Lattice` exposes the same calls by the same names so a Python driver
reads like the reference's ``main``.  There is no CPU fallback: importing
this module on a machine without the built library raises, and every call
reports CUDA errors as :class:`SymError`.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import Dict, Optional

import numpy as np

from .params import (FIELD_ID, INT_FIELDS, POP_FIELDS, SYM_JOB_SLAB, SYM_JOB_THREAD, SymJobResult, SymJobSpec,
                     SymParams, SymParticles)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsymmetry_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "symmetry.h")

_lib = None


class SymError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def header_functions(path: str = HEADER):
    """Names of every function declared in include/symmetry.h."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(sym_[a-z0-9_]+)\s*\(",
                                 src, flags=re.M)))


def lib() -> ctypes.CDLL:
    """Load the library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                              "(make -C symmetry_b200/csrc)")
        L = ctypes.CDLL(LIB_PATH)
        H = ctypes.c_void_p
        L.sym_create.argtypes = [ctypes.POINTER(SymParams), ctypes.c_int, ctypes.POINTER(H)]
        L.sym_destroy.argtypes = [H]
        L.sym_last_error.restype = ctypes.c_char_p
        L.sym_last_error.argtypes = [H]
        L.sym_params_reference.argtypes = [ctypes.POINTER(SymParams), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sym_params_check.argtypes = [ctypes.POINTER(SymParams), ctypes.c_char_p, ctypes.c_size_t]
        L.sym_footprint.argtypes = [ctypes.POINTER(SymParams), ctypes.POINTER(ctypes.c_size_t)]
        L.sym_set_field.argtypes = [H, ctypes.c_int, ctypes.c_void_p]
        L.sym_get_field.argtypes = [H, ctypes.c_int, ctypes.c_void_p]
        L.sym_set_populations.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p]
        L.sym_get_macros.argtypes = [H] + [ctypes.c_void_p] * 5
        L.sym_energy.argtypes = [H, ctypes.c_void_p]
        L.sym_output_results.argtypes = [H, ctypes.c_char_p]
        L.sym_output_result2.argtypes = [H, ctypes.c_char_p, ctypes.c_int, ctypes.c_double]
        L.sym_output3_write.argtypes = [H, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double]
        L.sym_output4.argtypes = [H, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.POINTER(ctypes.c_double)]
        L.sym_checkpoint_save.argtypes = [H, ctypes.c_char_p]
        L.sym_checkpoint_load.argtypes = [H, ctypes.c_char_p]
        L.sym_set_particles.argtypes = [H, ctypes.POINTER(SymParticles)]
        L.sym_get_particles.argtypes = [H, ctypes.POINTER(SymParticles)]
        L.sym_get_lagrange.argtypes = [H] + [ctypes.c_void_p] * 9
        L.sym_init_phase.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p]
        L.sym_init_thread.argtypes = [H] + [ctypes.c_double] * 5 + [ctypes.c_uint64]
        L.sym_init_slab.argtypes = [H] + [ctypes.c_double] * 4 + [ctypes.c_uint64]
        for n in ["initia_center", "initialization", "set_walls", "calmacros", "derivatives", "collision",
                  "recolor", "boundary", "curve", "lagrange_points", "capillary_force2", "momentum",
                  "repulsive", "movement", "refilling"]:
            getattr(L, "sym_" + n).argtypes = [H]
        L.sym_streaming.argtypes = [H, ctypes.c_int]
        L.sym_step.argtypes = [H, ctypes.c_int]
        L.sym_step_timed.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.sym_output3.argtypes = [H, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)]
        L.sym_neck_radius.argtypes = [H, ctypes.POINTER(ctypes.c_double)]
        L.sym_mass_momentum.argtypes = [H, ctypes.c_void_p]
        L.sym_device_status.argtypes = [H, ctypes.POINTER(ctypes.c_int32)]
        L.sym_selftest_wait_timeout.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                                ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_size_t]
        L.sym_batch_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.sym_batch_destroy.argtypes = [ctypes.c_void_p]
        L.sym_batch_last_error.restype = ctypes.c_char_p
        L.sym_batch_last_error.argtypes = [ctypes.c_void_p]
        L.sym_batch_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.sym_batch_step_timed.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.sym_batch_set_xchunk.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.sym_batch_get_xchunk.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.sym_batch_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.sym_batch_set_ctas_per_sm.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.sym_batch_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]
        L.sym_batch_step_kernels.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.sym_batch_kernels_per_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        V = ctypes.c_void_p
        L.sym_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(V)]
        L.sym_server_destroy.argtypes = [V]
        L.sym_server_last_error.restype = ctypes.c_char_p
        L.sym_server_last_error.argtypes = [V]
        L.sym_server_submit.argtypes = [V, ctypes.POINTER(SymJobSpec), ctypes.POINTER(ctypes.c_int64)]
        L.sym_server_tick.argtypes = [V, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.sym_server_result.argtypes = [V, ctypes.c_int64, ctypes.POINTER(SymJobResult)]
        L.sym_server_set_xchunk.argtypes = [V, ctypes.c_int, ctypes.c_int]
        L.sym_server_stats.argtypes = [V, ctypes.c_void_p]
        L.sym_mass_momentum_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
        _lib = L
    return _lib


def params_check(p: SymParams) -> Optional[str]:
    buf = ctypes.create_string_buffer(256)
    rc = lib().sym_params_check(ctypes.byref(p), buf, 256)
    return None if rc == 0 else buf.value.decode()


DEV_NONFINITE = 1   # sym_device_status flags (include/symmetry.h)
DEV_TIMEOUT = 2


def selftest_wait_timeout(polls: int, device: int = 0):
    """Run the timeout path of the fused kernels' bounded mbarrier wait:
    returns (flags, ms) -- the flags a timed-out tile load records and the
    event-timed duration of the launch."""
    st, ms = ctypes.c_int32(), ctypes.c_double()
    buf = ctypes.create_string_buffer(256)
    rc = lib().sym_selftest_wait_timeout(device, polls, ctypes.byref(st), ctypes.byref(ms), buf, 256)
    if rc:
        raise SymError(rc, "selftest_wait_timeout: " + buf.value.decode())
    return st.value, ms.value


def footprint(p: SymParams) -> int:
    n = ctypes.c_size_t()
    rc = lib().sym_footprint(ctypes.byref(p), ctypes.byref(n))
    if rc:
        raise SymError(rc, "footprint")
    return n.value


class Lattice:
    """One device-resident domain (a sym_handle)."""

    def __init__(self, params: SymParams, device: int = 0):
        self.p = params.copy()
        self.h = ctypes.c_void_p()
        rc = lib().sym_create(ctypes.byref(self.p), device, ctypes.byref(self.h))
        if rc:
            raise SymError(rc, "sym_create failed: " + (params_check(self.p) or "see stderr"))
        self.shape = (params.nx, params.ny, params.nz)

    def close(self):
        if self.h:
            lib().sym_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str):
        if rc:
            raise SymError(rc, f"{what}: {lib().sym_last_error(self.h).decode()}")

    # ---- state transfer --------------------------------------------------
    def set(self, name: str, arr: np.ndarray):
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        want = self.p.n_nodes * (19 if name in POP_FIELDS else 1)
        if a.size != want:
            raise ValueError(f"{name}: expected {want} elements, got {a.size}")
        self._ck(lib().sym_set_field(self.h, FIELD_ID[name], a.ctypes.data), f"set {name}")

    def get(self, name: str) -> np.ndarray:
        dt = np.int32 if name in INT_FIELDS else np.float64
        shape = self.shape + ((19,) if name in POP_FIELDS else ())
        out = np.empty(shape, dtype=dt)
        self._ck(lib().sym_get_field(self.h, FIELD_ID[name], out.ctypes.data), f"get {name}")
        return out

    def macros(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """rho, ux, uy, uz, rho_N of the current populations (calmacros),
        without changing the stepping state; `out` may supply the host arrays
        (contiguous float64 of the domain's size, e.g. pinned)."""
        names = ("rho", "ux", "uy", "uz", "rho_N")
        if out is None:
            out = {k: np.empty(self.shape, dtype=np.float64) for k in names}
        for k in names:
            a = out[k]
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != self.p.n_nodes:
                raise ValueError(f"{k}: contiguous float64 array of {self.p.n_nodes} values expected")
        self._ck(lib().sym_get_macros(self.h, *(out[k].ctypes.data for k in names)), "get_macros")
        return out

    def energy(self) -> np.ndarray:
        """output4's sums before normalisation (see sym_energy)."""
        out = np.zeros(6)
        self._ck(lib().sym_energy(self.h, out.ctypes.data), "energy")
        return out

    def output_results(self, path: str):
        self._ck(lib().sym_output_results(self.h, os.fsencode(path)), "output_results")

    def output_result2(self, prefix: str, t: int, tr: float):
        self._ck(lib().sym_output_result2(self.h, os.fsencode(prefix), t, tr), "output_result2")

    def output3_write(self, path: str, t: int, tr: float, rad_c: float, lamda_d: float):
        self._ck(lib().sym_output3_write(self.h, os.fsencode(path), t, tr, rad_c, lamda_d), "output3")

    def output4(self, path: str, t: int, tr: float, rad_c: float, wcap: float) -> float:
        """Append the Energy.dat record; returns the accumulated capillary work."""
        w = ctypes.c_double(wcap)
        self._ck(lib().sym_output4(self.h, os.fsencode(path), t, tr, rad_c, ctypes.byref(w)), "output4")
        return w.value

    def save(self, path: str):
        """Checkpoint the complete stepping state to `path`."""
        self._ck(lib().sym_checkpoint_save(self.h, os.fsencode(path)), "checkpoint save")

    def load(self, path: str):
        """Restore a checkpoint written by a handle with the same parameters."""
        self._ck(lib().sym_checkpoint_load(self.h, os.fsencode(path)), "checkpoint load")

    def set_populations(self, ri: np.ndarray, bi: np.ndarray):
        """Both colours from host arrays (pinned memory gives full PCIe rate)."""
        for a in (ri, bi):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != 19 * self.p.n_nodes:
                raise ValueError("populations must be contiguous float64 (nx,ny,nz,19)")
        self._ck(lib().sym_set_populations(self.h, ri.ctypes.data, bi.ctypes.data), "set_populations")

    def get_into(self, name: str, out: np.ndarray):
        """Download a field into a preallocated (e.g. pinned) host array."""
        self._ck(lib().sym_get_field(self.h, FIELD_ID[name], out.ctypes.data), f"get {name}")

    def set_particles(self, s: SymParticles):
        self._ck(lib().sym_set_particles(self.h, ctypes.byref(s)), "set_particles")

    def particles(self) -> SymParticles:
        s = SymParticles()
        self._ck(lib().sym_get_particles(self.h, ctypes.byref(s)), "get_particles")
        return s

    def lagrange(self) -> Dict[str, np.ndarray]:
        n = self.la_num * self.p.par
        names = ["Lax", "Lay", "Laz", "La_rhoN", "La_nx", "La_ny", "La_nz", "La_flag", "ds"]
        out = {k: np.zeros(n, dtype=np.int32 if k == "La_flag" else np.float64) for k in names}
        self._ck(lib().sym_get_lagrange(self.h, *[out[k].ctypes.data for k in names]), "get_lagrange")
        return out

    @property
    def la_num(self) -> int:
        if self.p.par == 0:
            return 0
        import math
        lam = self.p.la_m or int(2.0 * math.pi / self.p.alpha)
        lan = self.p.la_n or int(math.pi / self.p.alpha)
        return lam * (lan + 1)

    # ---- initial state -----------------------------------------------------
    def initia_center(self):
        self._ck(lib().sym_initia_center(self.h), "initia_center")

    def initialization(self):
        self._ck(lib().sym_initialization(self.h), "initialization")

    def init_phase(self, phi: np.ndarray, rho: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        self._ck(lib().sym_init_phase(self.h, phi.ctypes.data, rho.ctypes.data), "init_phase")

    def init_thread(self, radius, amp, wavelength, width=2.0, noise=1e-4, seed=0):
        self._ck(lib().sym_init_thread(self.h, radius, amp, wavelength, width, noise, seed), "init_thread")

    def init_slab(self, z0, z1, width=2.0, noise=1e-4, seed=0):
        self._ck(lib().sym_init_slab(self.h, z0, z1, width, noise, seed), "init_slab")

    # ---- the reference's subroutines -------------------------------------------
    def call(self, name: str):
        self._ck(getattr(lib(), "sym_" + name)(self.h), name)

    def streaming(self, which: int):
        self._ck(lib().sym_streaming(self.h, which), "streaming")

    def step(self, n: int = 1):
        self._ck(lib().sym_step(self.h, n), "step")

    def step_timed(self, n: int, use_graph: bool = False) -> np.ndarray:
        """Run n steps with CUDA events on the library stream; returns ms
        [total, phase kernel, particle+pin work, collide kernel] (-1 = not timed)."""
        ms = np.zeros(4)
        self._ck(lib().sym_step_timed(self.h, n, 1 if use_graph else 0, ms.ctypes.data), "step_timed")
        return ms

    # ---- diagnostics -------------------------------------------------------------
    def output3(self):
        h, y = ctypes.c_double(), ctypes.c_int32()
        self._ck(lib().sym_output3(self.h, ctypes.byref(h), ctypes.byref(y)), "output3")
        return h.value, y.value

    def neck_radius(self) -> float:
        r = ctypes.c_double()
        self._ck(lib().sym_neck_radius(self.h, ctypes.byref(r)), "neck_radius")
        return r.value

    def mass_momentum(self) -> np.ndarray:
        out = np.zeros(5)
        self._ck(lib().sym_mass_momentum(self.h, out.ctypes.data), "mass_momentum")
        return out

    def device_status(self) -> int:
        """Error flags the fused kernels recorded (DEV_NONFINITE | DEV_TIMEOUT)."""
        v = ctypes.c_int32()
        self._ck(lib().sym_device_status(self.h, ctypes.byref(v)), "device_status")
        return v.value


class Batch:
    """Many Lattice domains stepped together (sym_batch_*)."""

    def __init__(self, lattices):
        self.members = list(lattices)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        self.b = ctypes.c_void_p()
        rc = lib().sym_batch_create(arr, len(self.members), ctypes.byref(self.b))
        if rc:
            raise SymError(rc, "sym_batch_create: members must share device, CONFIG mode and storage")

    def _ck(self, rc, what):
        if rc:
            raise SymError(rc, f"{what}: {lib().sym_batch_last_error(self.b).decode()}")

    def step(self, n: int = 1):
        self._ck(lib().sym_batch_step(self.b, n), "batch step")

    def step_timed(self, n: int) -> float:
        ms = ctypes.c_double()
        self._ck(lib().sym_batch_step_timed(self.b, n, ctypes.byref(ms)), "batch step_timed")
        return ms.value

    def set_xchunk(self, i: int, x: int):
        self._ck(lib().sym_batch_set_xchunk(self.b, i, x), "set_xchunk")

    def set_ctas_per_sm(self, c: int):
        self._ck(lib().sym_batch_set_ctas_per_sm(self.b, c), "set_ctas_per_sm")

    def xchunk(self, i: int) -> int:
        v = ctypes.c_int()
        self._ck(lib().sym_batch_get_xchunk(self.b, i, ctypes.byref(v)), "get_xchunk")
        return v.value

    def autotune(self, trial_steps: int = 5) -> int:
        taken = ctypes.c_int()
        self._ck(lib().sym_batch_autotune(self.b, trial_steps, ctypes.byref(taken)), "autotune")
        return taken.value

    def step_kernels(self, n: int) -> np.ndarray:
        """n eager steps with CUDA events: ms [total, phase, particle/wall chains, collide]."""
        ms = np.zeros(4)
        self._ck(lib().sym_batch_step_kernels(self.b, n, ms.ctypes.data), "batch step_kernels")
        return ms

    def kernels_per_step(self) -> int:
        k = ctypes.c_int()
        self._ck(lib().sym_batch_kernels_per_step(self.b, ctypes.byref(k)), "kernels_per_step")
        return k.value

    def info(self):
        n, t, g = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int()
        self._ck(lib().sym_batch_info(self.b, ctypes.byref(n), ctypes.byref(t), ctypes.byref(g)), "info")
        return dict(nodes=n.value, tiles=t.value, grid=g.value)

    def close(self):
        if self.b:
            lib().sym_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def job_spec(w, max_steps: int, stop_radius: float = 1.0, t_arrival: float = -1.0, drift_tol: float = 0.0,
             wall_budget_s: float = 0.0) -> SymJobSpec:
    """The sym_job_spec of a workload (same initial state as setup_workload)."""
    js = SymJobSpec()
    js.p = w.params.copy()
    g = w.gen
    if w.kind == "thread":
        js.kind = SYM_JOB_THREAD
        vals = [g["radius"], g["amp"], g["wavelength"], g.get("width", 2.0), g.get("noise", 1e-4)]
    else:
        js.kind = SYM_JOB_SLAB
        vals = [g["z0"], g["z1"], g.get("width", 2.0), g.get("noise", 1e-4), 0.0]
    for k, v in enumerate(vals):
        js.gen[k] = float(v)
    js.seed = int(g.get("seed", 0))
    js.max_steps = int(max_steps)
    js.stop_radius = float(stop_radius)
    if w.params.par:
        q = w.particles[0]
        for k in range(3):
            js.center[k] = float(q["center"][k])
            js.up[k] = float(q.get("up", [0.0, 0.0, 0.0])[k])
    js.t_arrival = float(t_arrival)
    js.drift_tol = float(drift_tol)
    js.wall_budget_s = float(wall_budget_s)
    return js


class Server:
    """Continuous-batching job server (sym_server_*)."""

    def __init__(self, device: int = 0, budget_bytes: int = 160 * 10**9, slots: int = 256, check_every: int = 10):
        self.s = ctypes.c_void_p()
        rc = lib().sym_server_create(device, int(budget_bytes), int(slots), int(check_every), ctypes.byref(self.s))
        if rc:
            raise SymError(rc, "sym_server_create")

    def _ck(self, rc, what):
        if rc:
            raise SymError(rc, f"{what}: {lib().sym_server_last_error(self.s).decode()}")

    def submit(self, spec: SymJobSpec) -> int:
        i = ctypes.c_int64()
        self._ck(lib().sym_server_submit(self.s, ctypes.byref(spec), ctypes.byref(i)), "submit")
        return i.value

    def tick(self, max_steps: int = 0):
        r, p = ctypes.c_int(), ctypes.c_int()
        self._ck(lib().sym_server_tick(self.s, int(max_steps), ctypes.byref(r), ctypes.byref(p)), "tick")
        return r.value, p.value

    def result(self, job_id: int) -> SymJobResult:
        out = SymJobResult()
        self._ck(lib().sym_server_result(self.s, int(job_id), ctypes.byref(out)), "result")
        return out

    def set_xchunk(self, size_class: int, x: int):
        self._ck(lib().sym_server_set_xchunk(self.s, size_class, x), "set_xchunk")

    def stats(self):
        out = np.zeros(8)
        self._ck(lib().sym_server_stats(self.s, out.ctypes.data), "stats")
        keys = ["node_updates", "device_ms", "done", "failed", "running", "pending", "resident_bytes", "clock_s"]
        return dict(zip(keys, out.tolist()))

    def run_until_idle(self, max_steps: int = 0):
        while True:
            r, p = self.tick(max_steps)
            if r == 0 and p == 0:
                return

    def close(self):
        if self.s:
            lib().sym_server_destroy(self.s)
            self.s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_workload(w, device: int = 0) -> Lattice:
    """A Lattice initialised like main (Source1.f90:208-214) for a CONFIG workload,
    with the phase field generated on the device."""
    from .params import particles_set
    L = Lattice(w.params, device)
    if w.params.par:
        s = SymParticles()
        particles_set(s, "center", w.params.par, [q["center"] for q in w.particles])
        particles_set(s, "center0", w.params.par, [q["center"] for q in w.particles])
        particles_set(s, "up", w.params.par, [q.get("up", [0, 0, 0]) for q in w.particles])
        L.set_particles(s)
    L.call("set_walls")
    g = w.gen
    if w.kind == "thread":
        L.init_thread(g["radius"], g["amp"], g["wavelength"], g.get("width", 2.0), g.get("noise", 1e-4),
                      g.get("seed", 0))
    else:
        L.init_slab(g["z0"], g["z1"], g.get("width", 2.0), g.get("noise", 1e-4), g.get("seed", 0))
    L.call("derivatives")
    return L
