"""ctypes mirrors of the C ABI structs in include/symmetry.h and the
parameter sets of the reference and of the config workloads.

The reference (Source1.f90) fixes its constants at compile time
(Source1.f90:7-26) and by assignments in ``main`` (Source1.f90:57-103);
:func:`reference_params` reproduces those values for a runtime domain size.
"""
from __future__ import annotations

import ctypes
import math

SYM_MODE_REFERENCE = 0
SYM_MODE_CONFIG = 1
SYM_STORE_FP64 = 0
SYM_STORE_FP32 = 1
SYM_STORE_FP16 = 2
SYM_MAX_PAR = 32

STORAGE_NAMES = {"fp64": SYM_STORE_FP64, "fp32": SYM_STORE_FP32, "fp16": SYM_STORE_FP16}

# field ids (enum in symmetry.h)
FIELDS = [
    "ri", "bi", "fi", "ffi",
    "rho", "ux", "uy", "uz",
    "rho_N", "rho_R", "rho_B",
    "n_x", "n_y", "n_z", "gradx", "grady", "gradz",
    "flag",
    "walls", "walls_old", "walls_all", "pin", "pout",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
POP_FIELDS = {"ri", "bi", "fi", "ffi"}
INT_FIELDS = {"flag", "walls", "walls_old", "walls_all", "pin", "pout"}


class SymParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("mode", ctypes.c_int32), ("wall_x", ctypes.c_int32), ("storage", ctypes.c_int32),
        ("par", ctypes.c_int32), ("la_m", ctypes.c_int32), ("la_n", ctypes.c_int32),
        ("bounce", ctypes.c_int32),
        ("rho0", ctypes.c_double), ("nu_r", ctypes.c_double), ("nu_b", ctypes.c_double),
        ("s_e", ctypes.c_double), ("s_eps", ctypes.c_double), ("s_q", ctypes.c_double),
        ("s_pi", ctypes.c_double), ("s_m", ctypes.c_double),
        ("sigma", ctypes.c_double), ("beta", ctypes.c_double), ("cita", ctypes.c_double),
        ("body", ctypes.c_double * 3),
        ("rad", ctypes.c_double), ("rho_p", ctypes.c_double), ("mass", ctypes.c_double),
        ("inertia", ctypes.c_double), ("fg", ctypes.c_double), ("alpha", ctypes.c_double),
        ("evap_lim", ctypes.c_double),
    ]

    def copy(self) -> "SymParams":
        c = SymParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(SymParams))
        return c

    @property
    def n_nodes(self) -> int:
        return int(self.nx) * int(self.ny) * int(self.nz)


V3 = ctypes.c_double * (3 * SYM_MAX_PAR)


class SymParticles(ctypes.Structure):
    _fields_ = [
        ("center", V3), ("center_old", V3), ("center0", V3), ("up", V3), ("rp", V3),
        ("fp", V3), ("tp", V3), ("fre", V3), ("tension", V3), ("tension_t", V3),
        ("shb", ctypes.c_double * SYM_MAX_PAR),
    ]


def particles_get(s: SymParticles, name: str, par: int):
    """Return a (par, 3) nested list view of one (par,3) column-major array."""
    a = getattr(s, name)
    return [[a[k * par + p] for k in range(3)] for p in range(par)]


def particles_set(s: SymParticles, name: str, par: int, values) -> None:
    a = getattr(s, name)
    for p in range(par):
        for k in range(3):
            a[k * par + p] = float(values[p][k])


def reference_params(nx: int = 152, ny: int = 152, nz: int = 152, par: int = 12) -> SymParams:
    """The reference's built-in constants (Source1.f90:9-26, 57-103)."""
    p = SymParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.mode = SYM_MODE_REFERENCE
    p.par = par
    oh, lamda, rad_c = 0.1, 10.0, 30.0
    sigma, rho0 = 0.05, 0.05
    nu_r = oh / math.sqrt(rho0 / (rad_c * sigma))
    p.rho0 = rho0
    p.nu_r, p.nu_b = nu_r, nu_r / lamda
    p.s_e = p.s_eps = p.s_q = p.s_pi = p.s_m = 0.0
    p.sigma, p.beta = sigma, 0.7
    p.cita = 90.0 / 180.0 * math.pi
    p.rad = 7.5
    p.rho_p = 1.0 * rho0
    p.mass = 4.0 / 3.0 * p.rho_p * math.pi * (p.rad * p.rad * p.rad)
    p.inertia = 2.0 / 5.0 * p.mass * (p.rad * p.rad)
    p.fg = -math.pi * 2.0 * p.rad * sigma
    p.alpha = 2.0 / 180.0 * math.pi
    p.evap_lim = 1.0e-8
    return p


def config_params(nx, ny, nz, *, tau_r=1.0, tau_b=None, sigma=5e-3, beta=0.7, rho0=1.0,
                  s_e=0.0, s_eps=0.0, s_q=0.0, s_pi=0.0, s_m=0.0, wall_x=False,
                  cita_deg=90.0, par=0, rad=0.0, rho_p_ratio=1.0, body=(0.0, 0.0, 0.0),
                  storage="fp64", alpha_deg=2.0) -> SymParams:
    """A CONFIG-mode parameter set: periodic box, optional x wall planes."""
    tau_b = tau_r if tau_b is None else tau_b
    p = SymParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.mode = SYM_MODE_CONFIG
    p.wall_x = 1 if wall_x else 0
    p.storage = STORAGE_NAMES[storage] if isinstance(storage, str) else int(storage)
    p.par = par
    p.rho0 = rho0
    p.nu_r, p.nu_b = (tau_r - 0.5) / 3.0, (tau_b - 0.5) / 3.0
    p.s_e, p.s_eps, p.s_q, p.s_pi, p.s_m = s_e, s_eps, s_q, s_pi, s_m
    p.sigma, p.beta = sigma, beta
    p.cita = cita_deg / 180.0 * math.pi
    p.body[0], p.body[1], p.body[2] = body
    p.rad = rad
    p.rho_p = rho_p_ratio * rho0
    if rad > 0:
        p.mass = 4.0 / 3.0 * p.rho_p * math.pi * (rad * rad * rad)
        p.inertia = 2.0 / 5.0 * p.mass * (rad * rad)
    p.fg = -math.pi * 2.0 * max(rad, 1.0) * sigma
    p.alpha = alpha_deg / 180.0 * math.pi
    p.evap_lim = 1.0e-8
    return p


# ---- serving (sym_server_*) ------------------------------------------------------
SYM_JOB_THREAD = 0
SYM_JOB_SLAB = 1
JOB_STATUS = {0: "pending", 1: "running", 2: "breakup", 3: "limit", 4: "failed"}


class SymJobSpec(ctypes.Structure):
    """One served job (sym_job_spec): a CONFIG domain, its initial state and stop rule."""
    _fields_ = [
        ("p", SymParams),
        ("kind", ctypes.c_int32), ("max_steps", ctypes.c_int32),
        ("gen", ctypes.c_double * 5),
        ("seed", ctypes.c_uint64),
        ("stop_radius", ctypes.c_double),
        ("center", ctypes.c_double * 3), ("up", ctypes.c_double * 3),
        ("t_arrival", ctypes.c_double),
        ("drift_tol", ctypes.c_double), ("wall_budget_s", ctypes.c_double),
    ]


class SymJobResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32), ("error", ctypes.c_int32), ("steps", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("breakup_step", ctypes.c_double), ("rmin", ctypes.c_double),
        ("t_arrival", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
        ("node_updates", ctypes.c_int64),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["status"] = JOB_STATUS.get(self.status, str(self.status))
        return d
