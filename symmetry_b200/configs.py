"""Synthetic workloads of the lattice-update library (no dataset is involved).

Each workload is a seeded CONFIG-mode domain.  The phase-field generators
here are the host-side definition of the initial state; the library's device
initialisers (``sym_init_thread`` / ``sym_init_slab``) compute the same
formula on the GPU for domains too large to build on the host.

Initial state, following the reference's ``initialization``
(Source1.f90:850-896) with a configurable interface profile:
  phi = tanh(2 (r - d) / W) + noise, clamped to [-1, 1]
  rho = rho0 + 3 sigma / r(z) where phi > 0 (Laplace jump, :875-881), else rho0
  rho_R = rho (1 + phi) / 2, populations at SRT equilibrium with u = 0.
Noise: uniform in [-a, a], a = 1e-4, from splitmix64(seed ^ L) where
L = z + nz*(y + ny*x) is the 0-based node index.
"""
from __future__ import annotations

import dataclasses
import json
import math
from typing import List, Optional

import numpy as np

from .params import SymParams, config_params

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _MASK
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK
        return z ^ (z >> np.uint64(31))


def node_noise(nx: int, ny: int, nz: int, amp: float, seed: int) -> np.ndarray:
    """Per-node uniform noise in [-amp, amp), shape (nx, ny, nz)."""
    L = np.arange(nx * ny * nz, dtype=np.uint64)
    h = splitmix64(np.uint64(seed) ^ L)
    u = (h >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
    return (u * (2.0 * amp) - amp).reshape(nx, ny, nz)


def thread_phase(nx, ny, nz, radius, amp, wavelength, width=2.0, noise=1e-4, seed=0,
                 rho0=1.0, sigma=0.0):
    """Rayleigh-Plateau thread along z: returns (phi, rho), shape (nx,ny,nz)."""
    x = np.arange(nx, dtype=np.float64)[:, None, None]
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    z = np.arange(nz, dtype=np.float64)[None, None, :]
    xc, yc = (nx - 1) / 2.0, (ny - 1) / 2.0
    rz = radius * (1.0 + amp * np.cos(2.0 * math.pi * z / wavelength))
    d = np.sqrt((x - xc) ** 2 + (y - yc) ** 2)
    phi = np.tanh(2.0 * (rz - d) / width)
    if noise > 0:
        phi = phi + node_noise(nx, ny, nz, noise, seed)
    phi = np.clip(phi, -1.0, 1.0)
    rho = np.where(phi > 0.0, rho0 + 3.0 * sigma / rz, rho0) * np.ones_like(phi)
    return phi, rho


def slab_phase(nx, ny, nz, z0, z1, width=2.0, noise=1e-4, seed=0, rho0=1.0):
    """Red slab z0 <= z <= z1 (periodic in z), flat interfaces, no Laplace jump."""
    z = np.arange(nz, dtype=np.float64)
    dz = np.minimum(z - z0, z1 - z)
    phi = np.broadcast_to(np.tanh(2.0 * dz / width)[None, None, :], (nx, ny, nz)).copy()
    if noise > 0:
        phi = phi + node_noise(nx, ny, nz, noise, seed)
    phi = np.clip(phi, -1.0, 1.0)
    return phi, np.full_like(phi, rho0)


@dataclasses.dataclass
class Workload:
    """One seeded domain: its parameters, its initial phase generator and particles."""
    name: str
    params: SymParams
    kind: str                      # "thread" or "slab"
    gen: dict                      # generator arguments
    steps: int
    particles: List[dict] = dataclasses.field(default_factory=list)  # centre/up

    def phase(self):
        p = self.params
        if self.kind == "thread":
            return thread_phase(p.nx, p.ny, p.nz, rho0=p.rho0, sigma=p.sigma, **self.gen)
        return slab_phase(p.nx, p.ny, p.nz, rho0=p.rho0, **self.gen)

    @property
    def nodes(self) -> int:
        return self.params.n_nodes


def c1_thread(nx=32, ny=32, nz=96, steps=2000, storage="fp64", radius=6.0) -> Workload:
    """Plain method, periodic 32x32x96 Rayleigh-Plateau thread, FP64."""
    p = config_params(nx, ny, nz, tau_r=1.0, sigma=5e-3, beta=0.7, rho0=1.0,
                      s_e=1.19, s_eps=1.4, s_q=1.2, s_pi=1.0, storage=storage)
    gen = dict(radius=radius, amp=0.05, wavelength=float(nz),
               width=2.0, noise=1e-4, seed=1001)
    return Workload("c1_thread", p, "thread", gen, steps)


def c2_wall_particle(nx=64, ny=64, nz=128, steps=5000, storage="fp64", rad=8.0,
                     centre=(32.0, 32.0, 40.0), z0=40.0, z1=88.0) -> Workload:
    """Wetting x walls (60 deg) + one moving sphere, FP64, 64x64x128."""
    p = config_params(nx, ny, nz, tau_r=0.8, sigma=5e-3, beta=0.7, rho0=1.0, wall_x=True,
                      cita_deg=60.0, par=1, rad=rad, rho_p_ratio=1.5,
                      body=(0.0, 0.0, -1e-6), storage=storage)
    gen = dict(z0=z0, z1=z1, width=2.0, noise=1e-4, seed=1002)
    return Workload("c2_wall_particle", p, "slab", gen, steps,
                    particles=[dict(center=list(centre), up=[0.0, 0.0, 0.01])])


def c3_thread(nx=256, ny=256, nz=512, steps=40000, storage="fp64", radius=24.0) -> Workload:
    """Precision study: periodic 256x256x512 thread, R=24, tau=0.7, A=8e-3."""
    p = config_params(nx, ny, nz, tau_r=0.7, sigma=8e-3, beta=0.7, rho0=1.0, storage=storage)
    gen = dict(radius=radius, amp=0.02, wavelength=float(nz), width=2.0,
               noise=1e-4, seed=1003)
    return Workload("c3_thread", p, "thread", gen, steps)


def _c4_domain(rng, name, seed, storage, steps, wall_cita_deg=None, sphere_override=None) -> Workload:
    """One domain of the batched-mix distribution (draw order fixed; the
    sphere draw is consumed even when `sphere_override` decides it)."""
    n = int(rng.integers(24, 65))
    nz_raw = int(rng.integers(64, 385))
    R = float(rng.uniform(4.0, 0.3 * n))
    lam_ratio = float(rng.uniform(0.7, 2.0))
    A = float(rng.uniform(2e-3, 1e-2))
    tau = float(rng.uniform(0.6, 1.5))
    sphere = bool(rng.integers(0, 2))
    if sphere_override is not None:
        sphere = bool(sphere_override)
    lam = lam_ratio * 2.0 * math.pi * R
    nwave = max(1, int(round(nz_raw / lam)))
    nz = int(round(nwave * lam))
    nz = max(nz, 16)
    lam = nz / nwave
    walls = wall_cita_deg is not None
    p = config_params(n, n, nz, tau_r=tau, sigma=A, beta=0.7, rho0=1.0, storage=storage,
                      par=1 if sphere else 0, rad=R / 2.0 if sphere else 0.0,
                      rho_p_ratio=1.2, wall_x=walls, cita_deg=wall_cita_deg if walls else 90.0)
    gen = dict(radius=R, amp=0.05, wavelength=lam, width=2.0, noise=1e-4, seed=seed)
    parts = []
    if sphere:
        parts = [dict(center=[(n - 1) / 2.0, (n - 1) / 2.0, nz / 2.0], up=[0.0, 0.0, 0.0])]
    return Workload(name, p, "thread", gen, steps, parts)


def c4_manifest(n_domains=96, seed=4, storage="fp16", steps=3000) -> List[Workload]:
    """Batched uneven Rayleigh-Plateau domains (frozen from default_rng(seed));
    exactly half of them (the odd-numbered ones) carry the sphere."""
    rng = np.random.default_rng(seed)
    return [_c4_domain(rng, f"c4_{k:03d}", 1004000 + k, storage, steps, sphere_override=(k % 2 == 1))
            for k in range(n_domains)]


@dataclasses.dataclass
class Job:
    """One served job: its workload and its arrival time in seconds."""
    workload: Workload
    t_arrival: float
    cita_deg: Optional[float]


def c5_jobs(rate=20.0, duration=120.0, seed=5, storage="fp16", max_steps=50000) -> List[Job]:
    """Open-loop Poisson arrivals (rate jobs/s for `duration` s), frozen from
    default_rng(seed): 90% domains of the batched-mix distribution, 10%
    128x128x512 threads with R=16 (the precision-study thread scaled down:
    tau=0.7, A=8e-3, 2% perturbation over one 512 wavelength); each job has
    wetting x walls with probability 0.3, contact angle uniform in [30,150]
    degrees.  Seeds 1005000+j."""
    rng = np.random.default_rng(seed)
    out, t, j = [], 0.0, 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        big = bool(rng.random() < 0.1)
        walls = bool(rng.random() < 0.3)
        cita = float(rng.uniform(30.0, 150.0)) if walls else None
        if big:
            p = config_params(128, 128, 512, tau_r=0.7, sigma=8e-3, beta=0.7, rho0=1.0, storage=storage,
                              wall_x=walls, cita_deg=cita if walls else 90.0)
            gen = dict(radius=16.0, amp=0.02, wavelength=512.0, width=2.0, noise=1e-4, seed=1005000 + j)
            w = Workload(f"c5_{j:04d}", p, "thread", gen, max_steps)
        else:
            w = _c4_domain(rng, f"c5_{j:04d}", 1005000 + j, storage, max_steps, cita)
        out.append(Job(w, t, cita))
        j += 1
    return out


def manifest_json(ws: List[Workload]) -> str:
    rows = []
    for w in ws:
        p = w.params
        rows.append(dict(name=w.name, nx=p.nx, ny=p.ny, nz=p.nz, tau=3 * p.nu_r + 0.5,
                         sigma=p.sigma, par=p.par, rad=p.rad, gen=w.gen, particles=w.particles))
    return json.dumps(rows, indent=1)
