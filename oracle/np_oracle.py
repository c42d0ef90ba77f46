"""Second, independent restatement of the lattice update in numpy --
TEST INFRASTRUCTURE ONLY (cross-checks the C++ oracle on small grids).

Written directly from Source1.f90 for the CONFIG geometry (periodic box,
optional solid wetting wall planes at x=0 and x=nx-1, no particles),
vectorised with whole-array shifts instead of loops, and reading the moment
matrix from the golden fixture parsed out of the reference's data statement.
Summation orders differ from the C++ oracle, so agreement is to rounding
(~1e-13), not bit-exact.
"""
from __future__ import annotations

import json
import os

import numpy as np

_G = json.load(open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                 "tests", "golden", "reference_constants.json")))
C = np.array([_G["cix"], _G["ciy"], _G["ciz"]], dtype=np.int64).T        # (19,3)
OPC = np.array(_G["opc"])
W = np.array(_G["wi"])
M = np.array(_G["M"], dtype=np.float64)
MINV = (M / (M * M).sum(axis=1, keepdims=True)).T                        # :126-130


def shift(a, c):
    """value at node x + c (periodic), a indexed [..., x, y, z]"""
    return np.roll(a, shift=(-c[0], -c[1], -c[2]), axis=(-3, -2, -1))


class NpLattice:
    def __init__(self, p, phi, rho):
        self.p = p
        nx, ny, nz = p.nx, p.ny, p.nz
        self.walls_all = np.zeros((nx, ny, nz), dtype=np.int64)
        self.wall_id = np.zeros((nx, ny, nz), dtype=np.int64)
        if p.wall_x:
            self.walls_all[0] = 10; self.walls_all[-1] = 10
            self.wall_id[0] = 1; self.wall_id[-1] = 2
        solid = self.walls_all > 0
        # pout: fluid node with a solid neighbour; pin: solid node with a fluid neighbour (set_walls :352-373)
        self.pout = np.zeros_like(self.wall_id)
        self.pin = np.zeros_like(self.wall_id)
        for i in range(1, 19):
            nb = shift(self.wall_id, C[i])
            self.pout = np.where(~solid & (nb > 0), nb, self.pout)
            nbf = shift((~solid).astype(np.int64), C[i])
            self.pin = np.where(solid & (nbf > 0), self.wall_id, self.pin)
        rhoR = rho * (phi + 1.0) / 2.0
        rhoB = rho - rhoR
        self.ri = self.feq(rhoR, 0 * rho, 0 * rho, 0 * rho)
        self.bi = self.feq(rhoB, 0 * rho, 0 * rho, 0 * rho)
        self.rhoN = phi.copy()
        self.derivatives()

    @staticmethod
    def feq(rho, ux, uy, uz):   # equilf_SRT :833-848
        usq = ux * ux + uy * uy + uz * uz
        out = []
        for i in range(19):
            uc = ux * C[i, 0] + uy * C[i, 1] + uz * C[i, 2]
            out.append(rho * W[i] * (1 + 3 * uc + 4.5 * uc * uc - 1.5 * usq))
        return np.array(out)

    def calmacros(self):      # :770-831
        solid = self.walls_all >= 1
        self.fi = self.ri + self.bi
        self.rhoR = self.ri.sum(0)
        self.rhoB = self.bi.sum(0)
        self.rho = self.rhoR + self.rhoB
        u = np.einsum("i...,ik->k...", self.fi, C.astype(np.float64)) / self.rho
        self.u = np.where(solid, 0.0, u)
        self.rho = np.where(solid, self.p.rho0, self.rho)
        self.rhoN = np.where(solid, 0.0, (self.rhoR - self.rhoB) / np.where(solid, 1.0, self.rhoR + self.rhoB))

    def derivatives(self):    # :452-597
        np.seterr(divide="ignore", invalid="ignore")
        solid = self.walls_all > 0
        if solid.any():
            ws = np.zeros_like(self.rhoN); v = np.zeros_like(self.rhoN)
            for i in range(1, 19):
                fl = ~shift(solid, C[i])
                ws += np.where(fl, W[i], 0.0)
                v += np.where(fl, W[i] * shift(self.rhoN, C[i]), 0.0)
            self.rhoN = np.where(self.pin > 0, v / np.where(ws > 0, ws, 1.0), self.rhoN)
        g = np.zeros((3,) + self.rhoN.shape)
        for i in range(1, 19):
            g += W[i] * shift(self.rhoN, C[i])[None] * C[i][:, None, None, None]
        g *= 3.0
        g = np.where(solid[None], 0.0, g)
        fn = np.sqrt((g * g).sum(0))
        self.flag = (fn > self.p.evap_lim) & ~solid
        n = np.where(self.flag[None], g / np.where(fn > 0, fn, 1.0)[None], 0.0)
        if solid.any():
            cita = self.p.cita
            nw = np.zeros_like(n)
            nw[0] = np.where(self.pout == 1, 1.0, np.where(self.pout == 2, -1.0, 0.0))
            wet = (self.pout >= 1) & self.flag
            par = np.abs(nw - n).max(0) < 1e-5
            with np.errstate(invalid="ignore"):
                theta = np.where(par, 1e-5, np.arccos((nw * n).sum(0)))
            a1 = np.cos(cita) - np.sin(cita) * np.cos(theta) / np.sin(theta)
            a2 = np.cos(cita) + np.sin(cita) * np.cos(theta) / np.sin(theta)
            b1 = np.sin(cita) / np.sin(theta)
            v1 = a1 * nw + b1 * n
            v2 = a2 * nw - b1 * n
            d1 = ((v1 - n) ** 2).sum(0); d2 = ((v2 - n) ** 2).sum(0)
            rot = np.where((d1 < d2)[None], v1, v2)
            n = np.where(wet[None], rot, n)
            g = np.where(wet[None], fn[None] * rot, g)
        self.grad, self.n = g, n

    def collision(self):      # :599-695
        p = self.p
        solid = self.walls_all > 0
        dn = np.zeros((3, 3) + self.rhoN.shape)   # dn[a][b] = d n_a / d x_b
        for i in range(1, 19):
            nb = shift(self.n, C[i])
            for a in range(3):
                for b in range(3):
                    dn[a, b] += W[i] * nb[a] * C[i, b]
        dn *= 3.0
        nx, ny, nz = self.n
        kurv = (nx * ny * (dn[1, 0] + dn[0, 1]) + nx * nz * (dn[2, 0] + dn[0, 2]) + ny * nz * (dn[1, 2] + dn[2, 1])
                - (ny ** 2 + nz ** 2) * dn[0, 0] - (nx ** 2 + nz ** 2) * dn[1, 1] - (nx ** 2 + ny ** 2) * dn[2, 2])
        active = self.flag & (self.pout <= 0)
        F = np.where(active[None], 0.5 * p.sigma * kurv * self.grad, 0.0)
        F = F + self.rho[None] * np.array(list(p.body))[:, None, None, None]
        u = self.u + 0.5 * F / self.rho
        phi = self.rhoN
        nu = np.where(phi <= -1, p.nu_b, np.where(phi >= 1, p.nu_r, 2.0 / ((1 + phi) / p.nu_r + (1 - phi) / p.nu_b)))
        su = 1.0 / (3 * nu + 0.5)
        sq = 8 * (2 - su) / (8 - su)
        pick = lambda s, d: s if s > 0 else d
        s = [np.ones_like(su), pick(p.s_e, su), pick(p.s_eps, su), np.ones_like(su), pick(p.s_q, sq),
             np.ones_like(su), pick(p.s_q, sq), np.ones_like(su), pick(p.s_q, sq), su, pick(p.s_pi, su), su,
             pick(p.s_pi, su), su, su, su, pick(p.s_m, sq), pick(p.s_m, sq), pick(p.s_m, sq)]
        s = np.array([np.broadcast_to(v, su.shape) for v in s])
        m = np.einsum("rc,c...->r...", M, self.fi)
        ux, uy, uz = u
        usq = ux * ux + uy * uy + uz * uz
        z = np.zeros_like(ux)
        meq = self.rho * np.array([z + 1, 19 * usq - 11, 3 - 5.5 * usq, ux, -ux / 1.5, uy, -uy / 1.5, uz, -uz / 1.5,
                                   3 * ux * ux - usq, -0.5 * (3 * ux * ux - usq), uy * uy - uz * uz,
                                   -0.5 * (uy * uy - uz * uz), ux * uy, uy * uz, ux * uz, z, z, z])
        fx, fy, fz = F
        uf = ux * fx + uy * fy + uz * fz
        fk = np.array([z, 38 * uf, -11 * uf, fx, -fx / 1.5, fy, -fy / 1.5, fz, -fz / 1.5, 6 * ux * fx - 2 * uf,
                       -(3 * ux * fx - uf), 2 * (uy * fy - uz * fz), -(uy * fy - uz * fz), ux * fy + uy * fx,
                       uy * fz + uz * fy, ux * fz + uz * fx, z, z, z])
        m = m - s * (m - meq) + (1 - 0.5 * s) * fk
        f = np.einsum("rc,c...->r...", MINV, m)
        self.fi = np.where(solid[None], self.fi, f)
        self.u = np.where(solid[None], self.u, u)

    def recolor(self):        # :697-732
        p = self.p
        solid = self.walls_all >= 1
        R, B, rho = self.rhoR, self.rhoB, self.rho
        r = (R / rho)[None] * self.fi
        nc = np.einsum("k...,ik->i...", self.n, C.astype(np.float64))
        add = (R * B / rho * p.beta)[None] * W[:, None, None, None] * nc
        add[0] = 0.0
        r = np.where(self.flag[None], r + add, r)
        r = np.where((R <= p.evap_lim)[None], 0.0, r)
        r = np.where((B <= p.evap_lim)[None], self.fi, r)
        self.ri = np.where(solid[None], self.ri, r)
        self.bi = np.where(solid[None], self.bi, self.fi - r)

    def stream_and_bounce(self):   # streaming :735-768 + curve :990-1034 with wall velocity 0
        rs = np.array([shift(self.ri[i], -C[i]) for i in range(19)])
        bs = np.array([shift(self.bi[i], -C[i]) for i in range(19)])
        if (self.walls_all > 0).any():
            for i in range(1, 19):
                from_wall = (shift(self.wall_id, -C[i]) > 0) & (self.pout >= 1)
                rs[i] = np.where(from_wall, shift(rs[OPC[i]], -C[i]), rs[i])
                bs[i] = np.where(from_wall, shift(bs[OPC[i]], -C[i]), bs[i])
        self.ri, self.bi = rs, bs

    def step(self, n=1):
        for _ in range(n):
            self.calmacros()
            self.derivatives()
            self.collision()
            self.recolor()
            self.stream_and_bounce()
