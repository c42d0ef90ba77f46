/*
 * sym_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the per-timestep lattice update of the reference
 * (X-Sheen/Symmetry, Source1.f90), used as the checker by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py.  Nothing in
 * the library links or calls this file.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists on
 * this image, so it cannot be built.  This restatement is pinned against the
 * reference's own source executed instead: oracle/f90py.py translates
 * Source1.f90 statement by statement (main up to its time loop and every
 * subroutine, as written) into oracle/_ref/, and tests/test_reference_pin.py
 * runs main's set-up and the whole time-loop body beside this file, routine
 * by routine, with every array and particle variable equal bit for bit.
 * Also: golden constants parsed from Source1.f90 (tests/golden/), an
 * independent numpy restatement, and invariants derived from the code.
 *
 * Each routine follows the reference subroutine cited above it: same loop
 * ranges, same order of floating-point operations (left-to-right evaluation of
 * Fortran expressions, sequential SUM/MATMUL/DOT_PRODUCT), compiled with
 * -ffp-contract=off so no multiply-add is fused.  Loops whose result does not
 * depend on order run under OpenMP; reductions are done in a fixed order
 * (the reference's loop order where it leaves the order to OpenMP).
 *
 * Arrays use the Fortran layout: scalars (z,y,x) with z fastest, populations
 * (0:18,z,y,x); x,y,z below are 1-based like the reference.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/symmetry.h"

namespace {

// D3Q19 velocity set, opposite and mirror maps (Source1.f90:132-138).
const int CIX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int CIY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
const int CIZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int OPC[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
const int SYMX[19] = {0, 2, 1, 3, 4, 5, 6, 8, 7, 10, 9, 12, 11, 14, 13, 15, 16, 17, 18};
const int SYMY[19] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 16, 15, 18, 17};
const int SYMZ[19] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};

// Moment matrix of the reference's data statement (Source1.f90:105-123), built
// here from the polynomial each row holds (d'Humieres D3Q19 basis; row order as
// in the reference: rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww,
// pxy, pyz, pxz, mx, my, mz).  tests/golden/ pins it entry by entry against the
// data statement.
double moment_row(int r, int c) {
  const double x = CIX[c], y = CIY[c], z = CIZ[c];
  const double c2 = x * x + y * y + z * z;
  switch (r) {
    case 0: return 1.0;
    case 1: return 19.0 * c2 - 30.0;
    case 2: return (21.0 * c2 * c2 - 53.0 * c2 + 24.0) / 2.0;
    case 3: return x;
    case 4: return (5.0 * c2 - 9.0) * x;
    case 5: return y;
    case 6: return (5.0 * c2 - 9.0) * y;
    case 7: return z;
    case 8: return (5.0 * c2 - 9.0) * z;
    case 9: return 3.0 * x * x - c2;
    case 10: return (3.0 * c2 - 5.0) * (3.0 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3.0 * c2 - 5.0) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    default: return (x * x - y * y) * z;
  }
}

inline double sq(double a) { return a * a; }

struct Orc {
  sym_params p;
  int nx, ny, nz;
  size_t N;
  bool ref;
  int origin;        // node coordinate = index - 1 + origin
  int lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;  // update range (1-based, inclusive)
  int par, la_m, la_n, la_num;
  double wi[19];
  double M[19][19], Minv[19][19];
  double evap;
  double mass, inertia;

  std::vector<int32_t> walls, walls_old, walls_all, pin, pout, flag;
  std::vector<double> rho, ux, uy, uz, rhoN, rhoR, rhoB, nxv, nyv, nzv, gx, gy, gz;
  std::vector<double> fi, ffi, ri, bi, ft;
  sym_particles s;
  std::vector<double> Lax, Lay, Laz, La_rhoN, La_nx, La_ny, La_nz, ds;
  std::vector<int32_t> La_flag;

  inline size_t lin(int x, int y, int z) const {
    return (size_t)(z - 1) + (size_t)nz * ((size_t)(y - 1) + (size_t)ny * (size_t)(x - 1));
  }
  static inline int wrap(int v, int n) { return v < 1 ? v + n : (v > n ? v - n : v); }
  inline double coord(int i) const { return (double)(i - 1 + origin); }
  // component k (0..2) of particle pp (1-based) in sym_particles arrays
  inline double& C(double* a, int pp, int k) { return a[k * par + (pp - 1)]; }
  // displacement of a node coordinate from a centre along dim k (minimum
  // image in periodic CONFIG dimensions; plain difference in REFERENCE)
  inline double disp(double c, double cen, int k) const {
    double d = c - cen;
    if (!ref) {
      const int n = k == 0 ? nx : (k == 1 ? ny : nz);
      const bool periodic = !(k == 0 && p.wall_x);
      if (periodic) d -= (double)n * std::nearbyint(d / (double)n);
    }
    return d;
  }
};

void sym_phi_x(Orc& o, std::vector<double>& v) {  // symmetry_X_phi :1455-1462
  for (int y = 1; y <= o.ny; y++)
    for (int z = 1; z <= o.nz; z++) v[o.lin(o.nx, y, z)] = v[o.lin(o.nx - 1, y, z)];
}
void sym_phi_y(Orc& o, std::vector<double>& v) {  // symmetry_Y_phi :1489-1497
  for (int x = 1; x <= o.nx; x++)
    for (int z = 1; z <= o.nz; z++) {
      v[o.lin(x, o.ny, z)] = v[o.lin(x, o.ny - 1, z)];
      v[o.lin(x, 1, z)] = v[o.lin(x, 2, z)];
    }
}
void sym_phi_z(Orc& o, std::vector<double>& v) {  // symmetry_Z_phi :1525-1532
  for (int x = 1; x <= o.nx; x++)
    for (int y = 1; y <= o.ny; y++) v[o.lin(x, y, o.nz)] = v[o.lin(x, y, o.nz - 1)];
}
void sym_u_x(Orc& o, std::vector<double>& a, std::vector<double>& b, std::vector<double>& c) {
  for (int y = 1; y <= o.ny; y++)  // symmetry_X_u :1464-1473
    for (int z = 1; z <= o.nz; z++) {
      size_t d = o.lin(o.nx, y, z), s = o.lin(o.nx - 1, y, z);
      a[d] = -a[s]; b[d] = b[s]; c[d] = c[s];
    }
}
void sym_u_y(Orc& o, std::vector<double>& a, std::vector<double>& b, std::vector<double>& c) {
  for (int x = 1; x <= o.nx; x++)  // symmetry_Y_u :1499-1511
    for (int z = 1; z <= o.nz; z++) {
      size_t d = o.lin(x, o.ny, z), s = o.lin(x, o.ny - 1, z);
      a[d] = a[s]; b[d] = -b[s]; c[d] = c[s];
      d = o.lin(x, 1, z); s = o.lin(x, 2, z);
      a[d] = a[s]; b[d] = -b[s]; c[d] = c[s];
    }
}
void sym_u_z(Orc& o, std::vector<double>& a, std::vector<double>& b, std::vector<double>& c) {
  for (int x = 1; x <= o.nx; x++)  // symmetry_Z_u :1534-1542
    for (int y = 1; y <= o.ny; y++) {
      size_t d = o.lin(x, y, o.nz), s = o.lin(x, y, o.nz - 1);
      a[d] = a[s]; b[d] = b[s]; c[d] = -c[s];
    }
}
void sym_fi_x(Orc& o, std::vector<double>& f) {  // symmetry_X_fi :1443-1453
  for (int i = 0; i < 19; i++)
    for (int y = 1; y <= o.ny; y++)
      for (int z = 1; z <= o.nz; z++)
        f[19 * o.lin(o.nx, y, z) + i] = f[19 * o.lin(o.nx - 1, y, z) + SYMX[i]];
}
void sym_fi_y(Orc& o, std::vector<double>& f) {  // symmetry_Y_fi :1475-1487
  for (int i = 0; i < 19; i++)
    for (int x = 1; x <= o.nx; x++)
      for (int z = 1; z <= o.nz; z++) {
        f[19 * o.lin(x, o.ny, z) + i] = f[19 * o.lin(x, o.ny - 1, z) + SYMY[i]];
        f[19 * o.lin(x, 1, z) + i] = f[19 * o.lin(x, 2, z) + SYMY[i]];
      }
}
void sym_fi_z(Orc& o, std::vector<double>& f) {  // symmetry_Z_fi :1513-1523
  for (int i = 0; i < 19; i++)
    for (int x = 1; x <= o.nx; x++)
      for (int y = 1; y <= o.ny; y++)
        f[19 * o.lin(x, y, o.nz) + i] = f[19 * o.lin(x, y, o.nz - 1) + SYMZ[i]];
}
void mirror_macros(Orc& o) {  // the mirror sequence of calmacros :809-828 / refilling :1397-1416
  sym_phi_x(o, o.rhoN); sym_phi_x(o, o.rhoR); sym_phi_x(o, o.rhoB); sym_phi_x(o, o.rho);
  sym_u_x(o, o.ux, o.uy, o.uz); sym_fi_x(o, o.fi);
  sym_phi_y(o, o.rhoN); sym_phi_y(o, o.rhoR); sym_phi_y(o, o.rhoB); sym_phi_y(o, o.rho);
  sym_u_y(o, o.ux, o.uy, o.uz); sym_fi_y(o, o.fi);
  sym_phi_z(o, o.rhoN); sym_phi_z(o, o.rhoR); sym_phi_z(o, o.rhoB); sym_phi_z(o, o.rho);
  sym_u_z(o, o.ux, o.uy, o.uz); sym_fi_z(o, o.fi);
}

// equilf (Source1.f90:397-450)
void equilf(double meq[19], double fk[19], double rho, double ux, double uy, double uz, double fx,
            double fy, double fz) {
  const double usqr = ux * ux + uy * uy + uz * uz;
  meq[0] = 1.0;
  meq[1] = 19.0 * usqr - 11.0;
  meq[2] = 3.0 - 5.5 * usqr;
  meq[3] = ux;
  meq[4] = -ux / 1.5;
  meq[5] = uy;
  meq[6] = -uy / 1.5;
  meq[7] = uz;
  meq[8] = -uz / 1.5;
  meq[9] = 3.0 * ux * ux - usqr;
  meq[10] = -0.5 * (3.0 * ux * ux - usqr);
  meq[11] = uy * uy - uz * uz;
  meq[12] = -0.5 * (uy * uy - uz * uz);
  meq[13] = ux * uy;
  meq[14] = uy * uz;
  meq[15] = ux * uz;
  meq[16] = 0.0;
  meq[17] = 0.0;
  meq[18] = 0.0;
  for (int k = 0; k < 19; k++) meq[k] = rho * meq[k];
  const double uf = ux * fx + uy * fy + uz * fz;
  fk[0] = 0.0;
  fk[1] = 38.0 * uf;
  fk[2] = -11.0 * uf;
  fk[3] = fx;
  fk[4] = -fx / 1.5;
  fk[5] = fy;
  fk[6] = -fy / 1.5;
  fk[7] = fz;
  fk[8] = -fz / 1.5;
  fk[9] = 6.0 * ux * fx - 2.0 * uf;
  fk[10] = -(3.0 * ux * fx - uf);
  fk[11] = 2.0 * (uy * fy - uz * fz);
  fk[12] = -(uy * fy - uz * fz);
  fk[13] = ux * fy + uy * fx;
  fk[14] = uy * fz + uz * fy;
  fk[15] = ux * fz + uz * fx;
  fk[16] = 0.0;
  fk[17] = 0.0;
  fk[18] = 0.0;
}

// equilf_SRT (Source1.f90:833-848)
void equilf_srt(const double wi[19], double* feq, double rho, double ux, double uy, double uz) {
  const double usqr = ux * ux + uy * uy + uz * uz;
  for (int i = 0; i < 19; i++) {
    const double uc = ux * CIX[i] + uy * CIY[i] + uz * CIZ[i];
    feq[i] = rho * wi[i] * (1.0 + 3.0 * uc + 4.5 * uc * uc - 1.5 * usqr);
  }
}

void unitization(double a[3]) {  // :979-988
  double star = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  star = std::sqrt(star);
  a[0] = a[0] / star; a[1] = a[1] / star; a[2] = a[2] / star;
}
void veccross(const double a[3], const double b[3], double c[3]) {  // VecCross :1168-1175
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = -(a[0] * b[2] - a[2] * b[0]);
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Akai-2018 rotation of n toward the contact angle (derivatives :547-587 and
// Lagrange_points :1921-1947).  `guard` applies the 1e-5 parallel guard (the
// Lagrange copy overwrites it, :1929).
void akai_rotate(double cita, const double nw[3], const double n[3], bool guard, double out[3]) {
  double theta;
  double mx = std::max(std::fabs(nw[0] - n[0]), std::max(std::fabs(nw[1] - n[1]), std::fabs(nw[2] - n[2])));
  if (guard && mx < 1.0e-5) theta = 1.0e-5;
  else theta = std::acos(nw[0] * n[0] + nw[1] * n[1] + nw[2] * n[2]);
  const double a1 = std::cos(cita) - std::sin(cita) * std::cos(theta) / std::sin(theta);
  const double a2 = std::cos(cita) + std::sin(cita) * std::cos(theta) / std::sin(theta);
  const double b1 = std::sin(cita) / std::sin(theta);
  const double b2 = -std::sin(cita) / std::sin(theta);
  double v1[3], v2[3];
  for (int k = 0; k < 3; k++) { v1[k] = a1 * nw[k] + b1 * n[k]; v2[k] = a2 * nw[k] + b2 * n[k]; }
  const double db1 = sq(v1[0] - n[0]) + sq(v1[1] - n[1]) + sq(v1[2] - n[2]);
  const double db2 = sq(v2[0] - n[0]) + sq(v2[1] - n[1]) + sq(v2[2] - n[2]);
  if (db1 < db2) { out[0] = v1[0]; out[1] = v1[1]; out[2] = v1[2]; }
  else { out[0] = v2[0]; out[1] = v2[1]; out[2] = v2[2]; }
}

// wall normal at node (x,y,z) for the solid object `id` (particle or CONFIG wall)
void wall_normal(Orc& o, int id, int x, int y, int z, double nw[3]) {
  if (id <= o.par) {
    nw[0] = o.disp(o.coord(x), o.C(o.s.center, id, 0), 0);
    nw[1] = o.disp(o.coord(y), o.C(o.s.center, id, 1), 1);
    nw[2] = o.disp(o.coord(z), o.C(o.s.center, id, 2), 2);
    unitization(nw);
  } else {
    nw[0] = (id == SYM_WALL_ID_XLO(o.par)) ? 1.0 : -1.0;
    nw[1] = 0.0; nw[2] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// set_walls (Source1.f90:326-395)
void set_walls(Orc& o) {
  o.walls_old = o.walls_all;
  std::fill(o.walls_all.begin(), o.walls_all.end(), 0);
  std::fill(o.walls.begin(), o.walls.end(), 0);
  std::fill(o.pin.begin(), o.pin.end(), 0);
  std::fill(o.pout.begin(), o.pout.end(), 0);
  std::vector<int> ids;
  if (!o.ref && o.p.wall_x) {  // CONFIG solid wall planes x=0, x=nx-1
    for (int y = 1; y <= o.ny; y++)
      for (int z = 1; z <= o.nz; z++) {
        size_t a = o.lin(1, y, z), b = o.lin(o.nx, y, z);
        o.walls[a] = SYM_WALL_ID_XLO(o.par); o.walls_all[a] = 10;
        o.walls[b] = SYM_WALL_ID_XHI(o.par); o.walls_all[b] = 10;
      }
    ids.push_back(SYM_WALL_ID_XLO(o.par));
    ids.push_back(SYM_WALL_ID_XHI(o.par));
  }
  const double r2 = o.p.rad * o.p.rad;
  for (int pp = 1; pp <= o.par; pp++) {
    ids.push_back(pp);
    const double cx = o.C(o.s.center, pp, 0), cy = o.C(o.s.center, pp, 1), cz = o.C(o.s.center, pp, 2);
#pragma omp parallel for schedule(static)
    for (int x = 1; x <= o.nx; x++)
      for (int y = 1; y <= o.ny; y++)
        for (int z = 1; z <= o.nz; z++) {
          const double d = sq(o.disp(o.coord(x), cx, 0)) + sq(o.disp(o.coord(y), cy, 1)) +
                           sq(o.disp(o.coord(z), cz, 2));
          if (d <= r2) {
            o.walls[o.lin(x, y, z)] = pp;
            o.walls_all[o.lin(x, y, z)] = 10;
          }
        }
  }
  for (int id : ids) {
    // x-slabs write pin at neighbours in adjacent slabs with the same value id
    for (int x = o.lo_x; x <= o.hi_x; x++)
      for (int y = o.lo_y; y <= o.hi_y; y++)
        for (int z = o.lo_z; z <= o.hi_z; z++) {
          const size_t L = o.lin(x, y, z);
          if (o.walls_all[L] != 0) continue;
          for (int i = 1; i < 19; i++) {
            const size_t nb = o.lin(Orc::wrap(x + CIX[i], o.nx), Orc::wrap(y + CIY[i], o.ny),
                                    Orc::wrap(z + CIZ[i], o.nz));
            if (o.walls[nb] == id) { o.pout[L] = id; o.pin[nb] = id; }
          }
        }
  }
  if (o.ref) {
    std::vector<int32_t>* arrs[4] = {&o.walls, &o.walls_all, &o.pin, &o.pout};
    for (auto* a : arrs)
      for (int y = 1; y <= o.ny; y++)
        for (int z = 1; z <= o.nz; z++) (*a)[o.lin(o.nx, y, z)] = (*a)[o.lin(o.nx - 1, y, z)];
    for (auto* a : arrs)
      for (int x = 1; x <= o.nx; x++)
        for (int z = 1; z <= o.nz; z++) (*a)[o.lin(x, o.ny, z)] = (*a)[o.lin(x, o.ny - 1, z)];
    for (auto* a : arrs)
      for (int x = 1; x <= o.nx; x++)
        for (int z = 1; z <= o.nz; z++) (*a)[o.lin(x, 1, z)] = (*a)[o.lin(x, 2, z)];
    for (auto* a : arrs)
      for (int x = 1; x <= o.nx; x++)
        for (int y = 1; y <= o.ny; y++) (*a)[o.lin(x, y, o.nz)] = (*a)[o.lin(x, y, o.nz - 1)];
  }
}

// calmacros (Source1.f90:770-831)
void calmacros(Orc& o) {
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.walls_all[L] >= 1) {
          o.rhoN[L] = 0.0; o.ux[L] = 0.0; o.uy[L] = 0.0; o.uz[L] = 0.0; o.rho[L] = o.p.rho0;
        } else {
          double* f = &o.fi[19 * L];
          const double* r = &o.ri[19 * L];
          const double* b = &o.bi[19 * L];
          for (int i = 0; i < 19; i++) f[i] = r[i] + b[i];
          double sr = 0.0, sb = 0.0;
          for (int i = 0; i < 19; i++) sr += r[i];
          for (int i = 0; i < 19; i++) sb += b[i];
          o.rhoR[L] = sr; o.rhoB[L] = sb;
          const double rho = sr + sb;
          o.rho[L] = rho;
          double mx = 0.0, my = 0.0, mz = 0.0;
          for (int i = 0; i < 19; i++) mx += f[i] * CIX[i];
          for (int i = 0; i < 19; i++) my += f[i] * CIY[i];
          for (int i = 0; i < 19; i++) mz += f[i] * CIZ[i];
          o.ux[L] = mx / rho; o.uy[L] = my / rho; o.uz[L] = mz / rho;
          o.rhoN[L] = (sr - sb) / rho;
        }
      }
  if (o.ref) {
    for (int x = 1; x <= o.nx; x++)  // z=1 is wall (:806)
      for (int y = 1; y <= o.ny; y++) o.rhoN[o.lin(x, y, 1)] = o.rhoN[o.lin(x, y, 2)];
    for (int y = 1; y <= o.ny; y++)  // x=1 is wall (:807)
      for (int z = 1; z <= o.nz; z++) o.rhoN[o.lin(1, y, z)] = o.rhoN[o.lin(2, y, z)];
    mirror_macros(o);
  }
}

// derivatives (Source1.f90:452-597)
void derivatives(Orc& o) {
  // fictitious phi at pin nodes (:467-492); pin nodes are solid so they never
  // read one another
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.pin[L] > 0) {
          double ws = 0.0, v = 0.0;
          for (int i = 1; i < 19; i++) {
            const size_t nb = o.lin(Orc::wrap(x + CIX[i], o.nx), Orc::wrap(y + CIY[i], o.ny),
                                    Orc::wrap(z + CIZ[i], o.nz));
            if (o.walls_all[nb] <= 0) { ws = ws + o.wi[i]; v = v + o.wi[i] * o.rhoN[nb]; }
          }
          o.rhoN[L] = v / ws;
        }
      }
  if (o.ref) { sym_phi_x(o, o.rhoN); sym_phi_y(o, o.rhoN); sym_phi_z(o, o.rhoN); }
  // colour gradient and unit normal (:497-533)
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        o.gx[L] = 0.0; o.gy[L] = 0.0; o.gz[L] = 0.0;
        o.nxv[L] = 0.0; o.nyv[L] = 0.0; o.nzv[L] = 0.0;
        o.flag[L] = 0;
        if (o.walls_all[L] <= 0) {
          double gx = 0.0, gy = 0.0, gz = 0.0;
          for (int i = 1; i < 19; i++) {
            const size_t nb = o.lin(Orc::wrap(x + CIX[i], o.nx), Orc::wrap(y + CIY[i], o.ny),
                                    Orc::wrap(z + CIZ[i], o.nz));
            const double val = o.wi[i] * o.rhoN[nb];
            gx = gx + val * CIX[i]; gy = gy + val * CIY[i]; gz = gz + val * CIZ[i];
          }
          gx = 3.0 * gx; gy = 3.0 * gy; gz = 3.0 * gz;
          o.gx[L] = gx; o.gy[L] = gy; o.gz[L] = gz;
          const double fnorm = std::sqrt(gx * gx + gy * gy + gz * gz);
          if (fnorm > o.evap) {
            o.nxv[L] = gx / fnorm; o.nyv[L] = gy / fnorm; o.nzv[L] = gz / fnorm;
            o.flag[L] = 1;
          }
        }
      }
  // wetting boundary condition (:535-587)
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.pout[L] >= 1 && o.flag[L]) {
          double nw[3], n[3] = {o.nxv[L], o.nyv[L], o.nzv[L]}, v[3];
          wall_normal(o, o.pout[L], x, y, z, nw);
          akai_rotate(o.p.cita, nw, n, true, v);
          o.nxv[L] = v[0]; o.nyv[L] = v[1]; o.nzv[L] = v[2];
          const double fnorm = std::sqrt(o.gx[L] * o.gx[L] + o.gy[L] * o.gy[L] + o.gz[L] * o.gz[L]);
          o.gx[L] = fnorm * v[0]; o.gy[L] = fnorm * v[1]; o.gz[L] = fnorm * v[2];
        }
      }
  if (o.ref) {
    sym_u_x(o, o.nxv, o.nyv, o.nzv); sym_u_y(o, o.nxv, o.nyv, o.nzv); sym_u_z(o, o.nxv, o.nyv, o.nzv);
    sym_u_x(o, o.gx, o.gy, o.gz); sym_u_y(o, o.gx, o.gy, o.gz); sym_u_z(o, o.gx, o.gy, o.gz);
  }
}

// relaxation rates of one node (Source1.f90:674-684, runtime MRT rates)
void rates(const Orc& o, double rhoN, double si[19]) {
  double nu;
  if (rhoN <= -1.0) nu = o.p.nu_b;
  else if (rhoN >= 1.0) nu = o.p.nu_r;
  else nu = 2.0 / ((1.0 + rhoN) / o.p.nu_r + (1.0 - rhoN) / o.p.nu_b);
  const double su = 1.0 / (3.0 * nu + 0.5);
  const double sq_ = 8.0 * (2.0 - su) / (8.0 - su);
  const double se = o.p.s_e > 0 ? o.p.s_e : su;
  const double seps = o.p.s_eps > 0 ? o.p.s_eps : su;
  const double sqq = o.p.s_q > 0 ? o.p.s_q : sq_;
  const double spi = o.p.s_pi > 0 ? o.p.s_pi : su;
  const double sm = o.p.s_m > 0 ? o.p.s_m : sq_;
  const double s[19] = {1.0, se, seps, 1.0, sqq, 1.0, sqq, 1.0, sqq, su, spi, su, spi, su, su, su, sm, sm, sm};
  for (int k = 0; k < 19; k++) si[k] = s[k];
}

// collision (Source1.f90:599-695)
void collision(Orc& o) {
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.walls_all[L] > 0) continue;
        double force[3] = {0.0, 0.0, 0.0};
        const bool edge_ok = o.ref ? (z >= 3 && x >= 3) : true;
        if (o.flag[L] && o.pout[L] <= 0 && edge_ok) {
          double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // d[a][b] = d n_a / d x_b
          for (int i = 1; i < 19; i++) {
            const size_t nb = o.lin(Orc::wrap(x + CIX[i], o.nx), Orc::wrap(y + CIY[i], o.ny),
                                    Orc::wrap(z + CIZ[i], o.nz));
            double tmp = o.wi[i] * o.nxv[nb];
            d[0][0] = d[0][0] + tmp * CIX[i]; d[0][1] = d[0][1] + tmp * CIY[i]; d[0][2] = d[0][2] + tmp * CIZ[i];
            tmp = o.wi[i] * o.nyv[nb];
            d[1][0] = d[1][0] + tmp * CIX[i]; d[1][1] = d[1][1] + tmp * CIY[i]; d[1][2] = d[1][2] + tmp * CIZ[i];
            tmp = o.wi[i] * o.nzv[nb];
            d[2][0] = d[2][0] + tmp * CIX[i]; d[2][1] = d[2][1] + tmp * CIY[i]; d[2][2] = d[2][2] + tmp * CIZ[i];
          }
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) d[a][b] = 3.0 * d[a][b];
          const double nx = o.nxv[L], ny = o.nyv[L], nz = o.nzv[L];
          const double kurv = nx * ny * (d[1][0] + d[0][1]) + nx * nz * (d[2][0] + d[0][2]) +
                              ny * nz * (d[1][2] + d[2][1]) - (ny * ny + nz * nz) * d[0][0] -
                              (nx * nx + nz * nz) * d[1][1] - (nx * nx + ny * ny) * d[2][2];
          const double val = 0.5 * o.p.sigma * kurv;
          force[0] = val * o.gx[L]; force[1] = val * o.gy[L]; force[2] = val * o.gz[L];
        }
        if (!o.ref) {  // CONFIG body acceleration, Guo forcing
          force[0] = force[0] + o.rho[L] * o.p.body[0];
          force[1] = force[1] + o.rho[L] * o.p.body[1];
          force[2] = force[2] + o.rho[L] * o.p.body[2];
        }
        o.ux[L] = o.ux[L] + 0.5 * force[0] / o.rho[L];
        o.uy[L] = o.uy[L] + 0.5 * force[1] / o.rho[L];
        o.uz[L] = o.uz[L] + 0.5 * force[2] / o.rho[L];
        double si[19], mi[19], meq[19], fk[19];
        rates(o, o.rhoN[L], si);
        double* f = &o.fi[19 * L];
        for (int r = 0; r < 19; r++) {
          double acc = 0.0;
          for (int c = 0; c < 19; c++) acc += o.M[r][c] * f[c];
          mi[r] = acc;
        }
        equilf(meq, fk, o.rho[L], o.ux[L], o.uy[L], o.uz[L], force[0], force[1], force[2]);
        for (int k = 0; k < 19; k++) mi[k] = mi[k] - si[k] * (mi[k] - meq[k]) + (1.0 - 0.5 * si[k]) * fk[k];
        for (int r = 0; r < 19; r++) {
          double acc = 0.0;
          for (int c = 0; c < 19; c++) acc += o.Minv[r][c] * mi[c];
          f[r] = acc;
        }
        for (int i = 0; i < 19; i++) o.ffi[19 * L + i] = f[i];
      }
}

// Recolor (Source1.f90:697-732)
void recolor(Orc& o) {
  const double beta = o.p.beta;
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.walls_all[L] >= 1) continue;
        const double* f = &o.fi[19 * L];
        double* r = &o.ri[19 * L];
        double* b = &o.bi[19 * L];
        const double R = o.rhoR[L], B = o.rhoB[L], rho = o.rho[L];
        const double ratio = R / rho;
        for (int i = 0; i < 19; i++) r[i] = ratio * f[i];
        if (o.flag[L]) {
          for (int i = 1; i < 19; i++)
            r[i] = r[i] + R * B / rho * beta * o.wi[i] *
                              (o.nxv[L] * CIX[i] + o.nyv[L] * CIY[i] + o.nzv[L] * CIZ[i]);
        }
        if (R <= o.evap)
          for (int i = 0; i < 19; i++) r[i] = 0.0;
        if (B <= o.evap)
          for (int i = 0; i < 19; i++) r[i] = f[i];
        for (int i = 0; i < 19; i++) b[i] = f[i] - r[i];
      }
}

// boundary (Source1.f90:1544-1592): REFERENCE geometry only
void boundary(Orc& o) {
  if (!o.ref) return;
  sym_fi_x(o, o.ri); sym_fi_x(o, o.bi);
  sym_fi_y(o, o.ri); sym_fi_y(o, o.bi);
  sym_fi_z(o, o.ri); sym_fi_z(o, o.bi);
  {  // bottom wall z=1
    const int z = 2;
    for (int x = 1; x <= o.nx; x++)
      for (int y = 1; y <= o.ny; y++)
        for (int i = 1; i < 19; i++) {
          const int xn = Orc::wrap(x + CIX[i], o.nx), yn = Orc::wrap(y + CIY[i], o.ny),
                    zn = Orc::wrap(z + CIZ[i], o.nz);
          if (zn == 1) {
            o.ri[19 * o.lin(xn, yn, zn) + OPC[i]] = o.ri[19 * o.lin(x, y, z) + i];
            o.bi[19 * o.lin(xn, yn, zn) + OPC[i]] = o.bi[19 * o.lin(x, y, z) + i];
          }
        }
  }
  {  // back wall x=1
    const int x = 2;
    for (int y = 1; y <= o.ny; y++)
      for (int z = 1; z <= o.nz; z++)
        for (int i = 1; i < 19; i++) {
          const int xn = Orc::wrap(x + CIX[i], o.nx), yn = Orc::wrap(y + CIY[i], o.ny),
                    zn = Orc::wrap(z + CIZ[i], o.nz);
          if (xn == 1) {
            o.ri[19 * o.lin(xn, yn, zn) + OPC[i]] = o.ri[19 * o.lin(x, y, z) + i];
            o.bi[19 * o.lin(xn, yn, zn) + OPC[i]] = o.bi[19 * o.lin(x, y, z) + i];
          }
        }
  }
}

// streaming (Source1.f90:735-768): periodic pull over all nodes, i = 1..18
void streaming(Orc& o, std::vector<double>& f) {
#pragma omp parallel for schedule(static)
  for (int x = 1; x <= o.nx; x++)
    for (int y = 1; y <= o.ny; y++)
      for (int z = 1; z <= o.nz; z++) {
        const size_t L = o.lin(x, y, z);
        o.ft[19 * L] = f[19 * L];
        for (int i = 1; i < 19; i++) {
          const int j = OPC[i];
          const size_t src = o.lin(Orc::wrap(x + CIX[j], o.nx), Orc::wrap(y + CIY[j], o.ny),
                                   Orc::wrap(z + CIZ[j], o.nz));
          o.ft[19 * L + i] = f[19 * src + i];
        }
      }
  f.swap(o.ft);
}

// rigid-body velocity of particle pp at a node (curve :1009-1014)
inline void rigid_u(Orc& o, const double* centre, int pp, double xr, double yr, double zr, double uw[3]) {
  (void)centre;
  const double upx = o.C(o.s.up, pp, 0), upy = o.C(o.s.up, pp, 1), upz = o.C(o.s.up, pp, 2);
  const double rpx = o.C(o.s.rp, pp, 0), rpy = o.C(o.s.rp, pp, 1), rpz = o.C(o.s.rp, pp, 2);
  uw[0] = upx + zr * rpy - yr * rpz;
  uw[1] = upy + xr * rpz - zr * rpx;
  uw[2] = upz + yr * rpx - xr * rpy;
}

// curve (Source1.f90:990-1034): moving-particle halfway bounce-back.  CONFIG
// wall planes bounce back with zero velocity on every link into them.
void curve(Orc& o) {
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        const int pp = o.pout[L];
        if (pp < 1) continue;
        for (int i = 1; i < 19; i++) {
          const int xb = o.ref ? x - CIX[i] : Orc::wrap(x - CIX[i], o.nx);
          const int yb = o.ref ? y - CIY[i] : Orc::wrap(y - CIY[i], o.ny);
          const int zb = o.ref ? z - CIZ[i] : Orc::wrap(z - CIZ[i], o.nz);
          const size_t B = o.lin(xb, yb, zb);
          const int wb = o.walls[B];
          const bool flat = !o.ref && wb > o.par;
          if (wb == pp || flat) {
            double star = 0.0;
            if (wb <= o.par) {
              double uw[3];
              const double xr = o.disp(o.coord(x), o.C(o.s.center, wb, 0), 0);
              const double yr = o.disp(o.coord(y), o.C(o.s.center, wb, 1), 1);
              const double zr = o.disp(o.coord(z), o.C(o.s.center, wb, 2), 2);
              rigid_u(o, o.s.center, wb, xr, yr, zr, uw);
              star = uw[0] * (double)CIX[i] + uw[1] * (double)CIY[i] + uw[2] * (double)CIZ[i];
            }
            o.ri[19 * L + i] = o.ri[19 * B + OPC[i]] + 6.0 * o.wi[i] * o.rhoR[L] * star;
            o.bi[19 * L + i] = o.bi[19 * B + OPC[i]] + 6.0 * o.wi[i] * o.rhoB[L] * star;
          }
        }
      }
  if (o.ref) {
    sym_fi_x(o, o.ri); sym_fi_x(o, o.bi);
    sym_fi_y(o, o.ri); sym_fi_y(o, o.bi);
    sym_fi_z(o, o.ri); sym_fi_z(o, o.bi);
  }
}

// curve2 (Source1.f90:1036-1101): moving-particle bounce-back interpolated with
// the link fraction qq (the distance from the node to the sphere along the link
// over the link length), the wall velocity taken at the wall point.  Links into
// CONFIG wall planes keep the halfway bounce-back of curve.  One node's links
// are updated in index order, as in the reference's loop (a link may read a
// population of the same node updated before it).
void curve2(Orc& o) {
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        const int pp = o.pout[L];
        if (pp < 1) continue;
        for (int i = 1; i < 19; i++) {
          const int xb = o.ref ? x - CIX[i] : Orc::wrap(x - CIX[i], o.nx);
          const int yb = o.ref ? y - CIY[i] : Orc::wrap(y - CIY[i], o.ny);
          const int zb = o.ref ? z - CIZ[i] : Orc::wrap(z - CIZ[i], o.nz);
          const size_t B = o.lin(xb, yb, zb);
          const int wb = o.walls[B];
          if (wb == pp && pp <= o.par) {
            const int xf = o.ref ? x + CIX[i] : Orc::wrap(x + CIX[i], o.nx);
            const int yf = o.ref ? y + CIY[i] : Orc::wrap(y + CIY[i], o.ny);
            const int zf = o.ref ? z + CIZ[i] : Orc::wrap(z + CIZ[i], o.nz);
            const size_t F = o.lin(xf, yf, zf);
            const double cx = CIX[i], cy = CIY[i], cz = CIZ[i];
            const double x0 = o.disp(o.coord(x), o.C(o.s.center, pp, 0), 0);
            const double y0 = o.disp(o.coord(y), o.C(o.s.center, pp, 1), 1);
            const double z0 = o.disp(o.coord(z), o.C(o.s.center, pp, 2), 2);
            double star = cx * x0 + cy * y0 + cz * z0;
            const double R2 = o.p.rad * o.p.rad;
            double star1 = cx * cx * (R2 - y0 * y0 - z0 * z0) + cy * cy * (R2 - x0 * x0 - z0 * z0) +
                           cz * cz * (R2 - x0 * x0 - y0 * y0);
            star1 = star1 + 2.0 * (cx * cy * x0 * y0 + cy * cz * y0 * z0 + cz * cx * z0 * x0);
            star1 = std::sqrt(star1);
            const double star2 = cx * cx + cy * cy + cz * cz;
            const double xw = x0 + cx * (star1 - star) / star2;
            const double yw = y0 + cy * (star1 - star) / star2;
            const double zw = z0 + cz * (star1 - star) / star2;
            const double dis = sq(xw - x0) + sq(yw - y0) + sq(zw - z0);
            const double qq = std::sqrt(dis) / std::sqrt(star2);
            const double xr = o.disp(o.coord(x) - cx * qq, o.C(o.s.center, pp, 0), 0);
            const double yr = o.disp(o.coord(y) - cy * qq, o.C(o.s.center, pp, 1), 1);
            const double zr = o.disp(o.coord(z) - cz * qq, o.C(o.s.center, pp, 2), 2);
            double uw[3];
            rigid_u(o, o.s.center, pp, xr, yr, zr, uw);
            star = uw[0] * cx + uw[1] * cy + uw[2] * cz;
            const int j = OPC[i];
            o.ri[19 * L + i] = 1.0 / (1.0 + qq) *
                               (qq * (o.ri[19 * F + i] + o.ri[19 * B + j]) + (1.0 - qq) * o.ri[19 * L + j] +
                                6.0 * o.wi[i] * o.rhoR[L] * star);
            o.bi[19 * L + i] = 1.0 / (1.0 + qq) *
                               (qq * (o.bi[19 * F + i] + o.bi[19 * B + j]) + (1.0 - qq) * o.bi[19 * L + j] +
                                6.0 * o.wi[i] * o.rhoB[L] * star);
          } else if (wb == pp || (!o.ref && wb > o.par)) {
            // halfway (curve) for the CONFIG wall planes
            o.ri[19 * L + i] = o.ri[19 * B + OPC[i]];
            o.bi[19 * L + i] = o.bi[19 * B + OPC[i]];
          }
        }
      }
  if (o.ref) {
    sym_fi_x(o, o.ri); sym_fi_x(o, o.bi);
    sym_fi_y(o, o.ri); sym_fi_y(o, o.bi);
    sym_fi_z(o, o.ri); sym_fi_z(o, o.bi);
  }
}

// momentum (Source1.f90:1178-1261): Galilean-invariant momentum exchange.
// The reference adds the force and torque under an OpenMP REDUCTION, whose
// order of additions is left to the threads; here they are added in its loop
// order (x, y, z, i) into one accumulator per particle -- the order of a
// one-thread run, which the tests reproduce bit for bit.
void momentum(Orc& o) {
  const int P = o.par;
  std::vector<double> sums((size_t)P * 6, 0.0);
  for (int x = o.lo_x; x <= o.hi_x; x++) {
    double* acc = sums.data();
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        const int pp = o.pout[L];
        if (pp < 1 || pp > P) continue;
        for (int i = 1; i < 19; i++) {
          const int xb = o.ref ? x - CIX[i] : Orc::wrap(x - CIX[i], o.nx);
          const int yb = o.ref ? y - CIY[i] : Orc::wrap(y - CIY[i], o.ny);
          const int zb = o.ref ? z - CIZ[i] : Orc::wrap(z - CIZ[i], o.nz);
          if (o.walls[o.lin(xb, yb, zb)] != pp) continue;
          const double xr = o.disp(o.coord(x), o.C(o.s.center, pp, 0), 0);
          const double yr = o.disp(o.coord(y), o.C(o.s.center, pp, 1), 1);
          const double zr = o.disp(o.coord(z), o.C(o.s.center, pp, 2), 2);
          double uw[3];
          rigid_u(o, o.s.center, pp, xr, yr, zr, uw);
          const int j = OPC[i];
          const double f = o.fi[19 * L + i], g = o.ffi[19 * L + j];
          const double fmx = ((double)CIX[i] - uw[0]) * f - ((double)CIX[j] - uw[0]) * g;
          const double fmy = ((double)CIY[i] - uw[1]) * f - ((double)CIY[j] - uw[1]) * g;
          const double fmz = ((double)CIZ[i] - uw[2]) * f - ((double)CIZ[j] - uw[2]) * g;
          const double tqx = yr * fmz - zr * fmy;
          const double tqy = zr * fmx - xr * fmz;
          const double tqz = xr * fmy - yr * fmx;
          double* a = &acc[(pp - 1) * 6];
          a[0] = a[0] - fmx; a[1] = a[1] - fmy; a[2] = a[2] - fmz;
          a[3] = a[3] - tqx; a[4] = a[4] - tqy; a[5] = a[5] - tqz;
        }
      }
  }
  for (int pp = 1; pp <= P; pp++) {
    const double* t = &sums[(size_t)(pp - 1) * 6];
    for (int k = 0; k < 3; k++) { o.C(o.s.fp, pp, k) = t[k]; o.C(o.s.tp, pp, k) = t[3 + k]; }
  }
}

// Lagrange_points (Source1.f90:1799-1978); the per-step Laglange.dat write is not reproduced
void lagrange_points(Orc& o) {
  static const int EX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
  static const int EY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
  static const int EZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  const int P = o.par;
  const double Rad = o.p.rad, alpha = o.p.alpha;
  std::fill(o.La_flag.begin(), o.La_flag.end(), 0);
  std::fill(o.La_rhoN.begin(), o.La_rhoN.end(), 0.0);
  std::fill(o.La_nx.begin(), o.La_nx.end(), 0.0);
  std::fill(o.La_ny.begin(), o.La_ny.end(), 0.0);
  std::fill(o.La_nz.begin(), o.La_nz.end(), 0.0);
#pragma omp parallel for schedule(static)
  for (int pp = 1; pp <= P; pp++) {
    const double cx = o.C(o.s.center, pp, 0), cy = o.C(o.s.center, pp, 1), cz = o.C(o.s.center, pp, 2);
    double shb = 0.0;
    int num = 0;
    long x0 = 0, y0 = 0, z0 = 0;
    for (int na = 1; na <= o.la_m; na++)
      for (int nb = 1; nb <= o.la_n + 1; nb++) {
        const size_t q = (size_t)num * P + (pp - 1);  // (par, La_num) column-major
        const double aa = (double)(na - 1) * alpha, bb = (double)(nb - 1) * alpha;
        const double lx = cx + Rad * std::sin(bb) * std::cos(aa);
        const double ly = cy + Rad * std::sin(bb) * std::sin(aa);
        const double lz = cz + Rad * std::cos(bb);
        o.Lax[q] = lx; o.Lay[q] = ly; o.Laz[q] = lz;
        o.ds[q] = Rad * Rad * std::sin(bb) * (alpha * alpha);
        bool in_domain;
        if (o.ref) in_domain = lx < o.nx - 0.5 && ly >= 1.5 && ly < o.ny - 0.5 && lz < o.nz - 0.5;
        else in_domain = true;
        // node index of a (possibly unwrapped) node coordinate
        auto idx = [&](long c, int n, int k) -> int {
          if (o.ref) return (int)c;
          long i = c - o.origin + 1;  // 1-based, unwrapped
          const bool periodic = !(k == 0 && o.p.wall_x);
          if (periodic) { i = ((i - 1) % n + n) % n + 1; }
          else { i = std::min<long>(std::max<long>(i, 1), n); }
          return (int)i;
        };
        if (in_domain) {
          if (o.ref) { x0 = (long)lx; y0 = (long)ly; z0 = (long)lz; }  // int() truncation
          else { x0 = (long)std::floor(lx); y0 = (long)std::floor(ly); z0 = (long)std::floor(lz); }
          double wsum = 0.0, acc = 0.0;
          for (int i = 0; i < 8; i++) {
            const long xf = x0 + EX[i], yf = y0 + EY[i], zf = z0 + EZ[i];
            const size_t F = o.lin(idx(xf, o.nx, 0), idx(yf, o.ny, 1), idx(zf, o.nz, 2));
            if (o.walls[F] <= 0) {
              const double star = o.rhoN[F] + o.gx[F] * (lx - (double)xf) + o.gy[F] * (ly - (double)yf) +
                                  o.gz[F] * (lz - (double)zf);
              const double dis = sq((double)xf - lx) + sq((double)yf - ly) + sq((double)zf - lz);
              const double w = 1.0 / dis;
              acc = acc + w * star;
              wsum = wsum + w;
            }
          }
          double v = acc / wsum;
          if (v < -1.0) v = -1.0;
          if (v > 1.0) v = 1.0;
          o.La_rhoN[q] = v;
          if (std::fabs(v) < 0.99) o.La_flag[q] = 1;
        }
        if (o.La_rhoN[q] > 0.0) shb = shb + o.ds[q];
        if (o.La_flag[q]) {
          double nw[3] = {lx - cx, ly - cy, lz - cz};
          unitization(nw);
          double mn = 100.0;
          long xx = x0, yy = y0, zz = z0;
          for (int i = 0; i < 8; i++) {
            const long xf = x0 + EX[i], yf = y0 + EY[i], zf = z0 + EZ[i];
            const bool inside = o.ref ? (xf <= o.nx && yf >= 1 && yf <= o.ny && zf <= o.nz) : true;
            if (!inside) continue;
            const size_t F = o.lin(idx(xf, o.nx, 0), idx(yf, o.ny, 1), idx(zf, o.nz, 2));
            if (o.walls[F] <= 0) {
              if (std::fabs(o.nxv[F] * o.nxv[F] + o.nyv[F] * o.nyv[F] + o.nzv[F] * o.nzv[F]) > 0.0) {
                const double dis = sq((double)xf - lx) + sq((double)yf - ly) + sq((double)zf - lz);
                if (std::sqrt(dis) < mn) { mn = std::sqrt(dis); xx = xf; yy = yf; zz = zf; }
              }
            }
          }
          const size_t G = o.lin(idx(xx, o.nx, 0), idx(yy, o.ny, 1), idx(zz, o.nz, 2));
          double nt[3] = {o.nxv[G], o.nyv[G], o.nzv[G]};
          unitization(nt);
          double v[3];
          akai_rotate(o.p.cita, nw, nt, false, v);
          o.La_nx[q] = v[0]; o.La_ny[q] = v[1]; o.La_nz[q] = v[2];
        }
        num++;
      }
    o.s.shb[pp - 1] = shb;
  }
}

// capillary_force2 (Source1.f90:1980-2028)
void capillary_force2(Orc& o) {
  const int P = o.par;
  const double k = 0.134 * 1.43;
  const bool right = (o.p.cita == M_PI / 2.0);
  for (int pp = 1; pp <= P; pp++) {
    const double cx = o.C(o.s.center, pp, 0), cy = o.C(o.s.center, pp, 1), cz = o.C(o.s.center, pp, 2);
    double T[3] = {0, 0, 0}, TT[3] = {0, 0, 0};
    for (int num = 0; num < o.la_num; num++) {
      const size_t q = (size_t)num * P + (pp - 1);
      if (!o.La_flag[q]) continue;
      double nw[3] = {o.Lax[q] - cx, o.Lay[q] - cy, o.Laz[q] - cz};
      const double xr[3] = {nw[0], nw[1], nw[2]};
      unitization(nw);
      const double ie[3] = {-o.La_nx[q], -o.La_ny[q], -o.La_nz[q]};
      double temp[3], nt[3], tt[3];
      veccross(ie, nw, temp);
      const double projector = std::sqrt(temp[0] * temp[0] + temp[1] * temp[1] + temp[2] * temp[2]);
      veccross(temp, ie, nt);
      unitization(nt);
      const double rn = o.La_rhoN[q];
      const double star = 4.5 * k * o.p.beta * sq(1.0 - rn * rn) * o.ds[q] * projector;
      for (int c = 0; c < 3; c++) temp[c] = right ? star * nw[c] * o.p.sigma : star * nt[c] * o.p.sigma;
      for (int c = 0; c < 3; c++) T[c] = T[c] + temp[c];
      veccross(xr, temp, tt);
      for (int c = 0; c < 3; c++) TT[c] = TT[c] + tt[c];
    }
    for (int c = 0; c < 3; c++) { o.C(o.s.tension, pp, c) = T[c]; o.C(o.s.tension_t, pp, c) = TT[c]; }
  }
}

// repulsive (Source1.f90:1594-1671)
void repulsive(Orc& o) {
  const int P = o.par;
  const double range = 3.0, order = 0.01, Fg = o.p.fg, rad = o.p.rad;
  for (int c = 0; c < 3 * P; c++) o.s.fre[c] = 0.0;
  for (int pp = 1; pp <= P; pp++) {
    const double cx = o.C(o.s.center, pp, 0), cy = o.C(o.s.center, pp, 1), cz = o.C(o.s.center, pp, 2);
    double& fx = o.C(o.s.fre, pp, 0);
    double& fy = o.C(o.s.fre, pp, 1);
    double& fz = o.C(o.s.fre, pp, 2);
    if (o.ref) {
      const double dtop = (double)o.nz - 0.5 - cz - rad, dbot = cz - 1.5 - rad;
      const double dleft = cy - 1.5 - rad, dright = (double)o.ny - 1.5 - cy - rad;
      const double dfront = cx - 1.5 - rad, dback = (double)o.nx - 1.5 - cx - rad;
      if (dtop < range) fz = fz + 2.0 * (Fg / order) * sq(dtop - range) / sq(range);
      if (dbot < range) fz = fz - 2.0 * (Fg / order) * sq(dbot - range) / sq(range);
      if (dleft < range) fy = fy - 2.0 * (Fg / order) * sq(dleft - range) / sq(range);
      if (dright < range) fy = fy + 2.0 * (Fg / order) * sq(dright - range) / sq(range);
      if (dfront < range) fx = fx - 2.0 * (Fg / order) * sq(dfront - range) / sq(range);
      if (dback < range) fx = fx + 2.0 * (Fg / order) * sq(dback - range) / sq(range);
    } else if (o.p.wall_x) {  // CONFIG wall planes: halfway surfaces at x=0.5, x=nx-1.5
      const double dlo = cx - 0.5 - rad, dhi = (double)(o.nx - 1) - 0.5 - cx - rad;
      if (dlo < range) fx = fx - 2.0 * (Fg / order) * sq(dlo - range) / sq(range);
      if (dhi < range) fx = fx + 2.0 * (Fg / order) * sq(dhi - range) / sq(range);
    }
  }
  for (int i = 1; i <= P; i++)
    for (int j = 1; j <= P; j++) {
      if (i == j) continue;
      double d[3];
      for (int c = 0; c < 3; c++) d[c] = o.C(o.s.center, i, c) - o.C(o.s.center, j, c);
      if (!o.ref)
        for (int c = 0; c < 3; c++) {
          const int n = c == 0 ? o.nx : (c == 1 ? o.ny : o.nz);
          if (!(c == 0 && o.p.wall_x)) d[c] -= (double)n * std::nearbyint(d[c] / (double)n);
        }
      const double dis = std::sqrt(sq(d[0]) + sq(d[1]) + sq(d[2])) - rad * 2.0;
      if (dis < range)
        for (int c = 0; c < 3; c++)
          o.C(o.s.fre, i, c) = o.C(o.s.fre, i, c) - (Fg / order) * sq(dis - range) / sq(range) * d[c] / dis;
    }
}

// movement (Source1.f90:1263-1349)
void movement(Orc& o) {
  const int P = o.par;
  auto& s = o.s;
  if (o.ref) {
    for (int pp = 1; pp <= P; pp++) {
      if (std::fabs(o.C(s.center0, pp, 0) - ((double)o.nx - 0.5)) < 0.1) {
        o.C(s.fp, pp, 0) = 0.0; o.C(s.fp, pp, 1) = 2.0 * o.C(s.fp, pp, 1); o.C(s.fp, pp, 2) = 2.0 * o.C(s.fp, pp, 2);
        o.C(s.tp, pp, 0) = 2.0 * o.C(s.tp, pp, 0); o.C(s.tp, pp, 1) = 0.0; o.C(s.tp, pp, 2) = 0.0;
        o.C(s.fre, pp, 0) = 0.0;
        o.C(s.tension, pp, 0) = 0.0; o.C(s.tension, pp, 1) = o.C(s.tension, pp, 1) * 2.0;
        o.C(s.tension, pp, 2) = o.C(s.tension, pp, 2) * 2.0;
        o.C(s.tension_t, pp, 0) = 2.0 * o.C(s.tension_t, pp, 0);
        o.C(s.tension_t, pp, 1) = 0.0; o.C(s.tension_t, pp, 2) = 0.0;
      }
      const double c0y = o.C(s.center0, pp, 1);
      if (std::fabs(c0y - ((double)o.ny - 0.5)) < 0.1 || std::fabs(c0y - 1.5) < 0.1) {
        o.C(s.fp, pp, 0) = 2.0 * o.C(s.fp, pp, 0); o.C(s.fp, pp, 1) = 0.0; o.C(s.fp, pp, 2) = 2.0 * o.C(s.fp, pp, 2);
        o.C(s.tp, pp, 0) = 0.0; o.C(s.tp, pp, 1) = 2.0 * o.C(s.tp, pp, 1); o.C(s.tp, pp, 2) = 0.0;
        o.C(s.fre, pp, 1) = 0.0;
        o.C(s.tension, pp, 0) = 2.0 * o.C(s.tension, pp, 0); o.C(s.tension, pp, 1) = 0.0;
        o.C(s.tension, pp, 2) = 2.0 * o.C(s.tension, pp, 2);
        o.C(s.tension_t, pp, 0) = 0.0; o.C(s.tension_t, pp, 1) = 0.0; o.C(s.tension_t, pp, 2) = 0.0;
      }
      if (std::fabs(o.C(s.center0, pp, 2) - ((double)o.nz - 0.5)) < 0.1) {
        o.C(s.fp, pp, 0) = 2.0 * o.C(s.fp, pp, 0); o.C(s.fp, pp, 1) = 2.0 * o.C(s.fp, pp, 1); o.C(s.fp, pp, 2) = 0.0;
        o.C(s.tp, pp, 0) = 0.0; o.C(s.tp, pp, 1) = 0.0; o.C(s.tp, pp, 2) = 2.0 * o.C(s.tp, pp, 2);
        o.C(s.fre, pp, 2) = 0.0;
        o.C(s.tension, pp, 0) = o.C(s.tension, pp, 0) * 2.0; o.C(s.tension, pp, 1) = o.C(s.tension, pp, 1) * 2.0;
        o.C(s.tension, pp, 2) = 0.0;
        o.C(s.tension_t, pp, 0) = 0.0; o.C(s.tension_t, pp, 1) = 0.0;
        o.C(s.tension_t, pp, 2) = 2.0 * o.C(s.tension_t, pp, 2);
      }
    }
    for (int pp = 1; pp <= P; pp++) {
      if (pp == P / 3 + 1) {
        double t = (o.C(s.tension, pp, 0) + o.C(s.tension, pp, 2)) / 2.0;
        o.C(s.tension, pp, 0) = t; o.C(s.tension, pp, 2) = t;
        o.C(s.tension_t, pp, 1) = 0.0;
        t = (o.C(s.fp, pp, 0) + o.C(s.fp, pp, 2)) / 2.0;
        o.C(s.fp, pp, 0) = t; o.C(s.fp, pp, 2) = t;
        o.C(s.tp, pp, 1) = 0.0;
        t = (o.C(s.fre, pp, 0) + o.C(s.fre, pp, 2)) / 2.0;
        o.C(s.fre, pp, 0) = t; o.C(s.fre, pp, 2) = t;
      }
    }
  }
  const double m = o.mass, I = o.inertia;
  double F[3 * SYM_MAX_PAR];
  for (int pp = 1; pp <= P; pp++)
    for (int c = 0; c < 3; c++) {
      double f = o.C(s.fp, pp, c) + o.C(s.fre, pp, c) + o.C(s.tension, pp, c);
      if (!o.ref) f = f + m * o.p.body[c];
      F[c * P + pp - 1] = f;
      o.C(s.up, pp, c) = o.C(s.up, pp, c) + f / m;
      o.C(s.rp, pp, c) = o.C(s.rp, pp, c) + (o.C(s.tp, pp, c) + o.C(s.tension_t, pp, c)) / I;
    }
  for (int c = 0; c < 3 * P; c++) s.center_old[c] = s.center[c];
  for (int pp = 1; pp <= P; pp++)
    for (int c = 0; c < 3; c++)
      o.C(s.center, pp, c) = o.C(s.center, pp, c) + o.C(s.up, pp, c) + 0.5 * F[c * P + pp - 1] / m;
}

// refilling (Source1.f90:1351-1418)
void refilling(Orc& o) {
#pragma omp parallel for schedule(static)
  for (int x = o.lo_x; x <= o.hi_x; x++)
    for (int y = o.lo_y; y <= o.hi_y; y++)
      for (int z = o.lo_z; z <= o.hi_z; z++) {
        const size_t L = o.lin(x, y, z);
        const int pp = o.pout[L];
        if (!(pp >= 1 && o.walls_old[L] >= 1) || pp > o.par) continue;
        const double xr = o.disp(o.coord(x), o.C(o.s.center_old, pp, 0), 0);
        const double yr = o.disp(o.coord(y), o.C(o.s.center_old, pp, 1), 1);
        const double zr = o.disp(o.coord(z), o.C(o.s.center_old, pp, 2), 2);
        double uw[3];
        rigid_u(o, o.s.center_old, pp, xr, yr, zr, uw);
        o.ux[L] = uw[0]; o.uy[L] = uw[1]; o.uz[L] = uw[2];
        double sr = 0.0, sb = 0.0, num = 0.0;
        for (int i = 1; i < 19; i++) {
          const size_t nb = o.lin(Orc::wrap(x + CIX[i], o.nx), Orc::wrap(y + CIY[i], o.ny),
                                  Orc::wrap(z + CIZ[i], o.nz));
          if (o.walls_old[nb] <= 0) { sr = sr + o.rhoR[nb]; sb = sb + o.rhoB[nb]; num = num + 1.0; }
        }
        o.rhoR[L] = sr / num; o.rhoB[L] = sb / num;
        o.rho[L] = o.rhoR[L] + o.rhoB[L];
        o.rhoN[L] = (o.rhoR[L] - o.rhoB[L]) / o.rho[L];
        equilf_srt(o.wi, &o.ri[19 * L], o.rhoR[L], uw[0], uw[1], uw[2]);
        equilf_srt(o.wi, &o.bi[19 * L], o.rhoB[L], uw[0], uw[1], uw[2]);
        for (int i = 0; i < 19; i++) o.fi[19 * L + i] = o.ri[19 * L + i] + o.bi[19 * L + i];
      }
  if (o.ref) mirror_macros(o);
}

// initialization (Source1.f90:850-896), REFERENCE geometry
void initialization_ref(Orc& o) {
  const double Rad_c = 30.0;
  const double lamda_d = ((double)o.ny - 2.0) * 2.0;
  const double x0 = (double)o.nx - 0.5, z0 = (double)o.nz - 0.5;
  std::fill(o.ux.begin(), o.ux.end(), 0.0);
  std::fill(o.uy.begin(), o.uy.end(), 0.0);
  std::fill(o.uz.begin(), o.uz.end(), 0.0);
#pragma omp parallel for schedule(static)
  for (int x = 1; x <= o.nx; x++)
    for (int y = 1; y <= o.ny; y++)
      for (int z = 1; z <= o.nz; z++) {
        const size_t L = o.lin(x, y, z);
        const double dis = sq((double)x - x0) + sq((double)z - z0);
        const double dis_x = 0.1 * Rad_c * std::cos(2.0 * M_PI * ((double)y - 1.5) / lamda_d);
        const double star = Rad_c + dis_x - std::sqrt(dis);
        o.rhoN[L] = std::tanh(star * 6.0 * o.p.beta * 0.134);
        const double plus = o.p.sigma / (Rad_c + dis_x) * 3.0;
        o.rho[L] = o.rhoN[L] > 0.0 ? o.p.rho0 + plus : o.p.rho0;
        o.rhoR[L] = o.rho[L] * (o.rhoN[L] + 1.0) / 2.0;
        o.rhoB[L] = o.rho[L] - o.rhoR[L];
        equilf_srt(o.wi, &o.ri[19 * L], o.rhoR[L], 0.0, 0.0, 0.0);
        equilf_srt(o.wi, &o.bi[19 * L], o.rhoB[L], 0.0, 0.0, 0.0);
        for (int i = 0; i < 19; i++) {
          o.fi[19 * L + i] = o.ri[19 * L + i] + o.bi[19 * L + i];
          o.ffi[19 * L + i] = o.fi[19 * L + i];
        }
      }
}

// initia_center (Source1.f90:926-976), REFERENCE geometry with par=12
void initia_center(Orc& o) {
  const int P = o.par;
  const int col[3] = {4, 8, 12}, row[3] = {4, 4, 4};
  const double Rad_c = 30.0, lamda_d = ((double)o.ny - 2.0) * 2.0, rad = o.p.rad;
  const double tab = (double)(o.ny - 2) / ((double)P / 3.0 - 0.5);
  const double x0 = (double)o.nx - 0.5, z0 = (double)o.nz - 0.5;
  int num_col = 1, num = 0;
  for (int pp = 1; pp <= P; pp++) {
    num = num + 1;
    if (num_col <= 3 && pp > col[num_col - 1]) num_col = num_col + 1;
    const double a = 0.0 - (double)(num_col - 1) * M_PI / 4.0;
    double b;
    if (num_col % 2 == 0) b = 1.5 + ((double)num - 1.0) * tab;
    else b = 1.5 + ((double)num - 0.5) * tab;
    if (num_col <= 3 && num == row[num_col - 1]) num = 0;
    const double dis_x = 0.1 * Rad_c * std::cos(2.0 * M_PI * (b - 1.5) / lamda_d);
    double star = Rad_c + dis_x;
    star = std::sqrt(rad * rad + star * star + 2.0 * rad * star * std::cos(o.p.cita));
    o.C(o.s.center, pp, 0) = x0 - star * std::cos(a);
    o.C(o.s.center, pp, 1) = b;
    o.C(o.s.center, pp, 2) = z0 + star * std::sin(a);
  }
  for (int c = 0; c < 3 * P; c++) o.s.center0[c] = o.s.center[c];
}

// CONFIG: equilibrium fill from a phase field and a density field (the fill of :883-894)
void init_phase(Orc& o, const double* phi, const double* rho) {
  std::fill(o.ux.begin(), o.ux.end(), 0.0);
  std::fill(o.uy.begin(), o.uy.end(), 0.0);
  std::fill(o.uz.begin(), o.uz.end(), 0.0);
#pragma omp parallel for schedule(static)
  for (long L = 0; L < (long)o.N; L++) {
    o.rhoN[L] = phi[L];
    o.rho[L] = rho[L];
    o.rhoR[L] = o.rho[L] * (o.rhoN[L] + 1.0) / 2.0;
    o.rhoB[L] = o.rho[L] - o.rhoR[L];
    equilf_srt(o.wi, &o.ri[19 * L], o.rhoR[L], 0.0, 0.0, 0.0);
    equilf_srt(o.wi, &o.bi[19 * L], o.rhoB[L], 0.0, 0.0, 0.0);
    for (int i = 0; i < 19; i++) {
      o.fi[19 * L + i] = o.ri[19 * L + i] + o.bi[19 * L + i];
      o.ffi[19 * L + i] = o.fi[19 * L + i];
    }
  }
}

void has_particles_step(Orc& o) {
  lagrange_points(o);
  capillary_force2(o);
  momentum(o);
  repulsive(o);
  movement(o);
}

// one loop body of main (Source1.f90:216-251), output gate excluded
void step(Orc& o) {
  calmacros(o);
  if (o.par > 0) has_particles_step(o);
  set_walls(o);
  if (o.par > 0) refilling(o);
  derivatives(o);
  collision(o);
  recolor(o);
  boundary(o);
  streaming(o, o.ri);
  streaming(o, o.bi);
  if (o.p.bounce) curve2(o);
  else curve(o);
}

}  // namespace

// ------------------------------------------------------------------------
// C API for ctypes (tests/, bench.py cpu_baseline)
extern "C" {

void* orc_create(const sym_params* p) {
  Orc* o = new Orc();
  o->p = *p;
  o->nx = p->nx; o->ny = p->ny; o->nz = p->nz;
  o->N = (size_t)p->nx * p->ny * p->nz;
  o->ref = p->mode == SYM_MODE_REFERENCE;
  o->origin = o->ref ? 1 : 0;
  if (o->ref) {
    o->lo_x = 2; o->hi_x = o->nx - 1; o->lo_y = 2; o->hi_y = o->ny - 1; o->lo_z = 2; o->hi_z = o->nz - 1;
  } else {
    o->lo_x = 1; o->hi_x = o->nx; o->lo_y = 1; o->hi_y = o->ny; o->lo_z = 1; o->hi_z = o->nz;
  }
  o->par = p->par;
  o->la_m = p->la_m > 0 ? p->la_m : (int)(2.0 * M_PI / p->alpha);
  o->la_n = p->la_n > 0 ? p->la_n : (int)(M_PI / p->alpha);
  o->la_num = o->par > 0 ? o->la_m * (o->la_n + 1) : 0;
  o->evap = p->evap_lim > 0 ? p->evap_lim : 1.0e-8;
  o->mass = p->mass > 0 ? p->mass : 4.0 / 3.0 * p->rho_p * M_PI * (p->rad * p->rad * p->rad);
  o->inertia = p->inertia > 0 ? p->inertia : 2.0 / 5.0 * o->mass * (p->rad * p->rad);
  o->wi[0] = 1.0 / 3.0;
  for (int i = 1; i <= 6; i++) o->wi[i] = 1.0 / 18.0;
  for (int i = 7; i < 19; i++) o->wi[i] = 1.0 / 36.0;
  for (int r = 0; r < 19; r++)
    for (int c = 0; c < 19; c++) o->M[r][c] = moment_row(r, c);
  for (int i = 0; i < 19; i++)  // M_inv(i,j) = M(j,i)/DOT_PRODUCT(M(j,:),M(j,:)) (:126-130)
    for (int j = 0; j < 19; j++) {
      double nrm = 0.0;
      for (int c = 0; c < 19; c++) nrm += o->M[j][c] * o->M[j][c];
      o->Minv[i][j] = o->M[j][i] / nrm;
    }
  const size_t N = o->N;
  for (auto* v : {&o->walls, &o->walls_old, &o->walls_all, &o->pin, &o->pout, &o->flag}) v->assign(N, 0);
  for (auto* v : {&o->rho, &o->ux, &o->uy, &o->uz, &o->rhoN, &o->rhoR, &o->rhoB, &o->nxv, &o->nyv, &o->nzv,
                  &o->gx, &o->gy, &o->gz})
    v->assign(N, 0.0);
  for (auto* v : {&o->fi, &o->ffi, &o->ri, &o->bi, &o->ft}) v->assign(19 * N, 0.0);
  std::memset(&o->s, 0, sizeof(o->s));
  const size_t NL = (size_t)o->la_num * o->par;
  for (auto* v : {&o->Lax, &o->Lay, &o->Laz, &o->La_rhoN, &o->La_nx, &o->La_ny, &o->La_nz, &o->ds})
    v->assign(NL, 0.0);
  o->La_flag.assign(NL, 0);
  return o;
}

void orc_destroy(void* h) { delete (Orc*)h; }

// Access to internal arrays by name: returns a pointer and element count.
void* orc_array(void* h, const char* name, int64_t* count, int32_t* is_int) {
  Orc* o = (Orc*)h;
  struct D { const char* n; std::vector<double>* v; };
  struct I { const char* n; std::vector<int32_t>* v; };
  D ds[] = {{"rho", &o->rho}, {"ux", &o->ux}, {"uy", &o->uy}, {"uz", &o->uz}, {"rho_N", &o->rhoN},
            {"rho_R", &o->rhoR}, {"rho_B", &o->rhoB}, {"n_x", &o->nxv}, {"n_y", &o->nyv}, {"n_z", &o->nzv},
            {"gradx", &o->gx}, {"grady", &o->gy}, {"gradz", &o->gz}, {"fi", &o->fi}, {"ffi", &o->ffi},
            {"ri", &o->ri}, {"bi", &o->bi}, {"Lax", &o->Lax}, {"Lay", &o->Lay}, {"Laz", &o->Laz},
            {"La_rhoN", &o->La_rhoN}, {"La_nx", &o->La_nx}, {"La_ny", &o->La_ny}, {"La_nz", &o->La_nz},
            {"ds", &o->ds}};
  I is[] = {{"walls", &o->walls}, {"walls_old", &o->walls_old}, {"walls_all", &o->walls_all},
            {"pin", &o->pin}, {"pout", &o->pout}, {"flag", &o->flag}, {"La_flag", &o->La_flag}};
  for (auto& d : ds)
    if (!std::strcmp(d.n, name)) { *count = (int64_t)d.v->size(); *is_int = 0; return d.v->data(); }
  for (auto& d : is)
    if (!std::strcmp(d.n, name)) { *count = (int64_t)d.v->size(); *is_int = 1; return d.v->data(); }
  *count = 0;
  return nullptr;
}

sym_particles* orc_particles(void* h) { return &((Orc*)h)->s; }
void orc_matrices(void* h, double* M, double* Minv) {
  Orc* o = (Orc*)h;
  for (int r = 0; r < 19; r++)
    for (int c = 0; c < 19; c++) { M[r * 19 + c] = o->M[r][c]; Minv[r * 19 + c] = o->Minv[r][c]; }
}
int orc_la_num(void* h) { return ((Orc*)h)->la_num; }
void orc_tables(int32_t* t, double* w) {
  for (int i = 0; i < 19; i++) {
    t[i] = CIX[i]; t[19 + i] = CIY[i]; t[38 + i] = CIZ[i]; t[57 + i] = OPC[i];
    t[76 + i] = SYMX[i]; t[95 + i] = SYMY[i]; t[114 + i] = SYMZ[i];
  }
  Orc tmp;
  for (int i = 0; i < 19; i++) w[i] = i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
  (void)tmp;
}

void orc_set_walls(void* h) { set_walls(*(Orc*)h); }
void orc_calmacros(void* h) { calmacros(*(Orc*)h); }
void orc_derivatives(void* h) { derivatives(*(Orc*)h); }
void orc_collision(void* h) { collision(*(Orc*)h); }
void orc_recolor(void* h) { recolor(*(Orc*)h); }
void orc_boundary(void* h) { boundary(*(Orc*)h); }
void orc_streaming(void* h, int which) { Orc* o = (Orc*)h; streaming(*o, which == 0 ? o->ri : o->bi); }
void orc_curve(void* h) {
  Orc& o = *(Orc*)h;
  if (o.p.bounce) curve2(o);
  else curve(o);
}
void orc_lagrange_points(void* h) { lagrange_points(*(Orc*)h); }
void orc_capillary_force2(void* h) { capillary_force2(*(Orc*)h); }
void orc_momentum(void* h) { momentum(*(Orc*)h); }
void orc_repulsive(void* h) { repulsive(*(Orc*)h); }
void orc_movement(void* h) { movement(*(Orc*)h); }
void orc_refilling(void* h) { refilling(*(Orc*)h); }
void orc_initialization(void* h) { initialization_ref(*(Orc*)h); }
void orc_initia_center(void* h) { initia_center(*(Orc*)h); }
void orc_init_phase(void* h, const double* phi, const double* rho) { init_phase(*(Orc*)h, phi, rho); }
void orc_step(void* h, int n) {
  for (int t = 0; t < n; t++) step(*(Orc*)h);
}
int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// output3 (Source1.f90:1673-1717), REFERENCE geometry
void orc_output3(void* h, double* hmin_out, int32_t* y0_out) {
  Orc& o = *(Orc*)h;
  const int x = o.nx - 1;
  double hmin = (double)o.nz;
  int y0 = 0;
  std::vector<double> bottom(o.ny + 1, 1.0);
  const double top = (double)o.nz - 0.5;
  for (int y = 2; y <= o.ny - 1; y++)
    for (int z = 2; z <= o.nz - 1; z++) {
      const size_t L = o.lin(x, y, z);
      if (o.pout[L] == 0 && o.walls_all[L] == 0) {
        const int zn = z + 1;
        const size_t Ln = o.lin(x, y, zn);
        if (o.pout[Ln] == 0 && o.walls_all[Ln] == 0)
          if (o.rhoN[L] * o.rhoN[Ln] < 0.0) bottom[y] = (double)zn - o.rhoN[Ln] / (o.rhoN[Ln] - o.rhoN[L]);
      }
    }
  for (int y = 2; y <= o.ny - 1; y++) {
    const double hh = top - bottom[y];
    if (hh < hmin) { hmin = hh; y0 = y; }
  }
  *hmin_out = hmin;
  *y0_out = y0;
}

// output4 field sums (Source1.f90:1729-1750) on the arrays of the last
// calmacros: out[0] = sum (rho - rho0)/3 and out[1] = sum rho |u|^2 / 2 over
// red fluid nodes, out[2] = fluid nodes with a fluid neighbour of the other
// colour.  The reference's walls_all(z,y,z), rho(z,y,z), uz(z,y,z) (:1736,
// :1739) are read at (z,y,x).  REFERENCE: x,y,z in 2..n-1 (:1730-1732);
// CONFIG: every node with periodic neighbours.
void orc_energy(void* h, double* out) {
  Orc& o = *(Orc*)h;
  double epv = 0.0, emov = 0.0, area = 0.0;
  const int lo = o.ref ? 2 : 1, dx = o.ref ? 1 : 0;
  for (int x = lo; x <= o.nx - dx; x++)
    for (int y = lo; y <= o.ny - dx; y++)
      for (int z = lo; z <= o.nz - dx; z++) {
        const size_t L = o.lin(x, y, z);
        if (o.walls_all[L] > 0) continue;
        if (o.rhoN[L] > 0.0) {
          epv = epv + (o.rho[L] - o.p.rho0) / 3.0;
          emov = emov + 0.5 * o.rho[L] * (sq(o.ux[L]) + sq(o.uy[L]) + sq(o.uz[L]));
        }
        for (int i = 1; i < 19; i++) {
          int xn = x + CIX[i], yn = y + CIY[i], zn = z + CIZ[i];
          if (!o.ref) { xn = Orc::wrap(xn, o.nx); yn = Orc::wrap(yn, o.ny); zn = Orc::wrap(zn, o.nz); }
          const size_t Ln = o.lin(xn, yn, zn);
          if (o.rhoN[L] * o.rhoN[Ln] < 0.0 && o.walls_all[Ln] <= 0) {
            area = area + 1.0;
            break;
          }
        }
      }
  out[0] = epv;
  out[1] = emov;
  out[2] = area;
}

// CONFIG stop rule: min_z sqrt(sum_xy (1+phi)/2 / pi), phi = rho_N after calmacros
double orc_neck_radius(void* h) {
  Orc& o = *(Orc*)h;
  double mn = 1e300;
  for (int z = 1; z <= o.nz; z++) {
    double s = 0.0;
    for (int x = 1; x <= o.nx; x++)
      for (int y = 1; y <= o.ny; y++) {
        const size_t L = o.lin(x, y, z);
        if (o.walls_all[L] <= 0) s += (1.0 + o.rhoN[L]) * 0.5;
      }
    mn = std::min(mn, std::sqrt(s / M_PI));
  }
  return mn;
}

}  // extern "C"
