// lattice.cuh -- D3Q19 constants and per-node physics shared by every kernel.
//
// Constants are constexpr functions so that, inside fully unrolled loops, the
// compiler folds them to immediates: the 19x19 moment transform becomes ~200
// adds/multiplies with no zero terms and no memory operands.
#pragma once
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>
#include "../../include/symmetry.h"

namespace symb200 {

// D3Q19 velocities, opposites, mirror maps (Source1.f90:132-138)
__host__ __device__ __forceinline__ constexpr int CX(int i) {
  constexpr int a[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int CY(int i) {
  constexpr int a[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int CZ(int i) {
  constexpr int a[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int OPC(int i) {
  constexpr int a[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int SYMX(int i) {
  constexpr int a[19] = {0, 2, 1, 3, 4, 5, 6, 8, 7, 10, 9, 12, 11, 14, 13, 15, 16, 17, 18};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int SYMY(int i) {
  constexpr int a[19] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 16, 15, 18, 17};
  return a[i];
}
__host__ __device__ __forceinline__ constexpr int SYMZ(int i) {
  constexpr int a[19] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
  return a[i];
}
// weights wi (Source1.f90:140-142)
__host__ __device__ __forceinline__ constexpr double W(int i) {
  return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// Moment matrix rows (the polynomials behind the data statement at
// Source1.f90:105-123; row order rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx,
// 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz).
__host__ __device__ __forceinline__ constexpr double MROW(int r, int c) {
  const double x = CX(c), y = CY(c), z = CZ(c);
  const double c2 = x * x + y * y + z * z;
  return r == 0 ? 1.0
       : r == 1 ? 19.0 * c2 - 30.0
       : r == 2 ? (21.0 * c2 * c2 - 53.0 * c2 + 24.0) / 2.0
       : r == 3 ? x
       : r == 4 ? (5.0 * c2 - 9.0) * x
       : r == 5 ? y
       : r == 6 ? (5.0 * c2 - 9.0) * y
       : r == 7 ? z
       : r == 8 ? (5.0 * c2 - 9.0) * z
       : r == 9 ? 3.0 * x * x - c2
       : r == 10 ? (3.0 * c2 - 5.0) * (3.0 * x * x - c2)
       : r == 11 ? y * y - z * z
       : r == 12 ? (3.0 * c2 - 5.0) * (y * y - z * z)
       : r == 13 ? x * y
       : r == 14 ? y * z
       : r == 15 ? x * z
       : r == 16 ? (y * y - z * z) * x
       : r == 17 ? (z * z - x * x) * y
       : (x * x - y * y) * z;
}
// squared row norms |M(j,:)|^2: 19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8
__host__ __device__ __forceinline__ constexpr double MNORM(int r) {
  constexpr double a[19] = {19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8};
  return a[r];
}
// M_inv(i,j) = M(j,i) / |M(j,:)|^2 (Source1.f90:126-130)
__host__ __device__ __forceinline__ constexpr double MINV(int i, int j) { return MROW(j, i) / MNORM(j); }

// ---------------------------------------------------------------------------
// Device view of the parameters (filled on the host from sym_params).
struct DevParams {
  int nx, ny, nz;
  long long N;
  int ref;                 // REFERENCE geometry
  int origin;              // node coordinate = 0-based index + origin
  int lo[3], hi[3];        // update range, 0-based inclusive, per axis (x,y,z)
  int wall_x;
  int par, la_m, la_n, la_num;
  int bounce;              // 0 halfway bounce-back (curve), 1 interpolated (curve2)
  double rho0, nu_r, nu_b;
  double s_e, s_eps, s_q, s_pi, s_m;
  double sigma, beta, cita;
  double body[3];
  double rad, mass, inertia, fg, alpha, evap;
  double sin_cita, cos_cita;   // of the contact angle (fused path)
  double inu_r, inu_b;     // 1/nu_r, 1/nu_b (fused path)
};

template <typename T>
__device__ __forceinline__ T wrapi(T v, T n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// a / b: IEEE division in FP64; in FP32 arithmetic (the FP32 and 16-bit
// storage paths) the fast reciprocal-based quotient (2 ulp), whose error is far
// below the storage rounding
template <typename R>
__device__ __forceinline__ R qdiv(R a, R b) { return a / b; }
template <>
__device__ __forceinline__ float qdiv<float>(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ long long lin(const DevParams& P, int x, int y, int z) {
  return (long long)z + (long long)P.nz * ((long long)y + (long long)P.ny * (long long)x);
}

// Displacement of node coordinate c from centre `cen` along axis k (minimum
// image in periodic CONFIG axes).
__device__ __forceinline__ double disp(const DevParams& P, double c, double cen, int k) {
  double d = c - cen;
  if (!P.ref) {
    const int n = k == 0 ? P.nx : (k == 1 ? P.ny : P.nz);
    const bool periodic = !(k == 0 && P.wall_x);
    if (periodic) d -= (double)n * nearbyint(d / (double)n);
  }
  return d;
}

// equilf (Source1.f90:397-450): equilibrium moments and Guo forcing moments.
// EXACT keeps the reference's divisions by 1.5; the fused path multiplies by
// 2/3 instead (same value up to one rounding).
template <typename R, bool EXACT = true>
__device__ __forceinline__ void equilf(R meq[19], R fk[19], R rho, R ux, R uy, R uz, R fx, R fy, R fz) {
  const R usqr = ux * ux + uy * uy + uz * uz;
  meq[0] = R(1);
  meq[1] = R(19) * usqr - R(11);
  meq[2] = R(3) - R(5.5) * usqr;
  meq[3] = ux;
  meq[4] = EXACT ? -ux / R(1.5) : ux * R(-2.0 / 3.0);
  meq[5] = uy;
  meq[6] = EXACT ? -uy / R(1.5) : uy * R(-2.0 / 3.0);
  meq[7] = uz;
  meq[8] = EXACT ? -uz / R(1.5) : uz * R(-2.0 / 3.0);
  meq[9] = R(3) * ux * ux - usqr;
  meq[10] = R(-0.5) * (R(3) * ux * ux - usqr);
  meq[11] = uy * uy - uz * uz;
  meq[12] = R(-0.5) * (uy * uy - uz * uz);
  meq[13] = ux * uy;
  meq[14] = uy * uz;
  meq[15] = ux * uz;
  meq[16] = R(0);
  meq[17] = R(0);
  meq[18] = R(0);
#pragma unroll
  for (int k = 0; k < 19; k++) meq[k] = rho * meq[k];
  const R uf = ux * fx + uy * fy + uz * fz;
  fk[0] = R(0);
  fk[1] = R(38) * uf;
  fk[2] = R(-11) * uf;
  fk[3] = fx;
  fk[4] = EXACT ? -fx / R(1.5) : fx * R(-2.0 / 3.0);
  fk[5] = fy;
  fk[6] = EXACT ? -fy / R(1.5) : fy * R(-2.0 / 3.0);
  fk[7] = fz;
  fk[8] = EXACT ? -fz / R(1.5) : fz * R(-2.0 / 3.0);
  fk[9] = R(6) * ux * fx - R(2) * uf;
  fk[10] = -(R(3) * ux * fx - uf);
  fk[11] = R(2) * (uy * fy - uz * fz);
  fk[12] = -(uy * fy - uz * fz);
  fk[13] = ux * fy + uy * fx;
  fk[14] = uy * fz + uz * fy;
  fk[15] = ux * fz + uz * fx;
  fk[16] = R(0);
  fk[17] = R(0);
  fk[18] = R(0);
}

// equilf_SRT (Source1.f90:833-848)
template <typename R>
__device__ __forceinline__ R feq_srt(int i, R rho, R ux, R uy, R uz, R usqr) {
  const R uc = ux * R(CX(i)) + uy * R(CY(i)) + uz * R(CZ(i));
  return rho * R(W(i)) * (R(1) + R(3) * uc + R(4.5) * uc * uc - R(1.5) * usqr);
}

// node-local relaxation rates (Source1.f90:674-684, runtime MRT rates)
template <typename R>
__device__ __forceinline__ void node_rates(const DevParams& P, R rhoN, R& su, R& se, R& seps, R& sq, R& spi, R& sm) {
  R nu;
  if (rhoN <= R(-1)) nu = R(P.nu_b);
  else if (rhoN >= R(1)) nu = R(P.nu_r);
  else nu = R(2) / ((R(1) + rhoN) / R(P.nu_r) + (R(1) - rhoN) / R(P.nu_b));
  su = R(1) / (R(3) * nu + R(0.5));
  const R sq_ = R(8) * (R(2) - su) / (R(8) - su);
  se = P.s_e > 0 ? R(P.s_e) : su;
  seps = P.s_eps > 0 ? R(P.s_eps) : su;
  sq = P.s_q > 0 ? R(P.s_q) : sq_;
  spi = P.s_pi > 0 ? R(P.s_pi) : su;
  sm = P.s_m > 0 ? R(P.s_m) : sq_;
}

// The same rates with two divisions (fused path): with phi clamped to
// [-1, 1] and D = (1+phi)/nu_r + (1-phi)/nu_b, nu = 2/D gives the branches
// of the reference at the ends, so su = 1/(3 nu + 1/2) = 2D/(12 + D).
template <typename R>
__device__ __forceinline__ void node_rates_fast(const DevParams& P, R rhoN, R& su, R& se, R& seps, R& sq, R& spi,
                                                R& sm) {
  const R ph = fmin(fmax(rhoN, R(-1)), R(1));
  const R D = (R(1) + ph) * R(P.inu_r) + (R(1) - ph) * R(P.inu_b);
  su = qdiv<R>(R(2) * D, R(12) + D);
  const R sq_ = qdiv<R>(R(8) * (R(2) - su), R(8) - su);
  se = P.s_e > 0 ? R(P.s_e) : su;
  seps = P.s_eps > 0 ? R(P.s_eps) : su;
  sq = P.s_q > 0 ? R(P.s_q) : sq_;
  spi = P.s_pi > 0 ? R(P.s_pi) : su;
  sm = P.s_m > 0 ? R(P.s_m) : sq_;
}

// MRT collision with Guo forcing in moment space on f[0..18] in place
// (collision :685-688): m = M f; m -= s (m - meq) - (1 - s/2) fk; f = M^-1 m.
template <typename R>
__device__ __forceinline__ void mrt_collide(const DevParams& P, R f[19], R rho, R ux, R uy, R uz, R fx, R fy,
                                            R fz, R rhoN) {
  R su, se, seps, sq, spi, sm;
  node_rates<R>(P, rhoN, su, se, seps, sq, spi, sm);
  R m[19];
#pragma unroll
  for (int r = 0; r < 19; r++) {
    R acc = R(0);
#pragma unroll
    for (int c = 0; c < 19; c++) {
      constexpr double zero = 0.0;
      if (MROW(r, c) != zero) {
        if (MROW(r, c) == 1.0) acc = acc + f[c];
        else if (MROW(r, c) == -1.0) acc = acc - f[c];
        else acc = acc + R(MROW(r, c)) * f[c];
      }
    }
    m[r] = acc;
  }
  R meq[19], fk[19];
  equilf<R>(meq, fk, rho, ux, uy, uz, fx, fy, fz);
  const R s[19] = {R(1), se, seps, R(1), sq, R(1), sq, R(1), sq, su, spi, su, spi, su, su, su, sm, sm, sm};
#pragma unroll
  for (int k = 0; k < 19; k++) m[k] = m[k] - s[k] * (m[k] - meq[k]) + (R(1) - R(0.5) * s[k]) * fk[k];
#pragma unroll
  for (int r = 0; r < 19; r++) {
    R acc = R(0);
#pragma unroll
    for (int c = 0; c < 19; c++) {
      if (MINV(r, c) != 0.0) acc = acc + R(MINV(r, c)) * m[c];
    }
    f[r] = acc;
  }
}

// The same collision in the opposite-pair basis (fused path).  Row r of M is
// even (M(r,opc(c)) = M(r,c)) or odd (= -M(r,c)) under velocity reversal, so
// with p_k = f_i + f_opc(i) and q_k = f_i - f_opc(i) over the 9 pairs the even
// moments need only p (and f_0) and the odd ones only q; back-transformed,
// f_i = E_i + O_i and f_opc(i) = E_i - O_i with E (O) the sum over even (odd)
// rows.  Half the multiply-adds of the dense form; the result differs from it
// only by rounding order.
__host__ __device__ __forceinline__ constexpr int PREP(int k) {   // pair representatives, k = 0..8
  constexpr int a[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
  return a[k];
}
__host__ __device__ __forceinline__ constexpr bool MEVEN(int r) {
  for (int c = 0; c < 19; c++)
    if (MROW(r, OPC(c)) != MROW(r, c)) return false;
  return true;
}

// rows relaxed with the fixed rate 1 (density, momentum)
__host__ __device__ __forceinline__ constexpr bool MCONS(int r) { return r == 0 || r == 3 || r == 5 || r == 7; }

template <int... Is, typename F>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
// f(std::integral_constant<int, i>) for i = 0..N-1: i is a constant expression
// inside f, so every coefficient below is folded by the front end
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <typename R>
__device__ __forceinline__ void mrt_collide_pairs(const DevParams& P, R f[19], R rho, R ux, R uy, R uz, R fx, R fy,
                                                  R fz, R rhoN) {
  R su, se, seps, sq, spi, sm;
  node_rates_fast<R>(P, rhoN, su, se, seps, sq, spi, sm);
  R pp[9], qq[9];
  static_for<9>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    pp[k] = f[PREP(k)] + f[OPC(PREP(k))];
    qq[k] = f[PREP(k)] - f[OPC(PREP(k))];
  });
  R m[19];
  static_for<19>([&](auto rc) {
    constexpr int r = decltype(rc)::value;
    constexpr bool even = MEVEN(r);
    R acc = R(0);
    if constexpr (MCONS(r)) return;   // relaxed with rate 1: not needed (below)
    if constexpr (even && MROW(r, 0) != 0.0) acc = R(MROW(r, 0)) * f[0];
    static_for<9>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      constexpr double c = MROW(r, PREP(k));
      const R v = even ? pp[k] : qq[k];
      if constexpr (c == 1.0) acc = acc + v;
      else if constexpr (c == -1.0) acc = acc - v;
      else if constexpr (c != 0.0) acc = acc + R(c) * v;
    });
    m[r] = acc;
  });
  R meq[19], fk[19];
  equilf<R, false>(meq, fk, rho, ux, uy, uz, fx, fy, fz);
  const R s[19] = {R(1), se, seps, R(1), sq, R(1), sq, R(1), sq, su, spi, su, spi, su, su, su, sm, sm, sm};
  // density and momentum relax with rate 1 (:684): m - (m - meq) + fk/2 = meq + fk/2
  static_for<19>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if constexpr (MCONS(k)) m[k] = meq[k] + R(0.5) * fk[k];
    else m[k] = m[k] - s[k] * (m[k] - meq[k]) + (R(1) - R(0.5) * s[k]) * fk[k];
  });
  static_for<9>([&](auto kc) {
    constexpr int i = PREP(decltype(kc)::value);
    R e = R(0), o = R(0);
    static_for<19>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      if constexpr (MINV(i, r) != 0.0) {
        if constexpr (MEVEN(r)) e = e + R(MINV(i, r)) * m[r];
        else o = o + R(MINV(i, r)) * m[r];
      }
    });
    f[i] = e + o;
    f[OPC(i)] = e - o;
  });
  if constexpr (sizeof(R) == 4) {
    // FP32 arithmetic: the rest population closes the mass balance, so the
    // post-collision populations sum to rho up to the rounding of these
    // additions.  The rounded inverse-transform coefficients would otherwise
    // bias every node's mass the same way, step after step (a drift of about
    // 1e-9 per step).
    R s = R(0);
#pragma unroll
    for (int i = 1; i < 19; i++) s = s + f[i];
    f[0] = rho - s;
  } else {
    R e = R(0);
    static_for<19>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      if constexpr (MEVEN(r) && MINV(0, r) != 0.0) e = e + R(MINV(0, r)) * m[r];
    });
    f[0] = e;
  }
}

// Link fraction of curve2 (Source1.f90:1055-1070): node at displacement
// (x0,y0,z0) from the centre of a sphere of radius rad, link c pointing out of
// the sphere: qq = distance from the node back along -c to the sphere surface,
// over |c|.
__device__ __forceinline__ double link_fraction(double x0, double y0, double z0, double cx, double cy, double cz,
                                                double rad) {
  const double star = cx * x0 + cy * y0 + cz * z0;
  const double R2 = rad * rad;
  double star1 = cx * cx * (R2 - y0 * y0 - z0 * z0) + cy * cy * (R2 - x0 * x0 - z0 * z0) +
                 cz * cz * (R2 - x0 * x0 - y0 * y0);
  star1 = star1 + 2.0 * (cx * cy * x0 * y0 + cy * cz * y0 * z0 + cz * cx * z0 * x0);
  star1 = sqrt(star1);
  const double star2 = cx * cx + cy * cy + cz * cz;
  const double xw = x0 + cx * (star1 - star) / star2;
  const double yw = y0 + cy * (star1 - star) / star2;
  const double zw = z0 + cz * (star1 - star) / star2;
  const double dis = (xw - x0) * (xw - x0) + (yw - y0) * (yw - y0) + (zw - z0) * (zw - z0);
  return sqrt(dis) / sqrt(star2);
}

__device__ __forceinline__ void unitization(double a[3]) {
  double star = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  star = sqrt(star);
  a[0] = a[0] / star; a[1] = a[1] / star; a[2] = a[2] / star;
}
__device__ __forceinline__ void veccross(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = -(a[0] * b[2] - a[2] * b[0]);
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Akai-2018 rotation toward the contact angle (derivatives :547-587,
// Lagrange_points :1921-1947; the Lagrange copy has no parallel guard, :1929)
//
// In FP32 arithmetic (the FP32 and 16-bit storage paths) cos(theta) and
// sin(theta) are taken as nw.n and |nw x n| (equal to the reference's
// cos(acos(.)) and sin(acos(.)) for unit vectors) with sin(theta) held at or
// above sin(1e-5) at both ends: in single precision nw.n rounds to exactly +-1
// for angles up to ~3.5e-4, where the acos form divides by sin(0) = 0.
// FP64 keeps the reference's expressions unchanged.
template <typename R>
__device__ __forceinline__ void akai_rotate_sc(R sc, R cc, const R nw[3], const R n[3], bool guard, R out[3]);
template <typename R>
__device__ __forceinline__ void akai_rotate(R cita, const R nw[3], const R n[3], bool guard, R out[3]) {
  akai_rotate_sc<R>(sin(cita), cos(cita), nw, n, guard, out);
}
// the same with sin(cita) and cos(cita) given
template <typename R>
__device__ __forceinline__ void akai_rotate_sc(R sc, R cc, const R nw[3], const R n[3], bool guard, R out[3]) {
  const R mx = fmax(fabs(nw[0] - n[0]), fmax(fabs(nw[1] - n[1]), fabs(nw[2] - n[2])));
  R ct, st;
  if (sizeof(R) == 4) {
    if (guard && mx < R(1e-5)) {
      ct = cos(R(1e-5));
      st = sin(R(1e-5));
    } else {
      const R cx = nw[1] * n[2] - nw[2] * n[1], cy = nw[2] * n[0] - nw[0] * n[2], cz = nw[0] * n[1] - nw[1] * n[0];
      ct = fmin(fmax(nw[0] * n[0] + nw[1] * n[1] + nw[2] * n[2], R(-1)), R(1));
      st = fmax(sqrt(cx * cx + cy * cy + cz * cz), R(1e-5));
    }
  } else {
    R theta;
    if (guard && mx < R(1e-5)) theta = R(1e-5);
    else theta = acos(nw[0] * n[0] + nw[1] * n[1] + nw[2] * n[2]);
    ct = cos(theta);
    st = sin(theta);
  }
  const R a1 = cc - sc * ct / st;
  const R a2 = cc + sc * ct / st;
  const R b1 = sc / st;
  const R b2 = -sc / st;
  R v1[3], v2[3];
#pragma unroll
  for (int k = 0; k < 3; k++) { v1[k] = a1 * nw[k] + b1 * n[k]; v2[k] = a2 * nw[k] + b2 * n[k]; }
  const R db1 = (v1[0] - n[0]) * (v1[0] - n[0]) + (v1[1] - n[1]) * (v1[1] - n[1]) + (v1[2] - n[2]) * (v1[2] - n[2]);
  const R db2 = (v2[0] - n[0]) * (v2[0] - n[0]) + (v2[1] - n[1]) * (v2[1] - n[1]) + (v2[2] - n[2]) * (v2[2] - n[2]);
  if (db1 < db2) { out[0] = v1[0]; out[1] = v1[1]; out[2] = v1[2]; }
  else { out[0] = v2[0]; out[1] = v2[1]; out[2] = v2[2]; }
}

// wall normal for solid object `id` seen from node (x,y,z) (0-based indices)
__device__ __forceinline__ void wall_normal_dev(const DevParams& P, const sym_particles* S, int id, int x, int y,
                                                int z, double nw[3]) {
  if (id <= P.par) {
    const int par = P.par;
    nw[0] = disp(P, (double)(x + P.origin), S->center[0 * par + id - 1], 0);
    nw[1] = disp(P, (double)(y + P.origin), S->center[1 * par + id - 1], 1);
    nw[2] = disp(P, (double)(z + P.origin), S->center[2 * par + id - 1], 2);
    unitization(nw);
  } else {
    nw[0] = (id == P.par + 1) ? 1.0 : -1.0;
    nw[1] = 0.0; nw[2] = 0.0;
  }
}

}  // namespace symb200
