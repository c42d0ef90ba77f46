// ref_kernels.cu -- the reference's per-timestep subroutines as device kernels
// on the canonical state (FP64 SoA arrays mirroring the reference's arrays).
//
// These kernels keep the reference's subroutine boundaries one to one so that
// each Fortran call site maps to one library call (the drop-in path).  Each
// kernel cites the loop it replaces.  Indices are 0-based: a reference node
// (x,y,z) (1-based) is (x-1,y-1,z-1) here.
#include <cstdio>
#include <vector>
#include "state.cuh"

namespace symb200 {

namespace {

constexpr int TPB = 256;

inline unsigned blocks_for(long long n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

// thread t -> node of the update range (z fastest)
__device__ __forceinline__ bool range_node(const DevParams& P, long long t, int& x, int& y, int& z) {
  const int rx = P.hi[0] - P.lo[0] + 1, ry = P.hi[1] - P.lo[1] + 1, rz = P.hi[2] - P.lo[2] + 1;
  if (t >= (long long)rx * ry * rz) return false;
  z = P.lo[2] + (int)(t % rz);
  t /= rz;
  y = P.lo[1] + (int)(t % ry);
  x = P.lo[0] + (int)(t / ry);
  return true;
}
inline long long range_count(const DevParams& P) {
  return (long long)(P.hi[0] - P.lo[0] + 1) * (P.hi[1] - P.lo[1] + 1) * (P.hi[2] - P.lo[2] + 1);
}

__device__ __forceinline__ long long nbr(const DevParams& P, int x, int y, int z, int i) {
  return lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
}

// ---- mirror-plane copies (symmetry_X/Y/Z_phi/_u/_fi, Source1.f90:1443-1542) ----
// Copy plane `src` onto plane `dst` along `axis` for every node of the other two axes.
__device__ __forceinline__ bool plane_node(const DevParams& P, int axis, int t, int dst, int src, long long& Ld,
                                           long long& Ls) {
  int a, b, na, nb;
  if (axis == 0) { na = P.ny; nb = P.nz; }
  else if (axis == 1) { na = P.nx; nb = P.nz; }
  else { na = P.nx; nb = P.ny; }
  if (t >= na * nb) return false;
  a = t / nb; b = t % nb;
  if (axis == 0) { Ld = lin(P, dst, a, b); Ls = lin(P, src, a, b); }
  else if (axis == 1) { Ld = lin(P, a, dst, b); Ls = lin(P, a, src, b); }
  else { Ld = lin(P, a, b, dst); Ls = lin(P, a, b, src); }
  return true;
}
template <typename T>
__global__ void k_plane_scalar(DevParams P, T* v, int axis, int dst, int src) {
  long long Ld, Ls;
  if (plane_node(P, axis, blockIdx.x * blockDim.x + threadIdx.x, dst, src, Ld, Ls)) v[Ld] = v[Ls];
}
__global__ void k_plane_u(DevParams P, double* a, double* b, double* c, int axis, int dst, int src) {
  long long Ld, Ls;
  if (!plane_node(P, axis, blockIdx.x * blockDim.x + threadIdx.x, dst, src, Ld, Ls)) return;
  a[Ld] = axis == 0 ? -a[Ls] : a[Ls];
  b[Ld] = axis == 1 ? -b[Ls] : b[Ls];
  c[Ld] = axis == 2 ? -c[Ls] : c[Ls];
}
__global__ void k_plane_pop(DevParams P, double* f, int axis, int dst, int src) {
  long long Ld, Ls;
  if (!plane_node(P, axis, blockIdx.x * blockDim.x + threadIdx.x, dst, src, Ld, Ls)) return;
  const long long N = P.N;
  double tmp[19];
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const int s = axis == 0 ? SYMX(i) : (axis == 1 ? SYMY(i) : SYMZ(i));
    tmp[i] = f[s * N + Ls];
  }
#pragma unroll
  for (int i = 0; i < 19; i++) f[i * N + Ld] = tmp[i];
}

int plane_threads(const DevParams& P, int axis) {
  return axis == 0 ? P.ny * P.nz : (axis == 1 ? P.nx * P.nz : P.nx * P.ny);
}
template <typename T>
void mirror_scalar(sym_handle* h, T* v, int axis) {
  const DevParams& P = h->dp;
  const int n = axis == 0 ? P.nx : (axis == 1 ? P.ny : P.nz);
  const unsigned g = blocks_for(plane_threads(P, axis));
  k_plane_scalar<T><<<g, TPB, 0, h->st>>>(P, v, axis, n - 1, n - 2);
  if (axis == 1) k_plane_scalar<T><<<g, TPB, 0, h->st>>>(P, v, axis, 0, 1);
}
void mirror_u(sym_handle* h, double* a, double* b, double* c, int axis) {
  const DevParams& P = h->dp;
  const int n = axis == 0 ? P.nx : (axis == 1 ? P.ny : P.nz);
  const unsigned g = blocks_for(plane_threads(P, axis));
  k_plane_u<<<g, TPB, 0, h->st>>>(P, a, b, c, axis, n - 1, n - 2);
  if (axis == 1) k_plane_u<<<g, TPB, 0, h->st>>>(P, a, b, c, axis, 0, 1);
}
void mirror_pop(sym_handle* h, double* f, int axis) {
  const DevParams& P = h->dp;
  const int n = axis == 0 ? P.nx : (axis == 1 ? P.ny : P.nz);
  const unsigned g = blocks_for(plane_threads(P, axis));
  k_plane_pop<<<g, TPB, 0, h->st>>>(P, f, axis, n - 1, n - 2);
  if (axis == 1) k_plane_pop<<<g, TPB, 0, h->st>>>(P, f, axis, 0, 1);
}

// ---- calmacros (Source1.f90:770-831) --------------------------------------
__global__ void k_calmacros(DevParams P, const double* __restrict__ ri, const double* __restrict__ bi,
                            double* __restrict__ fi, double* rho, double* ux, double* uy, double* uz, double* rhoN,
                            double* rhoR, double* rhoB, const int32_t* __restrict__ walls_all) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  if (walls_all[L] >= 1) {
    rhoN[L] = 0.0; ux[L] = 0.0; uy[L] = 0.0; uz[L] = 0.0; rho[L] = P.rho0;
    return;
  }
  double f[19], sr = 0.0, sb = 0.0;
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const double r = ri[i * N + L], b = bi[i * N + L];
    f[i] = r + b;
    fi[i * N + L] = f[i];
    sr = sr + r;
  }
#pragma unroll
  for (int i = 0; i < 19; i++) sb = sb + bi[i * N + L];
  rhoR[L] = sr; rhoB[L] = sb;
  const double rh = sr + sb;
  rho[L] = rh;
  double mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
  for (int i = 0; i < 19; i++) {
    if (CX(i)) mx = mx + f[i] * (double)CX(i);
    if (CY(i)) my = my + f[i] * (double)CY(i);
    if (CZ(i)) mz = mz + f[i] * (double)CZ(i);
  }
  ux[L] = mx / rh; uy[L] = my / rh; uz[L] = mz / rh;
  rhoN[L] = (sr - sb) / rh;
}

void mirror_macros(sym_handle* h, bool with_fi) {
  for (int ax = 0; ax < 3; ax++) {
    mirror_scalar(h, h->rhoN, ax); mirror_scalar(h, h->rhoR, ax); mirror_scalar(h, h->rhoB, ax);
    mirror_scalar(h, h->rho, ax); mirror_u(h, h->ux, h->uy, h->uz, ax);
    if (with_fi) mirror_pop(h, h->fi, ax);
  }
}

// ---- derivatives (Source1.f90:452-597) ------------------------------------
__global__ void k_pin_fill(DevParams P, const int32_t* __restrict__ pin, const int32_t* __restrict__ walls_all,
                           double* rhoN) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z);
  if (pin[L] <= 0) return;
  double ws = 0.0, v = 0.0;
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const long long nb = nbr(P, x, y, z, i);
    if (walls_all[nb] <= 0) { ws = ws + W(i); v = v + W(i) * rhoN[nb]; }
  }
  rhoN[L] = v / ws;
}

__global__ void k_gradient(DevParams P, const int32_t* __restrict__ walls_all, const double* __restrict__ rhoN,
                           double* gx, double* gy, double* gz, double* nx, double* ny, double* nz, int32_t* flag) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z);
  double g0 = 0.0, g1 = 0.0, g2 = 0.0, n0 = 0.0, n1 = 0.0, n2 = 0.0;
  int fl = 0;
  if (walls_all[L] <= 0) {
#pragma unroll
    for (int i = 1; i < 19; i++) {
      const double val = W(i) * rhoN[nbr(P, x, y, z, i)];
      if (CX(i)) g0 = g0 + val * (double)CX(i);
      if (CY(i)) g1 = g1 + val * (double)CY(i);
      if (CZ(i)) g2 = g2 + val * (double)CZ(i);
    }
    g0 = 3.0 * g0; g1 = 3.0 * g1; g2 = 3.0 * g2;
    const double fnorm = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
    if (fnorm > P.evap) { n0 = g0 / fnorm; n1 = g1 / fnorm; n2 = g2 / fnorm; fl = 1; }
  }
  gx[L] = g0; gy[L] = g1; gz[L] = g2; nx[L] = n0; ny[L] = n1; nz[L] = n2; flag[L] = fl;
}

__global__ void k_wetting(DevParams P, const sym_particles* __restrict__ S, const int32_t* __restrict__ pout,
                          const int32_t* __restrict__ flag, double* gx, double* gy, double* gz, double* nx, double* ny,
                          double* nz) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z);
  const int pp = pout[L];
  if (!(pp >= 1 && flag[L])) return;
  double nw[3], n[3] = {nx[L], ny[L], nz[L]}, v[3];
  wall_normal_dev(P, S, pp, x, y, z, nw);
  akai_rotate<double>(P.cita, nw, n, true, v);
  nx[L] = v[0]; ny[L] = v[1]; nz[L] = v[2];
  const double fnorm = sqrt(gx[L] * gx[L] + gy[L] * gy[L] + gz[L] * gz[L]);
  gx[L] = fnorm * v[0]; gy[L] = fnorm * v[1]; gz[L] = fnorm * v[2];
}

// ---- collision (Source1.f90:599-695) --------------------------------------
__global__ void __launch_bounds__(128) k_collision(
    DevParams P, const int32_t* __restrict__ walls_all, const int32_t* __restrict__ pout,
    const int32_t* __restrict__ flag, const double* __restrict__ nxv, const double* __restrict__ nyv,
    const double* __restrict__ nzv, const double* __restrict__ gx, const double* __restrict__ gy,
    const double* __restrict__ gz, const double* __restrict__ rho, const double* __restrict__ rhoN, double* ux,
    double* uy, double* uz, double* fi, double* ffi) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  if (walls_all[L] > 0) return;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  const bool edge_ok = P.ref ? (z >= 2 && x >= 2) : true;  // z>=3 .and. x>=3 (1-based), :624
  if (flag[L] && pout[L] <= 0 && edge_ok) {
    double d00 = 0, d01 = 0, d02 = 0, d10 = 0, d11 = 0, d12 = 0, d20 = 0, d21 = 0, d22 = 0;
#pragma unroll
    for (int i = 1; i < 19; i++) {
      const long long nb = nbr(P, x, y, z, i);
      double tmp = W(i) * nxv[nb];
      if (CX(i)) d00 = d00 + tmp * (double)CX(i);
      if (CY(i)) d01 = d01 + tmp * (double)CY(i);
      if (CZ(i)) d02 = d02 + tmp * (double)CZ(i);
      tmp = W(i) * nyv[nb];
      if (CX(i)) d10 = d10 + tmp * (double)CX(i);
      if (CY(i)) d11 = d11 + tmp * (double)CY(i);
      if (CZ(i)) d12 = d12 + tmp * (double)CZ(i);
      tmp = W(i) * nzv[nb];
      if (CX(i)) d20 = d20 + tmp * (double)CX(i);
      if (CY(i)) d21 = d21 + tmp * (double)CY(i);
      if (CZ(i)) d22 = d22 + tmp * (double)CZ(i);
    }
    d00 *= 3.0; d01 *= 3.0; d02 *= 3.0; d10 *= 3.0; d11 *= 3.0; d12 *= 3.0; d20 *= 3.0; d21 *= 3.0; d22 *= 3.0;
    const double nx = nxv[L], ny = nyv[L], nz = nzv[L];
    const double kurv = nx * ny * (d10 + d01) + nx * nz * (d20 + d02) + ny * nz * (d12 + d21) -
                        (ny * ny + nz * nz) * d00 - (nx * nx + nz * nz) * d11 - (nx * nx + ny * ny) * d22;
    const double val = 0.5 * P.sigma * kurv;
    fx = val * gx[L]; fy = val * gy[L]; fz = val * gz[L];
  }
  const double rh = rho[L];
  if (!P.ref) { fx = fx + rh * P.body[0]; fy = fy + rh * P.body[1]; fz = fz + rh * P.body[2]; }
  const double u0 = ux[L] + 0.5 * fx / rh, u1 = uy[L] + 0.5 * fy / rh, u2 = uz[L] + 0.5 * fz / rh;
  ux[L] = u0; uy[L] = u1; uz[L] = u2;
  double f[19];
#pragma unroll
  for (int i = 0; i < 19; i++) f[i] = fi[i * N + L];
  mrt_collide<double>(P, f, rh, u0, u1, u2, fx, fy, fz, rhoN[L]);
#pragma unroll
  for (int i = 0; i < 19; i++) { fi[i * N + L] = f[i]; ffi[i * N + L] = f[i]; }
}

// ---- Recolor (Source1.f90:697-732) ----------------------------------------
__global__ void k_recolor(DevParams P, const int32_t* __restrict__ walls_all, const int32_t* __restrict__ flag,
                          const double* __restrict__ fi, double* ri, double* bi, const double* __restrict__ rhoR,
                          const double* __restrict__ rhoB, const double* __restrict__ rho,
                          const double* __restrict__ nxv, const double* __restrict__ nyv,
                          const double* __restrict__ nzv) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  if (walls_all[L] >= 1) return;
  const double R = rhoR[L], B = rhoB[L], rh = rho[L];
  const double ratio = R / rh;
  const bool fl = flag[L] != 0;
  const double coef = R * B / rh * P.beta;
  const double n0 = nxv[L], n1 = nyv[L], n2 = nzv[L];
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const double f = fi[i * N + L];
    double r = ratio * f;
    if (i > 0 && fl) r = r + coef * W(i) * (n0 * (double)CX(i) + n1 * (double)CY(i) + n2 * (double)CZ(i));
    if (R <= P.evap) r = 0.0;
    if (B <= P.evap) r = f;
    ri[i * N + L] = r;
    bi[i * N + L] = f - r;
  }
}

// ---- boundary (Source1.f90:1544-1592), REFERENCE geometry -------------------
__global__ void k_bb_bottom(DevParams P, double* ri, double* bi) {  // bottom wall z=1 (1-based)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.nx * P.ny) return;
  const int x = t / P.ny, y = t % P.ny, z = 1;
  const long long N = P.N, L = lin(P, x, y, z);
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const int zn = wrapi(z + CZ(i), P.nz);
    if (zn == 0) {
      const long long Ln = lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), zn);
      ri[OPC(i) * N + Ln] = ri[i * N + L];
      bi[OPC(i) * N + Ln] = bi[i * N + L];
    }
  }
}
__global__ void k_bb_back(DevParams P, double* ri, double* bi) {  // back wall x=1 (1-based)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.ny * P.nz) return;
  const int y = t / P.nz, z = t % P.nz, x = 1;
  const long long N = P.N, L = lin(P, x, y, z);
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const int xn = wrapi(x + CX(i), P.nx);
    if (xn == 0) {
      const long long Ln = lin(P, xn, wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
      ri[OPC(i) * N + Ln] = ri[i * N + L];
      bi[OPC(i) * N + Ln] = bi[i * N + L];
    }
  }
}

// ---- streaming (Source1.f90:735-768): periodic pull, i = 1..18 ---------------
__global__ void k_stream_pull(DevParams P, const double* __restrict__ f, double* __restrict__ ft) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz), y = (int)((L / P.nz) % P.ny), x = (int)(L / ((long long)P.nz * P.ny));
  const long long N = P.N;
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const long long src = lin(P, wrapi(x - CX(i), P.nx), wrapi(y - CY(i), P.ny), wrapi(z - CZ(i), P.nz));
    ft[i * N + L] = f[i * N + src];
  }
}

// ---- curve (Source1.f90:990-1034) -----------------------------------------
__global__ void k_curve(DevParams P, const sym_particles* __restrict__ S, const int32_t* __restrict__ walls,
                        const int32_t* __restrict__ pout, double* ri, double* bi, const double* __restrict__ rhoR,
                        const double* __restrict__ rhoB) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  const int pp = pout[L];
  if (pp < 1) return;
  const int par = P.par;
#pragma unroll 1
  for (int i = 1; i < 19; i++) {
    const int xb = P.ref ? x - CX(i) : wrapi(x - CX(i), P.nx);
    const int yb = P.ref ? y - CY(i) : wrapi(y - CY(i), P.ny);
    const int zb = P.ref ? z - CZ(i) : wrapi(z - CZ(i), P.nz);
    const long long B = lin(P, xb, yb, zb);
    const int wb = walls[B];
    const bool flat = !P.ref && wb > par;
    if (wb == pp || flat) {
      double star = 0.0;
      if (wb <= par) {
        const double xr = disp(P, (double)(x + P.origin), S->center[0 * par + wb - 1], 0);
        const double yr = disp(P, (double)(y + P.origin), S->center[1 * par + wb - 1], 1);
        const double zr = disp(P, (double)(z + P.origin), S->center[2 * par + wb - 1], 2);
        const double* up = S->up;
        const double* rp = S->rp;
        const double uw0 = up[0 * par + wb - 1] + zr * rp[1 * par + wb - 1] - yr * rp[2 * par + wb - 1];
        const double uw1 = up[1 * par + wb - 1] + xr * rp[2 * par + wb - 1] - zr * rp[0 * par + wb - 1];
        const double uw2 = up[2 * par + wb - 1] + yr * rp[0 * par + wb - 1] - xr * rp[1 * par + wb - 1];
        star = uw0 * (double)CX(i) + uw1 * (double)CY(i) + uw2 * (double)CZ(i);
      }
      const int j = OPC(i);
      ri[i * N + L] = ri[j * N + B] + 6.0 * W(i) * rhoR[L] * star;
      bi[i * N + L] = bi[j * N + B] + 6.0 * W(i) * rhoB[L] * star;
    }
  }
}

// curve2 (Source1.f90:1036-1101): bounce-back interpolated with the link
// fraction, the wall velocity at the wall point; one thread per node updates
// its links in index order like the reference's loop.  CONFIG wall planes keep
// the halfway bounce-back.
__global__ void k_curve2(DevParams P, const sym_particles* __restrict__ S, const int32_t* __restrict__ walls,
                         const int32_t* __restrict__ pout, double* ri, double* bi, const double* __restrict__ rhoR,
                         const double* __restrict__ rhoB) {
  int x, y, z;
  if (!range_node(P, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  const int pp = pout[L];
  if (pp < 1) return;
  const int par = P.par;
#pragma unroll 1
  for (int i = 1; i < 19; i++) {
    const int xb = P.ref ? x - CX(i) : wrapi(x - CX(i), P.nx);
    const int yb = P.ref ? y - CY(i) : wrapi(y - CY(i), P.ny);
    const int zb = P.ref ? z - CZ(i) : wrapi(z - CZ(i), P.nz);
    const long long B = lin(P, xb, yb, zb);
    const int wb = walls[B];
    const int j = OPC(i);
    if (wb == pp && pp <= par) {
      const int xf = P.ref ? x + CX(i) : wrapi(x + CX(i), P.nx);
      const int yf = P.ref ? y + CY(i) : wrapi(y + CY(i), P.ny);
      const int zf = P.ref ? z + CZ(i) : wrapi(z + CZ(i), P.nz);
      const long long F = lin(P, xf, yf, zf);
      const double cx = CX(i), cy = CY(i), cz = CZ(i);
      const double* c = S->center;
      const double x0 = disp(P, (double)(x + P.origin), c[0 * par + pp - 1], 0);
      const double y0 = disp(P, (double)(y + P.origin), c[1 * par + pp - 1], 1);
      const double z0 = disp(P, (double)(z + P.origin), c[2 * par + pp - 1], 2);
      const double qq = link_fraction(x0, y0, z0, cx, cy, cz, P.rad);
      const double xr = disp(P, (double)(x + P.origin) - cx * qq, c[0 * par + pp - 1], 0);
      const double yr = disp(P, (double)(y + P.origin) - cy * qq, c[1 * par + pp - 1], 1);
      const double zr = disp(P, (double)(z + P.origin) - cz * qq, c[2 * par + pp - 1], 2);
      const double* up = S->up;
      const double* rp = S->rp;
      const double uw0 = up[0 * par + pp - 1] + zr * rp[1 * par + pp - 1] - yr * rp[2 * par + pp - 1];
      const double uw1 = up[1 * par + pp - 1] + xr * rp[2 * par + pp - 1] - zr * rp[0 * par + pp - 1];
      const double uw2 = up[2 * par + pp - 1] + yr * rp[0 * par + pp - 1] - xr * rp[1 * par + pp - 1];
      const double star = uw0 * cx + uw1 * cy + uw2 * cz;
      ri[i * N + L] = 1.0 / (1.0 + qq) *
                      (qq * (ri[i * N + F] + ri[j * N + B]) + (1.0 - qq) * ri[j * N + L] + 6.0 * W(i) * rhoR[L] * star);
      bi[i * N + L] = 1.0 / (1.0 + qq) *
                      (qq * (bi[i * N + F] + bi[j * N + B]) + (1.0 - qq) * bi[j * N + L] + 6.0 * W(i) * rhoB[L] * star);
    } else if (wb == pp || (!P.ref && wb > par)) {
      ri[i * N + L] = ri[j * N + B];
      bi[i * N + L] = bi[j * N + B];
    }
  }
}

// ---- initial state -----------------------------------------------------------
// initialization (Source1.f90:850-896), REFERENCE geometry
__global__ void k_initialization(DevParams P, double* rhoN, double* rho, double* rhoR, double* rhoB, double* ux,
                                 double* uy, double* uz, double* ri, double* bi, double* fi, double* ffi) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz) + 1, y = (int)((L / P.nz) % P.ny) + 1,
            x = (int)(L / ((long long)P.nz * P.ny)) + 1;  // 1-based like the reference
  const double Rad_c = 30.0, lamda_d = ((double)P.ny - 2.0) * 2.0;
  const double x0 = (double)P.nx - 0.5, z0 = (double)P.nz - 0.5;
  const double dis = ((double)x - x0) * ((double)x - x0) + ((double)z - z0) * ((double)z - z0);
  const double dis_x = 0.1 * Rad_c * cos(2.0 * M_PI * ((double)y - 1.5) / lamda_d);
  const double star = Rad_c + dis_x - sqrt(dis);
  const double phi = tanh(star * 6.0 * P.beta * 0.134);
  const double plus = P.sigma / (Rad_c + dis_x) * 3.0;
  const double rh = phi > 0.0 ? P.rho0 + plus : P.rho0;
  const double R = rh * (phi + 1.0) / 2.0;
  const double B = rh - R;
  rhoN[L] = phi; rho[L] = rh; rhoR[L] = R; rhoB[L] = B; ux[L] = 0.0; uy[L] = 0.0; uz[L] = 0.0;
  const long long N = P.N;
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const double r = feq_srt<double>(i, R, 0.0, 0.0, 0.0, 0.0), b = feq_srt<double>(i, B, 0.0, 0.0, 0.0, 0.0);
    ri[i * N + L] = r; bi[i * N + L] = b;
    if (fi) { fi[i * N + L] = r + b; ffi[i * N + L] = r + b; }
  }
}

// equilibrium fill from rhoN and rho (the fill of :883-894)
__global__ void k_init_fill(DevParams P, const double* rhoN, const double* rho, double* rhoR, double* rhoB,
                            double* ux, double* uy, double* uz, double* ri, double* bi, double* fi, double* ffi) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= P.N) return;
  const double phi = rhoN[L], rh = rho[L];
  const double R = rh * (phi + 1.0) / 2.0;
  const double B = rh - R;
  rhoR[L] = R; rhoB[L] = B; ux[L] = 0.0; uy[L] = 0.0; uz[L] = 0.0;
  const long long N = P.N;
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const double r = feq_srt<double>(i, R, 0.0, 0.0, 0.0, 0.0), b = feq_srt<double>(i, B, 0.0, 0.0, 0.0, 0.0);
    ri[i * N + L] = r; bi[i * N + L] = b;
    if (fi) { fi[i * N + L] = r + b; ffi[i * N + L] = r + b; }
  }
}

// splitmix64 finaliser (Steele, Lea, Flood 2014)
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  unsigned long long z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double node_noise(long long L, double amp, unsigned long long seed) {
  const unsigned long long hsh = splitmix64(seed ^ (unsigned long long)L);
  const double u = (double)(hsh >> 11) * 0x1.0p-53;
  return u * (2.0 * amp) - amp;
}
// CONFIG Rayleigh-Plateau thread along z (same formula as configs.thread_phase)
__global__ void k_init_thread(DevParams P, double* rhoN, double* rho, double radius, double amp, double wavelength,
                              double width, double noise, unsigned long long seed) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz), y = (int)((L / P.nz) % P.ny), x = (int)(L / ((long long)P.nz * P.ny));
  const double xc = (P.nx - 1) / 2.0, yc = (P.ny - 1) / 2.0;
  const double rz = radius * (1.0 + amp * cos(2.0 * M_PI * (double)z / wavelength));
  const double d = sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
  double phi = tanh(2.0 * (rz - d) / width);
  if (noise > 0) phi = phi + node_noise(L, noise, seed);
  phi = fmin(fmax(phi, -1.0), 1.0);
  rhoN[L] = phi;
  rho[L] = phi > 0.0 ? P.rho0 + 3.0 * P.sigma / rz : P.rho0;
}
__global__ void k_init_slab(DevParams P, double* rhoN, double* rho, double z0, double z1, double width, double noise,
                            unsigned long long seed) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz);
  const double dz = fmin((double)z - z0, z1 - (double)z);
  double phi = tanh(2.0 * dz / width);
  if (noise > 0) phi = phi + node_noise(L, noise, seed);
  phi = fmin(fmax(phi, -1.0), 1.0);
  rhoN[L] = phi;
  rho[L] = P.rho0;
}

// ---- diagnostics -----------------------------------------------------------
// deterministic block reduction of doubles (fixed tree for a fixed blockDim)
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// per-z-plane sum of (1+phi)/2 over fluid nodes: one block per z
__global__ void k_plane_red(DevParams P, const double* __restrict__ rhoN, const int32_t* __restrict__ walls_all,
                            double* out) {
  __shared__ double sh[256];
  const int z = blockIdx.x;
  double s = 0.0;
  for (int t = threadIdx.x; t < P.nx * P.ny; t += 256) {
    const int x = t / P.ny, y = t % P.ny;
    const long long L = lin(P, x, y, z);
    if (walls_all[L] <= 0) s += (1.0 + rhoN[L]) * 0.5;
  }
  s = block_sum<256>(s, sh);
  if (threadIdx.x == 0) out[z] = s;
}

// output3 (Source1.f90:1686-1699): per y, the last phi sign change along z on plane x = xl-1
__global__ void k_output3(DevParams P, const double* __restrict__ rhoN, const int32_t* __restrict__ walls_all,
                          const int32_t* __restrict__ pout, double* bottom) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x + 1;  // 0-based y = 1..ny-2
  if (y > P.ny - 2) return;
  const int x = P.nx - 2;
  double b = 1.0;
  for (int z = 1; z <= P.nz - 2; z++) {
    const long long L = lin(P, x, y, z);
    if (pout[L] == 0 && walls_all[L] == 0) {
      const long long Ln = lin(P, x, y, z + 1);
      if (pout[Ln] == 0 && walls_all[Ln] == 0)
        if (rhoN[L] * rhoN[Ln] < 0.0) b = (double)(z + 2) - rhoN[Ln] / (rhoN[Ln] - rhoN[L]);
    }
  }
  bottom[y] = b;
}

// FP64 mass and momentum over fluid nodes: per-block partials
__global__ void k_mass_mom(DevParams P, const double* __restrict__ ri, const double* __restrict__ bi,
                           const int32_t* __restrict__ walls_all, double* part) {
  __shared__ double sh[256];
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  double v[5] = {0, 0, 0, 0, 0};
  if (L < P.N && walls_all[L] <= 0) {
    const long long N = P.N;
#pragma unroll
    for (int i = 0; i < 19; i++) {
      const double r = ri[i * N + L], b = bi[i * N + L], f = r + b;
      v[0] += r; v[1] += b;
      v[2] += f * CX(i); v[3] += f * CY(i); v[4] += f * CZ(i);
    }
  }
  for (int k = 0; k < 5; k++) {
    const double s = block_sum<256>(v[k], sh);
    if (threadIdx.x == 0) part[blockIdx.x * 5LL + k] = s;
  }
}
__global__ void k_sum_partials(const double* part, long long nblk, int width, double* out) {
  __shared__ double sh[256];
  for (int k = 0; k < width; k++) {
    double s = 0.0;
    for (long long b = threadIdx.x; b < nblk; b += 256) s += part[b * width + k];
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) out[k] = s;
  }
}

__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, long long N) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 19 * N) return;
  const long long L = t / 19;
  const int i = (int)(t % 19);
  soa[i * N + L] = aos[t];
}
__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, long long N) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 19 * N) return;
  const long long L = t / 19;
  const int i = (int)(t % 19);
  aos[t] = soa[i * N + L];
}

}  // namespace

// ===========================================================================
// host launchers
int ref_calmacros(sym_handle* h) {
  const DevParams& P = h->dp;
  k_calmacros<<<blocks_for(range_count(P)), TPB, 0, h->st>>>(P, h->ri, h->bi, h->fi, h->rho, h->ux, h->uy, h->uz,
                                                              h->rhoN, h->rhoR, h->rhoB, h->walls_all);
  if (P.ref) {
    k_plane_scalar<double><<<blocks_for(plane_threads(P, 2)), TPB, 0, h->st>>>(P, h->rhoN, 2, 0, 1);  // z=1 wall
    k_plane_scalar<double><<<blocks_for(plane_threads(P, 0)), TPB, 0, h->st>>>(P, h->rhoN, 0, 0, 1);  // x=1 wall
    mirror_macros(h, true);
  }
  return check_cuda(h, cudaGetLastError(), "calmacros");
}

int ref_derivatives(sym_handle* h) {
  const DevParams& P = h->dp;
  const unsigned g = blocks_for(range_count(P));
  k_pin_fill<<<g, TPB, 0, h->st>>>(P, h->pin, h->walls_all, h->rhoN);
  if (P.ref)
    for (int ax = 0; ax < 3; ax++) mirror_scalar(h, h->rhoN, ax);
  k_gradient<<<g, TPB, 0, h->st>>>(P, h->walls_all, h->rhoN, h->gx, h->gy, h->gz, h->nx, h->ny, h->nz, h->flag);
  k_wetting<<<g, TPB, 0, h->st>>>(P, h->dpart, h->pout, h->flag, h->gx, h->gy, h->gz, h->nx, h->ny, h->nz);
  if (P.ref) {
    for (int ax = 0; ax < 3; ax++) mirror_u(h, h->nx, h->ny, h->nz, ax);
    for (int ax = 0; ax < 3; ax++) mirror_u(h, h->gx, h->gy, h->gz, ax);
  }
  return check_cuda(h, cudaGetLastError(), "derivatives");
}

int ref_collision(sym_handle* h) {
  const DevParams& P = h->dp;
  k_collision<<<blocks_for(range_count(P), 128), 128, 0, h->st>>>(P, h->walls_all, h->pout, h->flag, h->nx, h->ny,
                                                                   h->nz, h->gx, h->gy, h->gz, h->rho, h->rhoN,
                                                                   h->ux, h->uy, h->uz, h->fi, h->ffi);
  return check_cuda(h, cudaGetLastError(), "collision");
}

int ref_recolor(sym_handle* h) {
  const DevParams& P = h->dp;
  k_recolor<<<blocks_for(range_count(P)), TPB, 0, h->st>>>(P, h->walls_all, h->flag, h->fi, h->ri, h->bi, h->rhoR,
                                                            h->rhoB, h->rho, h->nx, h->ny, h->nz);
  return check_cuda(h, cudaGetLastError(), "recolor");
}

int ref_boundary(sym_handle* h) {
  const DevParams& P = h->dp;
  if (!P.ref) return SYM_OK;
  for (int ax = 0; ax < 3; ax++) { mirror_pop(h, h->ri, ax); mirror_pop(h, h->bi, ax); }
  k_bb_bottom<<<blocks_for((long long)P.nx * P.ny), TPB, 0, h->st>>>(P, h->ri, h->bi);
  k_bb_back<<<blocks_for((long long)P.ny * P.nz), TPB, 0, h->st>>>(P, h->ri, h->bi);
  return check_cuda(h, cudaGetLastError(), "boundary");
}

int ref_streaming(sym_handle* h, int which) {
  const DevParams& P = h->dp;
  double* f = which == 0 ? h->ri : h->bi;
  k_stream_pull<<<blocks_for(P.N), TPB, 0, h->st>>>(P, f, h->ft);
  cudaMemcpyAsync(f + P.N, h->ft + P.N, sizeof(double) * 18 * P.N, cudaMemcpyDeviceToDevice, h->st);
  return check_cuda(h, cudaGetLastError(), "streaming");
}

int ref_curve(sym_handle* h) {
  const DevParams& P = h->dp;
  if (P.bounce)
    k_curve2<<<blocks_for(range_count(P)), TPB, 0, h->st>>>(P, h->dpart, h->walls, h->pout, h->ri, h->bi, h->rhoR,
                                                             h->rhoB);
  else
    k_curve<<<blocks_for(range_count(P)), TPB, 0, h->st>>>(P, h->dpart, h->walls, h->pout, h->ri, h->bi, h->rhoR,
                                                            h->rhoB);
  if (P.ref)
    for (int ax = 0; ax < 3; ax++) { mirror_pop(h, h->ri, ax); mirror_pop(h, h->bi, ax); }
  return check_cuda(h, cudaGetLastError(), "curve");
}

int ref_initialization(sym_handle* h) {
  const DevParams& P = h->dp;
  k_initialization<<<blocks_for(P.N), TPB, 0, h->st>>>(P, h->rhoN, h->rho, h->rhoR, h->rhoB, h->ux, h->uy, h->uz,
                                                        h->ri, h->bi, h->fi, h->ffi);
  return check_cuda(h, cudaGetLastError(), "initialization");
}

int ref_init_fill(sym_handle* h) {
  const DevParams& P = h->dp;
  k_init_fill<<<blocks_for(P.N), TPB, 0, h->st>>>(P, h->rhoN, h->rho, h->rhoR, h->rhoB, h->ux, h->uy, h->uz, h->ri,
                                                   h->bi, h->fi, h->ffi);
  return check_cuda(h, cudaGetLastError(), "init_fill");
}

int ref_init_thread(sym_handle* h, double radius, double amp, double wavelength, double width, double noise,
                    unsigned long long seed) {
  const DevParams& P = h->dp;
  k_init_thread<<<blocks_for(P.N), TPB, 0, h->st>>>(P, h->rhoN, h->rho, radius, amp, wavelength, width, noise, seed);
  return ref_init_fill(h);
}

int ref_init_slab(sym_handle* h, double z0, double z1, double width, double noise, unsigned long long seed) {
  const DevParams& P = h->dp;
  k_init_slab<<<blocks_for(P.N), TPB, 0, h->st>>>(P, h->rhoN, h->rho, z0, z1, width, noise, seed);
  return ref_init_fill(h);
}

int ref_neck_radius(sym_handle* h, double* rmin) {
  const DevParams& P = h->dp;
  k_plane_red<<<P.nz, 256, 0, h->st>>>(P, h->rhoN, h->walls_all, h->red);
  std::vector<double> s(P.nz);
  cudaMemcpyAsync(s.data(), h->red, sizeof(double) * P.nz, cudaMemcpyDeviceToHost, h->st);
  if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "neck_radius")) return e;
  double mn = 1e300;
  for (int z = 0; z < P.nz; z++) mn = fmin(mn, sqrt(s[z] / M_PI));
  *rmin = mn;
  return SYM_OK;
}

int ref_output3(sym_handle* h, double* hmin, int32_t* y0) {
  const DevParams& P = h->dp;
  k_output3<<<blocks_for(P.ny), TPB, 0, h->st>>>(P, h->rhoN, h->walls_all, h->pout, h->red);
  std::vector<double> b(P.ny);
  cudaMemcpyAsync(b.data(), h->red, sizeof(double) * P.ny, cudaMemcpyDeviceToHost, h->st);
  if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "output3")) return e;
  double hm = (double)P.nz;
  int yy = 0;
  const double top = (double)P.nz - 0.5;
  for (int y = 1; y <= P.ny - 2; y++) {
    const double hh = top - b[y];
    if (hh < hm) { hm = hh; yy = y + 1; }
  }
  *hmin = hm;
  *y0 = yy;
  return SYM_OK;
}

int ref_mass_momentum(sym_handle* h, double out[5]) {
  const DevParams& P = h->dp;
  const long long nblk = (P.N + 255) / 256;
  if ((size_t)(nblk * 5 + 8) > h->red_len) return set_error(h, SYM_ERR_STATE, "reduction scratch too small");
  k_mass_mom<<<(unsigned)nblk, 256, 0, h->st>>>(P, h->ri, h->bi, h->walls_all, h->red);
  k_sum_partials<<<1, 256, 0, h->st>>>(h->red, nblk, 5, h->red + nblk * 5);
  cudaMemcpyAsync(out, h->red + nblk * 5, sizeof(double) * 5, cudaMemcpyDeviceToHost, h->st);
  return check_cuda(h, cudaStreamSynchronize(h->st), "mass_momentum");
}

int aos_to_soa(sym_handle* h, const double* aos, double* soa) {
  k_aos_to_soa<<<blocks_for(19 * (long long)h->N), TPB, 0, h->st>>>(aos, soa, (long long)h->N);
  return check_cuda(h, cudaGetLastError(), "aos_to_soa");
}
int soa_to_aos(sym_handle* h, const double* soa, double* aos) {
  k_soa_to_aos<<<blocks_for(19 * (long long)h->N), TPB, 0, h->st>>>(soa, aos, (long long)h->N);
  return check_cuda(h, cudaGetLastError(), "soa_to_aos");
}

// exported for particles.cu (mirror sequences used by set_walls/refilling)
void mirror_int_all(sym_handle* h, int32_t* a, int axis) { mirror_scalar<int32_t>(h, a, axis); }
void mirror_macros_all(sym_handle* h) { mirror_macros(h, true); }

}  // namespace symb200
