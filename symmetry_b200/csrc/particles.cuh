// particles.cuh -- device bodies of the particle coupling (Source1.f90 L4):
// set_walls, Lagrange_points, capillary_force2, momentum, repulsive, movement,
// refilling.  The per-handle kernels of particles.cu (one launch per
// subroutine call, the drop-in path) and the batched kernels of sparse.cu
// (one launch per subroutine for every domain of a fused step) call the same
// bodies.
//
// Node scans are restricted to each sphere's bounding box (the reference scans
// the whole domain per particle, O(par*N)); every node the reference can touch
// lies inside the box, so results are the same.  FP64 reductions use fixed
// trees (per-block partials, then one ordered pass), so they are deterministic.
#pragma once
#include <cmath>
#include "state.cuh"

namespace symb200 {
namespace part {

__device__ __forceinline__ double PC(const double* a, int par, int pp, int k) { return a[k * par + pp - 1]; }

// Bounding box of a sphere in node indices, [c - R - m, c + R + m] per axis.
// The extent is fixed on the host (it depends on R and m only); the origin is
// computed in the kernel from the device-resident centre, so launches stay
// valid inside a captured CUDA graph while the particle moves.
struct Box {
  int n[3];
  int full[3];    // axis covered entirely (box wider than the domain)
  double margin;
  __host__ __device__ long long count() const { return (long long)n[0] * n[1] * n[2]; }
};

inline Box sphere_box(const DevParams& P, double margin) {
  Box b;
  const int dims[3] = {P.nx, P.ny, P.nz};
  b.margin = margin;
  for (int k = 0; k < 3; k++) {
    int n = (int)std::ceil(2.0 * (P.rad + margin)) + 2;
    b.full[k] = 0;
    if (n >= dims[k]) { n = dims[k]; b.full[k] = 1; }
    b.n[k] = n;
  }
  return b;
}

// box thread -> 0-based node index (wrapped in periodic axes); false when the
// node falls outside a non-periodic axis
__device__ __forceinline__ bool box_node(const DevParams& P, const Box& b, const double* centre, int pp,
                                         long long t, int& x, int& y, int& z) {
  if (t >= b.count()) return false;
  int id[3];
  id[2] = (int)(t % b.n[2]);
  t /= b.n[2];
  id[1] = (int)(t % b.n[1]);
  id[0] = (int)(t / b.n[1]);
  const int dims[3] = {P.nx, P.ny, P.nz};
  int v[3];
  for (int k = 0; k < 3; k++) {
    if (b.full[k]) { v[k] = id[k]; continue; }
    const double c = centre[k * P.par + pp - 1] - (double)P.origin;
    const int lo = (int)floor(c - P.rad - b.margin);
    int q = lo + id[k];
    const bool periodic = !P.ref && !(k == 0 && P.wall_x);
    if (periodic) q = ((q % dims[k]) + dims[k]) % dims[k];
    else if (q < 0 || q >= dims[k]) return false;
    v[k] = q;
  }
  x = v[0]; y = v[1]; z = v[2];
  return true;
}
__device__ __forceinline__ bool in_range(const DevParams& P, int x, int y, int z) {
  return x >= P.lo[0] && x <= P.hi[0] && y >= P.lo[1] && y <= P.hi[1] && z >= P.lo[2] && z <= P.hi[2];
}

// ---- set_walls (Source1.f90:326-395) -----------------------------------------
// the previous masks become walls_old and every mask of node L is cleared
__device__ __forceinline__ void walls_reset_node(long long L, int32_t* walls, int32_t* walls_old, int32_t* walls_all,
                                                 int32_t* pin, int32_t* pout) {
  walls_old[L] = walls_all[L];
  walls_all[L] = 0; walls[L] = 0; pin[L] = 0; pout[L] = 0;
}
// distance test with separately rounded products and sums (bit-exact masks)
__device__ __forceinline__ void walls_mark_node(const DevParams& P, const sym_particles* S, int pp, double r2, int x,
                                                int y, int z, int32_t* walls, int32_t* walls_all) {
  const int par = P.par;
  const double dx = disp(P, (double)(x + P.origin), PC(S->center, par, pp, 0), 0);
  const double dy = disp(P, (double)(y + P.origin), PC(S->center, par, pp, 1), 1);
  const double dz = disp(P, (double)(z + P.origin), PC(S->center, par, pp, 2), 2);
  const double d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (d <= r2) {
    const long long L = lin(P, x, y, z);
    walls[L] = pp;
    walls_all[L] = 10;
  }
}
__device__ __forceinline__ void pinpout_node(const DevParams& P, int x, int y, int z, int id,
                                             const int32_t* __restrict__ walls, const int32_t* __restrict__ walls_all,
                                             int32_t* pin, int32_t* pout) {
  if (!in_range(P, x, y, z)) return;
  const long long L = lin(P, x, y, z);
  if (walls_all[L] != 0) return;
  for (int i = 1; i < 19; i++) {
    const long long nb = lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
    if (walls[nb] == id) { pout[L] = id; pin[nb] = id; }
  }
}

// ---- Lagrange_points (Source1.f90:1799-1978) ----------------------------------
__device__ __forceinline__ int lag_idx(const DevParams& P, long long c, int n, int k) {
  if (P.ref) {  // 1-based coordinate -> 0-based index; a point outside the
                // arrays (the reference's domain test leaves x < 1 and z < 1
                // open, :1832) is clamped to the edge instead of read out of bounds
    const long long i = c - 1;
    return (int)(i < 0 ? 0 : (i > n - 1 ? n - 1 : i));
  }
  long long i = c - P.origin;
  const bool periodic = !(k == 0 && P.wall_x);
  if (periodic) {
    if (i < 0 || i >= n) i = ((i % n) + n) % n;
  } else {
    i = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
  }
  return (int)i;
}

// sin and cos of the two angles of Lagrange point `num` (:1826-1830): they
// depend on the point index only, so a step can read them from a table
__device__ __forceinline__ void lagrange_trig(const DevParams& P, int num, double& sa, double& ca, double& sb,
                                              double& cb) {
  const int na = num / (P.la_n + 1) + 1, nb = num % (P.la_n + 1) + 1;
  const double aa = (double)(na - 1) * P.alpha, bb = (double)(nb - 1) * P.alpha;
  sa = sin(aa); ca = cos(aa); sb = sin(bb); cb = cos(bb);
}

// Lagrange point `num` of particle pp: position, area element, interpolated
// phase, flag and rotated normal
__device__ __forceinline__ void lagrange_point(const DevParams& P, const sym_particles* __restrict__ S,
                                               const int32_t* __restrict__ walls, const double* __restrict__ rhoN,
                                               const double* __restrict__ gx, const double* __restrict__ gy,
                                               const double* __restrict__ gz, const double* __restrict__ nxv,
                                               const double* __restrict__ nyv, const double* __restrict__ nzv,
                                               double* Lax, double* Lay, double* Laz, double* La_rhoN, double* La_nx,
                                               double* La_ny, double* La_nz, int32_t* La_flag, double* ds, int num,
                                               int pp, const double* __restrict__ tab = nullptr) {
  const int EX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
  const int EY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
  const int EZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  const int par = P.par;
  if (num >= P.la_num) return;
  const long long q = (long long)num * par + (pp - 1);
  const double cx = PC(S->center, par, pp, 0), cy = PC(S->center, par, pp, 1), cz = PC(S->center, par, pp, 2);
  const double Rad = P.rad, alpha = P.alpha;
  // the point's angles: from the table of sin/cos per point (lagrange_trig)
  // when given, else computed here -- the same values either way
  double sa, ca, sb, cb;
  if (tab) {
    sa = tab[4LL * num]; ca = tab[4LL * num + 1]; sb = tab[4LL * num + 2]; cb = tab[4LL * num + 3];
  } else {
    lagrange_trig(P, num, sa, ca, sb, cb);
  }
  const double lx = cx + Rad * sb * ca;
  const double ly = cy + Rad * sb * sa;
  const double lz = cz + Rad * cb;
  Lax[q] = lx; Lay[q] = ly; Laz[q] = lz;
  ds[q] = Rad * Rad * sb * (alpha * alpha);
  const bool in_domain = P.ref ? (lx < P.nx - 0.5 && ly >= 1.5 && ly < P.ny - 0.5 && lz < P.nz - 0.5) : true;
  double v = 0.0;
  int fl = 0;
  long long x0 = 0, y0 = 0, z0 = 0;
  // array indices of the corners' coordinates: every corner takes c or c + 1
  // along each axis, so six lookups serve all eight corners
  int ix0 = 0, ix1 = 0, iy0 = 0, iy1 = 0, iz0 = 0, iz1 = 0;
  if (in_domain) {
    if (P.ref) { x0 = (long long)lx; y0 = (long long)ly; z0 = (long long)lz; }
    else { x0 = (long long)floor(lx); y0 = (long long)floor(ly); z0 = (long long)floor(lz); }
    ix0 = lag_idx(P, x0, P.nx, 0); ix1 = lag_idx(P, x0 + 1, P.nx, 0);
    iy0 = lag_idx(P, y0, P.ny, 1); iy1 = lag_idx(P, y0 + 1, P.ny, 1);
    iz0 = lag_idx(P, z0, P.nz, 2); iz1 = lag_idx(P, z0 + 1, P.nz, 2);
    double wsum = 0.0, acc = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const long long xf = x0 + EX[i], yf = y0 + EY[i], zf = z0 + EZ[i];
      const long long F = lin(P, EX[i] ? ix1 : ix0, EY[i] ? iy1 : iy0, EZ[i] ? iz1 : iz0);
      if (walls[F] <= 0) {
        const double star = rhoN[F] + gx[F] * (lx - (double)xf) + gy[F] * (ly - (double)yf) + gz[F] * (lz - (double)zf);
        const double dis = (double)(xf - lx) * (double)(xf - lx) + ((double)yf - ly) * ((double)yf - ly) +
                           ((double)zf - lz) * ((double)zf - lz);
        const double w = 1.0 / dis;
        acc = acc + w * star;
        wsum = wsum + w;
      }
    }
    v = acc / wsum;
    if (v < -1.0) v = -1.0;
    if (v > 1.0) v = 1.0;
    if (fabs(v) < 0.99) fl = 1;
  }
  La_rhoN[q] = v;
  La_flag[q] = fl;
  double o0 = 0.0, o1 = 0.0, o2 = 0.0;
  if (fl) {
    double nw[3] = {lx - cx, ly - cy, lz - cz};
    unitization(nw);
    double mn = 100.0;
    long long G = lin(P, ix0, iy0, iz0);   // corner 0 unless a nearer one qualifies
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
      const int ex = ((i + 1) >> 1) & 1, ey = (i >> 1) & 1, ez = (i >> 2) & 1;   // EX[i], EY[i], EZ[i]
      const long long xf = x0 + ex, yf = y0 + ey, zf = z0 + ez;
      const bool inside = P.ref ? (xf <= P.nx && yf >= 1 && yf <= P.ny && zf <= P.nz) : true;
      if (!inside) continue;
      const long long F = lin(P, ex ? ix1 : ix0, ey ? iy1 : iy0, ez ? iz1 : iz0);
      if (walls[F] <= 0) {
        if (fabs(nxv[F] * nxv[F] + nyv[F] * nyv[F] + nzv[F] * nzv[F]) > 0.0) {
          const double dis = ((double)xf - lx) * ((double)xf - lx) + ((double)yf - ly) * ((double)yf - ly) +
                             ((double)zf - lz) * ((double)zf - lz);
          if (sqrt(dis) < mn) { mn = sqrt(dis); G = F; }
        }
      }
    }
    double nt[3] = {nxv[G], nyv[G], nzv[G]};
    unitization(nt);
    double r[3];
    akai_rotate<double>(P.cita, nw, nt, false, r);
    o0 = r[0]; o1 = r[1]; o2 = r[2];
  }
  La_nx[q] = o0; La_ny[q] = o1; La_nz[q] = o2;
}

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

// K block sums at once, each added in block_sum's pairwise order (the same
// result bit for bit) with one barrier per level for all K; sh holds K * NT
// doubles.  The sums are left in sh[c * NT].
template <int NT, int K>
__device__ __forceinline__ void block_sums(const double (&v)[K], double* sh) {
#pragma unroll
  for (int c = 0; c < K; c++) sh[c * NT + threadIdx.x] = v[c];
  __syncthreads();
#pragma unroll
  for (int s = NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
#pragma unroll
      for (int c = 0; c < K; c++) sh[c * NT + threadIdx.x] = sh[c * NT + threadIdx.x] + sh[c * NT + threadIdx.x + s];
    }
    __syncthreads();
  }
}

// Shb (immersed area) and capillary_force2 (Source1.f90:1980-2028).  The
// 16,380 Lagrange points of a particle are split over kCapBlocks blocks that
// write fixed-order partial sums (part[(pp-1)*kCapBlocks + block][7]); the
// final pass adds them in block order (deterministic).  Block-level: every
// thread of the 256-thread block calls it, with kCapShared doubles of shared
// memory in sh.
constexpr int kCapBlocks = 32;
constexpr int kCapShared = 7 * 256;
__device__ __forceinline__ void capillary_partial(const DevParams& P, const sym_particles* __restrict__ S,
                                                  const double* __restrict__ Lax, const double* __restrict__ Lay,
                                                  const double* __restrict__ Laz, const double* __restrict__ La_rhoN,
                                                  const double* __restrict__ La_nx, const double* __restrict__ La_ny,
                                                  const double* __restrict__ La_nz,
                                                  const int32_t* __restrict__ La_flag, const double* __restrict__ ds,
                                                  int do_tension, double* part, int pp, int blk, double* sh) {
  const int par = P.par;
  const double cx = PC(S->center, par, pp, 0), cy = PC(S->center, par, pp, 1), cz = PC(S->center, par, pp, 2);
  const double k = 0.134 * 1.43;
  const bool right = (P.cita == M_PI / 2.0);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int num = blk * 256 + threadIdx.x; num < P.la_num; num += 256 * kCapBlocks) {
    const long long q = (long long)num * par + (pp - 1);
    if (La_rhoN[q] > 0.0) acc[6] += ds[q];
    if (!do_tension || !La_flag[q]) continue;
    double nw[3] = {Lax[q] - cx, Lay[q] - cy, Laz[q] - cz};
    const double xr[3] = {nw[0], nw[1], nw[2]};
    unitization(nw);
    const double ie[3] = {-La_nx[q], -La_ny[q], -La_nz[q]};
    double temp[3], nt[3], tt[3];
    veccross(ie, nw, temp);
    const double projector = sqrt(temp[0] * temp[0] + temp[1] * temp[1] + temp[2] * temp[2]);
    veccross(temp, ie, nt);
    unitization(nt);
    const double rn = La_rhoN[q];
    const double om = 1.0 - rn * rn;
    const double star = 4.5 * k * P.beta * (om * om) * ds[q] * projector;
    for (int c = 0; c < 3; c++) temp[c] = right ? star * nw[c] * P.sigma : star * nt[c] * P.sigma;
    veccross(xr, temp, tt);
    for (int c = 0; c < 3; c++) { acc[c] += temp[c]; acc[3 + c] += tt[c]; }
  }
  block_sums<256, 7>(acc, sh);
  if (threadIdx.x < 7) part[((size_t)(pp - 1) * kCapBlocks + blk) * 7 + threadIdx.x] = sh[threadIdx.x * 256];
}
// component c (0..6) of particle pp's capillary sums, in block order
__device__ __forceinline__ void capillary_final_body(const DevParams& P, sym_particles* S,
                                                     const double* __restrict__ part, int do_shb, int do_tension,
                                                     int pp, int c) {
  const int par = P.par;
  if (c >= 7) return;
  double s = 0.0;
  for (int b = 0; b < kCapBlocks; b++) s += part[((size_t)(pp - 1) * kCapBlocks + b) * 7 + c];
  if (c < 3 && do_tension) S->tension[c * par + pp - 1] = s;
  else if (c < 6 && c >= 3 && do_tension) S->tension_t[(c - 3) * par + pp - 1] = s;
  else if (c == 6 && do_shb) S->shb[pp - 1] = s;
}

// ---- momentum (Source1.f90:1178-1261) ------------------------------------------
// block `blk` of particle pp's box: 256 nodes, one fixed-order partial per block
__device__ __forceinline__ void momentum_partial(const DevParams& P, const Box& b, int pp,
                                                 const sym_particles* __restrict__ S,
                                                 const int32_t* __restrict__ walls, const int32_t* __restrict__ pout,
                                                 const double* __restrict__ fi, const double* __restrict__ ffi,
                                                 double* part, long long nblk, long long blk, double* sh) {
  const int par = P.par;
  int x, y, z;
  double a[6] = {0, 0, 0, 0, 0, 0};
  if (box_node(P, b, S->center, pp, blk * 256LL + threadIdx.x, x, y, z) && in_range(P, x, y, z)) {
    const long long L = lin(P, x, y, z), N = P.N;
    if (pout[L] == pp) {
      const double xr = disp(P, (double)(x + P.origin), PC(S->center, par, pp, 0), 0);
      const double yr = disp(P, (double)(y + P.origin), PC(S->center, par, pp, 1), 1);
      const double zr = disp(P, (double)(z + P.origin), PC(S->center, par, pp, 2), 2);
      const double uw0 = PC(S->up, par, pp, 0) + zr * PC(S->rp, par, pp, 1) - yr * PC(S->rp, par, pp, 2);
      const double uw1 = PC(S->up, par, pp, 1) + xr * PC(S->rp, par, pp, 2) - zr * PC(S->rp, par, pp, 0);
      const double uw2 = PC(S->up, par, pp, 2) + yr * PC(S->rp, par, pp, 0) - xr * PC(S->rp, par, pp, 1);
      for (int i = 1; i < 19; i++) {
        const int xb = P.ref ? x - CX(i) : wrapi(x - CX(i), P.nx);
        const int yb = P.ref ? y - CY(i) : wrapi(y - CY(i), P.ny);
        const int zb = P.ref ? z - CZ(i) : wrapi(z - CZ(i), P.nz);
        if (walls[lin(P, xb, yb, zb)] != pp) continue;
        const int j = OPC(i);
        const double f = fi[i * N + L], g = ffi[j * N + L];
        const double fmx = ((double)CX(i) - uw0) * f - ((double)CX(j) - uw0) * g;
        const double fmy = ((double)CY(i) - uw1) * f - ((double)CY(j) - uw1) * g;
        const double fmz = ((double)CZ(i) - uw2) * f - ((double)CZ(j) - uw2) * g;
        a[0] = a[0] - fmx; a[1] = a[1] - fmy; a[2] = a[2] - fmz;
        a[3] = a[3] - (yr * fmz - zr * fmy);
        a[4] = a[4] - (zr * fmx - xr * fmz);
        a[5] = a[5] - (xr * fmy - yr * fmx);
      }
    }
  }
  for (int k = 0; k < 6; k++) {
    const double s = block_sum<256>(a[k], sh);
    if (threadIdx.x == 0) part[((long long)(pp - 1) * nblk + blk) * 6 + k] = s;
  }
}
// block-level: force and torque of particle pp from its nblk partials
__device__ __forceinline__ void momentum_final_body(const DevParams& P, sym_particles* S, const double* part,
                                                    long long nblk, int pp, double* sh) {
  const int par = P.par;
  for (int k = 0; k < 6; k++) {
    double s = 0.0;
    for (long long bb = threadIdx.x; bb < nblk; bb += 256) s += part[((long long)(pp - 1) * nblk + bb) * 6 + k];
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) {
      if (k < 3) S->fp[k * par + pp - 1] = s;
      else S->tp[(k - 3) * par + pp - 1] = s;
    }
  }
}

// ---- momentum over link lists (fused and batched paths) ------------------------
// margin of the momentum box and of set_walls' pin/pout box (the same box)
constexpr double kLinkMargin = 3.0;
// margin of the box on which a fused step writes the canonical views (prep):
// every later reader of them in the step stays within R + 2 of the centre the
// box is placed on -- Lagrange corners (R + sqrt 3), link nodes (R + 1),
// refilled nodes and the fluid neighbours they average (R + 2 of the same,
// pre-move centre) -- and a particle moves far less than a node per step
constexpr double kPrepMargin = 3.0;
// The links of particle pp -- (fluid node, velocity i) with the node's
// neighbour x - c_i inside the particle -- are kept per block of pp's
// momentum box as a compact list: block b's entries are (node, 18-bit mask of
// its links into pp) of the nodes of that block that have any, in thread
// order, so the list and the sums over it are deterministic.  set_walls
// rebuilds the lists of a step while it marks pin/pout (walls, and so the
// links, change only there); the next step's momentum reads them.

// the links of fluid node (x,y,z) into solid id: bit i set when the
// neighbour x + c_i belongs to id
__device__ __forceinline__ unsigned link_mask(const DevParams& P, int x, int y, int z, int id,
                                              const int32_t* __restrict__ walls) {
  unsigned m = 0;
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const long long nb = lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
    if (walls[nb] == id) m |= 1u << i;
  }
  return m;
}

// block-wide compaction of (L, mask) for the threads with has = true into
// seg[0 .. count), in thread order; every thread of the block calls it
__device__ __forceinline__ void link_compact(bool has, unsigned L, unsigned mask, uint2* seg, int* count,
                                             int* sh /* [8] */) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, has);
  if (lane == 0) sh[warp] = __popc(bal);
  __syncthreads();
  int off = 0, tot = 0;
  for (int w = 0; w < 8; w++) {
    if (w < (int)warp) off += sh[w];
    tot += sh[w];
  }
  if (has) seg[off + __popc(bal & ((1u << lane) - 1u))] = make_uint2(L, mask);
  if (threadIdx.x == 0) *count = tot;
  __syncthreads();
}

// one block of pp's links: the momentum exchange of its entries (the terms of
// :1193-1259), reduced by warp shuffles and then over the block's 8 warps in
// a fixed order into part[pp-1][blk]
__device__ __forceinline__ void momentum_links_partial(const DevParams& P, int pp, const sym_particles* __restrict__ S,
                                                       const int32_t* __restrict__ pout,
                                                       const double* __restrict__ fi,
                                                       const double* __restrict__ ffi, const uint2* __restrict__ seg,
                                                       int count, double* part, long long nblk, long long blk,
                                                       double* sh /* [8][6] */) {
  const int par = P.par;
  double a[6] = {0, 0, 0, 0, 0, 0};
  if ((int)threadIdx.x < count) {
    const uint2 e = seg[threadIdx.x];
    const long long L = e.x, N = P.N;
    if (pout[L] == pp) {   // a later particle's set_walls may have taken the node
      const unsigned q = (unsigned)e.x / (unsigned)P.nz;
      const int z = (int)(e.x - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
      const double xr = disp(P, (double)(x + P.origin), PC(S->center, par, pp, 0), 0);
      const double yr = disp(P, (double)(y + P.origin), PC(S->center, par, pp, 1), 1);
      const double zr = disp(P, (double)(z + P.origin), PC(S->center, par, pp, 2), 2);
      const double uw0 = PC(S->up, par, pp, 0) + zr * PC(S->rp, par, pp, 1) - yr * PC(S->rp, par, pp, 2);
      const double uw1 = PC(S->up, par, pp, 1) + xr * PC(S->rp, par, pp, 2) - zr * PC(S->rp, par, pp, 0);
      const double uw2 = PC(S->up, par, pp, 2) + yr * PC(S->rp, par, pp, 0) - xr * PC(S->rp, par, pp, 1);
#pragma unroll
      for (int i = 1; i < 19; i++) {
        // the reference's link i (neighbour x - c_i inside, :1193-1203) is
        // bit OPC(i) of the mask; i ascending as there
        if (!(e.y >> OPC(i) & 1u)) continue;
        const int j = OPC(i);
        const double f = fi[i * N + L], g = ffi[j * N + L];
        const double fmx = ((double)CX(i) - uw0) * f - ((double)CX(j) - uw0) * g;
        const double fmy = ((double)CY(i) - uw1) * f - ((double)CY(j) - uw1) * g;
        const double fmz = ((double)CZ(i) - uw2) * f - ((double)CZ(j) - uw2) * g;
        a[0] = a[0] - fmx; a[1] = a[1] - fmy; a[2] = a[2] - fmz;
        a[3] = a[3] - (yr * fmz - zr * fmy);
        a[4] = a[4] - (zr * fmx - xr * fmz);
        a[5] = a[5] - (xr * fmy - yr * fmx);
      }
    }
  }
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 6; c++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[c] += __shfl_down_sync(0xffffffffu, a[c], o);
    if (lane == 0) sh[warp * 6 + c] = a[c];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int w = 0; w < 8; w++) v += sh[w * 6 + threadIdx.x];
    part[((long long)(pp - 1) * nblk + blk) * 6 + threadIdx.x] = v;
  }
}

// ---- repulsive (Source1.f90:1594-1671), one thread ---------------------------------
__device__ __forceinline__ void repulsive_body(const DevParams& P, sym_particles* S) {
  const int par = P.par;
  const double range = 3.0, order = 0.01, Fg = P.fg, rad = P.rad;
  for (int c = 0; c < 3 * par; c++) S->fre[c] = 0.0;
  auto sqd = [](double a) { return a * a; };
  for (int pp = 1; pp <= par; pp++) {
    const double cx = PC(S->center, par, pp, 0), cy = PC(S->center, par, pp, 1), cz = PC(S->center, par, pp, 2);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    if (P.ref) {
      const double dtop = (double)P.nz - 0.5 - cz - rad, dbot = cz - 1.5 - rad;
      const double dleft = cy - 1.5 - rad, dright = (double)P.ny - 1.5 - cy - rad;
      const double dfront = cx - 1.5 - rad, dback = (double)P.nx - 1.5 - cx - rad;
      if (dtop < range) fz = fz + 2.0 * (Fg / order) * sqd(dtop - range) / sqd(range);
      if (dbot < range) fz = fz - 2.0 * (Fg / order) * sqd(dbot - range) / sqd(range);
      if (dleft < range) fy = fy - 2.0 * (Fg / order) * sqd(dleft - range) / sqd(range);
      if (dright < range) fy = fy + 2.0 * (Fg / order) * sqd(dright - range) / sqd(range);
      if (dfront < range) fx = fx - 2.0 * (Fg / order) * sqd(dfront - range) / sqd(range);
      if (dback < range) fx = fx + 2.0 * (Fg / order) * sqd(dback - range) / sqd(range);
    } else if (P.wall_x) {
      const double dlo = cx - 0.5 - rad, dhi = (double)(P.nx - 1) - 0.5 - cx - rad;
      if (dlo < range) fx = fx - 2.0 * (Fg / order) * sqd(dlo - range) / sqd(range);
      if (dhi < range) fx = fx + 2.0 * (Fg / order) * sqd(dhi - range) / sqd(range);
    }
    S->fre[0 * par + pp - 1] = fx; S->fre[1 * par + pp - 1] = fy; S->fre[2 * par + pp - 1] = fz;
  }
  for (int i = 1; i <= par; i++)
    for (int j = 1; j <= par; j++) {
      if (i == j) continue;
      double d[3];
      for (int c = 0; c < 3; c++) d[c] = PC(S->center, par, i, c) - PC(S->center, par, j, c);
      if (!P.ref)
        for (int c = 0; c < 3; c++) {
          const int n = c == 0 ? P.nx : (c == 1 ? P.ny : P.nz);
          if (!(c == 0 && P.wall_x)) d[c] -= (double)n * nearbyint(d[c] / (double)n);
        }
      const double dis = sqrt(sqd(d[0]) + sqd(d[1]) + sqd(d[2])) - rad * 2.0;
      if (dis < range)
        for (int c = 0; c < 3; c++)
          S->fre[c * par + i - 1] = S->fre[c * par + i - 1] - (Fg / order) * sqd(dis - range) / sqd(range) * d[c] / dis;
    }
}

// ---- movement (Source1.f90:1263-1349), one thread ------------------------------------
__device__ __forceinline__ void movement_body(const DevParams& P, sym_particles* S) {
  const int par = P.par;
  auto A = [&](double* a, int pp, int k) -> double& { return a[k * par + pp - 1]; };
  if (P.ref) {
    for (int pp = 1; pp <= par; pp++) {
      if (fabs(A(S->center0, pp, 0) - ((double)P.nx - 0.5)) < 0.1) {
        A(S->fp, pp, 0) = 0.0; A(S->fp, pp, 1) = 2.0 * A(S->fp, pp, 1); A(S->fp, pp, 2) = 2.0 * A(S->fp, pp, 2);
        A(S->tp, pp, 0) = 2.0 * A(S->tp, pp, 0); A(S->tp, pp, 1) = 0.0; A(S->tp, pp, 2) = 0.0;
        A(S->fre, pp, 0) = 0.0;
        A(S->tension, pp, 0) = 0.0; A(S->tension, pp, 1) = A(S->tension, pp, 1) * 2.0;
        A(S->tension, pp, 2) = A(S->tension, pp, 2) * 2.0;
        A(S->tension_t, pp, 0) = 2.0 * A(S->tension_t, pp, 0);
        A(S->tension_t, pp, 1) = 0.0; A(S->tension_t, pp, 2) = 0.0;
      }
      const double c0y = A(S->center0, pp, 1);
      if (fabs(c0y - ((double)P.ny - 0.5)) < 0.1 || fabs(c0y - 1.5) < 0.1) {
        A(S->fp, pp, 0) = 2.0 * A(S->fp, pp, 0); A(S->fp, pp, 1) = 0.0; A(S->fp, pp, 2) = 2.0 * A(S->fp, pp, 2);
        A(S->tp, pp, 0) = 0.0; A(S->tp, pp, 1) = 2.0 * A(S->tp, pp, 1); A(S->tp, pp, 2) = 0.0;
        A(S->fre, pp, 1) = 0.0;
        A(S->tension, pp, 0) = 2.0 * A(S->tension, pp, 0); A(S->tension, pp, 1) = 0.0;
        A(S->tension, pp, 2) = 2.0 * A(S->tension, pp, 2);
        A(S->tension_t, pp, 0) = 0.0; A(S->tension_t, pp, 1) = 0.0; A(S->tension_t, pp, 2) = 0.0;
      }
      if (fabs(A(S->center0, pp, 2) - ((double)P.nz - 0.5)) < 0.1) {
        A(S->fp, pp, 0) = 2.0 * A(S->fp, pp, 0); A(S->fp, pp, 1) = 2.0 * A(S->fp, pp, 1); A(S->fp, pp, 2) = 0.0;
        A(S->tp, pp, 0) = 0.0; A(S->tp, pp, 1) = 0.0; A(S->tp, pp, 2) = 2.0 * A(S->tp, pp, 2);
        A(S->fre, pp, 2) = 0.0;
        A(S->tension, pp, 0) = A(S->tension, pp, 0) * 2.0; A(S->tension, pp, 1) = A(S->tension, pp, 1) * 2.0;
        A(S->tension, pp, 2) = 0.0;
        A(S->tension_t, pp, 0) = 0.0; A(S->tension_t, pp, 1) = 0.0;
        A(S->tension_t, pp, 2) = 2.0 * A(S->tension_t, pp, 2);
      }
    }
    for (int pp = 1; pp <= par; pp++) {
      if (pp == par / 3 + 1) {
        double t = (A(S->tension, pp, 0) + A(S->tension, pp, 2)) / 2.0;
        A(S->tension, pp, 0) = t; A(S->tension, pp, 2) = t;
        A(S->tension_t, pp, 1) = 0.0;
        t = (A(S->fp, pp, 0) + A(S->fp, pp, 2)) / 2.0;
        A(S->fp, pp, 0) = t; A(S->fp, pp, 2) = t;
        A(S->tp, pp, 1) = 0.0;
        t = (A(S->fre, pp, 0) + A(S->fre, pp, 2)) / 2.0;
        A(S->fre, pp, 0) = t; A(S->fre, pp, 2) = t;
      }
    }
  }
  const double m = P.mass, I = P.inertia;
  double F[3 * SYM_MAX_PAR];
  for (int pp = 1; pp <= par; pp++)
    for (int c = 0; c < 3; c++) {
      double f = A(S->fp, pp, c) + A(S->fre, pp, c) + A(S->tension, pp, c);
      if (!P.ref) f = f + m * P.body[c];
      F[c * par + pp - 1] = f;
      A(S->up, pp, c) = A(S->up, pp, c) + f / m;
      A(S->rp, pp, c) = A(S->rp, pp, c) + (A(S->tp, pp, c) + A(S->tension_t, pp, c)) / I;
    }
  for (int c = 0; c < 3 * par; c++) S->center_old[c] = S->center[c];
  for (int pp = 1; pp <= par; pp++)
    for (int c = 0; c < 3; c++)
      A(S->center, pp, c) = A(S->center, pp, c) + A(S->up, pp, c) + 0.5 * F[c * par + pp - 1] / m;
}

// ---- refilling (Source1.f90:1351-1418) --------------------------------------------
__device__ __forceinline__ void refill_node(const DevParams& P, int pp, const sym_particles* __restrict__ S,
                                            const int32_t* __restrict__ pout, const int32_t* __restrict__ walls_old,
                                            double* rho, double* rhoN, double* rhoR, double* rhoB, double* ux,
                                            double* uy, double* uz, double* ri, double* bi, double* fi, int x, int y,
                                            int z) {
  if (!in_range(P, x, y, z)) return;
  const long long L = lin(P, x, y, z), N = P.N;
  if (pout[L] != pp || walls_old[L] < 1) return;
  const int par = P.par;
  const double xr = disp(P, (double)(x + P.origin), PC(S->center_old, par, pp, 0), 0);
  const double yr = disp(P, (double)(y + P.origin), PC(S->center_old, par, pp, 1), 1);
  const double zr = disp(P, (double)(z + P.origin), PC(S->center_old, par, pp, 2), 2);
  const double u0 = PC(S->up, par, pp, 0) + zr * PC(S->rp, par, pp, 1) - yr * PC(S->rp, par, pp, 2);
  const double u1 = PC(S->up, par, pp, 1) + xr * PC(S->rp, par, pp, 2) - zr * PC(S->rp, par, pp, 0);
  const double u2 = PC(S->up, par, pp, 2) + yr * PC(S->rp, par, pp, 0) - xr * PC(S->rp, par, pp, 1);
  ux[L] = u0; uy[L] = u1; uz[L] = u2;
  double sr = 0.0, sb = 0.0, num = 0.0;
  for (int i = 1; i < 19; i++) {
    const long long nb = lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
    if (walls_old[nb] <= 0) { sr = sr + rhoR[nb]; sb = sb + rhoB[nb]; num = num + 1.0; }
  }
  const double R = sr / num, B = sb / num, rh = R + B;
  rhoR[L] = R; rhoB[L] = B; rho[L] = rh; rhoN[L] = (R - B) / rh;
  const double usqr = u0 * u0 + u1 * u1 + u2 * u2;
#pragma unroll
  for (int i = 0; i < 19; i++) {
    const double r = feq_srt<double>(i, R, u0, u1, u2, usqr), bb = feq_srt<double>(i, B, u0, u1, u2, usqr);
    ri[i * N + L] = r; bi[i * N + L] = bb; fi[i * N + L] = r + bb;
  }
}

}  // namespace part
}  // namespace symb200
