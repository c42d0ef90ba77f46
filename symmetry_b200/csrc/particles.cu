// particles.cu -- particle coupling on the canonical state (Source1.f90 L4):
// set_walls, Lagrange_points, capillary_force2, momentum, repulsive, movement,
// refilling, initia_center -- one launch per subroutine call of one handle
// (the drop-in path).  The node and point bodies are in particles.cuh.
#include <cmath>
#include "particles.cuh"

namespace symb200 {

void mirror_int_all(sym_handle* h, int32_t* a, int axis);
void mirror_macros_all(sym_handle* h);

namespace {

using namespace part;

constexpr int TPB = 256;
inline unsigned blocks_for(long long n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

Box sphere_box(const sym_handle* h, double margin) { return part::sphere_box(h->dp, margin); }

// ---- set_walls (Source1.f90:326-395) -----------------------------------------
__global__ void k_walls_reset(long long N, int32_t* walls, int32_t* walls_old, int32_t* walls_all, int32_t* pin,
                              int32_t* pout) {
  const long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (L >= N) return;
  walls_reset_node(L, walls, walls_old, walls_all, pin, pout);
}
__global__ void k_walls_flat(DevParams P, int32_t* walls, int32_t* walls_all) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.ny * P.nz) return;
  const int y = t / P.nz, z = t % P.nz;
  const long long a = lin(P, 0, y, z), b = lin(P, P.nx - 1, y, z);
  walls[a] = P.par + 1; walls_all[a] = 10;
  walls[b] = P.par + 2; walls_all[b] = 10;
}
__global__ void k_walls_mark(DevParams P, Box b, const sym_particles* __restrict__ S, int pp, double r2,
                             int32_t* walls, int32_t* walls_all) {
  int x, y, z;
  if (!box_node(P, b, S->center, pp, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  walls_mark_node(P, S, pp, r2, x, y, z, walls, walls_all);
}
__global__ void k_walls_pinpout_box(DevParams P, Box b, const sym_particles* __restrict__ S, int id,
                                    const int32_t* __restrict__ walls, const int32_t* __restrict__ walls_all,
                                    int32_t* pin, int32_t* pout) {
  int x, y, z;
  if (!box_node(P, b, S->center, id, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  pinpout_node(P, x, y, z, id, walls, walls_all, pin, pout);
}
__global__ void k_walls_pinpout_plane(DevParams P, int xplane, int id, const int32_t* __restrict__ walls,
                                      const int32_t* __restrict__ walls_all, int32_t* pin, int32_t* pout) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.ny * P.nz) return;
  pinpout_node(P, xplane, t / P.nz, t % P.nz, id, walls, walls_all, pin, pout);
}

// ---- Lagrange_points (Source1.f90:1799-1978) ----------------------------------
__global__ void k_lagrange(DevParams P, const sym_particles* __restrict__ S, const int32_t* __restrict__ walls,
                           const double* __restrict__ rhoN, const double* __restrict__ gx,
                           const double* __restrict__ gy, const double* __restrict__ gz,
                           const double* __restrict__ nxv, const double* __restrict__ nyv,
                           const double* __restrict__ nzv, double* Lax, double* Lay, double* Laz, double* La_rhoN,
                           double* La_nx, double* La_ny, double* La_nz, int32_t* La_flag, double* ds) {
  lagrange_point(P, S, walls, rhoN, gx, gy, gz, nxv, nyv, nzv, Lax, Lay, Laz, La_rhoN, La_nx, La_ny, La_nz, La_flag,
                 ds, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y + 1);
}

// Shb and capillary_force2 (Source1.f90:1980-2028): kCapBlocks blocks per particle
__global__ void k_capillary(DevParams P, const sym_particles* __restrict__ S, const double* __restrict__ Lax,
                            const double* __restrict__ Lay, const double* __restrict__ Laz,
                            const double* __restrict__ La_rhoN, const double* __restrict__ La_nx,
                            const double* __restrict__ La_ny, const double* __restrict__ La_nz,
                            const int32_t* __restrict__ La_flag, const double* __restrict__ ds, int do_tension,
                            double* part) {
  __shared__ double sh[kCapShared];
  capillary_partial(P, S, Lax, Lay, Laz, La_rhoN, La_nx, La_ny, La_nz, La_flag, ds, do_tension, part,
                    blockIdx.y + 1, blockIdx.x, sh);
}
__global__ void k_capillary_final(DevParams P, sym_particles* S, const double* __restrict__ part, int do_shb,
                                  int do_tension) {
  capillary_final_body(P, S, part, do_shb, do_tension, blockIdx.x + 1, threadIdx.x);
}

// ---- momentum (Source1.f90:1178-1261) ------------------------------------------
__global__ void k_momentum(DevParams P, Box b, int pp, const sym_particles* __restrict__ S,
                           const int32_t* __restrict__ walls, const int32_t* __restrict__ pout,
                           const double* __restrict__ fi, const double* __restrict__ ffi, double* part,
                           long long nblk) {
  __shared__ double sh[256];
  momentum_partial(P, b, pp, S, walls, pout, fi, ffi, part, nblk, blockIdx.x, sh);
}
__global__ void k_momentum_final(DevParams P, sym_particles* S, const double* part, long long nblk) {
  __shared__ double sh[256];
  momentum_final_body(P, S, part, nblk, blockIdx.x + 1, sh);
}

// ---- repulsive (Source1.f90:1594-1671) and movement (:1263-1349) -----------------
__global__ void k_repulsive(DevParams P, sym_particles* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  repulsive_body(P, S);
}
__global__ void k_movement(DevParams P, sym_particles* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  movement_body(P, S);
}

// ---- refilling (Source1.f90:1351-1418) --------------------------------------------
__global__ void k_refill(DevParams P, Box b, int pp, const sym_particles* __restrict__ S,
                         const int32_t* __restrict__ pout, const int32_t* __restrict__ walls_old, double* rho,
                         double* rhoN, double* rhoR, double* rhoB, double* ux, double* uy, double* uz, double* ri,
                         double* bi, double* fi) {
  int x, y, z;
  if (!box_node(P, b, S->center_old, pp, blockIdx.x * (long long)blockDim.x + threadIdx.x, x, y, z)) return;
  refill_node(P, pp, S, pout, walls_old, rho, rhoN, rhoR, rhoB, ux, uy, uz, ri, bi, fi, x, y, z);
}

// ---- initia_center (Source1.f90:926-976), REFERENCE geometry ----------------------
__global__ void k_initia_center(DevParams P, sym_particles* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int par = P.par;
  const int col[3] = {4, 8, 12}, row[3] = {4, 4, 4};
  const double Rad_c = 30.0, lamda_d = ((double)P.ny - 2.0) * 2.0, rad = P.rad;
  const double tab = (double)(P.ny - 2) / ((double)par / 3.0 - 0.5);
  const double x0 = (double)P.nx - 0.5, z0 = (double)P.nz - 0.5;
  int num_col = 1, num = 0;
  for (int pp = 1; pp <= par; pp++) {
    num = num + 1;
    if (num_col <= 3 && pp > col[num_col - 1]) num_col = num_col + 1;
    const double a = 0.0 - (double)(num_col - 1) * M_PI / 4.0;
    double b;
    if (num_col % 2 == 0) b = 1.5 + ((double)num - 1.0) * tab;
    else b = 1.5 + ((double)num - 0.5) * tab;
    if (num_col <= 3 && num == row[num_col - 1]) num = 0;
    const double dis_x = 0.1 * Rad_c * cos(2.0 * M_PI * (b - 1.5) / lamda_d);
    double star = Rad_c + dis_x;
    star = sqrt(rad * rad + star * star + 2.0 * rad * star * cos(P.cita));
    S->center[0 * par + pp - 1] = x0 - star * cos(a);
    S->center[1 * par + pp - 1] = b;
    S->center[2 * par + pp - 1] = z0 + star * sin(a);
  }
  for (int c = 0; c < 3 * par; c++) S->center0[c] = S->center[c];
}

}  // namespace

// ===========================================================================
// host launchers (no host synchronisation: every launch is graph-capturable)
int part_set_walls(sym_handle* h) {
  const DevParams& P = h->dp;
  k_walls_reset<<<blocks_for(P.N), TPB, 0, h->st>>>(P.N, h->walls, h->walls_old, h->walls_all, h->pin, h->pout);
  if (!P.ref && P.wall_x)
    k_walls_flat<<<blocks_for((long long)P.ny * P.nz), TPB, 0, h->st>>>(P, h->walls, h->walls_all);
  const double r2 = P.rad * P.rad;
  const Box bm = sphere_box(h, 1.0), bp = sphere_box(h, 3.0);
  for (int pp = 1; pp <= P.par; pp++)
    k_walls_mark<<<blocks_for(bm.count()), TPB, 0, h->st>>>(P, bm, h->dpart, pp, r2, h->walls, h->walls_all);
  if (!P.ref && P.wall_x) {
    const unsigned g = blocks_for((long long)P.ny * P.nz);
    k_walls_pinpout_plane<<<g, TPB, 0, h->st>>>(P, 1, P.par + 1, h->walls, h->walls_all, h->pin, h->pout);
    k_walls_pinpout_plane<<<g, TPB, 0, h->st>>>(P, P.nx - 2, P.par + 2, h->walls, h->walls_all, h->pin, h->pout);
  }
  for (int pp = 1; pp <= P.par; pp++)
    k_walls_pinpout_box<<<blocks_for(bp.count()), TPB, 0, h->st>>>(P, bp, h->dpart, pp, h->walls, h->walls_all,
                                                                    h->pin, h->pout);
  if (P.ref) {
    int32_t* arrs[4] = {h->walls, h->walls_all, h->pin, h->pout};
    for (int ax = 0; ax < 3; ax++)
      for (auto* a : arrs) mirror_int_all(h, a, ax);
  }
  return check_cuda(h, cudaGetLastError(), "set_walls");
}

int part_lagrange_points(sym_handle* h) {
  const DevParams& P = h->dp;
  if (P.par == 0) return SYM_OK;
  dim3 g(blocks_for(P.la_num, 128), P.par);
  k_lagrange<<<g, 128, 0, h->st>>>(P, h->dpart, h->walls, h->rhoN, h->gx, h->gy, h->gz, h->nx, h->ny, h->nz, h->lax,
                                   h->lay, h->laz, h->larhon, h->lanx, h->lany, h->lanz, h->laflag, h->lads);
  if ((size_t)kCapBlocks * 7 * P.par > h->red_len) return set_error(h, SYM_ERR_STATE, "capillary scratch too small");
  k_capillary<<<dim3(kCapBlocks, P.par), 256, 0, h->st>>>(P, h->dpart, h->lax, h->lay, h->laz, h->larhon, h->lanx,
                                                           h->lany, h->lanz, h->laflag, h->lads, 0, h->red);
  k_capillary_final<<<P.par, 32, 0, h->st>>>(P, h->dpart, h->red, 1, 0);
  return check_cuda(h, cudaGetLastError(), "Lagrange_points");
}

int part_capillary_force2(sym_handle* h) {
  const DevParams& P = h->dp;
  if (P.par == 0) return SYM_OK;
  if ((size_t)kCapBlocks * 7 * P.par > h->red_len) return set_error(h, SYM_ERR_STATE, "capillary scratch too small");
  k_capillary<<<dim3(kCapBlocks, P.par), 256, 0, h->st>>>(P, h->dpart, h->lax, h->lay, h->laz, h->larhon, h->lanx,
                                                           h->lany, h->lanz, h->laflag, h->lads, 1, h->red);
  k_capillary_final<<<P.par, 32, 0, h->st>>>(P, h->dpart, h->red, 0, 1);
  return check_cuda(h, cudaGetLastError(), "capillary_force2");
}

int part_momentum(sym_handle* h) {
  const DevParams& P = h->dp;
  if (P.par == 0) return SYM_OK;
  const Box b = sphere_box(h, 3.0);
  const long long nblk = (b.count() + 255) / 256;
  if ((size_t)(nblk * 6 * P.par) > h->red_len) return set_error(h, SYM_ERR_STATE, "momentum scratch too small");
  for (int pp = 1; pp <= P.par; pp++)
    k_momentum<<<(unsigned)nblk, 256, 0, h->st>>>(P, b, pp, h->dpart, h->walls, h->pout, h->fi, h->ffi, h->red,
                                                  nblk);
  k_momentum_final<<<P.par, 256, 0, h->st>>>(P, h->dpart, h->red, nblk);
  return check_cuda(h, cudaGetLastError(), "momentum");
}

int part_repulsive(sym_handle* h) {
  if (h->dp.par == 0) return SYM_OK;
  k_repulsive<<<1, 1, 0, h->st>>>(h->dp, h->dpart);
  return check_cuda(h, cudaGetLastError(), "repulsive");
}

int part_movement(sym_handle* h) {
  if (h->dp.par == 0) return SYM_OK;
  k_movement<<<1, 1, 0, h->st>>>(h->dp, h->dpart);
  return check_cuda(h, cudaGetLastError(), "movement");
}

int part_refilling(sym_handle* h) {
  const DevParams& P = h->dp;
  if (P.par == 0) return SYM_OK;
  const Box b = sphere_box(h, 4.0);
  for (int pp = 1; pp <= P.par; pp++)
    k_refill<<<blocks_for(b.count()), TPB, 0, h->st>>>(P, b, pp, h->dpart, h->pout, h->walls_old, h->rho, h->rhoN,
                                                        h->rhoR, h->rhoB, h->ux, h->uy, h->uz, h->ri, h->bi, h->fi);
  if (P.ref) mirror_macros_all(h);
  return check_cuda(h, cudaGetLastError(), "refilling");
}

int part_initia_center(sym_handle* h) {
  k_initia_center<<<1, 1, 0, h->st>>>(h->dp, h->dpart);
  return check_cuda(h, cudaGetLastError(), "initia_center");
}

}  // namespace symb200
