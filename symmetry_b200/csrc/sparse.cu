// sparse.cu -- the particle and wall work of a fused step (Source1.f90
// :237-243 and the pin fill of derivatives :467-492) for every domain of a
// batch, or the one domain of sym_step, at once.
//
// Each subroutine is one launch for all domains: a block table maps every
// block of the launch to (domain, particle, block within that particle's
// work), and a per-domain descriptor holds the domain's parameters, arrays
// and particle boxes.  Per step, in the reference's order:
//   prep            canonical views of the fused state on each particle box
//   lagrange        Lagrange points (Lagrange_points :1799-1978)
//   capillary       immersed area and capillary force, fixed-order partials
//                   (:1864-1866, capillary_force2 :1980-2028), then the sums
//   momentum        momentum exchange over the link lists (warp-shuffle
//                   partials per box block), then the sums (:1178-1261)
//   move            repulsion and Newton-Euler, one thread per domain
//                   (:1594-1671, :1263-1349)
//   set_walls       masks (:326-395): reset on the previous box, flat wall
//                   planes, sphere marks, pin/pout and the link lists of the
//                   next step's momentum
//   refilling       uncovered nodes (:1351-1418) and into the fused state
//   pin fill        fictitious phi on solid nodes next to fluid
// and, after the collide kernel, with the interpolated bounce-back:
//   curve2          links into a particle re-set with the link fraction
//                   (:1036-1101)
// Masks, refills and sums are written per particle in the same order as the
// per-handle kernels of particles.cu, so results are those of the drop-in
// path bit for bit -- except the momentum sums, which add the same per-node
// terms in another order (over the links instead of a box-wide tree): equal
// to rounding.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "state.cuh"
#include "fused.cuh"
#include "particles.cuh"

namespace symb200 {

using namespace fused;
using part::Box;

namespace {

constexpr int kT = 256;

struct SpDom {
  DevParams P;
  Pad pd;
  sym_particles* S;
  int32_t *walls, *walls_all, *walls_old, *pin, *pout;
  double *rho, *ux, *uy, *uz, *rhoN, *rhoR, *rhoB, *fi, *ffi, *ri, *bi;
  double *gx, *gy, *gz, *nx, *ny, *nz;
  double *lax, *lay, *laz, *larhon, *lanx, *lany, *lanz, *lads;
  int32_t* laflag;
  double* red;           // capillary partials, then momentum partials
  void* pops;            // fused populations of this step
  void* phic;            // this step's phase field (pin-filled below)
  void* phip;            // the previous step's phase field
  Ref* rr_old;           // 16-bit storage: reference pairs of the populations
  void* pnext;           // the populations this step's collide kernel writes
  const Ref* rr_cur;     // 16-bit storage: reference pairs they are encoded with
  void* acc;             // next step's accumulated colour densities
  const double* ltab;    // sin/cos of each Lagrange point's angles (4 per point)
  uint2* links;          // momentum link lists [particle][box block][kT] and their counts
  int* nlinks;
  long long link_blocks;
  int* status;
  Box bprep, bmom, bmark, bpin, bref, bpfill;
  long long nblk_mom;
  int full_reset;        // more than one particle: masks reset on the whole domain
  int pad_;
};

// one block of a launch: domain, particle (0 where none), block within the
// particle's work, variant (the wall plane for plane launches)
struct Blk {
  int d, pp, b, v;
};

// ---- kernels -------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(kT, 4) k_sp_prep(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  using R = typename Codec<S>::R;
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  int x, y, z;
  if (!part::box_node(D.P, D.bprep, D.S->center, e.pp, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
  prep_node<S>(D.P, D.pd, D.S, (const S*)D.pops, (const R*)D.phic, (const R*)D.phip, D.walls_all, D.pout, D.rhoN,
               D.rhoR, D.rhoB, D.fi, D.gx, D.gy, D.gz, D.nx, D.ny, D.nz, D.rr_old, x, y, z);
}

__global__ void __launch_bounds__(kT, 4) k_sp_lagrange(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  part::lagrange_point(D.P, D.S, D.walls, D.rhoN, D.gx, D.gy, D.gz, D.nx, D.ny, D.nz, D.lax, D.lay, D.laz, D.larhon,
                       D.lanx, D.lany, D.lanz, D.laflag, D.lads, e.b * kT + threadIdx.x, e.pp, D.ltab);
}

// the Lagrange points' sin/cos table of a domain, once per plan
__global__ void __launch_bounds__(kT) k_sp_lagrange_table(const SpDom* __restrict__ doms,
                                                           const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const int num = e.b * kT + threadIdx.x;
  if (num >= D.P.la_num) return;
  double* t = const_cast<double*>(D.ltab) + 4LL * num;
  part::lagrange_trig(D.P, num, t[0], t[1], t[2], t[3]);
}

__global__ void __launch_bounds__(kT) k_sp_capillary(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  __shared__ double sh[part::kCapShared];
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  part::capillary_partial(D.P, D.S, D.lax, D.lay, D.laz, D.larhon, D.lanx, D.lany, D.lanz, D.laflag, D.lads, 1,
                          D.red, e.pp, e.b, sh);
}

// immersed area (Lagrange_points) and capillary force and torque
// (capillary_force2) of one particle from the same partials
__global__ void k_sp_capillary_final(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  part::capillary_final_body(D.P, D.S, D.red, 1, 1, e.pp, threadIdx.x);
}

// momentum exchange over the link list of one block of the particle's box
// (written by the previous step's set_walls, or by the import)
__global__ void __launch_bounds__(kT) k_sp_momentum(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  __shared__ double sh[8 * 6];
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const long long seg = (long long)(e.pp - 1) * D.link_blocks + e.b;
  part::momentum_links_partial(D.P, e.pp, D.S, D.pout, D.fi, D.ffi, D.links + seg * kT, D.nlinks[seg], D.red,
                               D.nblk_mom, e.b, sh);
}

__global__ void __launch_bounds__(kT) k_sp_momentum_final(const SpDom* __restrict__ doms,
                                                          const Blk* __restrict__ map) {
  __shared__ double sh[kT];
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  part::momentum_final_body(D.P, D.S, D.red, D.nblk_mom, e.pp, sh);
}

// repulsion then Newton-Euler, one thread per domain with particles
__global__ void k_sp_move(const SpDom* __restrict__ doms, const int* __restrict__ list, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const SpDom& D = doms[list[t]];
  part::repulsive_body(D.P, D.S);
  part::movement_body(D.P, D.S);
}

// set_walls, reset: the masks of the previous step lie inside the previous
// box of the particle (pout reaches one link beyond the sphere), or, with
// more than one particle, anywhere: then the whole domain is reset
__global__ void __launch_bounds__(kT) k_sp_reset(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  long long L;
  if (D.full_reset) {
    L = (long long)e.b * kT + threadIdx.x;
    if (L >= D.P.N) return;
  } else {
    int x, y, z;
    if (!part::box_node(D.P, D.bpin, D.S->center_old, 1, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
    L = lin(D.P, x, y, z);
  }
  part::walls_reset_node(L, D.walls, D.walls_old, D.walls_all, D.pin, D.pout);
}

// set_walls, flat wetting walls (CONFIG): the planes x = 0 and x = nx-1 are
// solid at every step, so their previous mask (walls_old) is solid too
__global__ void __launch_bounds__(kT) k_sp_flat(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const int t = e.b * kT + threadIdx.x;
  if (t >= D.P.ny * D.P.nz) return;
  const int y = t / D.P.nz, z = t % D.P.nz;
  const long long a = lin(D.P, 0, y, z), b = lin(D.P, D.P.nx - 1, y, z);
  D.walls[a] = D.P.par + 1; D.walls_all[a] = 10; D.walls_old[a] = 10;
  D.walls[b] = D.P.par + 2; D.walls_all[b] = 10; D.walls_old[b] = 10;
}

__global__ void __launch_bounds__(kT) k_sp_mark(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  int x, y, z;
  if (!part::box_node(D.P, D.bmark, D.S->center, e.pp, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
  part::walls_mark_node(D.P, D.S, e.pp, D.P.rad * D.P.rad, x, y, z, D.walls, D.walls_all);
}

// pin/pout of the flat walls: v = 0 the plane x = 1 (wall x = 0), v = 1 the
// plane x = nx-2 (wall x = nx-1)
__global__ void __launch_bounds__(kT) k_sp_pin_plane(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const int t = e.b * kT + threadIdx.x;
  if (t >= D.P.ny * D.P.nz) return;
  const int xp = e.v == 0 ? 1 : D.P.nx - 2, id = D.P.par + 1 + e.v;
  part::pinpout_node(D.P, xp, t / D.P.nz, t % D.P.nz, id, D.walls, D.walls_all, D.pin, D.pout);
}

// pin/pout of particle pp on one block of its box, and that block's link list
// for the next step's momentum (every thread takes part in the compaction)
__global__ void __launch_bounds__(kT) k_sp_pin_box(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  __shared__ int sh[8];
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  int x, y, z;
  bool has = false;
  unsigned L = 0, mask = 0;
  if (part::box_node(D.P, D.bpin, D.S->center, e.pp, (long long)e.b * kT + threadIdx.x, x, y, z) &&
      part::in_range(D.P, x, y, z)) {
    part::pinpout_node(D.P, x, y, z, e.pp, D.walls, D.walls_all, D.pin, D.pout);
    const long long l = lin(D.P, x, y, z);
    if (D.walls_all[l] == 0) {
      mask = part::link_mask(D.P, x, y, z, e.pp, D.walls);
      has = mask != 0;
      L = (unsigned)l;
    }
  }
  const long long seg = (long long)(e.pp - 1) * D.link_blocks + e.b;
  part::link_compact(has, L, mask, D.links + seg * kT, D.nlinks + seg, sh);
}

// the link lists of particle pp from the current masks (after an import)
__global__ void __launch_bounds__(kT) k_links_build(DevParams P, part::Box b, int pp, const sym_particles* S,
                                                    const int32_t* __restrict__ walls,
                                                    const int32_t* __restrict__ walls_all, uint2* links,
                                                    int* nlinks, long long link_blocks) {
  __shared__ int sh[8];
  int x, y, z;
  bool has = false;
  unsigned L = 0, mask = 0;
  if (part::box_node(P, b, S->center, pp, (long long)blockIdx.x * kT + threadIdx.x, x, y, z) &&
      part::in_range(P, x, y, z)) {
    const long long l = lin(P, x, y, z);
    if (walls_all[l] == 0) {
      mask = part::link_mask(P, x, y, z, pp, walls);
      has = mask != 0;
      L = (unsigned)l;
    }
  }
  const long long seg = (long long)(pp - 1) * link_blocks + blockIdx.x;
  part::link_compact(has, L, mask, links + seg * kT, nlinks + seg, sh);
}

// refilling (uncovered nodes, :1351-1418) and the import of each refilled
// node into the fused state, by the same thread: a refilled node's import
// reads only what its own refill wrote, and no refill reads a refilled node
// (it averages fluid neighbours only), so nodes need no ordering
template <typename S>
__global__ void __launch_bounds__(kT) k_sp_refill_import(const SpDom* __restrict__ doms,
                                                         const Blk* __restrict__ map) {
  using R = typename Codec<S>::R;
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  int x, y, z;
  if (!part::box_node(D.P, D.bref, D.S->center_old, e.pp, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
  part::refill_node(D.P, e.pp, D.S, D.pout, D.walls_old, D.rho, D.rhoN, D.rhoR, D.rhoB, D.ux, D.uy, D.uz, D.ri,
                    D.bi, D.fi, x, y, z);
  refill_import_node<S>(D.P, D.pd, e.pp, (S*)D.pops, (R*)D.phic, D.pout, D.walls_old, D.ri, D.bi, D.rhoN,
                        D.rr_old, x, y, z);
}

// pin fill of the flat walls: v = 0 the plane x = 0, v = 1 the plane x = nx-1
template <typename R>
__global__ void __launch_bounds__(kT) k_sp_pinfill_plane(const SpDom* __restrict__ doms,
                                                         const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const int t = e.b * kT + threadIdx.x;
  if (t >= D.P.ny * D.P.nz) return;
  pinfill_node<R>(D.P, D.pd, (R*)D.phic, D.pin, D.walls_all, e.v == 0 ? 0 : D.P.nx - 1, t / D.P.nz, t % D.P.nz);
}

template <typename R>
__global__ void __launch_bounds__(kT) k_sp_pinfill_box(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  int x, y, z;
  if (!part::box_node(D.P, D.bpfill, D.S->center, e.pp, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
  pinfill_node<R>(D.P, D.pd, (R*)D.phic, D.pin, D.walls_all, x, y, z);
}

// curve2 (Source1.f90:1036-1101) on the fused state, after the collide kernel:
// the collide kernel bounced every link into particle pp halfway (curve) and
// kept the node's red post-collision populations behind ffi; here each such
// link of a node next to pp is replaced, in index order, by the
// interpolation of the reference with link fraction qq:
//   r_i = [qq (r*_i(x) + r*_opc(x)) + (1-qq) r_opc(x) + 6 w_i rhoR(x) uw.c_i] / (1+qq)
// with r* the node's post-collision values and r_opc(x) the population that
// arrived from x + c_i; likewise for blue.  The change of each updated
// population is added to the node's accumulated densities.
template <typename S>
__global__ void __launch_bounds__(kT) k_sp_curve2(const SpDom* __restrict__ doms, const Blk* __restrict__ map) {
  using R = typename Codec<S>::R;
  const Blk e = map[blockIdx.x];
  const SpDom& D = doms[e.d];
  const DevParams& P = D.P;
  const int pp = e.pp, par = P.par;
  int x, y, z;
  if (!part::box_node(P, D.bmom, D.S->center, pp, (long long)e.b * kT + threadIdx.x, x, y, z)) return;
  const long long L = lin(P, x, y, z);
  if (D.pout[L] != pp) return;
  const unsigned N = (unsigned)P.N;
  const double* ff = D.ffi;
  const double* rp = D.ffi + 19 * (size_t)N;
  const Ref rref = Codec<S>::kRef ? D.rr_cur[D.pd.idx(x, y, z)] : Ref{};
  S* pops = (S*)D.pnext;
  const double* c = D.S->center;
  const double x0 = disp(P, (double)(x + P.origin), c[0 * par + pp - 1], 0);
  const double y0 = disp(P, (double)(y + P.origin), c[1 * par + pp - 1], 1);
  const double z0 = disp(P, (double)(z + P.origin), c[2 * par + pp - 1], 2);
  const double rhoR = D.rhoR[L], rhoB = D.rhoB[L];
  double dr = 0.0, db = 0.0;
  static_for<18>([&](auto ic) {
    constexpr int i = decltype(ic)::value + 1;
    constexpr int j = OPC(i);
    const long long B = lin(P, wrapi(x - CX(i), P.nx), wrapi(y - CY(i), P.ny), wrapi(z - CZ(i), P.nz));
    if (D.walls[B] != pp) return;
    const double cx = CX(i), cy = CY(i), cz = CZ(i);
    const double qq = link_fraction(x0, y0, z0, cx, cy, cz, P.rad);
    const double xr = disp(P, (double)(x + P.origin) - cx * qq, c[0 * par + pp - 1], 0);
    const double yr = disp(P, (double)(y + P.origin) - cy * qq, c[1 * par + pp - 1], 1);
    const double zr = disp(P, (double)(z + P.origin) - cz * qq, c[2 * par + pp - 1], 2);
    const double* up = D.S->up;
    const double* rw = D.S->rp;
    const double uw0 = up[0 * par + pp - 1] + zr * rw[1 * par + pp - 1] - yr * rw[2 * par + pp - 1];
    const double uw1 = up[1 * par + pp - 1] + xr * rw[2 * par + pp - 1] - zr * rw[0 * par + pp - 1];
    const double uw2 = up[2 * par + pp - 1] + yr * rw[0 * par + pp - 1] - xr * rw[1 * par + pp - 1];
    const double star = uw0 * cx + uw1 * cy + uw2 * cz;
    const double ar = rp[(size_t)i * N + L], br = rp[(size_t)j * N + L];
    const double ab = ff[(size_t)i * N + L] - ar, bb = ff[(size_t)j * N + L] - br;
    R cr, cb, hr, hb;
    Codec<S>::template load<j>(pops, N, (unsigned)L, rref, cr, cb);
    Codec<S>::template load<i>(pops, N, (unsigned)L, rref, hr, hb);
    const double vr = 1.0 / (1.0 + qq) * (qq * (ar + br) + (1.0 - qq) * (double)cr + 6.0 * W(i) * rhoR * star);
    const double vb = 1.0 / (1.0 + qq) * (qq * (ab + bb) + (1.0 - qq) * (double)cb + 6.0 * W(i) * rhoB * star);
    Codec<S>::template store<i>(pops, N, (unsigned)L, rref, R(vr), R(vr) + R(vb));
    dr += vr - (double)hr;
    db += vb - (double)hb;
  });
  using AT = typename Acc<R>::T;
  if (kAccumulate<S> && (dr != 0.0 || db != 0.0)) {
    acc_add<R>((AT*)D.acc + L, R(dr), D.status);
    acc_add<R>((AT*)D.acc + P.N + L, R(db), D.status);
  }
}

long long nblocks(long long n) { return (n + kT - 1) / kT; }

}  // namespace

// ---- the plan ------------------------------------------------------------------
struct SparsePlan {
  int storage = -1;
  SpDom* d_dom[2] = {nullptr, nullptr};   // per parity
  // block tables, one per launch; several launches per particle index keep
  // the per-particle order of the masks and refills
  enum { PREP, LAG, CAP, CAPF, MOM, MOMF, RESET, FLAT, PINPLANE, PFPLANE, PFBOX, CURVE2, NFIX };
  struct Table {
    Blk* d = nullptr;
    int n = 0;
  };
  Table fix[NFIX];
  std::vector<Table> mark, pin, refill;   // [particle index - 1]
  int* d_move = nullptr;   // domains with particles
  double* d_ltab = nullptr;   // Lagrange sin/cos tables of every domain with particles
  int nmove = 0;
  int launches = 0;
};

namespace {

int plan_table(SparsePlan::Table& t, const std::vector<Blk>& v, cudaStream_t st) {
  t.n = (int)v.size();
  if (!t.n) return SYM_OK;
  if (cudaMalloc(&t.d, sizeof(Blk) * v.size()) != cudaSuccess) { (void)cudaGetLastError(); return SYM_ERR_OOM; }
  cudaMemcpyAsync(t.d, v.data(), sizeof(Blk) * v.size(), cudaMemcpyHostToDevice, st);
  return SYM_OK;
}

void* popp(sym_handle* h, int k) { return h->fast.pop[k]; }
void* phip(sym_handle* h, int k) {
  return h->fast.storage == SYM_STORE_FP64 ? (void*)h->fast.phi[k] : (void*)h->fast.phif[k];
}

SpDom make_dom(sym_handle* h, int cur, int pc) {
  SpDom d;
  std::memset(&d, 0, sizeof d);
  d.P = h->dp;
  d.pd = make_pad(h->dp);
  d.S = h->dpart;
  d.walls = h->walls; d.walls_all = h->walls_all; d.walls_old = h->walls_old; d.pin = h->pin; d.pout = h->pout;
  d.rho = h->rho; d.ux = h->ux; d.uy = h->uy; d.uz = h->uz;
  d.rhoN = h->rhoN; d.rhoR = h->rhoR; d.rhoB = h->rhoB; d.fi = h->fi; d.ffi = h->ffi; d.ri = h->ri; d.bi = h->bi;
  d.gx = h->gx; d.gy = h->gy; d.gz = h->gz; d.nx = h->nx; d.ny = h->ny; d.nz = h->nz;
  d.lax = h->lax; d.lay = h->lay; d.laz = h->laz; d.larhon = h->larhon;
  d.lanx = h->lanx; d.lany = h->lany; d.lanz = h->lanz; d.lads = h->lads; d.laflag = h->laflag;
  d.red = h->red;
  d.pops = popp(h, cur);
  d.phic = phip(h, pc);
  d.phip = phip(h, 1 - pc);
  d.rr_old = h->fast.rref[1 - pc];
  d.pnext = popp(h, 1 - cur);
  d.rr_cur = h->fast.rref[pc];
  d.acc = h->fast.acc;
  d.status = h->fast.status;
  d.links = h->fast.links;
  d.nlinks = h->fast.nlinks;
  d.link_blocks = h->fast.link_blocks;
  d.bprep = part::sphere_box(h->dp, part::kPrepMargin);
  d.bmom = part::sphere_box(h->dp, part::kLinkMargin);
  d.bmark = part::sphere_box(h->dp, 1.0);
  d.bpin = part::sphere_box(h->dp, part::kLinkMargin);
  d.bref = part::sphere_box(h->dp, 4.0);
  d.bpfill = part::sphere_box(h->dp, 2.0);
  d.nblk_mom = nblocks(d.bmom.count());
  d.full_reset = h->dp.par > 1 ? 1 : 0;
  return d;
}

}  // namespace

void sparse_plan_free(SparsePlan* p) {
  if (!p) return;
  for (int k = 0; k < 2; k++)
    if (p->d_dom[k]) cudaFree(p->d_dom[k]);
  for (auto& t : p->fix)
    if (t.d) cudaFree(t.d);
  for (auto* v : {&p->mark, &p->pin, &p->refill})
    for (auto& t : *v)
      if (t.d) cudaFree(t.d);
  if (p->d_move) cudaFree(p->d_move);
  if (p->d_ltab) cudaFree(p->d_ltab);
  delete p;
}

// The momentum link lists of a handle's particles from its current masks
// (the fused state was just built from the canonical one), enqueued on st.
int sparse_links_build(sym_handle* h, cudaStream_t st) {
  const DevParams& P = h->dp;
  if (P.par <= 0 || !h->fast.links) return SYM_OK;
  const part::Box b = part::sphere_box(P, part::kLinkMargin);
  for (int pp = 1; pp <= P.par; pp++)
    k_links_build<<<(unsigned)h->fast.link_blocks, kT, 0, st>>>(P, b, pp, h->dpart, h->walls, h->walls_all,
                                                                h->fast.links, h->fast.nlinks, h->fast.link_blocks);
  return cudaGetLastError() == cudaSuccess ? SYM_OK : SYM_ERR_CUDA;
}

// Plan of the sparse work of `doms` (each at buffer parity cur0/pc0 for step
// parity 0); null with *err set on failure.  The tables are copied on `st`.
SparsePlan* sparse_plan_build(const std::vector<sym_handle*>& doms, const std::vector<int>& cur0,
                              const std::vector<int>& pc0, cudaStream_t st, int* err) {
  SparsePlan* p = new SparsePlan();
  *err = SYM_OK;
  const int n = (int)doms.size();
  if (n) p->storage = doms[0]->fast.storage;
  std::vector<SpDom> dd[2];
  std::vector<Blk> tb[SparsePlan::NFIX];
  std::vector<Blk> ltb;            // blocks of the one-time Lagrange table launch
  std::vector<long long> ltoff;    // each domain's table offset (doubles), -1 without particles
  long long ltlen = 0;
  int maxpar = 0;
  std::vector<int> move;
  for (int i = 0; i < n; i++) {
    sym_handle* h = doms[i];
    for (int k = 0; k < 2; k++) dd[k].push_back(make_dom(h, (cur0[i] + k) & 1, (pc0[i] + k) & 1));
    const SpDom& D = dd[0].back();
    const DevParams& P = h->dp;
    const int plane_blk = (int)nblocks((long long)P.ny * P.nz);
    if (P.wall_x)
      for (int v = 0; v < 2; v++)
        for (int b = 0; b < plane_blk; b++) tb[SparsePlan::PFPLANE].push_back({i, 0, b, v});
    ltoff.push_back(P.par > 0 ? ltlen : -1);
    if (P.par <= 0) continue;
    for (long long b = 0; b < nblocks(P.la_num); b++) ltb.push_back({i, 0, (int)b, 0});
    ltlen += 4LL * P.la_num;
    maxpar = std::max(maxpar, P.par);
    move.push_back(i);
    if (P.wall_x) {
      for (int b = 0; b < plane_blk; b++) tb[SparsePlan::FLAT].push_back({i, 0, b, 0});
      for (int v = 0; v < 2; v++)
        for (int b = 0; b < plane_blk; b++) tb[SparsePlan::PINPLANE].push_back({i, 0, b, v});
    }
    if (D.full_reset) {
      for (long long b = 0; b < nblocks(P.N); b++) tb[SparsePlan::RESET].push_back({i, 0, (int)b, 0});
    } else {
      for (long long b = 0; b < nblocks(D.bpin.count()); b++) tb[SparsePlan::RESET].push_back({i, 1, (int)b, 0});
    }
    for (int pp = 1; pp <= P.par; pp++) {
      for (long long b = 0; b < nblocks(D.bprep.count()); b++) tb[SparsePlan::PREP].push_back({i, pp, (int)b, 0});
      for (long long b = 0; b < nblocks(P.la_num); b++) tb[SparsePlan::LAG].push_back({i, pp, (int)b, 0});
      for (int b = 0; b < part::kCapBlocks; b++) tb[SparsePlan::CAP].push_back({i, pp, b, 0});
      tb[SparsePlan::CAPF].push_back({i, pp, 0, 0});
      for (long long b = 0; b < D.nblk_mom; b++) tb[SparsePlan::MOM].push_back({i, pp, (int)b, 0});
      tb[SparsePlan::MOMF].push_back({i, pp, 0, 0});
      for (long long b = 0; b < nblocks(D.bpfill.count()); b++) tb[SparsePlan::PFBOX].push_back({i, pp, (int)b, 0});
      if (P.bounce)
        for (long long b = 0; b < nblocks(D.bmom.count()); b++) tb[SparsePlan::CURVE2].push_back({i, pp, (int)b, 0});
    }
  }
  std::vector<std::vector<Blk>> mk(maxpar), pn(maxpar), rf(maxpar);
  for (int i = 0; i < n; i++) {
    const SpDom& D = dd[0][i];
    for (int pp = 1; pp <= doms[i]->dp.par; pp++) {
      for (long long b = 0; b < nblocks(D.bmark.count()); b++) mk[pp - 1].push_back({i, pp, (int)b, 0});
      for (long long b = 0; b < nblocks(D.bpin.count()); b++) pn[pp - 1].push_back({i, pp, (int)b, 0});
      for (long long b = 0; b < nblocks(D.bref.count()); b++) rf[pp - 1].push_back({i, pp, (int)b, 0});
    }
  }
  int e = SYM_OK;
  if (ltlen > 0) {
    if (cudaMalloc(&p->d_ltab, sizeof(double) * ltlen) != cudaSuccess) {
      (void)cudaGetLastError();
      e = SYM_ERR_OOM;
    } else {
      for (int k = 0; k < 2; k++)
        for (int i = 0; i < n; i++)
          if (ltoff[i] >= 0) dd[k][i].ltab = p->d_ltab + ltoff[i];
    }
  }
  for (int k = 0; k < 2 && !e && n; k++) {
    if (cudaMalloc(&p->d_dom[k], sizeof(SpDom) * n) != cudaSuccess) {
      (void)cudaGetLastError();
      e = SYM_ERR_OOM;
      break;
    }
    cudaMemcpyAsync(p->d_dom[k], dd[k].data(), sizeof(SpDom) * n, cudaMemcpyHostToDevice, st);
  }
  for (int t = 0; t < SparsePlan::NFIX && !e; t++) e = plan_table(p->fix[t], tb[t], st);
  p->mark.resize(maxpar);
  p->pin.resize(maxpar);
  p->refill.resize(maxpar);
  for (int q = 0; q < maxpar && !e; q++) {
    e = plan_table(p->mark[q], mk[q], st);
    if (!e) e = plan_table(p->pin[q], pn[q], st);
    if (!e) e = plan_table(p->refill[q], rf[q], st);
  }
  if (!e && !move.empty()) {
    p->nmove = (int)move.size();
    if (cudaMalloc(&p->d_move, sizeof(int) * move.size()) != cudaSuccess) {
      (void)cudaGetLastError();
      e = SYM_ERR_OOM;
    } else {
      cudaMemcpyAsync(p->d_move, move.data(), sizeof(int) * move.size(), cudaMemcpyHostToDevice, st);
    }
  }
  SparsePlan::Table lt;
  if (!e && !ltb.empty()) {
    e = plan_table(lt, ltb, st);
    if (!e) k_sp_lagrange_table<<<(unsigned)lt.n, kT, 0, st>>>(p->d_dom[0], lt.d);
  }
  if (!e && cudaStreamSynchronize(st) != cudaSuccess) e = SYM_ERR_CUDA;
  if (lt.d) cudaFree(lt.d);
  if (e) {
    *err = e;
    sparse_plan_free(p);
    return nullptr;
  }
  // launches per step
  int l = 0;
  for (auto& t : p->fix) l += t.n ? 1 : 0;
  for (auto* v : {&p->mark, &p->pin, &p->refill})
    for (auto& t : *v) l += t.n ? 1 : 0;
  l += p->nmove ? 1 : 0;
  p->launches = l;
  return p;
}

namespace {
template <typename S>
void enqueue_plan(SparsePlan* p, int k, cudaStream_t st) {
  using R = typename Codec<S>::R;
  const SpDom* D = p->d_dom[k];
  auto& f = p->fix;
  auto go = [&](auto kern, const SparsePlan::Table& t, int threads = kT) {
    if (t.n) kern<<<t.n, threads, 0, st>>>(D, t.d);
  };
  go(k_sp_prep<S>, f[SparsePlan::PREP]);
  go(k_sp_lagrange, f[SparsePlan::LAG]);
  go(k_sp_capillary, f[SparsePlan::CAP]);
  go(k_sp_capillary_final, f[SparsePlan::CAPF], 32);
  go(k_sp_momentum, f[SparsePlan::MOM]);
  go(k_sp_momentum_final, f[SparsePlan::MOMF]);
  if (p->nmove) k_sp_move<<<(p->nmove + 31) / 32, 32, 0, st>>>(D, p->d_move, p->nmove);
  go(k_sp_reset, f[SparsePlan::RESET]);
  go(k_sp_flat, f[SparsePlan::FLAT]);
  for (auto& t : p->mark) go(k_sp_mark, t);
  go(k_sp_pin_plane, f[SparsePlan::PINPLANE]);
  for (auto& t : p->pin) go(k_sp_pin_box, t);
  for (auto& t : p->refill) go(k_sp_refill_import<S>, t);
  go(k_sp_pinfill_plane<R>, f[SparsePlan::PFPLANE]);
  go(k_sp_pinfill_box<R>, f[SparsePlan::PFBOX]);
}
}  // namespace

namespace {
template <typename S>
void enqueue_post(SparsePlan* p, int k, cudaStream_t st) {
  const auto& t = p->fix[SparsePlan::CURVE2];
  if (t.n) k_sp_curve2<S><<<t.n, kT, 0, st>>>(p->d_dom[k], t.d);
}
}  // namespace

// the work after the collide kernel of step parity k (the interpolated
// particle bounce-back), on `st`
int sparse_enqueue_post(SparsePlan* p, int k, cudaStream_t st) {
  if (!p || p->storage < 0 || !p->fix[SparsePlan::CURVE2].n) return SYM_OK;
  switch (p->storage) {
    case SYM_STORE_FP64: enqueue_post<double>(p, k, st); break;
    case SYM_STORE_FP32: enqueue_post<float>(p, k, st); break;
    default: enqueue_post<__half>(p, k, st);
  }
  return cudaGetLastError() == cudaSuccess ? SYM_OK : SYM_ERR_CUDA;
}

// the sparse work of step parity k on `st` (graph-capturable: no host sync)
int sparse_enqueue(SparsePlan* p, int k, cudaStream_t st) {
  if (!p || p->storage < 0) return SYM_OK;
  switch (p->storage) {
    case SYM_STORE_FP64: enqueue_plan<double>(p, k, st); break;
    case SYM_STORE_FP32: enqueue_plan<float>(p, k, st); break;
    default: enqueue_plan<__half>(p, k, st);
  }
  return cudaGetLastError() == cudaSuccess ? SYM_OK : SYM_ERR_CUDA;
}

int sparse_launches(const SparsePlan* p) { return p ? p->launches : 0; }

}  // namespace symb200
