// fused.cuh -- device code of the fused fast path, shared by the
// single-domain driver (fast.cu) and the batch engine (batch.cu).
// See fast.cu for the per-step kernel sequence.
#pragma once
#include <cuda_fp16.h>
#include <cmath>
#include <type_traits>
#include <utility>
#include "state.cuh"
#include "tma.cuh"

namespace symb200 {
namespace fused {

constexpr int BZ = 32;   // tile width along z: one warp per row
constexpr int XCHUNK = 32;   // x planes marched by one CTA

// ---- halo-padded phase field -----------------------------------------------------
struct Pad {
  int nxp, nyp, nzp;
  __host__ __device__ long long idx(int x, int y, int z) const {
    return (long long)(z + 2) + (long long)nzp * ((long long)(y + 2) + (long long)nyp * (long long)(x + 2));
  }
  __host__ __device__ long long size() const { return (long long)nxp * nyp * nzp; }
};
inline Pad make_pad(const DevParams& P) {
  Pad d;
  d.nxp = P.nx + 4;
  d.nyp = P.ny + 4;
  d.nzp = ((P.nz + 4) + 3) / 4 * 4;   // row stride a multiple of 16 bytes
  return d;
}

// store v at (x,y,z) and at each periodic image inside the 2-deep ghost layers
// (per axis: +n when within 2 of the low face, -n within 2 of the high face;
// both for n = 3).  Nodes 2 or more from every face store once.
template <typename R>
__device__ __forceinline__ void phi_store(const DevParams& P, const Pad& pd, R* phi, int x, int y, int z, R v) {
  if (x >= 2 && x < P.nx - 2 && y >= 2 && y < P.ny - 2 && z >= 2 && z < P.nz - 2) {
    phi[pd.idx(x, y, z)] = v;
    return;
  }
  int xs[3], ys[3], zs[3], nx = 1, ny = 1, nz = 1;
  xs[0] = x; ys[0] = y; zs[0] = z;
  if (x < 2) xs[nx++] = x + P.nx;
  if (x >= P.nx - 2) xs[nx++] = x - P.nx;
  if (y < 2) ys[ny++] = y + P.ny;
  if (y >= P.ny - 2) ys[ny++] = y - P.ny;
  if (z < 2) zs[nz++] = z + P.nz;
  if (z >= P.nz - 2) zs[nz++] = z - P.nz;
  for (int a = 0; a < nx; a++)
    for (int b = 0; b < ny; b++)
      for (int c = 0; c < nz; c++) phi[pd.idx(xs[a], ys[b], zs[c])] = v;
}

// ---- population storage codecs --------------------------------------------------
// Each velocity i holds an array of N slot pairs, pair index i*N + L: one
// aligned 2-slot load or store per velocity (8/16-byte pairs, 4-byte for the
// 16-bit storage), so a warp moves whole 128-byte lines per instruction.
// FP64 / FP32: the pair is (r, b).
// 16-bit storage (shifted storage, FP32 arithmetic): the pair is two FP16
// numbers relative to a reference pair (rho_ref, chi_ref) -- the density and
// red fraction of the node the population is stored at, from the step that
// wrote it (FP32):
//   q = 4096 (f - w rho_ref) / w    the total's deviation from its rest
//                                   equilibrium (the Laplace pressure jump
//                                   does not eat the significand; the 2^12
//                                   scale keeps deviations down to 1e-8 out
//                                   of the FP16 subnormal range)
//   d = 4096 (r - chi_ref f) / w    the red population's deviation from the
//                                   node's colour split of f: exactly 0 in a
//                                   pure phase, and the small colour
//                                   perturbations that seed an instability
//                                   keep FP16's 2^-11 relative precision
//                                   instead of a fixed step (no quotient)
// Encoder and decoder share the rounded rest equilibrium e = w rho_ref (one
// product, never contracted), so the rounding of the scale factors multiplies
// only the deviation and adds no bias to the mass.
// Indices are 32-bit pair offsets (the fused path requires 38*N < 2^32).
// load and store take the reference pair of the node the population is
// stored at (only the 16-bit codec uses it; kRef says whether it does).
using Ref = float2;
template <typename S>
struct Codec;
template <>
struct Codec<double> {
  using R = double;
  static constexpr bool kRef = false;
  template <int I>
  __device__ __forceinline__ static void load(const double* __restrict__ p, unsigned N, unsigned L, Ref, R& r, R& b) {
    const double2 v = reinterpret_cast<const double2*>(p)[I * N + L];
    r = v.x;
    b = v.y;
  }
  // total f = r + b and red r
  template <int I>
  __device__ __forceinline__ static void load_fr(const double* __restrict__ p, unsigned N, unsigned L, Ref, R& f,
                                                 R& r) {
    const double2 v = reinterpret_cast<const double2*>(p)[I * N + L];
    r = v.x;
    f = v.x + v.y;
  }
  template <int I>
  __device__ __forceinline__ static void store(double* p, unsigned N, unsigned L, Ref, R r, R f) {
    reinterpret_cast<double2*>(p)[I * N + L] = make_double2(r, f - r);
  }
};
template <>
struct Codec<float> {
  using R = float;
  static constexpr bool kRef = false;
  template <int I>
  __device__ __forceinline__ static void load(const float* __restrict__ p, unsigned N, unsigned L, Ref, R& r, R& b) {
    const float2 v = reinterpret_cast<const float2*>(p)[I * N + L];
    r = v.x;
    b = v.y;
  }
  template <int I>
  __device__ __forceinline__ static void load_fr(const float* __restrict__ p, unsigned N, unsigned L, Ref, R& f,
                                                 R& r) {
    const float2 v = reinterpret_cast<const float2*>(p)[I * N + L];
    r = v.x;
    f = v.x + v.y;
  }
  template <int I>
  __device__ __forceinline__ static void store(float* p, unsigned N, unsigned L, Ref, R r, R f) {
    reinterpret_cast<float2*>(p)[I * N + L] = make_float2(r, f - r);
  }
};
template <>
struct Codec<__half> {
  using R = float;
  static constexpr bool kRef = true;
  // total f and red r
  template <int I>
  __device__ __forceinline__ static void load_fr(const __half* __restrict__ p, unsigned N, unsigned L, Ref ref, R& f,
                                                 R& r) {
    const float2 q = __half22float2(reinterpret_cast<const __half2*>(p)[I * N + L]);
    f = fmaf(q.x, float(W(I) / 4096.0), __fmul_rn(float(W(I)), ref.x));
    r = fmaf(q.y, float(W(I) / 4096.0), ref.y * f);
  }
  template <int I>
  __device__ __forceinline__ static void load(const __half* __restrict__ p, unsigned N, unsigned L, Ref ref, R& r,
                                              R& b) {
    R f;
    load_fr<I>(p, N, L, ref, f, r);
    b = f - r;
  }
  template <int I>
  __device__ __forceinline__ static void store(__half* p, unsigned N, unsigned L, Ref ref, R r, R f) {
    constexpr float c = float(4096.0 / W(I));   // 12288, 73728 or 147456: exact
    const R q = (f - __fmul_rn(float(W(I)), ref.x)) * c;
    // exactly 0 in a pure phase: r = f with chi_ref = 1, r = 0 with chi_ref = 0
    const R d = fmaf(-ref.y, f, r) * c;
    reinterpret_cast<__half2*>(p)[I * N + L] = __floats2half2_rn(q, d);
  }
};
// the reference pair of node colour densities (sr, sb): density and red
// fraction (a pure phase exactly 1 or 0)
__device__ __forceinline__ Ref ref_pair(float sr, float sb) {
  const float rho = sr + sb;
  return make_float2(rho, sr / rho);
}
// the reference pair of a node with no populations of its own (solid): the
// rest density, half red
__device__ __forceinline__ Ref ref_rest(const DevParams& P) { return make_float2(float(P.rho0), 0.5f); }

// ---- next-step colour densities accumulated by the collide kernel ----------------
// The collide kernel of a step pushes every post-collision population to the
// node that holds it after streaming; it also adds the pushed values per
// destination node into two fixed-point accumulators (red, blue), so the next
// step's phase field (calmacros) reads 2 numbers per node instead of all 38
// populations.  Integer addition is associative, so the totals do not depend
// on the order in which the tiles' atomic adds land: the accumulated densities
// are deterministic.  FP64 storage: 64-bit integers in units of 2^-52
// (|rho| < 1024); FP32 arithmetic: 32-bit integers in units of 2^-26
// (|rho| < 31).  A value outside that range or not finite sets the domain's
// status word, and the next phase field is written as NaN (the NaN test of the
// stop rule then retires the run).
template <typename R>
struct Acc;
template <>
struct Acc<double> {
  using T = unsigned long long;
  __device__ __forceinline__ static T fix(double v) { return (T)__double2ll_rn(v * 0x1p52); }
  __device__ __forceinline__ static double val(T a) { return (double)(long long)a * 0x1p-52; }
  __device__ __forceinline__ static bool ok(double v) { return fabs(v) < 1024.0; }
};
template <>
struct Acc<float> {
  using T = unsigned int;
  __device__ __forceinline__ static T fix(float v) { return (T)__float2int_rn(v * 0x1p26f); }
  __device__ __forceinline__ static float val(T a) { return (float)(int)a * 0x1p-26f; }
  __device__ __forceinline__ static bool ok(float v) { return fabsf(v) < 31.0f; }
};
// Whether the collide kernel of storage S accumulates the next step's colour
// densities (the phase field then reads 2 values per node) or the phase field
// re-reads the populations (38 per node).  The accumulation costs arithmetic
// (warp shuffles, a shared-memory exchange, atomics), the re-read costs
// bytes: FP64 storage, bound by memory, accumulates; the 16-bit and FP32
// storages, bound by instruction issue, re-read.
template <typename S>
constexpr bool kAccumulate = sizeof(S) == 8;

// add v to accumulator p (a reduction: nothing is returned); out-of-range
// values set *status and add nothing
template <typename R>
__device__ __forceinline__ void acc_add(typename Acc<R>::T* p, R v, int* status) {
  if (Acc<R>::ok(v)) {
    atomicAdd(p, Acc<R>::fix(v));
  } else {
    atomicOr(status, 1);
  }
}

template <typename F, int... Is>
__device__ __forceinline__ void unroll19_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <typename F>
__device__ __forceinline__ void unroll19(F&& f) {
  unroll19_impl(f, std::make_integer_sequence<int, 19>{});
}

// ---- calmacros (Source1.f90:770-831) on the fused state ---------------------------
// Storages that do not accumulate: phi = (rhoR - rhoB) / rho from the node's
// own post-stream populations; 0 on solid nodes.  16-bit storage decodes with
// the reference pairs rr_old and records the node's (rho, red fraction) in rr_new:
// the references this step's encoders use and the next step decodes with.
template <typename S, bool SOLID>
__device__ __forceinline__ void phase_node(const DevParams& P, const Pad& pd, const S* __restrict__ pops,
                                           typename Codec<S>::R* __restrict__ phi,
                                           const int32_t* __restrict__ walls_all, const Ref* __restrict__ rr_old,
                                           Ref* __restrict__ rr_new, long long L) {
  using R = typename Codec<S>::R;
  if (L >= P.N) return;
  const unsigned Lu = (unsigned)L, q = Lu / (unsigned)P.nz;
  const int z = (int)(Lu - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
  R v = R(0);
  Ref nref = ref_rest(P);
  if (!(SOLID && walls_all[L] >= 1)) {
    const unsigned N = (unsigned)P.N;
    if constexpr (Codec<S>::kRef) {
      const Ref ref = rr_old[pd.idx(x, y, z)];
      R sr = R(0), sb = R(0);
      unroll19([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        R r, b;
        Codec<S>::template load<i>(pops, N, Lu, ref, r, b);
        sr = sr + r;
        sb = sb + b;
      });
      v = qdiv<R>(sr - sb, sr + sb);
      nref = ref_pair(float(sr), float(sb));
    } else {
      R sr = R(0), sf = R(0);
      unroll19([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        R f, r;
        Codec<S>::template load_fr<i>(pops, N, Lu, Ref{}, f, r);
        sr = sr + r;
        sf = sf + f;
      });
      v = qdiv<R>(sr - (sf - sr), sf);
    }
  }
  phi_store<R>(P, pd, phi, x, y, z, v);
  if constexpr (Codec<S>::kRef) phi_store<Ref>(P, pd, rr_new, x, y, z, nref);
}

template <typename S, bool SOLID>
__global__ void __launch_bounds__(256) k_phase(DevParams P, Pad pd, const S* __restrict__ pops,
                                               typename Codec<S>::R* __restrict__ phi,
                                               const int32_t* __restrict__ walls_all, const Ref* __restrict__ rr_old,
                                               Ref* __restrict__ rr_new) {
  phase_node<S, SOLID>(P, pd, pops, phi, walls_all, rr_old, rr_new, blockIdx.x * 256LL + threadIdx.x);
}

// From the accumulated colour densities (the steady-state phase field):
// phi = (rhoR - rhoB) / rho on fluid nodes, 0 on solid nodes, written with its
// periodic ghost images; the accumulators are cleared for the collide kernel
// of this step.  A storage with references (kRef) would also record the
// node's (rho, red fraction) in rr_new, as phase_node does.
// Nodes L0, L0 + 256, ..., L0 + 256 (NPT-1) per thread: every load of all of
// them is issued before the first store, so a thread keeps 2 NPT accumulator
// reads in flight (nothing waits on a store).
template <typename S, bool SOLID, int NPT>
__device__ __forceinline__ void finalize_nodes(const DevParams& P, const Pad& pd,
                                               typename Acc<typename Codec<S>::R>::T* __restrict__ acc,
                                               typename Codec<S>::R* __restrict__ phi,
                                               const int32_t* __restrict__ walls_all, Ref* __restrict__ rr_new,
                                               const int* __restrict__ status, long long L0) {
  using R = typename Codec<S>::R;
  using A = Acc<R>;
  const int bad = *status;
  typename A::T ar[NPT], ab[NPT];
  bool solid[NPT];
#pragma unroll
  for (int k = 0; k < NPT; k++) {
    const long long L = L0 + 256LL * k;
    ar[k] = ab[k] = 0;
    solid[k] = false;
    if (L < P.N) {
      ar[k] = acc[L];
      ab[k] = acc[L + P.N];
      solid[k] = SOLID && walls_all[L] >= 1;
    }
  }
#pragma unroll
  for (int k = 0; k < NPT; k++) {
    const long long L = L0 + 256LL * k;
    if (L >= P.N) break;
    acc[L] = 0;
    acc[L + P.N] = 0;
    // 32-bit index arithmetic (the fused path keeps 38*N < 2^32)
    const unsigned Lu = (unsigned)L, q = Lu / (unsigned)P.nz;
    const int z = (int)(Lu - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
    const R sr = A::val(ar[k]), sb = A::val(ab[k]);
    R v = R(0);
    Ref nref = ref_rest(P);
    if (!solid[k]) {
      v = qdiv<R>(sr - sb, sr + sb);
      nref = ref_pair(float(sr), float(sb));
    }
    if (bad) v = R(NAN);
    phi_store<R>(P, pd, phi, x, y, z, v);
    if constexpr (Codec<S>::kRef) phi_store<Ref>(P, pd, rr_new, x, y, z, nref);
  }
}

// nodes finalised per thread by the single-domain kernel
constexpr int kFinalizeNPT = 4;

template <typename S, bool SOLID>
__global__ void __launch_bounds__(256) k_finalize(DevParams P, Pad pd, typename Acc<typename Codec<S>::R>::T* acc,
                                                  typename Codec<S>::R* __restrict__ phi,
                                                  const int32_t* __restrict__ walls_all, Ref* __restrict__ rr_new,
                                                  const int* __restrict__ status) {
  finalize_nodes<S, SOLID, kFinalizeNPT>(P, pd, acc, phi, walls_all, rr_new, status,
                                         blockIdx.x * (256LL * kFinalizeNPT) + threadIdx.x);
}

// ---- wetting rotation of a node normal (derivatives :535-587) ---------------------
template <typename R>
__device__ __forceinline__ void wet_rotate(const DevParams& P, const sym_particles* S, int pp, int x, int y, int z,
                                           R& n0, R& n1, R& n2) {
  double nwd[3];
  wall_normal_dev(P, S, pp, x, y, z, nwd);
  const R nw[3] = {R(nwd[0]), R(nwd[1]), R(nwd[2])};
  const R n[3] = {n0, n1, n2};
  R v[3];
  akai_rotate_sc<R>(R(P.sin_cita), R(P.cos_cita), nw, n, true, v);
  n0 = v[0]; n1 = v[1]; n2 = v[2];
}

// ---- k_collide ------------------------------------------------------------------
// phi ring of 5 planes, normal ring of 4 planes, reference-pair ring of 6 planes:
// normals are computed one plane ahead and phi / reference-pair loaded three planes
// ahead, before the plane's single barrier.  A warp that has finished plane x
// runs those writes for plane x+1 while slower warps still read plane x's
// slots: phi at x, normals at x-1..x+1 and reference-pair at x-1..x+1 (the push
// targets).  The rings are sized so that the slots written for plane x+1
// (phi x+4 -> slot (x-1)%5, normals x+2 -> (x-2)%4, reference-pair x+4 -> (x-2)%6)
// are never among them.
constexpr int kIrrRing = 6;
// unit normal and |grad phi| of one node, read with one (FP32) or two (FP64)
// 16-byte shared-memory accesses
template <typename R>
struct alignas(4 * sizeof(R)) NormalV {
  R x, y, z, g;
};
// Tile height (rows of BZ nodes) of the collide kernels per storage: 16
// rows for the 16-bit codec, 8 for FP32 and FP64.  Measured on the batched
// mix: 16 rows (2 CTAs of 512 threads per SM) took the 16-bit collide from
// 4.79 to 4.28 ms against 8 rows (4 CTAs of 256) -- fewer halo normals, halo
// bytes and barriers per node -- and changed nothing in FP32; FP64 at 16 rows
// fits one CTA per SM and was slower (C3: 4.70 against 4.52 ms).
template <typename S>
constexpr int kBY = std::is_same<S, __half>::value ? 16 : 8;
template <typename S>
constexpr int kTPB = BZ * kBY<S>;
// the same for a storage mode chosen at run time (SYM_STORE_*)
inline int tile_rows(int storage) {
  return storage == SYM_STORE_FP16 ? kBY<__half> : (storage == SYM_STORE_FP32 ? kBY<float> : kBY<double>);
}
// phi and reference-pair plane tiles ((BY+4) x (BZ+4), z fastest) arrive by TMA:
// each slot starts on a 128-byte boundary
template <typename S>
constexpr int kPlaneTile = (kBY<S> + 4) * (BZ + 4);
template <typename S>
struct Smem {
  using R = typename Codec<S>::R;
  static constexpr int BY = kBY<S>;
  static constexpr int kPhiSlot = (kPlaneTile<S> * (int)sizeof(R) + 127) / 128 * 128 / (int)sizeof(R);
  static constexpr int kRefSlot = (kPlaneTile<S> * 8 + 127) / 128 * 128 / 8;
  alignas(128) R phi[5][kPhiSlot];
  alignas(128) Ref ref[Codec<S>::kRef ? kIrrRing : 1][kRefSlot];   // reference pairs of this step (16-bit storage)
  NormalV<R> n[4][BY + 2][BZ + 2];   // [plane][y][z]: n and |grad phi|
  // [cx+1][to row y+1, y-1][colour]: density sums crossing rows (accumulating
  // storages only; a single element otherwise)
  R xch[kAccumulate<S> ? 3 : 1][2][2][kAccumulate<S> ? BY : 1][kAccumulate<S> ? BZ : 1];
  uint64_t bar[kIrrRing];   // one mbarrier per plane load, used round robin
};
// dynamic shared memory of the collide kernels: the Smem block on a 128-byte
// boundary inside the allocation
template <typename S>
constexpr size_t smem_bytes() { return sizeof(Smem<S>) + 128; }
template <typename S>
__device__ __forceinline__ Smem<S>& smem_view(unsigned char* raw) {
  const uintptr_t a = (reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127);
  return *reinterpret_cast<Smem<S>*>(a);
}
// the CTA's mbarriers: initialised once per kernel by thread 0
template <typename S>
__device__ __forceinline__ void collide_init_barriers(Smem<S>& sm) {
  if (threadIdx.x == 0) {
    for (int k = 0; k < kIrrRing; k++) tma::mbar_init(&sm.bar[k], 1);
    tma::mbar_fence_init();
  }
  __syncthreads();
}
// push order of the collide kernel: groups of equal (cx, cy), cz = 0, +1, -1
// last (velocity numbering of Source1.f90:132-134)
__host__ __device__ __forceinline__ constexpr int PUSH_ORDER(int k) {
  constexpr int a[19] = {0, 5, 6, 1, 11, 13, 2, 12, 14, 3, 15, 17, 4, 16, 18, 7, 8, 9, 10};
  return a[k];
}

// One tile: the 32(z) x BY(y) footprint at (z0, y0), planes xa..xb-1.  Called
// by the single-domain kernel (tile from blockIdx) and by the batched
// persistent kernel (tile from the work-tile table).
template <typename S, bool SOLID>
__device__ __forceinline__ void collide_tile(const DevParams& P, const Pad& pd, const S* __restrict__ pin_,
                                             S* __restrict__ pout_, const typename Codec<S>::R* __restrict__ phi,
                                             const int32_t* __restrict__ walls,
                                             const int32_t* __restrict__ walls_all,
                                             const int32_t* __restrict__ pout,
                                             const sym_particles* __restrict__ Sp, double* __restrict__ ffi,
                                             const Ref* __restrict__ rr_old, const Ref* __restrict__ rr_new,
                                             typename Acc<typename Codec<S>::R>::T* acc, int* status,
                                             const CUtensorMap* tm_phi, const CUtensorMap* tm_ref,
                                             int z0, int y0, int xa, int xb, Smem<S>& sm, unsigned& nload,
                                             bool solid_rt = true) {
  using R = typename Codec<S>::R;
  constexpr int BY = kBY<S>, TPB = kTPB<S>, kTile = kPlaneTile<S>;
  // solid handling: compiled in (SOLID) and wanted by this domain (solid_rt);
  // the batched kernel compiles one variant and decides per tile
  const bool SOLIDX = SOLID && solid_rt;
  constexpr bool ACC = kAccumulate<S>;
  constexpr bool REF = Codec<S>::kRef;
  const int tz = threadIdx.x % BZ, ty = threadIdx.x / BZ;
  const unsigned N = (unsigned)P.N;
  const R evap = R(P.evap);
  const int sy = P.nz, sx = P.nz * P.ny;   // element strides of y and x

  // phi (and the reference pairs) of plane xp by TMA: one box of (BY+4) x (BZ+4) at the
  // padded origin (z0, y0, xp+2) -- z0 is a multiple of 32 elements, so the
  // innermost coordinate is 128-byte aligned; rows past the padded extent read
  // as zeros.  Plane xp is load number nl0 + xp - (xa - 2) of this CTA, on
  // mbarrier (number mod 6) with phase parity (number / 6) mod 2.
  const unsigned nl0 = nload;
  auto load_no = [&](int xp) { return nl0 + (unsigned)(xp - (xa - 2)); };
  constexpr uint32_t kTx = kTile * (sizeof(R) + (REF ? sizeof(Ref) : 0));
  auto load_phi = [&](int xp) {   // thread 0 only
    const unsigned q = load_no(xp);
    uint64_t* bar = &sm.bar[q % kIrrRing];
    tma::mbar_expect_tx(bar, kTx);
    tma::load_3d(sm.phi[((xp % 5) + 5) % 5], tm_phi, z0, y0, xp + 2, bar);
    if (REF) tma::load_3d(sm.ref[(unsigned)(xp + kIrrRing) % kIrrRing], tm_ref, z0, y0, xp + 2, bar);
  };
  auto wait_phi = [&](int xp) {   // every thread
    const unsigned q = load_no(xp);
    if (!tma::mbar_wait(&sm.bar[q % kIrrRing], (q / kIrrRing) & 1u)) atomicOr(status, 2);
  };
  auto PHI = [&](int xp, int py, int pz) -> R { return sm.phi[((xp % 5) + 5) % 5][py * (BZ + 4) + pz]; };
  // unit normal (rotated at wetting nodes) and |grad phi| of plane xp, halo 1
  auto compute_n = [&](int xp) {
    const int s = xp & 3;   // xp >= -1: the slot in the 4-plane normal ring
    // phi planes xp-1, xp, xp+1 in the 5-plane ring (xp >= -1)
    const R* const pm = sm.phi[(unsigned)(xp + 4) % 5u];
    const R* const p0 = sm.phi[(unsigned)(xp + 5) % 5u];
    const R* const pp1 = sm.phi[(unsigned)(xp + 6) % 5u];
    for (int t = threadIdx.x; t < (BY + 2) * (BZ + 2); t += TPB) {
      const int py = t / (BZ + 2), pz = t % (BZ + 2);
      const int y = y0 - 1 + py, z = z0 - 1 + pz;
      R n0 = R(0), n1 = R(0), n2 = R(0), fn = R(0);
      bool ok = y <= P.ny && z <= P.nz;
      int pp = 0;
      if (SOLIDX && ok) {
        const unsigned Lw = (unsigned)(wrapi(z, P.nz) + sy * wrapi(y, P.ny) + sx * wrapi(xp, P.nx));
        if (walls_all[Lw] > 0) ok = false;
        else pp = pout[Lw];
      }
      if (ok) {
        // grad phi = 3 sum_i w_i c_i phi(x + c_i) (:510-521), summed over the
        // nine opposite pairs: w_i c_i (phi(x + c_i) - phi(x - c_i))
        R g0 = R(0), g1 = R(0), g2 = R(0);
        static_for<9>([&](auto kc) {
          constexpr int i = PREP(decltype(kc)::value);
          constexpr int o = CY(i) * (BZ + 4) + CZ(i);
          const int b = (py + 1) * (BZ + 4) + pz + 1;
          const R* const pa = CX(i) > 0 ? pp1 : (CX(i) < 0 ? pm : p0);
          const R* const pb = CX(i) > 0 ? pm : (CX(i) < 0 ? pp1 : p0);
          const R d = pa[b + o] - pb[b - o];
          if (CX(i)) g0 = g0 + R(W(i) * CX(i)) * d;
          if (CY(i)) g1 = g1 + R(W(i) * CY(i)) * d;
          if (CZ(i)) g2 = g2 + R(W(i) * CZ(i)) * d;
        });
        g0 = R(3) * g0; g1 = R(3) * g1; g2 = R(3) * g2;
        const R g2s = g0 * g0 + g1 * g1 + g2 * g2;
        R rf = R(0);
        if constexpr (sizeof(R) == 4) {
          // FP32 arithmetic: |grad phi| and its reciprocal from one rsqrt
          if (g2s > evap * evap) { rf = rsqrtf(g2s); fn = g2s * rf; }
        } else {
          fn = sqrt(g2s);
          if (fn > evap) rf = R(1) / fn; else fn = R(0);
        }
        if (fn > R(0)) {
          n0 = g0 * rf; n1 = g1 * rf; n2 = g2 * rf;
          if (SOLIDX && pp >= 1) wet_rotate<R>(P, Sp, pp, wrapi(xp, P.nx), wrapi(y, P.ny), wrapi(z, P.nz), n0, n1, n2);
        }
      }
      sm.n[s][py][pz] = NormalV<R>{n0, n1, n2, fn};
    }
  };

  if (threadIdx.x == 0)
    for (int xp = xa - 2; xp <= xa + 2; xp++) load_phi(xp);
  for (int xp = xa - 2; xp <= xa + 2; xp++) wait_phi(xp);
  compute_n(xa - 1);
  compute_n(xa);
  // the first iteration's phi load reuses the slot of plane xa-2, which
  // compute_n(xa-1) above reads
  __syncthreads();
  nload = nl0 + (unsigned)(xb - xa + 4);   // loads of this tile: planes xa-2 .. xb+1

  const int y = y0 + ty, z = z0 + tz;
  const bool inr = y < P.ny && z < P.nz;
  // every lane runs the node arithmetic (lanes outside the domain on a
  // clamped node), so the warp shuffles of the density accumulation below see
  // the whole warp; `act` masks the stores and contributions
  const int yc = min(y, P.ny - 1), zc = min(z, P.nz - 1);
  // pushes whose destination lies outside this CTA's tile (or across a
  // periodic wrap) are added to the accumulators directly; the others are
  // combined inside the CTA first (z through warp shuffles, y through shared
  // memory, x in registers along the march) and added once per node
  const bool ezp = tz == BZ - 1 || z >= P.nz - 1, ezm = tz == 0 || z == 0;
  const bool eyp = ty == BY - 1 || y >= P.ny - 1, eym = ty == 0 || y == 0;
  using AT = typename Acc<R>::T;
  AT* const accR = acc;
  AT* const accB = acc + N;
  R aPr = R(0), aPb = R(0), aCr = R(0), aCb = R(0), aNr = R(0), aNb = R(0);   // planes x-1, x, x+1
  for (int x = xa; x < xb; x++) {
    // phi of plane x+3 on its way; normals of plane x+1 from phi planes x..x+2.
    // The slots the load overwrites (phi of plane x-2, reference pairs of plane x-3)
    // were last read before the previous plane's barriers.
    if (threadIdx.x == 0 && x + 3 <= xb + 1) load_phi(x + 3);
    wait_phi(x + 2);
    compute_n(x + 1);
    __syncthreads();
    const unsigned L = (unsigned)(zc + sy * yc + sx * x);
    int pp = 0;
    bool act = inr;
    if (SOLIDX) {
      if (walls_all[L] > 0) act = false;
      else pp = pout[L];
    }
    // g[cx+1][cy+1][colour]: in-tile pushes summed per destination column and
    // plane (cz = +-1 pushes arrive from the neighbouring lanes); sf: links
    // bounced back into this node
    R g[3][3][2];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
#pragma unroll
        for (int c = 0; c < 2; c++) g[a][b][c] = R(0);
    R sfr = R(0), sfb = R(0);
    // accumulating kernels run every lane of a warp with an active node (the
    // shuffles need the whole warp); the others skip inactive nodes
    if (sizeof(R) == 8 && x + 1 < xb && threadIdx.x < 19 * BY) {
      // FP64: the next plane's populations toward L2 while this plane
      // computes, one bulk prefetch per (velocity, row) of the tile, by
      // 19 x BY threads; the range is widened to 16-byte boundaries inside
      // the array.  (Measured: FP64 collide 4.71 ms with it, 4.87 with one
      // prefetch per population and thread, 4.89 without on the C3 thread;
      // the FP32-math kernels are faster without any.)
      constexpr size_t PB = 2 * sizeof(S);   // bytes per slot pair
      const int i = threadIdx.x / BY, yy = y0 + (int)threadIdx.x % BY;
      if (yy < P.ny) {
        const size_t a = ((size_t)i * N + (size_t)(z0 + sy * yy + sx * (x + 1))) * PB;
        const size_t e = min(a + (size_t)min(BZ, P.nz - z0) * PB + 15, (size_t)19 * N * PB) & ~size_t(15);
        const size_t b = a & ~size_t(15);
        if (e > b) tma::prefetch_l2(reinterpret_cast<const char*>(pin_) + b, (uint32_t)(e - b));
      }
    }
    if (ACC ? __any_sync(0xffffffffu, act) : act) {
    // calmacros on the own populations
    // (rho_B = rho - rho_R: a pure colour stays exactly pure, as r = f there)
    R f[19];
    R sr = R(0), rho = R(0);
    const Ref rref = REF ? rr_old[pd.idx(x, yc, zc)] : Ref{};
    unroll19([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      R r;
      Codec<S>::template load_fr<i>(pin_, N, L, rref, f[i], r);
      sr = sr + r;
      rho = rho + f[i];
    });
    const R sb = rho - sr;
    R ux = R(0), uy = R(0), uz = R(0);
#pragma unroll
    for (int i = 0; i < 19; i++) {
      if (CX(i)) ux = ux + f[i] * R(CX(i));
      if (CY(i)) uy = uy + f[i] * R(CY(i));
      if (CZ(i)) uz = uz + f[i] * R(CZ(i));
    }
    const R irho = qdiv<R>(R(1), rho);
    ux = ux * irho; uy = uy * irho; uz = uz * irho;
    const NormalV<R> nown = sm.n[x & 3][ty + 1][tz + 1];
    const R nx = nown.x, ny = nown.y, nz = nown.z, fn = nown.g;
    const bool flag = fn > evap;
    const R rhoN = PHI(x, ty + 2, tz + 2);
    // CSF surface tension from the curvature of the normal field (:624-667)
    R fx = R(0), fy = R(0), fz = R(0);
    if (flag && (!SOLIDX || pp <= 0)) {
      // d_ba = sum_i w_i c_ia n_b(x + c_i) (:635-660), over the nine opposite
      // pairs: w_i c_ia (n_b(x + c_i) - n_b(x - c_i))
      R d00 = 0, d01 = 0, d02 = 0, d10 = 0, d11 = 0, d12 = 0, d20 = 0, d21 = 0, d22 = 0;
      static_for<9>([&](auto kc) {
        constexpr int i = PREP(decltype(kc)::value);
        const NormalV<R> p = sm.n[(x + CX(i)) & 3][ty + 1 + CY(i)][tz + 1 + CZ(i)];
        const NormalV<R> m = sm.n[(x - CX(i)) & 3][ty + 1 - CY(i)][tz + 1 - CZ(i)];
        const R a = p.x - m.x, b = p.y - m.y, c = p.z - m.z;
        if (CX(i)) { constexpr double k = W(i) * CX(i); d00 = d00 + R(k) * a; d10 = d10 + R(k) * b; d20 = d20 + R(k) * c; }
        if (CY(i)) { constexpr double k = W(i) * CY(i); d01 = d01 + R(k) * a; d11 = d11 + R(k) * b; d21 = d21 + R(k) * c; }
        if (CZ(i)) { constexpr double k = W(i) * CZ(i); d02 = d02 + R(k) * a; d12 = d12 + R(k) * b; d22 = d22 + R(k) * c; }
      });
      d00 *= R(3); d01 *= R(3); d02 *= R(3); d10 *= R(3); d11 *= R(3); d12 *= R(3);
      d20 *= R(3); d21 *= R(3); d22 *= R(3);
      const R kurv = nx * ny * (d10 + d01) + nx * nz * (d20 + d02) + ny * nz * (d12 + d21) -
                     (ny * ny + nz * nz) * d00 - (nx * nx + nz * nz) * d11 - (nx * nx + ny * ny) * d22;
      const R val = R(0.5) * R(P.sigma) * kurv;
      fx = val * (fn * nx); fy = val * (fn * ny); fz = val * (fn * nz);
    }
    fx = fx + rho * R(P.body[0]);
    fy = fy + rho * R(P.body[1]);
    fz = fz + rho * R(P.body[2]);
    const R hirho = R(0.5) * irho;
    ux = ux + fx * hirho;
    uy = uy + fy * hirho;
    uz = uz + fz * hirho;
    mrt_collide_pairs<R>(P, f, rho, ux, uy, uz, fx, fy, fz, rhoN);
    // post-collision populations for the momentum exchange (:1241-1243), read
    // only next to particles (pout = particle id); wall planes (ids > par)
    // need none, and a handle without particles holds no ffi array
    if (SOLIDX && act && pp >= 1 && pp <= P.par) {
#pragma unroll
      for (int i = 0; i < 19; i++) ffi[(size_t)i * N + L] = (double)f[i];
    }
    // Latva-Kokko recolouring (:712-726): r_i = (rhoR/rho) f_i + beta rhoR rhoB /
    // rho w_i (n.c_i); a colour at or below EVAP_LIM empties (r_i = 0 when
    // rhoR is, r_i = f_i when rhoB is, the latter taking precedence), which the
    // two coefficients express once per node
    const bool rzero = sr <= evap, bzero = sb <= evap;
    const R ratio = bzero ? R(1) : (rzero ? R(0) : sr * irho);
    const R coef = (bzero || rzero || !flag) ? R(0) : sr * sb * irho * R(P.beta);
    const bool exp_ = x == xb - 1, exm = x == xa;
    // rigid-body velocity of particle pp at this node (curve :1009-1014), for
    // the links that bounce back from it
    R uw0 = R(0), uw1 = R(0), uw2 = R(0);
    if (SOLIDX && pp >= 1 && pp <= P.par) {
      const int par = P.par;
      const R xr = R(disp(P, (double)(x + P.origin), Sp->center[0 * par + pp - 1], 0));
      const R yr = R(disp(P, (double)(y + P.origin), Sp->center[1 * par + pp - 1], 1));
      const R zr = R(disp(P, (double)(z + P.origin), Sp->center[2 * par + pp - 1], 2));
      uw0 = R(Sp->up[0 * par + pp - 1]) + zr * R(Sp->rp[1 * par + pp - 1]) - yr * R(Sp->rp[2 * par + pp - 1]);
      uw1 = R(Sp->up[1 * par + pp - 1]) + xr * R(Sp->rp[2 * par + pp - 1]) - zr * R(Sp->rp[0 * par + pp - 1]);
      uw2 = R(Sp->up[2 * par + pp - 1]) + yr * R(Sp->rp[0 * par + pp - 1]) - xr * R(Sp->rp[1 * par + pp - 1]);
    }
    // neighbour offsets with the periodic wrap folded in (one select per face)
    const int oxp = (x == P.nx - 1) ? -(P.nx - 1) * sx : sx, oxm = (x == 0) ? (P.nx - 1) * sx : -sx;
    const int oyp = (yc == P.ny - 1) ? -(P.ny - 1) * sy : sy, oym = (yc == 0) ? (P.ny - 1) * sy : -sy;
    const int ozp = (zc == P.nz - 1) ? -(P.nz - 1) : 1, ozm = (zc == 0) ? (P.nz - 1) : -1;
    R zp[2] = {R(0), R(0)}, zm[2] = {R(0), R(0)};
    // directions in groups of equal (cx, cy): within a group only cz differs,
    // and the cz = +-1 pushes of the group move one lane up / down right after it
    static_for<19>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      constexpr int i = PUSH_ORDER(k);
      constexpr int a = CX(i) + 1, b = CY(i) + 1;
      [&] {
        R r = ratio * f[i];
        if (i > 0) r = r + coef * R(W(i)) * (nx * R(CX(i)) + ny * R(CY(i)) + nz * R(CZ(i)));
        const unsigned T = L + (CX(i) > 0 ? oxp : (CX(i) < 0 ? oxm : 0)) +
                           (CY(i) > 0 ? oyp : (CY(i) < 0 ? oym : 0)) + (CZ(i) > 0 ? ozp : (CZ(i) < 0 ? ozm : 0));
        if (!act) return;
        // interpolated bounce-back: the red post-collision populations of the
        // nodes next to particles, for the link update after this kernel
        if (SOLIDX && P.bounce && pp >= 1 && pp <= P.par) ffi[(size_t)(19 + i) * N + L] = (double)r;
        if (SOLIDX && i > 0 && pp >= 1) {
          const int wb = walls[T];
          const bool flat = wb > P.par;
          if (wb == pp || flat) {
            // curve (:1001-1019): link OPC(i) of this node comes back reversed
            constexpr int j = OPC(i);
            const R star = flat ? R(0) : uw0 * R(CX(j)) + uw1 * R(CY(j)) + uw2 * R(CZ(j));
            const R rr = r + R(6.0 * W(j)) * sr * star;
            const R bb = (f[i] - r) + R(6.0 * W(j)) * sb * star;
            const Ref rd = REF ? sm.ref[(unsigned)x % kIrrRing][(ty + 2) * (BZ + 4) + tz + 2] : Ref{};
            Codec<S>::template store<j>(pout_, N, L, rd, rr, rr + bb);
            sfr = sfr + rr;
            sfb = sfb + bb;
            return;
          }
        }
        const Ref rd = REF ? sm.ref[(unsigned)(x + CX(i) + kIrrRing) % kIrrRing]
                                   [(ty + 2 + CY(i)) * (BZ + 4) + tz + 2 + CZ(i)]
                           : Ref{};
        Codec<S>::template store<i>(pout_, N, T, rd, r, f[i]);
        if constexpr (!ACC) return;
        const R bv = f[i] - r;
        const bool ext = (CX(i) > 0 && exp_) || (CX(i) < 0 && exm) || (CY(i) > 0 && eyp) || (CY(i) < 0 && eym) ||
                         (CZ(i) > 0 && ezp) || (CZ(i) < 0 && ezm);
        if (ext) {
          acc_add<R>(accR + T, r, status);
          acc_add<R>(accB + T, bv, status);
        } else if (CZ(i) == 0) {
          g[a][b][0] = g[a][b][0] + r;
          g[a][b][1] = g[a][b][1] + bv;
        } else if (CZ(i) > 0) {
          zp[0] = r;
          zp[1] = bv;
        } else {
          zm[0] = r;
          zm[1] = bv;
        }
      }();
      if constexpr (ACC && CZ(i) < 0) {
        // last of a group with cz = 0, +1, -1: lane l receives the cz = +1 push
        // of lane l-1 and the cz = -1 push of lane l+1 (lane = tz)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const R up = __shfl_up_sync(0xffffffffu, zp[c], 1);
          const R dn = __shfl_down_sync(0xffffffffu, zm[c], 1);
          g[a][b][c] = g[a][b][c] + (tz > 0 ? up : R(0)) + (tz < BZ - 1 ? dn : R(0));
          zp[c] = R(0);
          zm[c] = R(0);
        }
      }
    });
    }
    if constexpr (ACC) {
      // along y through shared memory: row ty+1 receives the cy = +1 sums of row
      // ty and row ty-1 the cy = -1 sums, for each destination plane
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          sm.xch[a][0][c][ty][tz] = g[a][2][c];
          sm.xch[a][1][c][ty][tz] = g[a][0][c];
        }
      __syncthreads();
      R in[3][2];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          R v = g[a][1][c];
          if (ty > 0) v = v + sm.xch[a][0][c][ty - 1][tz];
          if (ty < BY - 1) v = v + sm.xch[a][1][c][ty + 1][tz];
          in[a][c] = v;
        }
      aPr = aPr + in[0][0]; aPb = aPb + in[0][1];
      aCr = aCr + in[1][0] + sfr; aCb = aCb + in[1][1] + sfb;
      aNr = aNr + in[2][0]; aNb = aNb + in[2][1];
      // plane x-1 of this column has all its in-tile contributions
      if (x > xa && inr && (aPr != R(0) || aPb != R(0))) {
        acc_add<R>(accR + (L - sx), aPr, status);
        acc_add<R>(accB + (L - sx), aPb, status);
      }
      aPr = aCr; aPb = aCb;
      aCr = aNr; aCb = aNb;
      aNr = R(0); aNb = R(0);
    }
  }
  if (ACC && xb > xa && inr && (aPr != R(0) || aPb != R(0))) {
    const unsigned L = (unsigned)(z + sy * y + sx * (xb - 1));
    acc_add<R>(accR + L, aPr, status);
    acc_add<R>(accB + L, aPb, status);
  }
}

// Resident CTAs per SM the collide kernels are compiled for: the FP32-math
// codecs fit 64 registers (32 warps per SM: 4 CTAs of 256 threads for FP32,
// 2 of 512 for the 16-bit codec; measured faster than 3 CTAs of 256 at 80
// registers, the latency-bound kernel gains from the extra warps), FP64 needs
// the 128 of 2 CTAs of 256.
template <typename S>
constexpr int collide_ctas() {
  return std::is_same<S, __half>::value ? 2 : (sizeof(typename Codec<S>::R) == 4 ? 4 : 2);
}

template <typename S, bool SOLID>
__global__ void __launch_bounds__(kTPB<S>, collide_ctas<S>()) k_collide(DevParams P, Pad pd, const S* __restrict__ pin_,
                                                   S* __restrict__ pout_,
                                                   const typename Codec<S>::R* __restrict__ phi,
                                                   const int32_t* __restrict__ walls,
                                                   const int32_t* __restrict__ walls_all,
                                                   const int32_t* __restrict__ pout,
                                                   const sym_particles* __restrict__ Sp, double* __restrict__ ffi,
                                                   const Ref* __restrict__ rr_old, const Ref* __restrict__ rr_new,
                                                   typename Acc<typename Codec<S>::R>::T* acc, int* status,
                                                   const __grid_constant__ CUtensorMap tm_phi,
                                                   const __grid_constant__ CUtensorMap tm_ref, int xchunk) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem<S>& sm = smem_view<S>(smem_raw);
  collide_init_barriers<S>(sm);
  unsigned nload = 0;
  const int xa = blockIdx.z * xchunk;
  collide_tile<S, SOLID>(P, pd, pin_, pout_, phi, walls, walls_all, pout, Sp, ffi, rr_old, rr_new, acc, status,
                         &tm_phi, &tm_ref, blockIdx.x * BZ, blockIdx.y * kBY<S>, xa, min(xa + xchunk, P.nx), sm,
                         nload);
}

// ---- the fused state's side of the particle and wall work ---------------------------
// (device bodies; the batched launches are in sparse.cu)

// pin fill (derivatives :467-492): fictitious phi of solid node (x,y,z) next
// to fluid = wi-weighted mean of its fluid neighbours
template <typename R>
__device__ __forceinline__ void pinfill_node(const DevParams& P, const Pad& pd, R* phi,
                                             const int32_t* __restrict__ pin, const int32_t* __restrict__ walls_all,
                                             int x, int y, int z) {
  const long long L = lin(P, x, y, z);
  if (pin[L] <= 0) return;
  R ws = R(0), v = R(0);
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const long long nb = lin(P, wrapi(x + CX(i), P.nx), wrapi(y + CY(i), P.ny), wrapi(z + CZ(i), P.nz));
    if (walls_all[nb] <= 0) { ws = ws + R(W(i)); v = v + R(W(i)) * phi[pd.idx(x + CX(i), y + CY(i), z + CZ(i))]; }
  }
  phi_store<R>(P, pd, phi, x, y, z, v / ws);
}

// particle preparation: canonical views of the fused state at a node of a
// particle box -- rho_N (this step's calmacros), rho_R/rho_B and, at nodes
// next to a particle, fi (current populations), and the previous step's
// gradient/normal (from the previous pin-filled phi): what Lagrange_points,
// momentum and refilling read.
// rr_old (16-bit storage): the reference pairs of the populations.
template <typename S>
__device__ __forceinline__ void prep_node(const DevParams& P, const Pad& pd, const sym_particles* __restrict__ Sp,
                                          const S* __restrict__ pops, const typename Codec<S>::R* __restrict__ phi_cur,
                                          const typename Codec<S>::R* __restrict__ phi_prev,
                                          const int32_t* __restrict__ walls_all, const int32_t* __restrict__ pout,
                                          double* rhoN, double* rhoR, double* rhoB, double* fi, double* gx,
                                          double* gy, double* gz, double* nxv, double* nyv, double* nzv,
                                          const Ref* __restrict__ rr_old, int x, int y, int z) {
  using R = typename Codec<S>::R;
  const long long L = lin(P, x, y, z);
  const unsigned N = (unsigned)P.N;
  const Ref rref = Codec<S>::kRef ? rr_old[pd.idx(x, y, z)] : Ref{};
  if (walls_all[L] > 0) {
    rhoN[L] = 0.0;
    gx[L] = 0.0; gy[L] = 0.0; gz[L] = 0.0; nxv[L] = 0.0; nyv[L] = 0.0; nzv[L] = 0.0;
    return;
  }
  // fi is read only by the momentum exchange, at nodes with links into a
  // particle (pout > 0): written there only
  const bool links = pout[L] > 0;
  R sr = R(0), sb = R(0);
  unroll19([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    R r, b;
    Codec<S>::template load<i>(pops, N, (unsigned)L, rref, r, b);
    if (links) fi[(size_t)i * N + L] = (double)(r + b);
    sr = sr + r;
    sb = sb + b;
  });
  rhoR[L] = (double)sr; rhoB[L] = (double)sb;
  rhoN[L] = (double)phi_cur[pd.idx(x, y, z)];
  R g0 = R(0), g1 = R(0), g2 = R(0);
#pragma unroll
  for (int i = 1; i < 19; i++) {
    const R val = R(W(i)) * phi_prev[pd.idx(x + CX(i), y + CY(i), z + CZ(i))];
    if (CX(i)) g0 = g0 + val * R(CX(i));
    if (CY(i)) g1 = g1 + val * R(CY(i));
    if (CZ(i)) g2 = g2 + val * R(CZ(i));
  }
  g0 = R(3) * g0; g1 = R(3) * g1; g2 = R(3) * g2;
  const R fn = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
  R n0 = R(0), n1 = R(0), n2 = R(0);
  if (fn > R(P.evap)) {
    n0 = g0 / fn; n1 = g1 / fn; n2 = g2 / fn;
    const int q = pout[L];
    if (q >= 1) {
      wet_rotate<R>(P, Sp, q, x, y, z, n0, n1, n2);
      g0 = fn * n0; g1 = fn * n1; g2 = fn * n2;
    }
  }
  gx[L] = g0; gy[L] = g1; gz[L] = g2; nxv[L] = n0; nyv[L] = n1; nzv[L] = n2;
}

// after refilling: a refilled node's canonical populations and phi into the
// fused state, encoded with a reference pair of its own (its colour
// densities), which it records in rr_old: the references this step's collide
// decodes with
template <typename S>
__device__ __forceinline__ void refill_import_node(const DevParams& P, const Pad& pd, int pp, S* pops,
                                                   typename Codec<S>::R* phi_cur, const int32_t* __restrict__ pout,
                                                   const int32_t* __restrict__ walls_old,
                                                   const double* __restrict__ ri, const double* __restrict__ bi,
                                                   const double* __restrict__ rhoN, Ref* __restrict__ rr_old,
                                                   int x, int y, int z) {
  using R = typename Codec<S>::R;
  const long long L = lin(P, x, y, z);
  const unsigned N = (unsigned)P.N;
  if (pout[L] != pp || walls_old[L] < 1) return;
  Ref ref{};
  if constexpr (Codec<S>::kRef) {
    double sr = 0.0, sb = 0.0;
    for (int i = 0; i < 19; i++) { sr += ri[(size_t)i * N + L]; sb += bi[(size_t)i * N + L]; }
    ref = sr + sb > 0.0 ? ref_pair(float(sr), float(sb)) : ref_rest(P);
    phi_store<Ref>(P, pd, rr_old, x, y, z, ref);
  }
  unroll19([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const R r = R(ri[(size_t)i * N + L]), b = R(bi[(size_t)i * N + L]);
    Codec<S>::template store<i>(pops, N, (unsigned)L, ref, r, r + b);
  });
  phi_store<R>(P, pd, phi_cur, x, y, z, R(rhoN[L]));
}

// whole-domain conversions between the canonical arrays and the fused state
// rr (16-bit storage, else null): receives each node's reference pair, its
// colour densities (the rest pair where both are 0: solid or empty nodes)
template <typename S>
__global__ void k_import_pops(DevParams P, Pad pd, const double* __restrict__ ri, const double* __restrict__ bi,
                              S* pops, Ref* rr, typename Acc<typename Codec<S>::R>::T* acc, int* status) {
  using R = typename Codec<S>::R;
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  if (L >= P.N) return;
  const unsigned N = (unsigned)P.N;
  Ref ref{};
  R sr = R(0), sb = R(0);
  if constexpr (Codec<S>::kRef) {
    double dr = 0.0, db = 0.0;
    for (int i = 0; i < 19; i++) { dr += ri[(size_t)i * N + L]; db += bi[(size_t)i * N + L]; }
    ref = dr + db > 0.0 ? ref_pair(float(dr), float(db)) : ref_rest(P);
    const unsigned Lu = (unsigned)L, q = Lu / (unsigned)P.nz;
    const int z = (int)(Lu - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
    phi_store<Ref>(P, pd, rr, x, y, z, ref);
  }
  unroll19([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const R r = R(ri[(size_t)i * N + L]), b = R(bi[(size_t)i * N + L]);
    Codec<S>::template store<i>(pops, N, (unsigned)L, ref, r, r + b);
    sr = sr + r;
    sb = sb + b;
  });
  // the accumulators the first phase field after the import reads (storages
  // that accumulate)
  using A = Acc<R>;
  if (acc) {
    if (!A::ok(sr) || !A::ok(sb)) atomicOr(status, 1);
    acc[L] = A::ok(sr) ? A::fix(sr) : 0;
    acc[L + P.N] = A::ok(sb) ? A::fix(sb) : 0;
  }
}
template <typename S>
__global__ void k_export_pops(DevParams P, Pad pd, const S* __restrict__ pops, const Ref* __restrict__ rr, double* ri,
                              double* bi) {
  using R = typename Codec<S>::R;
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  if (L >= P.N) return;
  const unsigned N = (unsigned)P.N;
  Ref rref{};
  if constexpr (Codec<S>::kRef) {
    const unsigned Lu = (unsigned)L, q = Lu / (unsigned)P.nz;
    const int z = (int)(Lu - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
    rref = rr[pd.idx(x, y, z)];
  }
  unroll19([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    R r, b;
    Codec<S>::template load<i>(pops, N, (unsigned)L, rref, r, b);
    ri[(size_t)i * N + L] = (double)r;
    bi[(size_t)i * N + L] = (double)b;
  });
}
// calmacros (Source1.f90:770-831) of the current fused populations without
// touching the fused state: rho, u = sum f c / rho (no force shift) and
// phi = (rhoR - rhoB) / rho on fluid nodes; phi = 0, u = 0, rho = rho0 on
// solid nodes.  rr (16-bit storage): the reference pairs of the populations.
template <typename S>
__global__ void k_macros(DevParams P, Pad pd, const S* __restrict__ pops, const Ref* __restrict__ rr,
                         const int32_t* __restrict__ walls_all, double* rho, double* ux, double* uy, double* uz,
                         double* rhoN) {
  using R = typename Codec<S>::R;
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  if (L >= P.N) return;
  if (walls_all[L] >= 1) {
    rhoN[L] = 0.0; ux[L] = 0.0; uy[L] = 0.0; uz[L] = 0.0; rho[L] = P.rho0;
    return;
  }
  const unsigned N = (unsigned)P.N;
  Ref rref{};
  if constexpr (Codec<S>::kRef) {
    const unsigned Lu = (unsigned)L, q = Lu / (unsigned)P.nz;
    const int z = (int)(Lu - q * (unsigned)P.nz), x = (int)(q / (unsigned)P.ny), y = (int)(q - (unsigned)x * P.ny);
    rref = rr[pd.idx(x, y, z)];
  }
  double sr = 0.0, sb = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
  unroll19([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    R r, b;
    Codec<S>::template load<i>(pops, N, (unsigned)L, rref, r, b);
    const double f = (double)r + (double)b;
    sr += (double)r;
    sb += (double)b;
    if (CX(i)) mx += f * CX(i);
    if (CY(i)) my += f * CY(i);
    if (CZ(i)) mz += f * CZ(i);
  });
  const double rh = sr + sb;
  rho[L] = rh;
  ux[L] = mx / rh; uy[L] = my / rh; uz[L] = mz / rh;
  rhoN[L] = (sr - sb) / rh;
}

template <typename R>
__global__ void k_import_phi(DevParams P, Pad pd, const double* __restrict__ rhoN, R* phi) {
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz), y = (int)((L / P.nz) % P.ny), x = (int)(L / ((long long)P.nz * P.ny));
  phi_store<R>(P, pd, phi, x, y, z, R(rhoN[L]));
}
template <typename R>
__global__ void k_export_phi(DevParams P, Pad pd, const R* __restrict__ phi, double* rhoN) {
  const long long L = blockIdx.x * 256LL + threadIdx.x;
  if (L >= P.N) return;
  const int z = (int)(L % P.nz), y = (int)((L / P.nz) % P.ny), x = (int)(L / ((long long)P.nz * P.ny));
  rhoN[L] = (double)phi[pd.idx(x, y, z)];
}


}  // namespace fused
}  // namespace symb200
