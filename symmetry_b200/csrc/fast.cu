// fast.cu -- fused fast path of the per-timestep lattice update (CONFIG mode).
//
// Per step (same order as the reference loop body, Source1.f90:216-251):
//   k_finalize   calmacros (a1): phi = (rhoR - rhoB) / rho from the two
//                colour densities per node that the previous step's collide
//                kernel accumulated, written into a halo-padded array (every
//                node also writes its periodic images in the 2-deep ghost
//                layers, so stencil tiles never wrap).
//   particles    sparse: Lagrange points, capillary force, momentum exchange,
//                repulsion, Newton-Euler, set_walls, refill -- on the
//                particle's bounding box only.
//   pin fill     sparse: fictitious phi on solid nodes next to fluid (:467-492).
//   k_collide    derivatives (:497-594) + collision (:599-695) + Recolor
//                (:697-732) + streaming (:735-768) + curve (:990-1034) fused:
//                a CTA owns a 32(z) x BY(y) footprint (BY per storage,
//                kBY) and marches along x with a 5-plane phi window and a
//                4-plane window of unit normals in
//                shared memory; it reads each node's populations once, and
//                pushes the recoloured post-collision populations to their
//                neighbours (push streaming), reflecting links that enter a
//                solid node back into the node itself (halfway bounce-back
//                with the wall velocity term of curve).  It also adds each
//                pushed value into its destination's colour-density
//                accumulators (combined inside the CTA, fixed-point atomics
//                across tiles), which the next step's k_finalize reads.
// Populations are stored post-stream as [colour-slot][velocity][node].
#include <cuda_fp16.h>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <utility>
#include <vector>
#include "state.cuh"
#include "fused.cuh"
#include "particles.cuh"

namespace symb200 {

namespace {

using namespace fused;

inline unsigned blocks_for(long long n, int tpb = 256) { return (unsigned)((n + tpb - 1) / tpb); }

// typed view of the fused buffers
template <typename S>
S* popbuf(sym_handle* h, int k) { return reinterpret_cast<S*>(h->fast.pop[k]); }
template <typename S>
typename Codec<S>::R* phibuf(sym_handle* h, int k);
template <>
double* phibuf<double>(sym_handle* h, int k) { return h->fast.phi[k]; }
template <>
float* phibuf<float>(sym_handle* h, int k) { return h->fast.phif[k]; }
template <>
float* phibuf<__half>(sym_handle* h, int k) { return h->fast.phif[k]; }

// reference densities of the 16-bit storage: decoded with rr[1 - pc], written
// by this step's phase kernel into rr[pc] (null for the other storages)
const float2* rr_old(const sym_handle* h, int pc) { return h->fast.rref[1 - pc]; }
float2* rr_new(sym_handle* h, int pc) { return h->fast.rref[pc]; }

bool has_solids(const sym_handle* h) { return h->dp.par > 0 || h->dp.wall_x; }

template <typename S>
typename Acc<typename Codec<S>::R>::T* accbuf(sym_handle* h) {
  return reinterpret_cast<typename Acc<typename Codec<S>::R>::T*>(h->fast.acc);
}

// the particle and wall work of this handle's fused steps (sparse.cu); built
// outside any stream capture
int ensure_sparse(sym_handle* h) {
  if (h->fast.sparse || !has_solids(h)) return SYM_OK;
  int err = SYM_OK;
  h->fast.sparse = sparse_plan_build({h}, {0}, {0}, h->st, &err);
  return h->fast.sparse ? SYM_OK : set_error(h, err, "sparse plan");
}

// ev (optional): 4 events recorded before k_finalize, after it, before
// k_collide and after k_collide, for per-kernel timing on the library stream
template <typename S>
int enqueue_step(sym_handle* h, int cur, int pc, cudaEvent_t* ev) {
  using R = typename Codec<S>::R;
  const DevParams& P = h->dp;
  const Pad pd = make_pad(P);
  const bool solid = has_solids(h);
  S* pin_ = popbuf<S>(h, cur);
  S* pnext = popbuf<S>(h, 1 - cur);
  R* phic = phibuf<S>(h, pc);
  R* phip = phibuf<S>(h, 1 - pc);
  // (a1) calmacros: from the colour densities the previous collide
  // accumulated, or from the populations
  if (ev) cudaEventRecord(ev[0], h->st);
  if constexpr (kAccumulate<S>) {
    const unsigned fin_blocks = blocks_for(P.N, 256 * kFinalizeNPT);
    if (solid)
      k_finalize<S, true><<<fin_blocks, 256, 0, h->st>>>(P, pd, accbuf<S>(h), phic, h->walls_all, rr_new(h, pc),
                                                         h->fast.status);
    else
      k_finalize<S, false><<<fin_blocks, 256, 0, h->st>>>(P, pd, accbuf<S>(h), phic, h->walls_all, rr_new(h, pc),
                                                          h->fast.status);
  } else {
    if (solid)
      k_phase<S, true><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, pin_, phic, h->walls_all, rr_old(h, pc),
                                                           rr_new(h, pc));
    else
      k_phase<S, false><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, pin_, phic, h->walls_all, rr_old(h, pc),
                                                            rr_new(h, pc));
  }
  if (ev) cudaEventRecord(ev[1], h->st);
  // particle coupling and pin fill (cur and pc advance together from 0)
  if (int e = sparse_enqueue(h->fast.sparse, cur, h->st)) return set_error(h, e, "sparse step");
  // (a3-a9) fused derivatives + collision + recolour + stream + bounce-back
  const int xc = h->fast.xchunk > 0 ? h->fast.xchunk : XCHUNK;
  dim3 grid((P.nz + BZ - 1) / BZ, (P.ny + kBY<S> - 1) / kBY<S>, (P.nx + xc - 1) / xc);
  const size_t shm = smem_bytes<S>();
  const CUtensorMap& tp = h->fast.tm_phi[pc];
  const CUtensorMap& tr = h->fast.tm_ref[pc];
  if (ev) cudaEventRecord(ev[2], h->st);
  if (solid)
    k_collide<S, true><<<grid, kTPB<S>, shm, h->st>>>(P, pd, pin_, pnext, phic, h->walls, h->walls_all, h->pout,
                                                  h->dpart, h->ffi, rr_old(h, pc), rr_new(h, pc), accbuf<S>(h),
                                                  h->fast.status, tp, tr, xc);
  else
    k_collide<S, false><<<grid, kTPB<S>, shm, h->st>>>(P, pd, pin_, pnext, phic, h->walls, h->walls_all, h->pout,
                                                   h->dpart, h->ffi, rr_old(h, pc), rr_new(h, pc), accbuf<S>(h),
                                                   h->fast.status, tp, tr, xc);
  if (int e = sparse_enqueue_post(h->fast.sparse, cur, h->st)) return set_error(h, e, "interpolated bounce-back");
  if (ev) cudaEventRecord(ev[3], h->st);
  return check_cuda(h, cudaGetLastError(), "fast step");
}

template <typename S>
int set_smem_attr(sym_handle* h) {
  const int shm = (int)smem_bytes<S>();
  cudaError_t e = cudaFuncSetAttribute(k_collide<S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_collide<S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  return check_cuda(h, e, "smem attribute");
}

// Stop-rule reduction on the fused phase field: per z plane, the sum over
// fluid nodes of (1+phi)/2 (the red area of the plane), one block per plane,
// in a fixed order (deterministic).  phi on solid nodes holds the pin fill
// and is skipped.
template <typename R>
__global__ void __launch_bounds__(256) k_neck_planes(DevParams P, Pad pd, const R* __restrict__ phi,
                                                     const int32_t* __restrict__ walls_all, double* out) {
  __shared__ double sh[256];
  const int z = blockIdx.x;
  double s = 0.0;
  const int nxy = P.nx * P.ny;
  for (int t = threadIdx.x; t < nxy; t += 256) {
    const int x = t / P.ny, y = t - x * P.ny;
    const long long L = (long long)z + (long long)P.nz * ((long long)y + (long long)P.ny * x);
    if (walls_all[L] <= 0) s += 0.5 * (1.0 + (double)phi[pd.idx(x, y, z)]);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[z] = sh[0];
}

int enqueue(sym_handle* h, int cur, int pc, cudaEvent_t* ev = nullptr) {
  switch (h->fast.storage) {
    case SYM_STORE_FP64: return enqueue_step<double>(h, cur, pc, ev);
    case SYM_STORE_FP32: return enqueue_step<float>(h, cur, pc, ev);
    default: return enqueue_step<__half>(h, cur, pc, ev);
  }
}

}  // namespace

// ===========================================================================
int fast_alloc(sym_handle* h) {
  FastState& F = h->fast;
  if (38.0 * (double)h->N >= 4294967296.0)
    return set_error(h, SYM_ERR_UNSUPPORTED, "fused path: 38*N must stay below 2^32 (N < 113M nodes)");
  F.storage = h->p.storage;
  const size_t s = F.storage == SYM_STORE_FP64 ? 8 : (F.storage == SYM_STORE_FP32 ? 4 : 2);
  const size_t popb = 38 * h->N * s;
  const size_t before = h->bytes;
  for (int k = 0; k < 2; k++)
    if (int e = dev_carve(h, &F.pop[k], popb)) return e;
  const Pad pd = make_pad(h->dp);
  for (int k = 0; k < 2; k++) {
    if (F.storage == SYM_STORE_FP64) {
      if (int e = dev_carve(h, (void**)&F.phi[k], sizeof(double) * pd.size())) return e;
    } else {
      if (int e = dev_carve(h, (void**)&F.phif[k], sizeof(float) * pd.size())) return e;
    }
    if (F.storage == SYM_STORE_FP16)
      if (int e = dev_carve(h, (void**)&F.rref[k], sizeof(float2) * pd.size())) return e;
  }
  if (F.storage == SYM_STORE_FP64)   // the storage whose collide kernel accumulates (kAccumulate)
    if (int e = dev_carve(h, &F.acc, 2 * h->N * 8)) return e;
  if (h->dp.par > 0) {
    // momentum link lists: one 256-entry segment per block of each particle's
    // momentum box (the box of set_walls' pin/pout marking)
    F.link_blocks = (part::sphere_box(h->dp, part::kLinkMargin).count() + 255) / 256;
    const size_t segs = (size_t)h->dp.par * F.link_blocks;
    if (int e = dev_carve(h, (void**)&F.links, segs * 256 * sizeof(uint2))) return e;
    if (int e = dev_carve(h, (void**)&F.nlinks, segs * sizeof(int))) return e;
  }
  if (int e = dev_carve(h, (void**)&F.status, sizeof(int))) return e;
  if (h->planning) return SYM_OK;
  F.bytes = h->bytes - before;
  // TMA descriptors of the phase-field (and 16-bit reference-pair) tiles the
  // collide kernel reads: boxes of (BZ+4) x (BY+4) x 1 over the padded arrays
  const int BY = tile_rows(F.storage);
  for (int k = 0; k < 2; k++) {
    const bool f64 = F.storage == SYM_STORE_FP64;
    void* phi = f64 ? (void*)F.phi[k] : (void*)F.phif[k];
    if (tma::encode_padded(&F.tm_phi[k], phi, f64 ? 8 : 4, h->dp.nz + 4, pd.nzp, pd.nyp, pd.nxp, BZ + 4, BY + 4))
      return set_error(h, SYM_ERR_CUDA, "TMA descriptor of the phase field");
    if (F.storage == SYM_STORE_FP16) {
      if (tma::encode_padded(&F.tm_ref[k], F.rref[k], 8, h->dp.nz + 4, pd.nzp, pd.nyp, pd.nxp, BZ + 4, BY + 4))
        return set_error(h, SYM_ERR_CUDA, "TMA descriptor of the reference densities");
    } else {
      F.tm_ref[k] = F.tm_phi[k];   // not read
    }
  }
  return F.storage == SYM_STORE_FP64 ? set_smem_attr<double>(h)
       : F.storage == SYM_STORE_FP32 ? set_smem_attr<float>(h) : set_smem_attr<__half>(h);
}

void fast_free(sym_handle* h) {
  FastState& F = h->fast;
  sparse_plan_free(F.sparse);
  F.sparse = nullptr;
  for (int k = 0; k < 2; k++) {
    dev_release(h, F.pop[k]);
    dev_release(h, F.phi[k]);
    dev_release(h, F.phif[k]);
    dev_release(h, F.rref[k]);
    if (k == 0) {
      dev_release(h, F.acc);
      dev_release(h, (void*)F.status);
      dev_release(h, (void*)F.links);
      dev_release(h, (void*)F.nlinks);
      F.acc = nullptr;
      F.status = nullptr;
      F.links = nullptr;
      F.nlinks = nullptr;
    }
    if (F.gexec[k]) cudaGraphExecDestroy(F.gexec[k]);
    if (F.graph[k]) cudaGraphDestroy(F.graph[k]);
    F.pop[k] = nullptr; F.phi[k] = nullptr; F.phif[k] = nullptr; F.rref[k] = nullptr;
    F.gexec[k] = nullptr; F.graph[k] = nullptr;
  }
}

// canonical -> fused: populations, and the pin-filled phi of the last
// derivatives call as the previous phase field
int fast_import(sym_handle* h) {
  FastState& F = h->fast;
  const DevParams& P = h->dp;
  const Pad pd = make_pad(P);
  F.cur = 0;
  F.pc = 0;
  cudaMemsetAsync(F.status, 0, sizeof(int), h->st);
  switch (F.storage) {
    case SYM_STORE_FP64:
      k_import_pops<double><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->ri, h->bi, popbuf<double>(h, 0), nullptr,
                                                                accbuf<double>(h), F.status);
      k_import_phi<double><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->rhoN, F.phi[1]);
      break;
    case SYM_STORE_FP32:
      k_import_pops<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->ri, h->bi, popbuf<float>(h, 0), nullptr,
                                                               accbuf<float>(h), F.status);
      k_import_phi<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->rhoN, F.phif[1]);
      break;
    default:
      // after import pc = 0: the next phase decodes with rref[1]
      k_import_pops<__half><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->ri, h->bi, popbuf<__half>(h, 0), F.rref[1],
                                                                accbuf<__half>(h), F.status);
      k_import_phi<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, h->rhoN, F.phif[1]);
  }
  if (int e = sparse_links_build(h, h->st)) return set_error(h, e, "momentum link lists");
  return check_cuda(h, cudaStreamSynchronize(h->st), "fast import");
}

// fused -> canonical: populations, the last pin-filled phi as rho_N, and the
// derivatives of that phi (what the next Lagrange_points call reads)
int fast_export(sym_handle* h) {
  FastState& F = h->fast;
  const DevParams& P = h->dp;
  const Pad pd = make_pad(P);
  switch (F.storage) {
    case SYM_STORE_FP64:
      k_export_pops<double><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<double>(h, F.cur), nullptr, h->ri, h->bi);
      k_export_phi<double><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, F.phi[1 - F.pc], h->rhoN);
      break;
    case SYM_STORE_FP32:
      k_export_pops<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<float>(h, F.cur), nullptr, h->ri, h->bi);
      k_export_phi<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, F.phif[1 - F.pc], h->rhoN);
      break;
    default:
      k_export_pops<__half><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<__half>(h, F.cur), F.rref[1 - F.pc],
                                                                 h->ri, h->bi);
      k_export_phi<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, F.phif[1 - F.pc], h->rhoN);
  }
  if (int e = check_cuda(h, cudaGetLastError(), "fast export")) return e;
  if (int e = ref_derivatives(h)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "fast export");
}

// calmacros of the current fused populations into the canonical macro arrays
// (rho, u, rho_N), leaving the fused state authoritative
int fast_macros(sym_handle* h) {
  FastState& F = h->fast;
  const DevParams& P = h->dp;
  const Pad pd = make_pad(P);
  switch (F.storage) {
    case SYM_STORE_FP64:
      k_macros<double><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<double>(h, F.cur), nullptr, h->walls_all,
                                                           h->rho, h->ux, h->uy, h->uz, h->rhoN);
      break;
    case SYM_STORE_FP32:
      k_macros<float><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<float>(h, F.cur), nullptr, h->walls_all,
                                                          h->rho, h->ux, h->uy, h->uz, h->rhoN);
      break;
    default:
      k_macros<__half><<<blocks_for(P.N), 256, 0, h->st>>>(P, pd, popbuf<__half>(h, F.cur), F.rref[1 - F.pc],
                                                           h->walls_all, h->rho, h->ux, h->uy, h->uz, h->rhoN);
  }
  return check_cuda(h, cudaGetLastError(), "fast macros");
}

// nsteps fused steps; each parity (which population/phi buffer is current) has
// its own captured graph
int fast_step(sym_handle* h, int nsteps) {
  FastState& F = h->fast;
  if (int e = ensure_sparse(h)) return e;
  for (int t = 0; t < nsteps; t++) {
    const int k = F.cur;   // cur and pc advance together
    if (!F.gexec[k]) {
      if (int e = check_cuda(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal), "capture"))
        return e;
      const int e1 = enqueue(h, F.cur, F.pc);
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
      if (e1) { if (g) cudaGraphDestroy(g); return e1; }
      if (int e = check_cuda(h, e2, "end capture")) return e;
      F.graph[k] = g;
      if (int e = check_cuda(h, cudaGraphInstantiate(&F.gexec[k], g, 0), "instantiate")) return e;
    }
    if (int e = check_cuda(h, cudaGraphLaunch(F.gexec[k], h->st), "graph launch")) return e;
    F.cur = 1 - F.cur;
    F.pc = 1 - F.pc;
  }
  return check_cuda(h, cudaStreamSynchronize(h->st), "fast step");
}

// nsteps eager (not graph) steps with CUDA events around the kernel classes.
// ms[0] = whole region, ms[1] = sum of k_finalize, ms[2] = sum of the sparse
// particle/pin-fill work, ms[3] = sum of k_collide.

int fast_step_timed(sym_handle* h, int nsteps, double ms[4]) {
  FastState& F = h->fast;
  if (int e = ensure_sparse(h)) return e;
  std::vector<cudaEvent_t> ev(4 * (size_t)nsteps + 2);
  for (auto& e : ev)
    if (int r = check_cuda(h, cudaEventCreate(&e), "event")) return r;
  int rc = SYM_OK;
  cudaEventRecord(ev[4 * nsteps], h->st);
  for (int t = 0; t < nsteps && !rc; t++) {
    rc = enqueue(h, F.cur, F.pc, &ev[4 * t]);
    F.cur = 1 - F.cur;
    F.pc = 1 - F.pc;
  }
  cudaEventRecord(ev[4 * nsteps + 1], h->st);
  if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->st), "timed steps");
  if (!rc) {
    float v;
    for (int k = 0; k < 4; k++) ms[k] = 0.0;
    cudaEventElapsedTime(&v, ev[4 * nsteps], ev[4 * nsteps + 1]);
    ms[0] = v;
    for (int t = 0; t < nsteps; t++) {
      cudaEventElapsedTime(&v, ev[4 * t], ev[4 * t + 1]); ms[1] += v;
      cudaEventElapsedTime(&v, ev[4 * t + 1], ev[4 * t + 2]); ms[2] += v;
      cudaEventElapsedTime(&v, ev[4 * t + 2], ev[4 * t + 3]); ms[3] += v;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}

namespace tma {
int encode_padded(CUtensorMap* map, void* base, int esize, int nz_ext, int nzp, int nyp, int nxp, int box_z,
                  int box_y) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  });
  if (!encode) return SYM_ERR_CUDA;
  // the rules a tiled TMA load relies on: 16-byte base and pitches, an inner
  // box extent that is a whole number of 16-byte units, at most 256 per box side
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((size_t)nzp * esize) % 16 || ((size_t)box_z * esize) % 16 ||
      box_z > 256 || box_y > 256 || nz_ext > nzp)
    return SYM_ERR_PARAM;
  const cuuint64_t dims[3] = {(cuuint64_t)nz_ext, (cuuint64_t)nyp, (cuuint64_t)nxp};
  const cuuint64_t strides[2] = {(cuuint64_t)nzp * esize, (cuuint64_t)nzp * nyp * esize};
  const cuuint32_t box[3] = {(cuuint32_t)box_z, (cuuint32_t)box_y, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(map, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                            base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SYM_OK : SYM_ERR_CUDA;
}
}  // namespace tma

}  // namespace symb200

namespace symb200 {

// Per-plane red area of the phase field written by the last fused step
// (phi of the populations that step started from), enqueued on `st` into
// device memory `out` (nz doubles).  r_eq(z) = sqrt(out[z] / pi).
int fast_neck_planes(sym_handle* h, double* out, cudaStream_t st) {
  FastState& F = h->fast;
  if (!F.valid) return set_error(h, SYM_ERR_STATE, "neck planes: the fused state is not current");
  const DevParams& P = h->dp;
  const Pad pd = make_pad(P);
  if (F.storage == SYM_STORE_FP64)
    k_neck_planes<double><<<P.nz, 256, 0, st>>>(P, pd, F.phi[1 - F.pc], h->walls_all, out);
  else
    k_neck_planes<float><<<P.nz, 256, 0, st>>>(P, pd, F.phif[1 - F.pc], h->walls_all, out);
  return check_cuda(h, cudaGetLastError(), "neck planes");
}

}  // namespace symb200
