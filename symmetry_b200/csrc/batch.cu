// batch.cu -- many independent CONFIG domains stepped together.
//
// One step of a batch is one CUDA graph:
//   phase field       calmacros of every domain in one launch (blocks map to
//                     domains through a prefix sum of per-domain block
//                     counts): from the colour densities the previous collide
//                     accumulated (FP64) or from the populations (16-bit, FP32);
//   sparse work       particle coupling and pin fill of every domain with
//                     solids, one launch per subroutine for all of them
//                     (sparse.cu);
//   k_collide_batch   one persistent launch (one CTA per SM slot) whose CTAs
//                     take 32x8xX tiles of any domain from a work-tile table
//                     through an atomic counter, largest tiles first, so
//                     domains of uneven size share the GPU without tails.
// Each domain keeps its own buffers and parity; two graphs (one per parity
// of the domain buffers) alternate.  The x extent X of the tiles is chosen per
// size class by sym_batch_autotune.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "state.cuh"
#include "fused.cuh"

using namespace symb200;
using namespace symb200::fused;

namespace {

struct DomainDesc {
  DevParams P;
  Pad pd;
  const void* pin;      // populations read this step
  void* pnext;          // populations written this step
  void* phic;           // phase field of this step
  const int32_t* walls;
  const int32_t* walls_all;
  const int32_t* pout;
  const sym_particles* Sp;
  double* ffi;
  const Ref* rr_old;  // 16-bit storage: reference pairs (see fused.cuh)
  Ref* rr_new;
  void* acc;            // accumulated colour densities of the next step (see fused.cuh)
  int* status;
  const CUtensorMap* tm_phi;    // TMA descriptors (device copies) of this step's phase field
  const CUtensorMap* tm_ref;   // and reference-pair arrays
  int solid;
  int pad_;
};

struct TileEntry {
  int dom, z0, y0, xa, xb, cost, r0, r1;
};


// blk[b] = (domain, block index within the domain) of phase block b
template <typename S>
__global__ void __launch_bounds__(256) k_phase_batch(const DomainDesc* __restrict__ descs,
                                                     const int2* __restrict__ blk) {
  using R = typename Codec<S>::R;
  const int2 e = blk[blockIdx.x];
  const DomainDesc& D = descs[e.x];
  const long long L = (long long)e.y * 256 + threadIdx.x;
  if (D.solid)
    phase_node<S, true>(D.P, D.pd, (const S*)D.pin, (R*)D.phic, D.walls_all, D.rr_old, D.rr_new, L);
  else
    phase_node<S, false>(D.P, D.pd, (const S*)D.pin, (R*)D.phic, D.walls_all, D.rr_old, D.rr_new, L);
}

template <typename S>
__global__ void __launch_bounds__(256) k_finalize_batch(const DomainDesc* __restrict__ descs,
                                                        const int2* __restrict__ blk) {
  using R = typename Codec<S>::R;
  using AT = typename Acc<R>::T;
  const int2 e = blk[blockIdx.x];
  const DomainDesc& D = descs[e.x];
  const long long L = (long long)e.y * 256 + threadIdx.x;
  if (D.solid)
    finalize_nodes<S, true, 1>(D.P, D.pd, (AT*)D.acc, (R*)D.phic, D.walls_all, D.rr_new, D.status, L);
  else
    finalize_nodes<S, false, 1>(D.P, D.pd, (AT*)D.acc, (R*)D.phic, D.walls_all, D.rr_new, D.status, L);
}

template <typename S>
__global__ void __launch_bounds__(kTPB<S>, collide_ctas<S>()) k_collide_batch(const DomainDesc* __restrict__ descs,
                                                           const TileEntry* __restrict__ tiles, int ntiles,
                                                           int* __restrict__ counter) {
  using R = typename Codec<S>::R;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem<S>& sm = smem_view<S>(smem_raw);
  __shared__ int s_tile;
  __shared__ __align__(16) DomainDesc s_desc;
  collide_init_barriers<S>(sm);
  unsigned nload = 0;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= ntiles) break;
    const TileEntry e = tiles[t];
    {  // stage the tile's domain descriptor in shared memory
      const int* src = reinterpret_cast<const int*>(&descs[e.dom]);
      int* dst = reinterpret_cast<int*>(&s_desc);
      for (int k = threadIdx.x; k < (int)(sizeof(DomainDesc) / sizeof(int)); k += kTPB<S>) dst[k] = src[k];
    }
    __syncthreads();
    const DomainDesc& D = s_desc;
    using AT = typename Acc<R>::T;
    // one compiled variant for every tile (solid handling switched per
    // domain): the instruction working set of the persistent kernel stays
    // that of one variant
    collide_tile<S, true>(D.P, D.pd, (const S*)D.pin, (S*)D.pnext, (const R*)D.phic, D.walls, D.walls_all, D.pout,
                          D.Sp, D.ffi, D.rr_old, D.rr_new, (AT*)D.acc, D.status, D.tm_phi, D.tm_ref, e.z0, e.y0,
                          e.xa, e.xb, sm, nload, D.solid != 0);
    __syncthreads();
  }
}

// the collide kernel's dynamic shared memory, and how many of its CTAs fit
// on one SM (*per_sm) of the device's *sms
template <typename S>
int set_batch_smem(int device, int* per_sm, int* sms) {
  const int shm = (int)smem_bytes<S>();
  if (cudaFuncSetAttribute(k_collide_batch<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm) != cudaSuccess)
    return SYM_ERR_CUDA;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_collide_batch<S>, kTPB<S>, shm);
  cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device);
  *per_sm = std::max(1, *per_sm);
  *sms = std::max(1, *sms);
  return SYM_OK;
}

}  // namespace

struct sym_batch {
  int device = 0;
  cudaStream_t st = nullptr;
  int storage = -1;
  std::vector<sym_handle*> doms;
  std::vector<int> xchunk;
  std::vector<int> built_cur, built_pc;   // domain parities graph 0 was built for
  int steps_since_build = 0;
  DomainDesc* d_desc[2] = {nullptr, nullptr};
  CUtensorMap* d_tmaps = nullptr;   // [parity][domain][phase field, reference pairs]
  int2* d_blk = nullptr;          // phase block -> (domain, block in domain)
  TileEntry* d_tiles = nullptr;
  int ntiles = 0;
  long long nblocks = 0;
  int* d_counter = nullptr;
  int grid = 0;                   // persistent collide CTAs: per_sm x sms
  int sms = 0, max_per_sm = 0, per_sm = 0;
  SparsePlan* sparse = nullptr;   // particle and wall work of every domain, batched
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool built = false;
  std::string err;
};

namespace {

int berr(sym_batch* b, int code, const char* msg) {
  if (b) b->err = msg;
  return code;
}
int bcuda(sym_batch* b, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SYM_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();   // not sticky: keep it out of later checks
  return berr(b, e == cudaErrorMemoryAllocation ? SYM_ERR_OOM : SYM_ERR_CUDA, m.c_str());
}

void free_graphs(sym_batch* b) {
  for (int k = 0; k < 2; k++) {
    if (b->gexec[k]) cudaGraphExecDestroy(b->gexec[k]);
    if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
    b->gexec[k] = nullptr;
    b->graph[k] = nullptr;
  }
  b->built = false;
}

void free_tables(sym_batch* b) {
  sparse_plan_free(b->sparse);
  b->sparse = nullptr;
  for (int k = 0; k < 2; k++)
    if (b->d_desc[k]) { cudaFree(b->d_desc[k]); b->d_desc[k] = nullptr; }
  if (b->d_blk) { cudaFree(b->d_blk); b->d_blk = nullptr; }
  if (b->d_tiles) { cudaFree(b->d_tiles); b->d_tiles = nullptr; }
  if (b->d_tmaps) { cudaFree(b->d_tmaps); b->d_tmaps = nullptr; }
}

void* popp(sym_handle* h, int k) { return h->fast.pop[k]; }
void* phip(sym_handle* h, int k) {
  return h->fast.storage == SYM_STORE_FP64 ? (void*)h->fast.phi[k] : (void*)h->fast.phif[k];
}

DomainDesc make_desc(sym_handle* h, int cur, int pc) {
  DomainDesc d;
  std::memset(&d, 0, sizeof d);
  d.P = h->dp;
  d.pd = make_pad(h->dp);
  d.pin = popp(h, cur);
  d.pnext = popp(h, 1 - cur);
  d.phic = phip(h, pc);
  d.walls = h->walls;
  d.walls_all = h->walls_all;
  d.pout = h->pout;
  d.Sp = h->dpart;
  d.ffi = h->ffi;
  d.rr_old = h->fast.rref[1 - pc];
  d.rr_new = h->fast.rref[pc];
  d.acc = h->fast.acc;
  d.status = h->fast.status;
  d.solid = (h->dp.par > 0 || h->dp.wall_x) ? 1 : 0;
  return d;
}

// One batch step on b->st (captured into a graph, or eager when timing):
// descriptor table k, domain i at buffer parity (built_cur[i] + k) & 1.
// ev (optional, eager only): 4 events recorded before the phase launch, after
// it, after the sparse work, and after the collide launch.
template <typename S>
int enqueue_batch_step(sym_batch* b, int k, cudaEvent_t* ev) {
  if (ev) cudaEventRecord(ev[0], b->st);
  if constexpr (kAccumulate<S>)
    k_finalize_batch<S><<<(unsigned)b->nblocks, 256, 0, b->st>>>(b->d_desc[k], b->d_blk);
  else
    k_phase_batch<S><<<(unsigned)b->nblocks, 256, 0, b->st>>>(b->d_desc[k], b->d_blk);
  if (ev) cudaEventRecord(ev[1], b->st);
  if (int e = sparse_enqueue(b->sparse, k, b->st)) return berr(b, e, "sparse step");
  if (ev) cudaEventRecord(ev[2], b->st);
  cudaMemsetAsync(b->d_counter + k, 0, sizeof(int), b->st);
  using R = typename Codec<S>::R;
  k_collide_batch<S><<<b->grid, kTPB<S>, smem_bytes<S>(), b->st>>>(b->d_desc[k], b->d_tiles, b->ntiles,
                                                                  b->d_counter + k);
  if (int e = sparse_enqueue_post(b->sparse, k, b->st)) return berr(b, e, "interpolated bounce-back");
  if (ev) cudaEventRecord(ev[3], b->st);
  return bcuda(b, cudaGetLastError(), "batch step");
}

int enqueue_any(sym_batch* b, int k, cudaEvent_t* ev) {
  return b->storage == SYM_STORE_FP64 ? enqueue_batch_step<double>(b, k, ev)
       : b->storage == SYM_STORE_FP32 ? enqueue_batch_step<float>(b, k, ev)
                                      : enqueue_batch_step<__half>(b, k, ev);
}

// (re)build the descriptor and tile tables and both step graphs
int build(sym_batch* b) {
  free_graphs(b);
  free_tables(b);
  const int n = (int)b->doms.size();
  b->built_cur.assign(n, 0);
  b->built_pc.assign(n, 0);
  std::vector<DomainDesc> desc[2];
  std::vector<long long> off(n + 1, 0);
  std::vector<TileEntry> tiles;
  for (int i = 0; i < n; i++) {
    sym_handle* h = b->doms[i];
    if (!h->fast.valid) {
      if (int e = fast_import(h)) return berr(b, e, h->err.c_str());
      h->fast.valid = true;
    }
    b->built_cur[i] = h->fast.cur;
    b->built_pc[i] = h->fast.pc;
    for (int k = 0; k < 2; k++) desc[k].push_back(make_desc(h, (h->fast.cur + k) & 1, (h->fast.pc + k) & 1));
    off[i + 1] = off[i] + (long long)((h->N + 255) / 256);
    const int xc = std::max(1, b->xchunk[i]);
    const DevParams& P = h->dp;
    const int BY = tile_rows(b->storage);
    for (int xa = 0; xa < P.nx; xa += xc)
      for (int y0 = 0; y0 < P.ny; y0 += BY)
        for (int z0 = 0; z0 < P.nz; z0 += BZ) {
          TileEntry e{};
          e.dom = i; e.z0 = z0; e.y0 = y0; e.xa = xa; e.xb = std::min(xa + xc, P.nx);
          e.cost = std::min(BZ, P.nz - z0) * std::min(BY, P.ny - y0) * (e.xb - e.xa);
          tiles.push_back(e);
        }
  }
  // largest tiles first: the persistent CTAs then finish together
  std::stable_sort(tiles.begin(), tiles.end(), [](const TileEntry& a, const TileEntry& c) { return a.cost > c.cost; });
  b->ntiles = (int)tiles.size();
  b->nblocks = off[n];
  // TMA descriptors: the device copies the domain descriptors point at
  std::vector<CUtensorMap> maps((size_t)4 * n);
  if (int e = bcuda(b, cudaMalloc(&b->d_tmaps, sizeof(CUtensorMap) * maps.size()), "descriptor maps")) return e;
  for (int k = 0; k < 2; k++)
    for (int i = 0; i < n; i++) {
      const int pc = (b->built_pc[i] + k) & 1;
      const size_t j = ((size_t)k * n + i) * 2;
      maps[j] = b->doms[i]->fast.tm_phi[pc];
      maps[j + 1] = b->doms[i]->fast.tm_ref[pc];
      desc[k][i].tm_phi = b->d_tmaps + j;
      desc[k][i].tm_ref = b->d_tmaps + j + 1;
    }
  cudaMemcpyAsync(b->d_tmaps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, b->st);
  for (int k = 0; k < 2; k++) {
    if (int e = bcuda(b, cudaMalloc(&b->d_desc[k], sizeof(DomainDesc) * n), "descriptors")) return e;
    cudaMemcpyAsync(b->d_desc[k], desc[k].data(), sizeof(DomainDesc) * n, cudaMemcpyHostToDevice, b->st);
  }
  std::vector<int2> blk((size_t)off[n]);
  for (int i = 0; i < n; i++)
    for (long long q = off[i]; q < off[i + 1]; q++) blk[(size_t)q] = make_int2(i, (int)(q - off[i]));
  if (int e = bcuda(b, cudaMalloc(&b->d_blk, sizeof(int2) * std::max<size_t>(1, blk.size())), "block table")) return e;
  cudaMemcpyAsync(b->d_blk, blk.data(), sizeof(int2) * blk.size(), cudaMemcpyHostToDevice, b->st);
  if (int e = bcuda(b, cudaMalloc(&b->d_tiles, sizeof(TileEntry) * std::max(1, b->ntiles)), "tiles")) return e;
  cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(TileEntry) * b->ntiles, cudaMemcpyHostToDevice, b->st);
  if (int e = bcuda(b, cudaStreamSynchronize(b->st), "tables")) return e;
  {
    int err = SYM_OK;
    b->sparse = sparse_plan_build(b->doms, b->built_cur, b->built_pc, b->st, &err);
    if (!b->sparse) return berr(b, err, "sparse plan");
  }
  for (int k = 0; k < 2; k++) {
    if (int e = bcuda(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal), "capture")) return e;
    int e1 = enqueue_any(b, k, nullptr);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
    if (e1) { if (g) cudaGraphDestroy(g); return e1; }
    if (int e = bcuda(b, e2, "end capture")) return e;
    b->graph[k] = g;
    if (int e = bcuda(b, cudaGraphInstantiate(&b->gexec[k], g, 0), "instantiate")) return e;
  }
  b->steps_since_build = 0;
  b->built = true;
  return SYM_OK;
}

// members stepped or exported outside the batch invalidate the graphs
bool stale(sym_batch* b) {
  if (!b->built) return true;
  for (size_t i = 0; i < b->doms.size(); i++) {
    const sym_handle* h = b->doms[i];
    if (!h->fast.valid) return true;
    if (h->fast.cur != ((b->built_cur[i] + b->steps_since_build) & 1)) return true;
    if (h->fast.pc != ((b->built_pc[i] + b->steps_since_build) & 1)) return true;
  }
  return false;
}

int launch_steps(sym_batch* b, int nsteps) {
  for (int t = 0; t < nsteps; t++) {
    const int k = b->steps_since_build & 1;
    if (int e = bcuda(b, cudaGraphLaunch(b->gexec[k], b->st), "graph launch")) return e;
    b->steps_since_build++;
    for (sym_handle* h : b->doms) {
      h->fast.cur ^= 1;
      h->fast.pc ^= 1;
    }
  }
  return SYM_OK;
}

}  // namespace

namespace symb200 {
// asynchronous batch steps on the batch stream (the server overlaps batches
// of different storage and enqueues its stop-rule reductions behind them)
int batch_launch(sym_batch* b, int nsteps) {
  cudaSetDevice(b->device);
  if (stale(b))
    if (int e = build(b)) return e;
  return launch_steps(b, nsteps);
}
cudaStream_t batch_stream(sym_batch* b) { return b->st; }
}  // namespace symb200

extern "C" {

int sym_batch_create(sym_handle* const* handles, int n, sym_batch** out) {
  if (!out || !handles || n <= 0) return SYM_ERR_PARAM;
  *out = nullptr;
  sym_batch* b = new sym_batch();
  b->device = handles[0]->device;
  b->storage = handles[0]->fast.storage;
  for (int i = 0; i < n; i++) {
    sym_handle* h = handles[i];
    if (!h || h->dp.ref || h->fast.storage < 0 || h->device != b->device || h->fast.storage != b->storage) {
      delete b;
      return SYM_ERR_PARAM;
    }
    b->doms.push_back(h);
    b->xchunk.push_back(32);
  }
  cudaSetDevice(b->device);
  int e = bcuda(b, cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "stream");
  if (!e) e = bcuda(b, cudaMalloc(&b->d_counter, 2 * sizeof(int)), "counter");
  if (!e) {
    e = b->storage == SYM_STORE_FP64 ? set_batch_smem<double>(b->device, &b->max_per_sm, &b->sms)
      : b->storage == SYM_STORE_FP32 ? set_batch_smem<float>(b->device, &b->max_per_sm, &b->sms)
                                     : set_batch_smem<__half>(b->device, &b->max_per_sm, &b->sms);
    b->per_sm = b->max_per_sm;
    b->grid = b->per_sm * b->sms;
  }
  if (e) {
    fprintf(stderr, "sym_batch_create: %s\n", b->err.c_str());
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return e;
  }
  *out = b;
  return SYM_OK;
}

int sym_batch_destroy(sym_batch* b) {
  if (!b) return SYM_OK;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  free_graphs(b);
  free_tables(b);
  if (b->d_counter) cudaFree(b->d_counter);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return SYM_OK;
}

const char* sym_batch_last_error(const sym_batch* b) { return b ? b->err.c_str() : "null batch"; }

int sym_batch_set_xchunk(sym_batch* b, int domain, int xchunk) {
  if (!b || domain < 0 || domain >= (int)b->doms.size() || xchunk < 1) return SYM_ERR_PARAM;
  if (b->xchunk[domain] != xchunk) {
    b->xchunk[domain] = xchunk;
    free_graphs(b);
  }
  return SYM_OK;
}

int sym_batch_set_ctas_per_sm(sym_batch* b, int per_sm) {
  if (!b || per_sm < 1 || per_sm > b->max_per_sm) return SYM_ERR_PARAM;
  if (b->per_sm != per_sm) {
    b->per_sm = per_sm;
    b->grid = per_sm * b->sms;
    free_graphs(b);
  }
  return SYM_OK;
}

int sym_batch_get_xchunk(sym_batch* b, int domain, int* xchunk) {
  if (!b || !xchunk || domain < 0 || domain >= (int)b->doms.size()) return SYM_ERR_PARAM;
  *xchunk = b->xchunk[domain];
  return SYM_OK;
}

int sym_batch_step(sym_batch* b, int nsteps) {
  if (!b || nsteps < 0) return SYM_ERR_PARAM;
  cudaSetDevice(b->device);
  if (stale(b))
    if (int e = build(b)) return e;
  if (int e = launch_steps(b, nsteps)) return e;
  return bcuda(b, cudaStreamSynchronize(b->st), "batch step");
}

int sym_batch_step_timed(sym_batch* b, int nsteps, double* ms) {
  if (!b || !ms || nsteps <= 0) return SYM_ERR_PARAM;
  cudaSetDevice(b->device);
  if (stale(b))
    if (int e = build(b)) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, b->st);
  int rc = launch_steps(b, nsteps);
  cudaEventRecord(e1, b->st);
  if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->st), "batch timed");
  float v = 0.f;
  if (!rc) cudaEventElapsedTime(&v, e0, e1);
  *ms = v;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Choose the tile x extent per size class (domains grouped by nx: <=32, <=48,
// larger) from {8, 12, 16, 24, 32, 64}, then the persistent collide grid
// (resident CTAs per SM, from the most that fit down to 1), each by timing trial_steps
// graph steps per candidate.  The trial steps advance every domain;
// *steps_taken reports how many.
int sym_batch_autotune(sym_batch* b, int trial_steps, int* steps_taken) {
  if (!b || trial_steps <= 0) return SYM_ERR_PARAM;
  const int cands[6] = {8, 12, 16, 24, 32, 64};
  auto cls = [](int nx) { return nx <= 32 ? 0 : (nx <= 48 ? 1 : 2); };
  int taken = 0;
  for (int c = 0; c < 3; c++) {
    bool any = false;
    for (sym_handle* h : b->doms) any |= cls(h->dp.nx) == c;
    if (!any) continue;
    double best = 1e300;
    int bestx = 32;
    for (int x : cands) {
      for (size_t i = 0; i < b->doms.size(); i++)
        if (cls(b->doms[i]->dp.nx) == c) sym_batch_set_xchunk(b, (int)i, x);
      double ms = 0;
      if (int e = sym_batch_step(b, 1)) return e;   // build + warm
      taken += 1;
      if (int e = sym_batch_step_timed(b, trial_steps, &ms)) return e;
      taken += trial_steps;
      if (ms < best) { best = ms; bestx = x; }
    }
    for (size_t i = 0; i < b->doms.size(); i++)
      if (cls(b->doms[i]->dp.nx) == c) sym_batch_set_xchunk(b, (int)i, bestx);
  }
  double best = 1e300;
  int bestc = b->max_per_sm;
  for (int c = b->max_per_sm; c >= 1; c--) {
    sym_batch_set_ctas_per_sm(b, c);
    double ms = 0;
    if (int e = sym_batch_step(b, 1)) return e;
    taken += 1;
    if (int e = sym_batch_step_timed(b, trial_steps, &ms)) return e;
    taken += trial_steps;
    if (ms < best) { best = ms; bestc = c; }
  }
  sym_batch_set_ctas_per_sm(b, bestc);
  if (steps_taken) *steps_taken = taken;
  return SYM_OK;
}

// nsteps eager (not graph) batch steps with CUDA events on the batch stream.
// ms[0] = whole region, ms[1] = phase launches, ms[2] = batched sparse
// work, ms[3] = collide launches (sums over the steps).
int sym_batch_step_kernels(sym_batch* b, int nsteps, double* ms) {
  if (!b || !ms || nsteps <= 0) return SYM_ERR_PARAM;
  cudaSetDevice(b->device);
  if (stale(b))
    if (int e = build(b)) return e;
  std::vector<cudaEvent_t> ev(4 * (size_t)nsteps + 2, nullptr);
  int rc = SYM_OK;
  for (auto& e : ev)
    if (!rc) rc = bcuda(b, cudaEventCreate(&e), "event");
  if (!rc) {
    cudaEventRecord(ev[4 * nsteps], b->st);
    for (int t = 0; t < nsteps && !rc; t++) {
      const int k = b->steps_since_build & 1;
      rc = enqueue_any(b, k, &ev[4 * t]);
      b->steps_since_build++;
      for (sym_handle* h : b->doms) {
        h->fast.cur ^= 1;
        h->fast.pc ^= 1;
      }
    }
    cudaEventRecord(ev[4 * nsteps + 1], b->st);
    if (!rc) rc = bcuda(b, cudaStreamSynchronize(b->st), "batch kernels");
  }
  if (!rc) {
    float v = 0.f;
    for (int k = 0; k < 4; k++) ms[k] = 0.0;
    cudaEventElapsedTime(&v, ev[4 * nsteps], ev[4 * nsteps + 1]);
    ms[0] = v;
    for (int t = 0; t < nsteps; t++) {
      cudaEventElapsedTime(&v, ev[4 * t], ev[4 * t + 1]); ms[1] += v;
      cudaEventElapsedTime(&v, ev[4 * t + 1], ev[4 * t + 2]); ms[2] += v;
      cudaEventElapsedTime(&v, ev[4 * t + 2], ev[4 * t + 3]); ms[3] += v;
    }
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

// Kernel launches in one captured batch step (kernel nodes of the graph).
int sym_batch_kernels_per_step(sym_batch* b, int* kernels) {
  if (!b || !kernels) return SYM_ERR_PARAM;
  cudaSetDevice(b->device);
  if (stale(b))
    if (int e = build(b)) return e;
  size_t n = 0;
  if (int e = bcuda(b, cudaGraphGetNodes(b->graph[0], nullptr, &n), "graph nodes")) return e;
  std::vector<cudaGraphNode_t> nodes(n);
  if (int e = bcuda(b, cudaGraphGetNodes(b->graph[0], nodes.data(), &n), "graph nodes")) return e;
  int cnt = 0;
  for (size_t i = 0; i < n; i++) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) cnt++;
  }
  *kernels = cnt;
  return SYM_OK;
}

int sym_batch_info(sym_batch* b, int64_t* nodes, int* ntiles, int* grid) {
  if (!b) return SYM_ERR_PARAM;
  long long n = 0;
  for (sym_handle* h : b->doms) n += (long long)h->N;
  if (nodes) *nodes = n;
  if (ntiles) *ntiles = b->ntiles;
  if (grid) *grid = b->grid;
  return SYM_OK;
}

}  // extern "C"
