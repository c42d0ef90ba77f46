// state.cuh -- device state behind a sym_handle.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/symmetry.h"
#include "lattice.cuh"

namespace symb200 {

struct SparsePlan;   // sparse.cu

// Fused fast-path state (CONFIG mode).  Populations are stored post-stream
// (push streaming), structure of arrays [colour][velocity][node], in the
// handle's storage type, double buffered.
struct FastState {
  int storage = -1;        // SYM_STORE_*
  void* pop[2] = {nullptr, nullptr};
  int cur = 0;             // buffer holding the current post-stream populations
  int pc = 0;              // phase-field buffer written by the next step
  int xchunk = 0;          // x planes per tile of the fused collide kernel (0 = default)
  double* phi[2] = {nullptr, nullptr};  // FP64 halo-padded phase field (pin-filled)
  float* phif[2] = {nullptr, nullptr};  // FP32 halo-padded phase field for FP32/FP16 storage
  float2* rref[2] = {nullptr, nullptr};  // 16-bit storage: halo-padded reference pairs (rho, red fraction), same parity as phi
  void* acc = nullptr;     // next step's colour densities, fixed point [red N][blue N] (see fused.cuh)
  uint2* links = nullptr;  // particles: momentum link lists [particle][box block][256] (see particles.cuh)
  int* nlinks = nullptr;   // entries of each [particle][box block]
  long long link_blocks = 0;   // blocks of one particle's momentum box
  int* status = nullptr;   // sticky: bit 0 an accumulated density was not finite or out of
                           // range, bit 1 a shared-memory tile load did not complete in time
  // TMA descriptors of the halo-padded phase field and reference-pair arrays, per parity
  CUtensorMap tm_phi[2] = {};
  CUtensorMap tm_ref[2] = {};
  bool valid = false;      // fast state holds the authoritative populations
  SparsePlan* sparse = nullptr;   // particle and wall work of sym_step (built on first use)
  size_t bytes = 0;
  cudaGraph_t graph[2] = {nullptr, nullptr};       // one captured step per buffer parity
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
};

}  // namespace symb200

struct sym_handle {
  sym_params p;
  symb200::DevParams dp;
  int device = 0;
  cudaStream_t st = nullptr;
  size_t N = 0;
  // canonical state (reference arrays, SoA, FP64)
  double *ri = nullptr, *bi = nullptr, *fi = nullptr, *ffi = nullptr, *ft = nullptr;
  double *rho = nullptr, *ux = nullptr, *uy = nullptr, *uz = nullptr;
  double *rhoN = nullptr, *rhoR = nullptr, *rhoB = nullptr;
  double *nx = nullptr, *ny = nullptr, *nz = nullptr, *gx = nullptr, *gy = nullptr, *gz = nullptr;
  int32_t *flag = nullptr, *walls = nullptr, *walls_old = nullptr, *walls_all = nullptr, *pin = nullptr,
          *pout = nullptr;
  // particles
  sym_particles* dpart = nullptr;   // device copy
  double *lax = nullptr, *lay = nullptr, *laz = nullptr, *larhon = nullptr, *lanx = nullptr, *lany = nullptr,
         *lanz = nullptr, *lads = nullptr;
  int32_t* laflag = nullptr;
  double* red = nullptr;            // reduction scratch (partials)
  size_t red_len = 0;
  double* hred = nullptr;           // pinned host scalars
  symb200::FastState fast;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_steps = 0;
  size_t bytes = 0;
  // Every array the handle holds from creation is carved from one device
  // allocation (the slab): one cudaMalloc and one cudaFree per handle, no
  // per-array rounding.  A planning pass sizes it (and answers sym_footprint)
  // without touching the device.
  bool planning = false;
  char* slab = nullptr;
  size_t slab_size = 0, slab_used = 0;
  std::string err;
};

namespace symb200 {
// launch helpers shared between translation units
int set_error(sym_handle* h, int code, const char* fmt, ...);
int check_cuda(sym_handle* h, cudaError_t e, const char* what);
void fill_devparams(const sym_params& p, DevParams& d);
int dev_carve(sym_handle* h, void** p, size_t bytes);   // zeroed device array from the slab (or cudaMalloc)
void dev_release(sym_handle* h, void* p);               // frees only what did not come from the slab

// canonical (reference-structured) kernels, ref_kernels.cu
int ref_calmacros(sym_handle* h);
int ref_derivatives(sym_handle* h);
int ref_collision(sym_handle* h);
int ref_recolor(sym_handle* h);
int ref_boundary(sym_handle* h);
int ref_streaming(sym_handle* h, int which);
int ref_curve(sym_handle* h);
int ref_initialization(sym_handle* h);
int ref_init_fill(sym_handle* h);    // rhoN, rho given -> populations
int ref_init_thread(sym_handle* h, double radius, double amp, double wavelength, double width, double noise,
                    unsigned long long seed);
int ref_init_slab(sym_handle* h, double z0, double z1, double width, double noise, unsigned long long seed);
int ref_neck_radius(sym_handle* h, double* rmin);
int ref_output3(sym_handle* h, double* hmin, int32_t* y0);
int ref_mass_momentum(sym_handle* h, double out[5]);
int aos_to_soa(sym_handle* h, const double* dev_aos, double* dev_soa);
int soa_to_aos(sym_handle* h, const double* dev_soa, double* dev_aos);

// particle kernels, particles.cu
int part_set_walls(sym_handle* h);
int part_lagrange_points(sym_handle* h);
int part_capillary_force2(sym_handle* h);
int part_momentum(sym_handle* h);
int part_repulsive(sym_handle* h);
int part_movement(sym_handle* h);
int part_refilling(sym_handle* h);
int part_initia_center(sym_handle* h);

// fused fast path, fast.cu
int fast_alloc(sym_handle* h);
void fast_free(sym_handle* h);
int fast_import(sym_handle* h);   // canonical -> fast
int fast_export(sym_handle* h);   // fast -> canonical
int fast_macros(sym_handle* h);   // calmacros of the fused populations into rho, u, rho_N (fused state kept)
int current_macros(sym_handle* h);   // calmacros of whichever state is current (capi.cu)
int fast_step(sym_handle* h, int nsteps);
int fast_step_timed(sym_handle* h, int nsteps, double ms[4]);
int fast_neck_planes(sym_handle* h, double* out, cudaStream_t st);   // per-z red area, nz doubles

// particle and wall work of fused steps, batched (sparse.cu): the plan for
// `doms` at buffer parities cur0/pc0 for step parity 0, its launches for step
// parity k, launches per step
SparsePlan* sparse_plan_build(const std::vector<sym_handle*>& doms, const std::vector<int>& cur0,
                              const std::vector<int>& pc0, cudaStream_t st, int* err);
int sparse_enqueue(SparsePlan* p, int k, cudaStream_t st);
int sparse_enqueue_post(SparsePlan* p, int k, cudaStream_t st);   // after the collide kernel
int sparse_launches(const SparsePlan* p);
void sparse_plan_free(SparsePlan* p);
// momentum link lists of h's particles from its current masks (after an import)
int sparse_links_build(sym_handle* h, cudaStream_t st);

// batch engine, batch.cu
int batch_launch(sym_batch* b, int nsteps);   // enqueue nsteps graph steps, no synchronisation
cudaStream_t batch_stream(sym_batch* b);
}  // namespace symb200
