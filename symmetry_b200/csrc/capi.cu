// capi.cu -- extern "C" entry points declared in include/symmetry.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>
#include "state.cuh"

using namespace symb200;

namespace symb200 {

int set_error(sym_handle* h, int code, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return code;
}

int check_cuda(sym_handle* h, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SYM_OK;
  return set_error(h, e == cudaErrorMemoryAllocation ? SYM_ERR_OOM : SYM_ERR_CUDA, "%s: %s", what,
                   cudaGetErrorString(e));
}

int dev_carve(sym_handle* h, void** p, size_t bytes) {
  const size_t b = (bytes + 255) / 256 * 256;
  *p = nullptr;
  if (h->planning) {
    h->slab_size += b;
    return SYM_OK;
  }
  if (h->slab && h->slab_used + b <= h->slab_size) {
    *p = h->slab + h->slab_used;
    h->slab_used += b;
  } else {
    const cudaError_t e = cudaMalloc(p, b);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();   // a failed allocation must not surface in a later launch check
      *p = nullptr;
      return check_cuda(h, e, "cudaMalloc");
    }
  }
  h->bytes += b;
  return check_cuda(h, cudaMemsetAsync(*p, 0, b, h->st), "memset");
}

void dev_release(sym_handle* h, void* p) {
  if (!p) return;
  if (h->slab && static_cast<char*>(p) >= h->slab && static_cast<char*>(p) < h->slab + h->slab_size) return;
  cudaFree(p);
}

void fill_devparams(const sym_params& p, DevParams& d) {
  d.nx = p.nx; d.ny = p.ny; d.nz = p.nz;
  d.N = (long long)p.nx * p.ny * p.nz;
  d.ref = p.mode == SYM_MODE_REFERENCE;
  d.origin = d.ref ? 1 : 0;
  const int dims[3] = {p.nx, p.ny, p.nz};
  for (int k = 0; k < 3; k++) {
    d.lo[k] = d.ref ? 1 : 0;
    d.hi[k] = d.ref ? dims[k] - 2 : dims[k] - 1;
  }
  d.wall_x = p.wall_x;
  d.par = p.par;
  d.la_m = p.la_m > 0 ? p.la_m : (p.alpha > 0 ? (int)(2.0 * M_PI / p.alpha) : 0);
  d.la_n = p.la_n > 0 ? p.la_n : (p.alpha > 0 ? (int)(M_PI / p.alpha) : 0);
  d.la_num = p.par > 0 ? d.la_m * (d.la_n + 1) : 0;
  d.rho0 = p.rho0; d.nu_r = p.nu_r; d.nu_b = p.nu_b;
  d.s_e = p.s_e; d.s_eps = p.s_eps; d.s_q = p.s_q; d.s_pi = p.s_pi; d.s_m = p.s_m;
  d.sigma = p.sigma; d.beta = p.beta; d.cita = p.cita;
  d.sin_cita = std::sin(p.cita); d.cos_cita = std::cos(p.cita);
  d.bounce = p.bounce;
  for (int k = 0; k < 3; k++) d.body[k] = p.body[k];
  d.rad = p.rad;
  d.mass = p.mass > 0 ? p.mass : 4.0 / 3.0 * p.rho_p * M_PI * (p.rad * p.rad * p.rad);
  d.inertia = p.inertia > 0 ? p.inertia : 2.0 / 5.0 * d.mass * (p.rad * p.rad);
  d.fg = p.fg; d.alpha = p.alpha;
  d.evap = p.evap_lim > 0 ? p.evap_lim : 1.0e-8;
  d.inu_r = p.nu_r > 0 ? 1.0 / p.nu_r : 0.0;
  d.inu_b = p.nu_b > 0 ? 1.0 / p.nu_b : 0.0;
}

}  // namespace symb200

namespace {

template <typename T>
int dalloc(sym_handle* h, T** p, size_t n) {
  void* v = nullptr;
  const int e = dev_carve(h, &v, sizeof(T) * n);
  *p = static_cast<T*>(v);
  return e;
}

size_t reduction_len(const sym_params& p) {
  const size_t N = (size_t)p.nx * p.ny * p.nz;
  size_t n = (N + 255) / 256 * 5 + 16;
  n = std::max(n, (size_t)p.nx + p.ny + p.nz + 16);
  if (p.par > 0) {
    // momentum partials: box (2(R+3)+3)^3 nodes per particle, 256 per block
    const double e = std::ceil(2.0 * (p.rad + 3.0)) + 2.0;
    const size_t box = (size_t)(e * e * e);
    n = std::max(n, ((box + 255) / 256) * 6 * (size_t)p.par + 16);
    n = std::max(n, (size_t)32 * 7 * p.par + 16);   // capillary partial sums
  }
  return n;
}

double* field_ptr_d(sym_handle* h, int f) {
  switch (f) {
    case SYM_F_RI: return h->ri;
    case SYM_F_BI: return h->bi;
    case SYM_F_FI: return h->fi;
    case SYM_F_FFI: return h->ffi;
    case SYM_F_RHO: return h->rho;
    case SYM_F_UX: return h->ux;
    case SYM_F_UY: return h->uy;
    case SYM_F_UZ: return h->uz;
    case SYM_F_RHO_N: return h->rhoN;
    case SYM_F_RHO_R: return h->rhoR;
    case SYM_F_RHO_B: return h->rhoB;
    case SYM_F_NX: return h->nx;
    case SYM_F_NY: return h->ny;
    case SYM_F_NZ: return h->nz;
    case SYM_F_GRADX: return h->gx;
    case SYM_F_GRADY: return h->gy;
    case SYM_F_GRADZ: return h->gz;
    default: return nullptr;
  }
}
int32_t* field_ptr_i(sym_handle* h, int f) {
  switch (f) {
    case SYM_F_FLAG: return h->flag;
    case SYM_F_WALLS: return h->walls;
    case SYM_F_WALLS_OLD: return h->walls_old;
    case SYM_F_WALLS_ALL: return h->walls_all;
    case SYM_F_PIN: return h->pin;
    case SYM_F_POUT: return h->pout;
    default: return nullptr;
  }
}

// Allocate the canonical arrays a CONFIG handle defers (fi, ffi, ft).  With
// the interpolated particle bounce-back the fused path also keeps the red
// post-collision populations of the nodes next to particles behind ffi
// (ffi + 19N), for the link update after the collide kernel.
int ensure_full(sym_handle* h) {
  double** pops[3] = {&h->fi, &h->ffi, &h->ft};
  const bool rpost = h->p.mode == SYM_MODE_CONFIG && h->p.bounce && h->p.par > 0;
  for (auto pp : pops)
    if (!*pp)
      if (int e = dalloc(h, pp, (pp == &h->ffi && rpost ? 38 : 19) * h->N)) return e;
  return SYM_OK;
}

// Make the canonical arrays authoritative (export the fused state if it holds
// the current populations).
int canonical(sym_handle* h) {
  if (h->fast.valid) {
    if (int e = fast_export(h)) return e;
    h->fast.valid = false;
  }
  return SYM_OK;
}

int guard(sym_handle* h) {
  if (!h) return SYM_ERR_PARAM;
  if (int e = check_cuda(h, cudaSetDevice(h->device), "cudaSetDevice")) return e;
  return SYM_OK;
}

// one loop body of main (Source1.f90:216-251) on the canonical state
int canonical_step_once(sym_handle* h) {
  int e;
  if ((e = ref_calmacros(h))) return e;
  if (h->p.par > 0) {
    if ((e = part_lagrange_points(h))) return e;
    if ((e = part_capillary_force2(h))) return e;
    if ((e = part_momentum(h))) return e;
    if ((e = part_repulsive(h))) return e;
    if ((e = part_movement(h))) return e;
  }
  if ((e = part_set_walls(h))) return e;
  if (h->p.par > 0)
    if ((e = part_refilling(h))) return e;
  if ((e = ref_derivatives(h))) return e;
  if ((e = ref_collision(h))) return e;
  if ((e = ref_recolor(h))) return e;
  if ((e = ref_boundary(h))) return e;
  if ((e = ref_streaming(h, 0))) return e;
  if ((e = ref_streaming(h, 1))) return e;
  return ref_curve(h);
}

int canonical_steps(sym_handle* h, int nsteps) {
  if (!h->gexec) {
    if (int e = check_cuda(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal), "begin capture"))
      return e;
    const int e1 = canonical_step_once(h);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e1) { if (g) cudaGraphDestroy(g); return e1; }
    if (int e = check_cuda(h, e2, "end capture")) return e;
    h->graph = g;
    if (int e = check_cuda(h, cudaGraphInstantiate(&h->gexec, g, 0), "graph instantiate")) return e;
  }
  for (int t = 0; t < nsteps; t++)
    if (int e = check_cuda(h, cudaGraphLaunch(h->gexec, h->st), "graph launch")) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "step");
}

// Every array a new handle holds, in one fixed order; with h->planning set it
// only sums the sizes.
int alloc_state(sym_handle* h) {
  const sym_params& p = h->p;
  const size_t N = h->N;
  int e = SYM_OK;
  // ri, bi always; fi, ffi and the streaming/transfer temporary ft only where
  // the mode needs them up front (REFERENCE subroutines, particle coupling),
  // otherwise on the first call that uses them (ensure_full)
  double** pops[2] = {&h->ri, &h->bi};
  for (auto pp : pops)
    if (!e) e = dalloc(h, pp, 19 * N);
  if (!e && (p.mode == SYM_MODE_REFERENCE || p.par > 0)) e = ensure_full(h);
  double** sc[13] = {&h->rho, &h->ux, &h->uy, &h->uz, &h->rhoN, &h->rhoR, &h->rhoB,
                     &h->nx, &h->ny, &h->nz, &h->gx, &h->gy, &h->gz};
  for (auto pp : sc)
    if (!e) e = dalloc(h, pp, N);
  int32_t** ms[6] = {&h->flag, &h->walls, &h->walls_old, &h->walls_all, &h->pin, &h->pout};
  for (auto pp : ms)
    if (!e) e = dalloc(h, pp, N);
  if (!e) e = dalloc(h, &h->dpart, 1);
  const size_t NL = (size_t)h->dp.la_num * h->dp.par;
  if (NL) {
    double** la[8] = {&h->lax, &h->lay, &h->laz, &h->larhon, &h->lanx, &h->lany, &h->lanz, &h->lads};
    for (auto pp : la)
      if (!e) e = dalloc(h, pp, NL);
    if (!e) e = dalloc(h, &h->laflag, NL);
  }
  h->red_len = reduction_len(p);
  if (!e) e = dalloc(h, &h->red, h->red_len);
  if (!e && p.mode == SYM_MODE_CONFIG) e = fast_alloc(h);
  return e;
}

}  // namespace

namespace symb200 {
// calmacros of the current populations into the canonical macro arrays
// (rho, u, rho_N) without changing the stepping state: from the fused
// populations when they are current, else from ri/bi (the canonical kernel
// also writes fi, which CONFIG handles without particles allocate lazily)
int current_macros(sym_handle* h) {
  if (h->fast.valid) return fast_macros(h);
  if (int e = ensure_full(h)) return e;
  return ref_calmacros(h);
}
}  // namespace symb200

extern "C" {

int sym_params_reference(sym_params* p, int nx, int ny, int nz) {
  if (!p) return SYM_ERR_PARAM;
  std::memset(p, 0, sizeof(*p));
  p->nx = nx; p->ny = ny; p->nz = nz;
  p->mode = SYM_MODE_REFERENCE;
  p->par = 12;                                    // :24
  const double oh = 0.1, lamda = 10.0, rad_c = 30.0;  // :58-63
  p->sigma = 0.05; p->rho0 = 0.05;                // :66-67
  p->nu_r = oh / std::sqrt(p->rho0 / (rad_c * p->sigma));
  p->nu_b = p->nu_r / lamda;                      // :69-70
  p->beta = 0.7;                                  // :17
  p->cita = 90.0 / 180.0 * M_PI;                  // :21
  p->rad = 7.5;                                   // :76
  p->rho_p = 1.0 * p->rho0;                       // :79
  p->mass = 4.0 / 3.0 * p->rho_p * M_PI * (p->rad * p->rad * p->rad);  // :81
  p->inertia = 2.0 / 5.0 * p->mass * (p->rad * p->rad);              // :82
  p->fg = -M_PI * 2.0 * p->rad * p->sigma;        // :84
  p->alpha = 2.0 / 180.0 * M_PI;                  // :22
  p->evap_lim = 1.0e-8;                           // :16
  return SYM_OK;
}

int sym_params_check(const sym_params* p, char* msg, size_t msg_len) {
  auto fail = [&](const char* m) {
    if (msg && msg_len) snprintf(msg, msg_len, "%s", m);
    return SYM_ERR_PARAM;
  };
  if (!p) return fail("null params");
  if (p->nx < 3 || p->ny < 3 || p->nz < 3) return fail("every dimension must be >= 3");
  if ((double)p->nx * p->ny * p->nz > 4.0e9) return fail("domain too large");
  if (p->mode != SYM_MODE_REFERENCE && p->mode != SYM_MODE_CONFIG) return fail("unknown mode");
  if (p->storage < SYM_STORE_FP64 || p->storage > SYM_STORE_FP16) return fail("unknown storage");
  if (p->par < 0 || p->par > SYM_MAX_PAR) return fail("par out of range");
  if (p->bounce != 0 && p->bounce != 1) return fail("bounce must be 0 (halfway) or 1 (interpolated)");
  if (!(p->nu_r > 0.0) || !(p->nu_b > 0.0) || !std::isfinite(p->nu_r) || !std::isfinite(p->nu_b))
    return fail("viscosities must be finite and > 0 (tau > 0.5)");
  if (!(p->rho0 > 0.0) || !std::isfinite(p->rho0)) return fail("rho0 must be finite and > 0");
  const double rates[5] = {p->s_e, p->s_eps, p->s_q, p->s_pi, p->s_m};
  for (double s : rates)
    if (!std::isfinite(s) || s >= 2.0) return fail("MRT rates must be finite and < 2");
  if (!std::isfinite(p->sigma) || !std::isfinite(p->beta) || !std::isfinite(p->cita)) return fail("non-finite sigma/beta/cita");
  for (int k = 0; k < 3; k++)
    if (!std::isfinite(p->body[k])) return fail("non-finite body force");
  if (p->par > 0) {
    if (!(p->rad > 0.0) || !std::isfinite(p->rad)) return fail("particle radius must be > 0");
    if (!(p->alpha > 0.0) && !(p->la_m > 0 && p->la_n > 0)) return fail("alpha or la_m/la_n required");
    if (!(p->rho_p > 0.0) && !(p->mass > 0.0)) return fail("particle density or mass required");
  }
  if (p->mode == SYM_MODE_CONFIG && p->wall_x && p->nx < 4) return fail("wall_x needs nx >= 4");
  if (p->mode == SYM_MODE_REFERENCE && p->wall_x) return fail("wall_x is a CONFIG-mode option");
  return SYM_OK;
}

int sym_footprint(const sym_params* p, size_t* bytes) {
  if (!p || !bytes) return SYM_ERR_PARAM;
  if (int e = sym_params_check(p, nullptr, 0)) return e;
  sym_handle h;   // planning pass: sizes only, no device calls
  h.p = *p;
  fill_devparams(*p, h.dp);
  h.N = (size_t)h.dp.N;
  h.planning = true;
  if (int e = alloc_state(&h)) return e;
  *bytes = h.slab_size;
  return SYM_OK;
}

int sym_create(const sym_params* p, int device, sym_handle** out) {
  if (!out) return SYM_ERR_PARAM;
  *out = nullptr;
  char msg[256];
  if (int e = sym_params_check(p, msg, sizeof msg)) {
    fprintf(stderr, "sym_create: %s\n", msg);
    return e;
  }
  sym_handle* h = new sym_handle();
  h->p = *p;
  h->device = device;
  fill_devparams(*p, h->dp);
  h->N = (size_t)h->dp.N;
  h->planning = true;
  int e = alloc_state(h);
  h->planning = false;
  h->bytes = 0;
  if (!e) e = check_cuda(h, cudaSetDevice(device), "cudaSetDevice");
  if (!e) e = check_cuda(h, cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking), "stream");
  if (!e) {
    const cudaError_t ce = cudaMalloc((void**)&h->slab, h->slab_size);
    if (ce != cudaSuccess) {
      (void)cudaGetLastError();
      h->slab = nullptr;
      e = check_cuda(h, ce, "device state");
    }
  }
  if (!e) e = alloc_state(h);
  if (!e) e = check_cuda(h, cudaStreamSynchronize(h->st), "create");
  if (e) {
    fprintf(stderr, "sym_create: %s\n", h->err.c_str());
    sym_destroy(h);
    return e;
  }
  *out = h;
  return SYM_OK;
}

int sym_destroy(sym_handle* h) {
  if (!h) return SYM_OK;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  fast_free(h);
  void* ptrs[] = {h->ri, h->bi, h->fi, h->ffi, h->ft, h->rho, h->ux, h->uy, h->uz, h->rhoN, h->rhoR, h->rhoB,
                  h->nx, h->ny, h->nz, h->gx, h->gy, h->gz, h->flag, h->walls, h->walls_old, h->walls_all,
                  h->pin, h->pout, h->dpart, h->lax, h->lay, h->laz, h->larhon, h->lanx, h->lany, h->lanz,
                  h->lads, h->laflag, h->red};
  for (void* q : ptrs) dev_release(h, q);
  if (h->slab) cudaFree(h->slab);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return SYM_OK;
}

const char* sym_last_error(const sym_handle* h) { return h ? h->err.c_str() : "null handle"; }

int sym_lattice_tables(int32_t tables[7 * 19], double wi[19], double m[19 * 19]) {
  for (int i = 0; i < 19; i++) {
    if (tables) {
      tables[i] = CX(i); tables[19 + i] = CY(i); tables[38 + i] = CZ(i); tables[57 + i] = OPC(i);
      tables[76 + i] = SYMX(i); tables[95 + i] = SYMY(i); tables[114 + i] = SYMZ(i);
    }
    if (wi) wi[i] = W(i);
    if (m)
      for (int c = 0; c < 19; c++) m[i * 19 + c] = MROW(i, c);
  }
  return SYM_OK;
}

int sym_set_field(sym_handle* h, int field, const void* host) {
  if (int e = guard(h)) return e;
  if (!host) return set_error(h, SYM_ERR_PARAM, "null host pointer");
  if (int e = canonical(h)) return e;
  const size_t N = h->N;
  if (field >= SYM_F_RI && field <= SYM_F_FFI) {
    if (int e = ensure_full(h)) return e;
    cudaMemcpyAsync(h->ft, host, sizeof(double) * 19 * N, cudaMemcpyHostToDevice, h->st);
    if (int e = aos_to_soa(h, h->ft, field_ptr_d(h, field))) return e;
  } else if (double* d = field_ptr_d(h, field)) {
    cudaMemcpyAsync(d, host, sizeof(double) * N, cudaMemcpyHostToDevice, h->st);
  } else if (int32_t* d = field_ptr_i(h, field)) {
    cudaMemcpyAsync(d, host, sizeof(int32_t) * N, cudaMemcpyHostToDevice, h->st);
  } else {
    return set_error(h, SYM_ERR_NOTFOUND, "unknown field %d", field);
  }
  return check_cuda(h, cudaStreamSynchronize(h->st), "set_field");
}

int sym_get_field(sym_handle* h, int field, void* host) {
  if (int e = guard(h)) return e;
  if (!host) return set_error(h, SYM_ERR_PARAM, "null host pointer");
  if (int e = canonical(h)) return e;
  const size_t N = h->N;
  if (field >= SYM_F_RI && field <= SYM_F_FFI) {
    if (int e = ensure_full(h)) return e;
    if (int e = soa_to_aos(h, field_ptr_d(h, field), h->ft)) return e;
    cudaMemcpyAsync(host, h->ft, sizeof(double) * 19 * N, cudaMemcpyDeviceToHost, h->st);
  } else if (double* d = field_ptr_d(h, field)) {
    cudaMemcpyAsync(host, d, sizeof(double) * N, cudaMemcpyDeviceToHost, h->st);
  } else if (int32_t* d = field_ptr_i(h, field)) {
    cudaMemcpyAsync(host, d, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, h->st);
  } else {
    return set_error(h, SYM_ERR_NOTFOUND, "unknown field %d", field);
  }
  return check_cuda(h, cudaStreamSynchronize(h->st), "get_field");
}

int sym_get_macros(sym_handle* h, double* rho, double* ux, double* uy, double* uz, double* rho_n) {
  if (int e = guard(h)) return e;
  if (int e = current_macros(h)) return e;
  double* src[5] = {h->rho, h->ux, h->uy, h->uz, h->rhoN};
  double* dst[5] = {rho, ux, uy, uz, rho_n};
  for (int k = 0; k < 5; k++)
    if (dst[k]) cudaMemcpyAsync(dst[k], src[k], sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->st);
  return check_cuda(h, cudaStreamSynchronize(h->st), "get_macros");
}

int sym_set_populations(sym_handle* h, const double* ri, const double* bi) {
  if (int e = guard(h)) return e;
  if (!ri || !bi) return set_error(h, SYM_ERR_PARAM, "null populations");
  if (int e = ensure_full(h)) return e;
  if (h->fast.valid) {
    // both colours are replaced: only the fused phase field is still needed
    if (int e = fast_export(h)) return e;
    h->fast.valid = false;
  }
  const size_t N = h->N;
  cudaMemcpyAsync(h->ft, ri, sizeof(double) * 19 * N, cudaMemcpyHostToDevice, h->st);
  if (int e = aos_to_soa(h, h->ft, h->ri)) return e;
  cudaMemcpyAsync(h->ft, bi, sizeof(double) * 19 * N, cudaMemcpyHostToDevice, h->st);
  if (int e = aos_to_soa(h, h->ft, h->bi)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "set_populations");
}

int sym_set_particles(sym_handle* h, const sym_particles* s) {
  if (int e = guard(h)) return e;
  if (!s) return set_error(h, SYM_ERR_PARAM, "null particles");
  cudaMemcpyAsync(h->dpart, s, sizeof(sym_particles), cudaMemcpyHostToDevice, h->st);
  return check_cuda(h, cudaStreamSynchronize(h->st), "set_particles");
}

int sym_get_particles(sym_handle* h, sym_particles* s) {
  if (int e = guard(h)) return e;
  if (!s) return set_error(h, SYM_ERR_PARAM, "null particles");
  cudaMemcpyAsync(s, h->dpart, sizeof(sym_particles), cudaMemcpyDeviceToHost, h->st);
  return check_cuda(h, cudaStreamSynchronize(h->st), "get_particles");
}

int sym_get_lagrange(sym_handle* h, double* lax, double* lay, double* laz, double* la_rhon, double* la_nx,
                     double* la_ny, double* la_nz, int32_t* la_flag, double* ds) {
  if (int e = guard(h)) return e;
  const size_t NL = (size_t)h->dp.la_num * h->dp.par;
  if (!NL) return SYM_OK;
  double* dst[8] = {lax, lay, laz, la_rhon, la_nx, la_ny, la_nz, ds};
  double* src[8] = {h->lax, h->lay, h->laz, h->larhon, h->lanx, h->lany, h->lanz, h->lads};
  for (int k = 0; k < 8; k++)
    if (dst[k]) cudaMemcpyAsync(dst[k], src[k], sizeof(double) * NL, cudaMemcpyDeviceToHost, h->st);
  if (la_flag) cudaMemcpyAsync(la_flag, h->laflag, sizeof(int32_t) * NL, cudaMemcpyDeviceToHost, h->st);
  return check_cuda(h, cudaStreamSynchronize(h->st), "get_lagrange");
}

// ---- initial state ---------------------------------------------------------
int sym_initia_center(sym_handle* h) {
  if (int e = guard(h)) return e;
  if (!h->dp.ref) return set_error(h, SYM_ERR_UNSUPPORTED, "initia_center is the REFERENCE particle layout");
  if (int e = part_initia_center(h)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "initia_center");
}
int sym_initialization(sym_handle* h) {
  if (int e = guard(h)) return e;
  if (!h->dp.ref) return set_error(h, SYM_ERR_UNSUPPORTED, "initialization is the REFERENCE initial state");
  h->fast.valid = false;
  if (int e = ref_initialization(h)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "initialization");
}
int sym_init_phase(sym_handle* h, const double* rho_n, const double* rho) {
  if (int e = guard(h)) return e;
  if (!rho_n || !rho) return set_error(h, SYM_ERR_PARAM, "null phase/density");
  h->fast.valid = false;
  cudaMemcpyAsync(h->rhoN, rho_n, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->st);
  cudaMemcpyAsync(h->rho, rho, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->st);
  if (int e = ref_init_fill(h)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "init_phase");
}
int sym_init_thread(sym_handle* h, double radius, double amp, double wavelength, double width, double noise,
                    uint64_t seed) {
  if (int e = guard(h)) return e;
  if (h->dp.ref) return set_error(h, SYM_ERR_UNSUPPORTED, "init_thread is a CONFIG initialiser");
  if (!(radius > 0) || !(wavelength > 0) || !(width > 0)) return set_error(h, SYM_ERR_PARAM, "bad thread geometry");
  h->fast.valid = false;
  if (int e = ref_init_thread(h, radius, amp, wavelength, width, noise, seed)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "init_thread");
}
int sym_init_slab(sym_handle* h, double z0, double z1, double width, double noise, uint64_t seed) {
  if (int e = guard(h)) return e;
  if (h->dp.ref) return set_error(h, SYM_ERR_UNSUPPORTED, "init_slab is a CONFIG initialiser");
  if (!(width > 0)) return set_error(h, SYM_ERR_PARAM, "bad slab width");
  h->fast.valid = false;
  if (int e = ref_init_slab(h, z0, z1, width, noise, seed)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "init_slab");
}

// ---- the reference's subroutines -----------------------------------------------
// `full`: the subroutine reads or writes fi, ffi or the temporary ft, which
// a CONFIG handle without particles allocates on first use
#define SYM_SUBROUTINE(name, call, full)                               \
  int name(sym_handle* h) {                                            \
    if (int e = guard(h)) return e;                                    \
    if (full)                                                          \
      if (int e = ensure_full(h)) return e;                            \
    if (int e = canonical(h)) return e;                                \
    if (int e = call) return e;                                        \
    return check_cuda(h, cudaStreamSynchronize(h->st), #name);         \
  }
SYM_SUBROUTINE(sym_set_walls, part_set_walls(h), false)
SYM_SUBROUTINE(sym_calmacros, ref_calmacros(h), true)
SYM_SUBROUTINE(sym_derivatives, ref_derivatives(h), false)
SYM_SUBROUTINE(sym_collision, ref_collision(h), true)
SYM_SUBROUTINE(sym_recolor, ref_recolor(h), true)
SYM_SUBROUTINE(sym_boundary, ref_boundary(h), true)
SYM_SUBROUTINE(sym_curve, ref_curve(h), true)
SYM_SUBROUTINE(sym_lagrange_points, part_lagrange_points(h), false)
SYM_SUBROUTINE(sym_capillary_force2, part_capillary_force2(h), false)
SYM_SUBROUTINE(sym_momentum, part_momentum(h), true)
SYM_SUBROUTINE(sym_repulsive, part_repulsive(h), false)
SYM_SUBROUTINE(sym_movement, part_movement(h), false)
SYM_SUBROUTINE(sym_refilling, part_refilling(h), true)
#undef SYM_SUBROUTINE

int sym_streaming(sym_handle* h, int which) {
  if (int e = guard(h)) return e;
  if (which != 0 && which != 1) return set_error(h, SYM_ERR_PARAM, "streaming: which must be 0 (ri) or 1 (bi)");
  if (int e = ensure_full(h)) return e;
  if (int e = canonical(h)) return e;
  if (int e = ref_streaming(h, which)) return e;
  return check_cuda(h, cudaStreamSynchronize(h->st), "sym_streaming");
}

int sym_step(sym_handle* h, int nsteps) {
  if (int e = guard(h)) return e;
  if (nsteps < 0) return set_error(h, SYM_ERR_PARAM, "nsteps < 0");
  if (nsteps == 0) return SYM_OK;
  if (!h->dp.ref && h->fast.storage >= 0) {
    if (!h->fast.valid) {
      if (int e = fast_import(h)) return e;
      h->fast.valid = true;
    }
    return fast_step(h, nsteps);
  }
  if (int e = ensure_full(h)) return e;
  if (int e = canonical(h)) return e;
  return canonical_steps(h, nsteps);
}

int sym_step_timed(sym_handle* h, int nsteps, int use_graph, double ms[4]) {
  if (int e = guard(h)) return e;
  if (!ms || nsteps <= 0) return set_error(h, SYM_ERR_PARAM, "step_timed: bad arguments");
  for (int k = 0; k < 4; k++) ms[k] = -1.0;
  if (h->dp.ref || h->fast.storage < 0) return set_error(h, SYM_ERR_UNSUPPORTED, "step_timed: CONFIG mode only");
  if (!h->fast.valid) {
    if (int e = fast_import(h)) return e;
    h->fast.valid = true;
  }
  if (!use_graph) return fast_step_timed(h, nsteps, ms);
  // graph replay with events around the whole region
  if (int e = fast_step(h, 1)) return e;   // make sure both parities are instantiated
  if (int e = fast_step(h, 1)) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, h->st);
  int rc = SYM_OK;
  for (int t = 0; t < nsteps && !rc; t++) {
    rc = check_cuda(h, cudaGraphLaunch(h->fast.gexec[h->fast.cur], h->st), "graph launch");
    h->fast.cur = 1 - h->fast.cur;
    h->fast.pc = 1 - h->fast.pc;
  }
  cudaEventRecord(b, h->st);
  if (!rc) rc = check_cuda(h, cudaStreamSynchronize(h->st), "timed graph");
  float v = 0.f;
  if (!rc) cudaEventElapsedTime(&v, a, b);
  ms[0] = v;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

// ---- diagnostics -----------------------------------------------------------
int sym_output3(sym_handle* h, double* hmin, int32_t* y0) {
  if (int e = guard(h)) return e;
  if (!hmin || !y0) return set_error(h, SYM_ERR_PARAM, "null output");
  if (int e = canonical(h)) return e;
  return ref_output3(h, hmin, y0);
}
int sym_neck_radius(sym_handle* h, double* rmin) {
  if (int e = guard(h)) return e;
  if (!rmin) return set_error(h, SYM_ERR_PARAM, "null output");
  if (h->fast.valid) {
    // the fused phase field is the rho_N an export would produce: reduce it
    // in place instead of exporting the populations
    const int nz = h->dp.nz;
    if (int e = fast_neck_planes(h, h->red, h->st)) return e;
    std::vector<double> a(nz);
    cudaMemcpyAsync(a.data(), h->red, sizeof(double) * nz, cudaMemcpyDeviceToHost, h->st);
    if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "neck_radius")) return e;
    double mn = 1e300;
    for (int z = 0; z < nz; z++) mn = std::fmin(mn, std::sqrt(a[z] / M_PI));
    *rmin = mn;
    return SYM_OK;
  }
  return ref_neck_radius(h, rmin);
}
int sym_mass_momentum(sym_handle* h, double out[5]) {
  if (int e = guard(h)) return e;
  if (!out) return set_error(h, SYM_ERR_PARAM, "null output");
  if (int e = canonical(h)) return e;
  return ref_mass_momentum(h, out);
}
int sym_device_status(sym_handle* h, int32_t* flags) {
  if (int e = guard(h)) return e;
  if (!flags) return set_error(h, SYM_ERR_PARAM, "null output");
  int32_t v = 0;
  if (h->fast.status) {
    cudaMemcpyAsync(&v, h->fast.status, sizeof(int32_t), cudaMemcpyDeviceToHost, h->st);
    if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "device status")) return e;
  }
  *flags = v;
  return SYM_OK;
}

}  // extern "C"
