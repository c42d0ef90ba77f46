// checkpoint.cu -- population checkpoint and restart of a handle.
//
// The reference keeps no restartable state: its OUT_t.dat files hold the
// macroscopic fields only (Source1.f90:898-924), and a run cannot resume from
// them.  A checkpoint here is the complete stepping state of a handle, so a
// run resumed from it continues bit for bit as if it had never stopped (a
// served job can be preempted and resumed, a long run survives a restart):
//   fused state (CONFIG handles stepped by sym_step): the current
//     populations in their storage format, the last phase field, the 16-bit
//     reference densities, the accumulated colour densities of the next step
//     and the status word, plus the masks, the post-collision populations the
//     next momentum exchange reads and the particle state;
//   canonical state (REFERENCE handles and handles driven per subroutine):
//     every reference array plus the particle state.
// File: the 8-byte magic "SYMCKPT1", a header (the handle's sym_params, the
// mode, buffer parities and node count), then named sections (16-byte name,
// 64-bit byte count, bytes).  A checkpoint loads only into a handle created
// with the same parameters.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "state.cuh"
#include "fused.cuh"

namespace symb200 {
namespace {

constexpr char kMagic[8] = {'S', 'Y', 'M', 'C', 'K', 'P', 'T', '1'};

struct Header {
  sym_params p;
  int32_t fused;     // 1: fused state, 0: canonical state
  int32_t storage;
  int32_t cur, pc;
  int64_t nodes;
};

struct Section {
  const char* name;
  void* dev;      // device array, or nullptr for the host particle block
  size_t bytes;
};

// the arrays of the handle's current state, in file order
std::vector<Section> sections(sym_handle* h, bool fused) {
  std::vector<Section> s;
  const size_t N = h->N;
  const size_t NI = sizeof(int32_t) * N;
  const size_t ND = sizeof(double) * N;
  if (fused) {
    FastState& F = h->fast;
    const size_t sp = F.storage == SYM_STORE_FP64 ? 8 : (F.storage == SYM_STORE_FP32 ? 4 : 2);
    const fused::Pad pd = fused::make_pad(h->dp);
    const size_t phib = (F.storage == SYM_STORE_FP64 ? 8 : 4) * (size_t)pd.size();
    s.push_back({"populations", F.pop[F.cur], 38 * N * sp});
    s.push_back({"phase_field", F.storage == SYM_STORE_FP64 ? (void*)F.phi[1 - F.pc] : (void*)F.phif[1 - F.pc],
                 phib});
    if (F.storage == SYM_STORE_FP16) s.push_back({"reference_pairs", F.rref[1 - F.pc], sizeof(float2) * pd.size()});
    if (F.acc) s.push_back({"accumulators", F.acc, 2 * N * 8});
    s.push_back({"status", F.status, sizeof(int)});
    if (h->dp.par > 0) s.push_back({"ffi", h->ffi, 19 * ND});   // held from creation
  } else {
    s.push_back({"ri", h->ri, 19 * ND});
    s.push_back({"bi", h->bi, 19 * ND});
    s.push_back({"fi", h->fi, 19 * ND});
    s.push_back({"ffi", h->ffi, 19 * ND});
    double* sc[13] = {h->rho, h->ux, h->uy, h->uz, h->rhoN, h->rhoR, h->rhoB,
                      h->nx, h->ny, h->nz, h->gx, h->gy, h->gz};
    const char* nm[13] = {"rho", "ux", "uy", "uz", "rho_N", "rho_R", "rho_B", "n_x", "n_y", "n_z",
                          "gradx", "grady", "gradz"};
    for (int k = 0; k < 13; k++) s.push_back({nm[k], sc[k], ND});
    s.push_back({"flag", h->flag, NI});
  }
  int32_t* ms[5] = {h->walls, h->walls_old, h->walls_all, h->pin, h->pout};
  const char* mn[5] = {"walls", "walls_old", "walls_all", "pin", "pout"};
  for (int k = 0; k < 5; k++) s.push_back({mn[k], ms[k], NI});
  s.push_back({"particles", nullptr, sizeof(sym_particles)});
  return s;
}

// the canonical population arrays a CONFIG handle allocates on first use
int ensure_canonical_pops(sym_handle* h) {
  double** pops[3] = {&h->fi, &h->ffi, &h->ft};
  for (auto pp : pops)
    if (!*pp)
      if (int e = dev_carve(h, (void**)pp, sizeof(double) * 19 * h->N)) return e;
  return SYM_OK;
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace
}  // namespace symb200

using namespace symb200;

extern "C" {

int sym_checkpoint_save(sym_handle* h, const char* path) {
  if (!h || !path) return SYM_ERR_PARAM;
  if (cudaSetDevice(h->device) != cudaSuccess) return set_error(h, SYM_ERR_CUDA, "cudaSetDevice");
  if (cudaStreamSynchronize(h->st) != cudaSuccess) return set_error(h, SYM_ERR_CUDA, "checkpoint: stream");
  const bool fused = h->fast.valid;
  if (!fused)
    if (int e = ensure_canonical_pops(h)) return e;
  Header hd;
  std::memset(&hd, 0, sizeof hd);
  hd.p = h->p;
  hd.fused = fused ? 1 : 0;
  hd.storage = h->fast.storage;
  hd.cur = h->fast.cur;
  hd.pc = h->fast.pc;
  hd.nodes = (int64_t)h->N;
  File out;
  out.f = fopen(path, "wb");
  if (!out.f) return set_error(h, SYM_ERR_PARAM, "checkpoint: cannot open %s for writing", path);
  bool ok = fwrite(kMagic, 1, 8, out.f) == 8 && fwrite(&hd, sizeof hd, 1, out.f) == 1;
  std::vector<char> buf;
  sym_particles sp;
  for (const Section& s : sections(h, fused)) {
    if (!ok) break;
    char name[16] = {0};
    std::strncpy(name, s.name, 15);
    const uint64_t n = s.bytes;
    ok = fwrite(name, 1, 16, out.f) == 16 && fwrite(&n, sizeof n, 1, out.f) == 1;
    const void* src = nullptr;
    if (s.dev) {
      buf.resize(s.bytes);
      if (int e = check_cuda(h, cudaMemcpy(buf.data(), s.dev, s.bytes, cudaMemcpyDeviceToHost), "checkpoint read"))
        return e;
      src = buf.data();
    } else {
      if (int e = check_cuda(h, cudaMemcpy(&sp, h->dpart, sizeof sp, cudaMemcpyDeviceToHost), "checkpoint read"))
        return e;
      src = &sp;
    }
    if (ok) ok = fwrite(src, 1, s.bytes, out.f) == s.bytes;
  }
  if (!ok || fflush(out.f) != 0) return set_error(h, SYM_ERR_PARAM, "checkpoint: write to %s failed", path);
  return SYM_OK;
}

int sym_checkpoint_load(sym_handle* h, const char* path) {
  if (!h || !path) return SYM_ERR_PARAM;
  if (cudaSetDevice(h->device) != cudaSuccess) return set_error(h, SYM_ERR_CUDA, "cudaSetDevice");
  if (cudaStreamSynchronize(h->st) != cudaSuccess) return set_error(h, SYM_ERR_CUDA, "checkpoint: stream");
  File in;
  in.f = fopen(path, "rb");
  if (!in.f) return set_error(h, SYM_ERR_PARAM, "checkpoint: cannot open %s", path);
  char magic[8];
  Header hd;
  if (fread(magic, 1, 8, in.f) != 8 || std::memcmp(magic, kMagic, 8) != 0 || fread(&hd, sizeof hd, 1, in.f) != 1)
    return set_error(h, SYM_ERR_PARAM, "checkpoint: %s is not a checkpoint file", path);
  if (std::memcmp(&hd.p, &h->p, sizeof(sym_params)) != 0 || hd.nodes != (int64_t)h->N)
    return set_error(h, SYM_ERR_PARAM, "checkpoint: written by a handle with other parameters");
  const bool fused = hd.fused != 0;
  if (fused && (hd.storage != h->fast.storage || h->fast.storage < 0 || hd.cur < 0 || hd.cur > 1 || hd.pc < 0 ||
                hd.pc > 1))
    return set_error(h, SYM_ERR_PARAM, "checkpoint: fused state of another storage mode");
  if (fused) {   // the sections name this parity's buffers
    h->fast.cur = hd.cur;
    h->fast.pc = hd.pc;
  } else {
    // canonical state replaces whatever the handle holds
    h->fast.valid = false;
    if (int e = ensure_canonical_pops(h)) return e;
  }
  std::vector<char> buf;
  for (const Section& s : sections(h, fused)) {
    char name[16];
    uint64_t n = 0;
    if (fread(name, 1, 16, in.f) != 16 || fread(&n, sizeof n, 1, in.f) != 1 ||
        std::strncmp(name, s.name, 16) != 0 || n != s.bytes)
      return set_error(h, SYM_ERR_PARAM, "checkpoint: section %s missing or of another size", s.name);
    buf.resize(n);
    if (fread(buf.data(), 1, n, in.f) != n) return set_error(h, SYM_ERR_PARAM, "checkpoint: %s is truncated", path);
    void* dst = s.dev ? s.dev : (void*)h->dpart;
    if (int e = check_cuda(h, cudaMemcpy(dst, buf.data(), n, cudaMemcpyHostToDevice), "checkpoint write")) return e;
  }
  if (fused) {   // the momentum link lists follow from the restored masks
    if (int e = sparse_links_build(h, h->st)) return set_error(h, e, "checkpoint: momentum link lists");
    if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "checkpoint links")) return e;
  }
  h->fast.valid = fused;
  return SYM_OK;
}

}  // extern "C"
