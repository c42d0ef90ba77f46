// server.cu -- continuous-batching job server over the batch engine.
//
// No counterpart in the reference, which runs one job per process.  The
// request loop (sym_server_tick) is, per round:
//   admit    at multiples of check_every server steps only, first come first
//            served while the job's footprint fits the byte budget and a slot
//            is free: create the handle, set walls and particles, build the
//            initial state on the device, import it into the fused state and
//            take the step-0 stop-rule reading;
//   rebuild  the batch of every storage mode whose membership changed;
//   run      every batch for n steps (to the next check, the nearest step
//            limit or the caller's cap) on its own stream, so batches of
//            different storage overlap on the device;
//   check    each job at a check step: per-z red area of its phase field
//            (fast_neck_planes) copied to pinned host memory, r_eq(z) =
//            sqrt(area/pi), min over z; breakup when it falls below the
//            job's stop radius (step interpolated between the last two
//            checks), failure when it is not finite;
//   retire   finished and failed jobs: results kept, device state freed.
// Because admission and checks fall on multiples of check_every since a
// job's own start, and a batch step equals a single-domain step bit for bit,
// a job's result does not depend on what runs beside it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>
#include "state.cuh"

using namespace symb200;

namespace {

struct Job {
  int64_t id = 0;
  sym_job_spec spec{};
  sym_handle* h = nullptr;
  size_t foot = 0;
  sym_job_result r{};
  // The phase field a check reads is the one the last step computed from
  // the populations it started from: after k steps it describes the state
  // after k-1 steps (the step-0 reading describes the initial state).
  int s_prev = -1;        // state step described by the previous check
  double r_prev = 0.0;    // min r_eq at the previous check
  int slot = -1;          // row of the pinned plane-sum buffer
  bool checking = false;  // a reading was enqueued this round
  double vol0 = 0.0;      // red-phase volume at admission (failure detection)
};

double stop_radius(const sym_job_spec& s) { return s.stop_radius > 0 ? s.stop_radius : 1.0; }

int size_class(int nx) { return nx <= 32 ? 0 : (nx <= 48 ? 1 : 2); }

}  // namespace

struct sym_server {
  int device = 0;
  size_t budget = 0;
  int slots = 0;
  int check_every = 10;
  long long gstep = 0;          // server steps run so far
  int64_t next_id = 1;
  std::deque<int64_t> pending;
  std::vector<int64_t> running;
  std::map<int64_t, Job> jobs;
  size_t resident = 0;
  sym_batch* batch[3] = {nullptr, nullptr, nullptr};   // one per storage mode
  bool dirty[3] = {false, false, false};
  int xchunk[3] = {32, 32, 32};
  // pinned host rows for the per-plane reductions, one row per slot
  double* hplanes = nullptr;
  int row_len = 0;
  int32_t* hflags = nullptr;    // pinned: each slot's device error flags at its last check
  std::vector<int> free_rows;
  cudaEvent_t ev[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  double node_updates = 0.0;
  double device_ms = 0.0;
  int done = 0, failed = 0;
  std::chrono::steady_clock::time_point t0;
  std::string err;
};

namespace {

int serr(sym_server* s, int code, const std::string& msg) {
  s->err = msg;
  return code;
}

double now(const sym_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

void finish(sym_server* s, Job& j, int status, int error) {
  j.r.status = status;
  j.r.error = error;
  j.r.t_done = now(s);
  if (status == SYM_JOB_FAILED) s->failed++;
  else s->done++;
}

void release(sym_server* s, Job& j) {
  if (j.h) {
    s->dirty[j.spec.p.storage] = true;
    sym_destroy(j.h);
    j.h = nullptr;
    s->resident -= j.foot;
  }
  if (j.slot >= 0) {
    s->free_rows.push_back(j.slot);
    j.slot = -1;
  }
}

// grow the pinned rows to `len` doubles (only between rounds: nothing in flight)
int ensure_rows(sym_server* s, int len) {
  if (!s->hflags) {
    if (cudaMallocHost(&s->hflags, sizeof(int32_t) * (size_t)s->slots) != cudaSuccess) {
      (void)cudaGetLastError();
      s->hflags = nullptr;
      return serr(s, SYM_ERR_OOM, "pinned host flags");
    }
  }
  if (len <= s->row_len && s->hplanes) return SYM_OK;
  const int nl = std::max(len, s->row_len);
  double* p = nullptr;
  if (cudaMallocHost(&p, sizeof(double) * (size_t)nl * s->slots) != cudaSuccess) {
    (void)cudaGetLastError();
    return serr(s, SYM_ERR_OOM, "pinned host rows");
  }
  if (s->hplanes) cudaFreeHost(s->hplanes);
  s->hplanes = p;
  s->row_len = nl;
  return SYM_OK;
}

// red-phase volume: the sum of the per-plane red areas of a job's pinned row
double vol_of(const sym_server* s, const Job& j) {
  const double* a = s->hplanes + (size_t)j.slot * s->row_len;
  double v = 0.0;
  for (int z = 0; z < j.spec.p.nz; z++) v += a[z];
  return v;
}

// min over z of sqrt(area/pi) from a job's pinned row
double rmin_of(const sym_server* s, const Job& j) {
  const double* a = s->hplanes + (size_t)j.slot * s->row_len;
  double m = INFINITY;
  for (int z = 0; z < j.spec.p.nz; z++) {
    const double r = std::sqrt(a[z] / M_PI);
    if (!(r == r)) return NAN;
    m = std::min(m, r);
  }
  return m;
}

// synchronous step-0 reading of an admitted job
int first_reading(sym_server* s, Job& j) {
  sym_handle* h = j.h;
  if (int e = fast_neck_planes(h, h->red, h->st)) return e;
  double* row = s->hplanes + (size_t)j.slot * s->row_len;
  cudaMemcpyAsync(row, h->red, sizeof(double) * j.spec.p.nz, cudaMemcpyDeviceToHost, h->st);
  if (int e = check_cuda(h, cudaStreamSynchronize(h->st), "first reading")) return e;
  j.r_prev = rmin_of(s, j);
  j.s_prev = 0;
  j.r.rmin = j.r_prev;
  j.vol0 = vol_of(s, j);
  return SYM_OK;
}

// create and initialise a job's device state; SYM_ERR_OOM leaves it pending
int start_job(sym_server* s, Job& j) {
  const sym_job_spec& sp = j.spec;
  sym_handle* h = nullptr;
  if (int e = sym_create(&sp.p, s->device, &h)) return e;
  j.h = h;
  int e = SYM_OK;
  if (sp.p.par > 0) {
    sym_particles pa;
    std::memset(&pa, 0, sizeof pa);
    const int par = sp.p.par;
    for (int k = 0; k < 3; k++) {
      pa.center[k * par] = sp.center[k];
      pa.center0[k * par] = sp.center[k];
      pa.up[k * par] = sp.up[k];
    }
    e = sym_set_particles(h, &pa);
  }
  if (!e) e = sym_set_walls(h);
  if (!e) {
    const double* g = sp.gen;
    e = sp.kind == SYM_JOB_THREAD ? sym_init_thread(h, g[0], g[1], g[2], g[3], g[4], sp.seed)
                                  : sym_init_slab(h, g[0], g[1], g[2], g[3], sp.seed);
  }
  if (!e) e = sym_derivatives(h);
  if (!e) e = fast_import(h);
  if (!e) h->fast.valid = true;
  if (!e) e = first_reading(s, j);
  if (e) s->err = h->err;
  return e;
}

void admit(sym_server* s) {
  while (!s->pending.empty() && (int)s->running.size() < s->slots) {
    Job& j = s->jobs[s->pending.front()];
    if (s->resident + j.foot > s->budget) {
      if (!s->running.empty()) break;   // wait for room
      s->pending.pop_front();           // can never fit
      finish(s, j, SYM_JOB_FAILED, SYM_ERR_OOM);
      continue;
    }
    if (ensure_rows(s, j.spec.p.nz)) break;
    j.slot = s->free_rows.back();
    s->free_rows.pop_back();
    j.r.t_admit = now(s);
    s->resident += j.foot;
    j.h = nullptr;
    const int e = start_job(s, j);
    if (e == SYM_ERR_OOM && !s->running.empty()) {   // device fuller than the budget says: retry later
      if (j.h) { sym_destroy(j.h); j.h = nullptr; }
      s->resident -= j.foot;
      s->free_rows.push_back(j.slot);
      j.slot = -1;
      j.r.t_admit = -1.0;
      break;
    }
    s->pending.pop_front();
    if (e) {
      s->resident -= j.foot;
      if (j.h) { sym_destroy(j.h); j.h = nullptr; }
      s->free_rows.push_back(j.slot);
      j.slot = -1;
      finish(s, j, SYM_JOB_FAILED, e);
      continue;
    }
    j.r.status = SYM_JOB_RUNNING;
    s->running.push_back(j.id);
    s->dirty[j.spec.p.storage] = true;
  }
}

int rebuild(sym_server* s) {
  for (int m = 0; m < 3; m++) {
    if (!s->dirty[m]) continue;
    s->dirty[m] = false;
    if (s->batch[m]) {
      sym_batch_destroy(s->batch[m]);
      s->batch[m] = nullptr;
    }
    std::vector<sym_handle*> hs;
    for (int64_t id : s->running) {
      Job& j = s->jobs[id];
      if (j.h && j.spec.p.storage == m) hs.push_back(j.h);
    }
    if (hs.empty()) continue;
    if (int e = sym_batch_create(hs.data(), (int)hs.size(), &s->batch[m]))
      return serr(s, e, "batch create failed");
    for (size_t i = 0; i < hs.size(); i++)
      sym_batch_set_xchunk(s->batch[m], (int)i, s->xchunk[size_class(hs[i]->dp.nx)]);
  }
  return SYM_OK;
}

}  // namespace

extern "C" {

int sym_server_create(int device, size_t budget_bytes, int slots, int check_every, sym_server** out) {
  if (!out || slots <= 0 || budget_bytes == 0) return SYM_ERR_PARAM;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return SYM_ERR_CUDA;
  sym_server* s = new sym_server();
  s->device = device;
  s->budget = budget_bytes;
  s->slots = slots;
  s->check_every = check_every > 0 ? check_every : 10;
  s->t0 = std::chrono::steady_clock::now();
  for (int r = slots - 1; r >= 0; r--) s->free_rows.push_back(r);
  for (int m = 0; m < 3; m++)
    for (int k = 0; k < 2; k++)
      if (cudaEventCreate(&s->ev[m][k]) != cudaSuccess) {
        sym_server_destroy(s);
        return SYM_ERR_CUDA;
      }
  *out = s;
  return SYM_OK;
}

int sym_server_destroy(sym_server* s) {
  if (!s) return SYM_OK;
  cudaSetDevice(s->device);
  for (int m = 0; m < 3; m++)
    if (s->batch[m]) sym_batch_destroy(s->batch[m]);
  for (auto& kv : s->jobs)
    if (kv.second.h) sym_destroy(kv.second.h);
  if (s->hplanes) cudaFreeHost(s->hplanes);
  if (s->hflags) cudaFreeHost(s->hflags);
  for (int m = 0; m < 3; m++)
    for (int k = 0; k < 2; k++)
      if (s->ev[m][k]) cudaEventDestroy(s->ev[m][k]);
  delete s;
  return SYM_OK;
}

const char* sym_server_last_error(const sym_server* s) { return s ? s->err.c_str() : "null server"; }

int sym_server_submit(sym_server* s, const sym_job_spec* spec, int64_t* id) {
  if (!s || !spec) return SYM_ERR_PARAM;
  char msg[256];
  if (spec->p.mode != SYM_MODE_CONFIG) return serr(s, SYM_ERR_PARAM, "jobs are CONFIG-mode domains");
  if (sym_params_check(&spec->p, msg, sizeof msg)) return serr(s, SYM_ERR_PARAM, msg);
  if (spec->p.storage < 0 || spec->p.storage > 2) return serr(s, SYM_ERR_PARAM, "bad storage");
  if (spec->p.par > 1) return serr(s, SYM_ERR_UNSUPPORTED, "jobs carry at most one particle");
  if (spec->max_steps <= 0) return serr(s, SYM_ERR_PARAM, "max_steps must be > 0");
  if (spec->kind != SYM_JOB_THREAD && spec->kind != SYM_JOB_SLAB) return serr(s, SYM_ERR_PARAM, "bad job kind");
  Job j;
  j.id = s->next_id++;
  j.spec = *spec;
  if (int e = sym_footprint(&spec->p, &j.foot)) return serr(s, e, "footprint");
  j.r.status = SYM_JOB_PENDING;
  j.r.breakup_step = -1.0;
  j.r.rmin = NAN;
  j.r.t_arrival = spec->t_arrival >= 0 ? spec->t_arrival : now(s);
  j.r.t_admit = -1.0;
  j.r.t_done = -1.0;
  s->jobs[j.id] = j;
  s->pending.push_back(j.id);
  if (id) *id = j.id;
  return SYM_OK;
}

int sym_server_tick(sym_server* s, int max_steps, int* running, int* pending) {
  if (!s) return SYM_ERR_PARAM;
  cudaSetDevice(s->device);
  const int C = s->check_every;
  if (s->gstep % C == 0) admit(s);
  if (int e = rebuild(s)) return e;
  if (!s->running.empty()) {
    // steps to the next event of any running job
    long long n = C - s->gstep % C;
    if (max_steps > 0) n = std::min<long long>(n, max_steps);
    for (int64_t id : s->running) {
      const Job& j = s->jobs[id];
      n = std::min<long long>(n, (long long)j.spec.max_steps - j.r.steps);
    }
    n = std::max<long long>(n, 1);
    for (int m = 0; m < 3; m++) {
      if (!s->batch[m]) continue;
      cudaStream_t st = batch_stream(s->batch[m]);
      cudaEventRecord(s->ev[m][0], st);
      if (int e = batch_launch(s->batch[m], (int)n))
        return serr(s, e, std::string("batch step: ") + sym_batch_last_error(s->batch[m]));
      cudaEventRecord(s->ev[m][1], st);
    }
    s->gstep += n;
    for (int64_t id : s->running) {
      Job& j = s->jobs[id];
      j.r.steps += (int)n;
      j.r.node_updates += (int64_t)n * (int64_t)j.h->N;
      s->node_updates += (double)n * (double)j.h->N;
      j.checking = (j.r.steps % C == 0) || j.r.steps >= j.spec.max_steps;
      if (!j.checking) continue;
      cudaStream_t st = batch_stream(s->batch[j.spec.p.storage]);
      if (int e = fast_neck_planes(j.h, j.h->red, st)) return serr(s, e, j.h->err);
      cudaMemcpyAsync(s->hplanes + (size_t)j.slot * s->row_len, j.h->red, sizeof(double) * j.spec.p.nz,
                      cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(s->hflags + j.slot, j.h->fast.status, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    }
    for (int m = 0; m < 3; m++) {
      if (!s->batch[m]) continue;
      const cudaError_t e = cudaStreamSynchronize(batch_stream(s->batch[m]));
      if (e != cudaSuccess) return serr(s, SYM_ERR_CUDA, std::string("server round: ") + cudaGetErrorString(e));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, s->ev[m][0], s->ev[m][1]);
      s->device_ms += ms;
    }
    // stop rule and retirement
    std::vector<int64_t> keep;
    for (int64_t id : s->running) {
      Job& j = s->jobs[id];
      bool end = false;
      if (j.checking) {
        const double r = rmin_of(s, j);
        j.r.rmin = r;
        const double thr = stop_radius(j.spec);
        const double dv = j.vol0 > 0.0 ? std::fabs(vol_of(s, j) - j.vol0) / j.vol0 : 0.0;
        const int32_t flags = s->hflags[j.slot];
        if (flags & SYM_DEV_TIMEOUT) {
          finish(s, j, SYM_JOB_FAILED, SYM_ERR_TIMEOUT);
          end = true;
        } else if (!(r == r) || (flags & SYM_DEV_NONFINITE)) {
          finish(s, j, SYM_JOB_FAILED, SYM_ERR_NAN);
          end = true;
        } else if (j.spec.drift_tol > 0.0 && dv > j.spec.drift_tol) {
          finish(s, j, SYM_JOB_FAILED, SYM_ERR_DRIFT);
          end = true;
        } else if (j.spec.wall_budget_s > 0.0 && now(s) - j.r.t_admit > j.spec.wall_budget_s) {
          finish(s, j, SYM_JOB_FAILED, SYM_ERR_TIMEOUT);
          end = true;
        } else if (r < thr) {
          const double f = (j.r_prev > r) ? (j.r_prev - thr) / (j.r_prev - r) : 1.0;
          j.r.breakup_step = j.s_prev + std::min(1.0, std::max(0.0, f)) * (double)(j.r.steps - 1 - j.s_prev);
          finish(s, j, SYM_JOB_BREAKUP, SYM_OK);
          end = true;
        } else if (j.r.steps >= j.spec.max_steps) {
          finish(s, j, SYM_JOB_LIMIT, SYM_OK);
          end = true;
        } else {
          j.r_prev = r;
          j.s_prev = j.r.steps - 1;
        }
      }
      if (end) release(s, j);
      else keep.push_back(id);
    }
    s->running.swap(keep);
  }
  if (running) *running = (int)s->running.size();
  if (pending) *pending = (int)s->pending.size();
  return SYM_OK;
}

int sym_server_result(sym_server* s, int64_t id, sym_job_result* out) {
  if (!s || !out) return SYM_ERR_PARAM;
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return serr(s, SYM_ERR_NOTFOUND, "unknown job id");
  *out = it->second.r;
  return SYM_OK;
}

int sym_server_set_xchunk(sym_server* s, int size_class, int xchunk) {
  if (!s || size_class < 0 || size_class > 2 || xchunk < 1) return SYM_ERR_PARAM;
  s->xchunk[size_class] = xchunk;
  for (int m = 0; m < 3; m++) s->dirty[m] = s->dirty[m] || s->batch[m] != nullptr;
  return SYM_OK;
}

int sym_server_stats(sym_server* s, double out[8]) {
  if (!s || !out) return SYM_ERR_PARAM;
  out[0] = s->node_updates;
  out[1] = s->device_ms;
  out[2] = s->done;
  out[3] = s->failed;
  out[4] = (double)s->running.size();
  out[5] = (double)s->pending.size();
  out[6] = (double)s->resident;
  out[7] = now(s);
  return SYM_OK;
}

}  // extern "C"
