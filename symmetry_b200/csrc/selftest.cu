// selftest.cu -- the timeout path of the bounded mbarrier wait, run on purpose.
//
// The collide kernels wait on mbarriers for their TMA tile loads.  A copy that
// never completes must not hang the kernel: the wait gives up after a bounded
// number of polls and the kernel records the timeout in its status word.
// This entry point exercises exactly that path without any lost copy: one
// thread waits on a barrier that nothing ever arrives on (its phase can never
// complete), with a caller-chosen poll limit, and reports the status word the
// collide kernels would have written, plus the time the wait took.  A second
// barrier that does complete checks the success path.  Nothing faults, traps
// or spins without a limit.
#include <cstdio>
#include "tma.cuh"
#include "../../include/symmetry.h"

namespace {

using namespace symb200;

__global__ void k_wait_timeout(int polls, int* status) {
  __shared__ alignas(8) uint64_t bar[2];
  if (threadIdx.x == 0) {
    tma::mbar_init(&bar[0], 1);  // never arrived on
    tma::mbar_init(&bar[1], 1);  // arrived on once below: phase 0 completes
    tma::mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  int st = 0;
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma::smem_addr(&bar[1])) : "memory");
  if (!tma::mbar_wait(&bar[1], 0u, polls)) st |= 4;  // must not happen
  if (!tma::mbar_wait(&bar[0], 0u, polls)) st |= 2;  // the status bit of a lost tile load
  *status = st;
}

}  // namespace

extern "C" int sym_selftest_wait_timeout(int device, int polls, int32_t* status, double* ms, char* msg,
                                         size_t msg_len) {
  auto fail = [&](int rc, const char* what, cudaError_t e) {
    if (msg && msg_len) snprintf(msg, msg_len, "%s: %s", what, e == cudaSuccess ? "" : cudaGetErrorString(e));
    return rc;
  };
  if (!status || !ms || polls < 1) return fail(SYM_ERR_PARAM, "status, ms and polls >= 1 are required", cudaSuccess);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(SYM_ERR_CUDA, "cudaSetDevice", e);
  int* d_st = nullptr;
  if ((e = cudaMalloc(&d_st, sizeof(int))) != cudaSuccess) return fail(SYM_ERR_CUDA, "cudaMalloc", e);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, 0);
  k_wait_timeout<<<1, 32>>>(polls, d_st);
  cudaEventRecord(b, 0);
  e = cudaEventSynchronize(b);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  int st = -1;
  if (e == cudaSuccess) e = cudaMemcpy(&st, d_st, sizeof(int), cudaMemcpyDeviceToHost);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d_st);
  if (e != cudaSuccess) return fail(SYM_ERR_CUDA, "wait self-test", e);
  *status = st;
  *ms = t;
  return SYM_OK;
}
