// tma.cuh -- tensor-memory-accelerator (TMA) tile loads of the halo-padded
// node arrays into shared memory, completed on mbarriers.
//
// Only plain tiled loads from this GPU's own memory are issued (no cluster
// multicast).  Every wait on an mbarrier is bounded: after kSpinLimit failed
// polls the waiting thread reports a timeout to its caller, which records it
// in the domain's status word and carries on, so a lost copy can never hang
// the kernel.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace symb200 {
namespace tma {

constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of transactions the copies will complete
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// bounded wait for the phase with the given parity; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = kSpinLimit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3-D tiled load of one box at coordinates (c0 innermost, c1, c2) into
// shared memory, completing on `bar`.  c0 times the element size must be a
// multiple of 16 bytes (the callers pass tile origins that are multiples of 32
// elements).
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// Ask the TMA unit to bring `bytes` of global memory at `src` into L2 (a hint:
// no data arrives in shared memory and nothing waits for it).  src and bytes
// must be multiples of 16.
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Host: encode the map of a halo-padded array (x slowest, z fastest) of
// `nz_ext` x `nyp` x `nxp` elements with row pitch `nzp` elements, read in
// boxes of box_z x box_y x 1.  Elements past nz_ext in a row (the pitch
// padding) read as zeros, like every other element outside the array.
int encode_padded(CUtensorMap* map, void* base, int esize, int nz_ext, int nzp, int nyp, int nxp, int box_z,
                  int box_y);

}  // namespace tma
}  // namespace symb200
