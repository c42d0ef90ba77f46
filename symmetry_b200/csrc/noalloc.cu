// noalloc.cu -- FP64 mass and momentum sums for callers that cannot allocate
// device memory.
//
// sym_mass_momentum (capi.cu) reduces into scratch that sym_create allocated.
// Some callers never create a handle and may not call cudaMalloc at all: a
// serving loop that reserved its whole device budget up front and must not
// allocate mid-run (an allocation can fail under fragmentation or stall the
// device), or a host program whose own memory manager owns every device byte.
// This entry point does the same reduction with its scratch in a fixed array
// that is part of the loaded library, so it allocates nothing.
#include <cstdio>
#include <mutex>
#include "state.cuh"

namespace {

constexpr long long kNodesPerBlock = 256;
// At most 65,536 blocks of 256 nodes: domains of up to 16,777,216 nodes.
constexpr long long kMaxBlocks = 65536;
constexpr long long kMaxNodes = kMaxBlocks * kNodesPerBlock;

// Per-block partial sums, 5 per block (2.6 MB).  Every GPU that loads the
// library holds this array until the process exits.  Each call overwrites
// every partial it later reads, so nothing has to start at zero; calls that
// overlap on the GPU share the array and race.
static __device__ __align__(256) double g_scratch[kMaxBlocks * 5];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Same per-node arithmetic and the same reduction tree as the handle-based
// kernels, so both entry points return identical sums for identical data.
__global__ void k_partials(const double* __restrict__ ri, const double* __restrict__ bi,
                           const int32_t* __restrict__ walls_all, long long N, double* part) {
  __shared__ double sh[256];
  const long long L = blockIdx.x * kNodesPerBlock + threadIdx.x;
  double v[5] = {0, 0, 0, 0, 0};
  if (L < N && (walls_all == nullptr || walls_all[L] <= 0)) {
#pragma unroll
    for (int i = 0; i < 19; i++) {
      const double r = ri[i * N + L], b = bi[i * N + L], f = r + b;
      v[0] += r; v[1] += b;
      v[2] += f * symb200::CX(i); v[3] += f * symb200::CY(i); v[4] += f * symb200::CZ(i);
    }
  }
  for (int k = 0; k < 5; k++) {
    const double s = block_sum<256>(v[k], sh);
    if (threadIdx.x == 0) part[blockIdx.x * 5LL + k] = s;
  }
}

__global__ void k_final(const double* part, long long nblk, double* out) {
  __shared__ double sh[256];
  for (int k = 0; k < 5; k++) {
    double s = 0.0;
    for (long long b = threadIdx.x; b < nblk; b += 256) s += part[b * 5 + k];
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) out[k] = s;
  }
}

int fail(char* msg, size_t len, int code, const char* text) {
  if (msg && len) snprintf(msg, len, "%s", text);
  return code;
}

}  // namespace

extern "C" int sym_mass_momentum_noalloc(const double* ri, const double* bi, const int32_t* walls_all,
                                         int64_t n_nodes, double* out, void* stream, char* msg,
                                         size_t msg_len) {
  if (n_nodes <= 0 || n_nodes > kMaxNodes) {
    char text[160];
    snprintf(text, sizeof text, "n_nodes = %lld is outside 1..%lld (the fixed scratch holds %lld block sums)",
             (long long)n_nodes, kMaxNodes, kMaxBlocks);
    return fail(msg, msg_len, SYM_ERR_PARAM, text);
  }
  if (!ri || !bi || !out) return fail(msg, msg_len, SYM_ERR_PARAM, "ri, bi and out must be device pointers");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(msg, msg_len, SYM_ERR_CUDA, "no current CUDA device");
  double* scratch = nullptr;
  {
    // first call on a device: look up the device address of the scratch array
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) return fail(msg, msg_len, SYM_ERR_CUDA, cudaGetErrorString(e));
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long nblk = (n_nodes + kNodesPerBlock - 1) / kNodesPerBlock;
  k_partials<<<(unsigned)nblk, 256, 0, st>>>(ri, bi, walls_all, n_nodes, scratch);
  k_final<<<1, 256, 0, st>>>(scratch, nblk, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(msg, msg_len, SYM_ERR_CUDA, cudaGetErrorString(e));
  return SYM_OK;
}
