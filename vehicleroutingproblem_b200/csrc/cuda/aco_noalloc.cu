// aco_noalloc.cu -- pheromone evaporation + deposit that allocates nothing.
//
// Some callers cannot allocate device memory once they are running: a host
// application that reserves all device memory up front and hands plugins
// only the buffers it owns (a framework with its own caching allocator, a
// solver service with a fixed memory budget), or a real-time loop that must
// not call cudaMalloc/cudaFree because they can synchronise the device and
// can fail under memory pressure.  For them this file offers
// aco_b200_evaporate_deposit_noalloc: the caller passes every input and
// output as a device pointer, and the kernel's scratch (its block ticket and
// the route offsets of the deposit) lives in a fixed file-scope device array
// instead of buffers owned by an aco_b200_ctx.
#include "aco_internal.cuh"

extern "C" {
#include "aco.h"
#include "aco_b200.h"
}

#include <cmath>
#include <cstdio>
#include <mutex>

using namespace acob200;

// Largest number of routes per solution the fixed scratch holds.
constexpr int kNoAllocMaxRoutes = 4096;
// Word 0: block ticket; the route offsets start at word 64 (byte 256).
constexpr int kTicketWords = 64;
constexpr int kScratchWords = kTicketWords + kNoAllocMaxRoutes + 1;

// The scratch of every call on a device (16.6 KB; every GPU that loads the
// library holds it until the process exits).  In host code this name is only
// a host-side handle: the kernel gets the device address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned int g_noalloc_scratch[kScratchWords];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned int *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device; looked up once per
// device (the first call on a device), which is why that first call must
// not be made while a stream is being captured.
cudaError_t scratch_address(unsigned int **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<unsigned int *>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

__global__ void __launch_bounds__(512) k_evap_deposit_noalloc(
    PheromoneView pv, int n, int K, const int *it_nodes, const int *it_lens, float dep_it,
    const int *gb_nodes, const int *gb_lens, float dep_gb, unsigned int *scratch) {
  // Saturating evaporation: max(q, q_min + delta) - delta.
  const int fl = (int)pv.q_min + (int)pv.delta;
  const unsigned long long nvec = pv.total / 16;
  uint4 *p4 = reinterpret_cast<uint4 *>(pv.tau);
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const uint32_t floor4 = 0x01010101u * (uint32_t)(fl > 255 ? 0 : fl);
  const uint32_t delta4 = 0x01010101u * (uint32_t)pv.delta;
  const uint32_t qmin4 = 0x01010101u * (uint32_t)pv.q_min;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < nvec;
       i += stride) {
    uint4 v = p4[i];
    if (fl > 255) {
      v = make_uint4(qmin4, qmin4, qmin4, qmin4);
    } else {
      v.x = __vsub4(__vmaxu4(v.x, floor4), delta4);
      v.y = __vsub4(__vmaxu4(v.y, floor4), delta4);
      v.z = __vsub4(__vmaxu4(v.z, floor4), delta4);
      v.w = __vsub4(__vmaxu4(v.w, floor4), delta4);
    }
    p4[i] = v;
  }
  if (blockIdx.x == 0) {
    for (unsigned long long i = nvec * 16 + threadIdx.x; i < pv.total; i += blockDim.x) {
      const uint8_t q = pv.tau[i];
      pv.tau[i] = ((int)q > fl) ? (uint8_t)(q - pv.delta) : pv.q_min;
    }
  }
  // The last block to finish the sweep deposits, with its route offsets in
  // the scratch array.
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned ticket = atomicAdd(scratch, 1u);
    s_last = (ticket == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int *offsets = reinterpret_cast<int *>(scratch + kTicketWords);
  const size_t stride_n = (size_t)n + 1;
  deposit_solution(pv, stride_n, CompactNodes{it_nodes}, it_lens, K, dep_it, offsets);
  __syncthreads();
  if (gb_nodes) deposit_solution(pv, stride_n, CompactNodes{gb_nodes}, gb_lens, K, dep_gb, offsets);
  if (threadIdx.x == 0) *scratch = 0u;
}

}  // namespace

extern "C" ACO_API int aco_b200_evaporate_deposit_noalloc(
    uint8_t *d_tau, int n, int K, const int *d_iter_nodes, const int *d_iter_lens,
    float dep_iter, const int *d_gbest_nodes, const int *d_gbest_lens, float dep_global,
    double rho, void *stream) {
  if (!d_tau || !d_iter_nodes || !d_iter_lens || n < 1 || K < 1 ||
      (d_gbest_nodes == nullptr) != (d_gbest_lens == nullptr) || !(rho > 0.0 && rho < 1.0)) {
    fprintf(stderr, "aco_b200_evaporate_deposit_noalloc: invalid arguments\n");
    return ACO_ERR_INVALID_INPUT;
  }
  if (((uintptr_t)d_tau & 15u) != 0u) {
    fprintf(stderr, "aco_b200_evaporate_deposit_noalloc: d_tau must be 16-byte aligned\n");
    return ACO_ERR_INVALID_INPUT;
  }
  if (K > kNoAllocMaxRoutes) {
    fprintf(stderr,
            "aco_b200_evaporate_deposit_noalloc: K=%d routes exceed the fixed scratch "
            "(at most %d routes per solution)\n",
            K, kNoAllocMaxRoutes);
    return ACO_ERR_INVALID_INPUT;
  }
  unsigned int *scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_evaporate_deposit_noalloc: scratch address: %s\n",
            cudaGetErrorString(e));
    return ACO_ERR_BACKEND;
  }
  // Quantization constants of the reference (src/cuda/aco_cuda.cu:209-215).
  const float lmin = logf(0.0001f);
  const float lmax = logf(100.0f);
  const float step = (lmax - lmin) / 255.0f;
  const float log_rho = logf(1.0f - (float)rho);
  PheromoneView pv;
  pv.tau = d_tau;
  pv.total = (unsigned long long)(n + 1) * (unsigned long long)(n + 1);
  pv.log_min = lmin;
  pv.log_step = step;
  pv.q_min = 0;
  pv.q_max = 255;
  pv.delta = (uint8_t)fmaxf(1.0f, roundf(-log_rho / step));
  pv.pad = 0;
  cudaStream_t s = (cudaStream_t)stream;
  // The ticket must start at zero; the previous call's contents stay in the
  // array otherwise.
  e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_evaporate_deposit_noalloc: %s\n", cudaGetErrorString(e));
    return ACO_ERR_BACKEND;
  }
  unsigned long long blocks = (pv.total / 16 + 511) / 512;
  if (blocks < 1) blocks = 1;
  if (blocks > 148ull * 4) blocks = 148ull * 4;
  k_evap_deposit_noalloc<<<(unsigned)blocks, 512, 0, s>>>(pv, n, K, d_iter_nodes, d_iter_lens,
                                                          dep_iter, d_gbest_nodes, d_gbest_lens,
                                                          dep_global, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_evaporate_deposit_noalloc: launch: %s\n", cudaGetErrorString(e));
    return ACO_ERR_BACKEND;
  }
  return ACO_OK;
}
