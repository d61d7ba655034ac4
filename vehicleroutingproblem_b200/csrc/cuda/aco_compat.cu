// aco_compat.cu -- the kernel-level interface of the reference
// (include/aco_cuda_kernels.h: 7 kernels, 7 launch_* wrappers) implemented
// with this library's kernels.  The native path is aco_b200.h; these entry
// points let code written against the reference header link unchanged.
#include "aco_internal.cuh"

#include "aco_cuda_kernels.h"

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

using namespace acob200;

namespace {

// Draw stream of the drop-in construct kernel (the 4th Philox counter word).
constexpr uint32_t kCompatStream = 0xC0FAu;

// Weight tables of the drop-in construct kernel, uploaded by
// launch_construct_solutions for the (alpha, beta, log_tau_step) it is given.
struct CompatTables {
  int32_t A[256];
  uint32_t lut[256];
  float thr[kThresholds];
  int ready;
};
__device__ CompatTables g_compat;

// Bits of the nodes 1..n in visited word w (aco_cuda_kernels.cu:105-121).
__device__ __forceinline__ uint64_t relevant_mask(int w, int n) {
  const int lo = w << 6;
  uint64_t mask = ~0ull;
  if (lo == 0) mask &= ~1ull;
  const int valid = n - lo + 1;
  if (valid <= 0) return 0ull;
  if (valid < 64) mask &= (1ull << valid) - 1ull;
  return mask;
}

__device__ __forceinline__ uint32_t evap_word(uint32_t x, uint32_t floor4, uint32_t delta4) {
  return __vsub4(__vmaxu4(x, floor4), delta4);
}

}  // namespace

// ---------------------------------------------------------------------------
// kernel_init_tau / kernel_evaporate_tau: 16-byte vector sweeps (any launch
// shape; bytes before the first 16-byte boundary and after the last one are
// done one at a time).
// ---------------------------------------------------------------------------

ACO_API __global__ void kernel_init_tau(uint8_t *d_tau, uint64_t total_elements, uint8_t q_tau0) {
  const uint64_t head = (uint64_t)((16 - ((uintptr_t)d_tau & 15)) & 15);
  const uint64_t h = head < total_elements ? head : total_elements;
  const uint64_t nvec = (total_elements - h) / 16;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t w = 0x01010101u * q_tau0;
  uint4 *p4 = reinterpret_cast<uint4 *>(d_tau + h);
  for (uint64_t i = tid; i < nvec; i += nthr) p4[i] = make_uint4(w, w, w, w);
  for (uint64_t i = tid; i < h; i += nthr) d_tau[i] = q_tau0;
  for (uint64_t i = h + nvec * 16 + tid; i < total_elements; i += nthr) d_tau[i] = q_tau0;
}

ACO_API __global__ void kernel_evaporate_tau(uint8_t *d_tau, uint64_t total_elements, uint8_t delta,
                                     uint8_t q_min) {
  // q > q_min + delta ? q - delta : q_min == max(q, q_min + delta) - delta
  const int fl = (int)q_min + (int)delta;
  const uint64_t head = (uint64_t)((16 - ((uintptr_t)d_tau & 15)) & 15);
  const uint64_t h = head < total_elements ? head : total_elements;
  const uint64_t nvec = (total_elements - h) / 16;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
  if (fl <= 255) {
    const uint32_t floor4 = 0x01010101u * (uint32_t)fl, delta4 = 0x01010101u * delta;
    uint4 *p4 = reinterpret_cast<uint4 *>(d_tau + h);
    for (uint64_t i = tid; i < nvec; i += nthr) {
      uint4 v = p4[i];
      v.x = evap_word(v.x, floor4, delta4);
      v.y = evap_word(v.y, floor4, delta4);
      v.z = evap_word(v.z, floor4, delta4);
      v.w = evap_word(v.w, floor4, delta4);
      p4[i] = v;
    }
  } else {
    const uint32_t q4 = 0x01010101u * q_min;
    uint4 *p4 = reinterpret_cast<uint4 *>(d_tau + h);
    for (uint64_t i = tid; i < nvec; i += nthr) p4[i] = make_uint4(q4, q4, q4, q4);
  }
  auto one = [&](uint64_t i) {
    const uint8_t q = d_tau[i];
    d_tau[i] = ((int)q > fl) ? (uint8_t)(q - delta) : q_min;
  };
  for (uint64_t i = tid; i < h; i += nthr) one(i);
  for (uint64_t i = h + nvec * 16 + tid; i < total_elements; i += nthr) one(i);
}

// ---------------------------------------------------------------------------
// kernel_build_candidate_lists: warp per node (grid-stride over warps), the
// same k-nearest order as the native kernel, with the reference's outputs:
// int ids and eta^beta = powf(1 / (d + 1e-9), beta) (aco_cuda_kernels.cu:204-213).
// ---------------------------------------------------------------------------

ACO_API __global__ void kernel_build_candidate_lists(const float2 *d_coords, int *d_candidate_idx,
                                             float *d_eta_beta, CudaParams params) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int k = params.cand_k;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i <= params.n; i += warps) {
    const unsigned long long key = warp_knn(d_coords, params.n, k, i, lane);
    if (lane < k) {
      const int node = (key == ~0ull) ? 0 : (int)(key & 0xffffffffu);
      d_candidate_idx[i * k + lane] = node;
      if (node > 0) {
        const float d = sqrtf(__uint_as_float((unsigned)(key >> 32)));
        const float eta = 1.0f / (d + CUDA_EPS);
        d_eta_beta[i * k + lane] = powf(eta, params.beta);
      } else {
        d_eta_beta[i * k + lane] = 0.0f;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// kernel_reset_ant_state: the reference's per-ant initial state
// (aco_cuda_kernels.cu:227-257), thread per ant.
// ---------------------------------------------------------------------------

ACO_API __global__ void kernel_reset_ant_state(int *d_routes, int *d_route_lengths, uint64_t *d_visited_l1,
                                       uint64_t *d_visited_l2, unsigned int *d_rng_states,
                                       CudaAntSummary *d_ant_summary, CudaParams params,
                                       unsigned int seed) {
  for (int ant = blockIdx.x * blockDim.x + threadIdx.x; ant < params.m;
       ant += gridDim.x * blockDim.x) {
    uint64_t *l1 = d_visited_l1 + (size_t)ant * (params.visited_row_stride / 8);
    uint64_t *l2 = d_visited_l2 + (size_t)ant * params.visited_l2_words;
    for (int w = 0; w < params.visited_l1_words; ++w) l1[w] = ~relevant_mask(w, params.n);
    for (int w = 0; w < params.visited_l2_words; ++w) l2[w] = 0ull;
    d_routes[ant] = 0;
    for (int v = 0; v < params.K; ++v) d_route_lengths[ant * params.K + v] = 1;
    d_rng_states[ant] = seed ^ (1664525u * (unsigned int)(ant + 1));
    d_ant_summary[ant].feasible = 0;
    d_ant_summary[ant].unvisited_count = params.n;
    d_ant_summary[ant].cost = 0.0f;
  }
}

// ---------------------------------------------------------------------------
// kernel_construct_solutions: warp per ant (grid-stride over warps) with the
// sequential path's rules and the exact integer roulette, on the reference's
// buffers: step-interleaved routes[step * m + ant] with shared depot steps,
// route lengths counting both depots, 64-bit visited words with the level-2
// summary, per-ant summaries.  Weights are derived per step from the
// pheromone row and the squared candidate distances with the tables of
// launch_construct_solutions.  Draw d of an ant is
// Philox({d/4, ant, 0, 0xC0FA}, {rng_state[ant], 0x5EEDC0DE})[d%4] >> 8.
// Capacity counts customers (the reference's unit demand), so the backward
// repair of the sequential path never has work to do and is not needed.
// ---------------------------------------------------------------------------

__device__ __forceinline__ int compat_level(float d2) {
  int lo = 0, hi = kThresholds;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (g_compat.thr[mid] <= d2) lo = mid + 1; else hi = mid;
  }
  return lo;
}

ACO_API __global__ void kernel_construct_solutions(const float2 *d_coords, const uint8_t *d_tau,
                                           const int *d_candidate_idx, const float *d_eta_beta,
                                           int *d_routes, int *d_route_lengths,
                                           uint64_t *d_visited_l1, uint64_t *d_visited_l2,
                                           unsigned int *d_rng_states,
                                           CudaAntSummary *d_ant_summary,
                                           CudaIterStats *d_iter_stats, CudaParams params) {
  (void)d_eta_beta;
  (void)d_iter_stats;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int n = params.n, K = params.K, m = params.m, k = params.cand_k;
  const int cap = params.cap > 0 ? params.cap : n;
  const size_t stride = (size_t)n + 1;
  if (!g_compat.ready) return;
  for (int ant = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ant < m; ant += warps) {
    uint64_t *l1 = d_visited_l1 + (size_t)ant * (params.visited_row_stride / 8);
    uint64_t *l2 = d_visited_l2 + (size_t)ant * params.visited_l2_words;
    const uint32_t key0 = d_rng_states[ant];
    uint32_t d = 0;
    int remaining = n, step = 0;
    double cost = 0.0;
    for (int v = 0; v < K; ++v) {
      int cur = 0, load = 0, len = 1;
      const long long fut64 = (long long)(K - v - 1) * cap;
      const int future = fut64 > 0x7fffffffLL ? 0x7fffffff : (int)fut64;
      while (remaining > 0 && remaining > future && load < cap) {
        const float2 pc = d_coords[cur];
        int c = 0, e = INT_MIN;
        if (lane < k) {
          c = d_candidate_idx[cur * k + lane];
          if (c > 0)
            e = g_compat.A[d_tau[(size_t)cur * stride + c]] - compat_level(dist2f(pc, d_coords[c]));
        }
        const int emax = __reduce_max_sync(kFull, e);
        uint32_t w = 0u;
        if (c > 0) {
          const int r = emax - e;
          w = g_compat.lut[r > kRelMax ? kRelMax : r];
          if ((l1[c >> 6] >> (c & 63)) & 1ull) w = 0u;
        }
        const uint32_t denom = __reduce_add_sync(kFull, w);
        const uint32_t cum = warp_incl_scan(w, lane);
        int next = 0;
        if (denom != 0u) {
          uint32_t blk[4];
          philox4x32_10(d >> 2, (uint32_t)ant, 0u, kCompatStream, key0, kDrawKey1, blk);
          const uint32_t r = blk[d & 3u] >> (32 - kDrawBits);
          ++d;
          const uint32_t thr =
              (uint32_t)(((unsigned long long)r * denom + 0xFFFFFFull) >> kDrawBits);
          const unsigned msk = __ballot_sync(kFull, w != 0u && cum >= thr);
          next = __shfl_sync(kFull, c, msk ? __ffs(msk) - 1 : 0);
        } else {
          // nearest unvisited node, lowest index on ties
          uint32_t bh = 0xffffffffu, bn = 0xffffffffu;
          for (int wi = lane; wi < params.visited_l1_words; wi += 32) {
            uint64_t fr = ~l1[wi] & relevant_mask(wi, n);
            while (fr) {
              const int b = __ffsll((long long)fr) - 1;
              fr &= fr - 1;
              const int node = (wi << 6) + b;
              const uint32_t h = __float_as_uint(dist2f(pc, d_coords[node]));
              if (h < bh) {
                bh = h;
                bn = (uint32_t)node;
              }
            }
          }
          const uint32_t mh = __reduce_min_sync(kFull, bh);
          const uint32_t mn = __reduce_min_sync(kFull, bh == mh ? bn : 0xffffffffu);
          next = (mh == 0xffffffffu) ? 0 : (int)mn;
        }
        if (next <= 0) break;
        if (lane == 0) {
          ++step;
          d_routes[(size_t)step * m + ant] = next;
          const int wi = next >> 6;
          l1[wi] |= 1ull << (next & 63);
          // The reference's level-2 test, kept as written (aco_cuda_kernels.cu:534).
          if (l1[wi] == ~relevant_mask(wi, n)) l2[wi >> 6] |= 1ull << (wi & 63);
          cost = __dadd_rn(cost, dist64(pc, d_coords[next]));
        }
        __syncwarp();
        ++len;
        ++load;
        --remaining;
        cur = next;
      }
      if (lane == 0) {
        ++step;
        d_routes[(size_t)step * m + ant] = 0;
        cost = __dadd_rn(cost, dist64(d_coords[cur], d_coords[0]));
        d_route_lengths[ant * K + v] = len + 1;
      }
      __syncwarp();
    }
    if (lane == 0) {
      d_ant_summary[ant].feasible = remaining == 0 ? 1 : 0;
      d_ant_summary[ant].unvisited_count = remaining;
      d_ant_summary[ant].cost = (float)cost;
    }
  }
}

// ---------------------------------------------------------------------------
// kernel_deposit_solution / kernel_deposit_flat_solution: the reference's
// per-vehicle walk (any launch shape); the launch_* wrappers use the
// block-parallel deposit instead.  Both give the reference's bytes.
// ---------------------------------------------------------------------------

__device__ __forceinline__ PheromoneView compat_pv(uint8_t *tau, const CudaParams &p) {
  PheromoneView pv;
  pv.tau = tau;
  pv.total = (unsigned long long)(p.n + 1) * (p.n + 1);
  pv.log_min = p.log_tau_min;
  pv.log_step = p.log_tau_step;
  pv.q_min = p.q_tau_min;
  pv.q_max = p.q_tau_max;
  pv.delta = p.q_evap_delta;
  pv.pad = 0;
  return pv;
}

ACO_API __global__ void kernel_deposit_solution(uint8_t *d_tau, const int *d_routes,
                                        const int *d_route_lengths, float deposit_amount,
                                        int best_ant, CudaParams params) {
  const PheromoneView pv = compat_pv(d_tau, params);
  const size_t stride = (size_t)params.n + 1;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < params.K; v += gridDim.x * blockDim.x) {
    int step = 0;
    for (int u = 0; u < v; ++u) step += d_route_lengths[best_ant * params.K + u] - 1;
    const int len = d_route_lengths[best_ant * params.K + v];
    int prev = 0;
    for (int t = 1; t < len; ++t) {
      ++step;
      const int cur = d_routes[(size_t)step * params.m + best_ant];
      deposit_arc(pv, stride, prev, cur, deposit_amount);
      prev = cur;
    }
  }
}

ACO_API __global__ void kernel_deposit_flat_solution(uint8_t *d_tau, const int *d_flat_routes,
                                             const int *d_flat_lengths, float deposit_amount,
                                             CudaParams params) {
  const PheromoneView pv = compat_pv(d_tau, params);
  const size_t stride = (size_t)params.n + 1;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < params.K; v += gridDim.x * blockDim.x) {
    const int len = d_flat_lengths[v];
    const int *r = d_flat_routes + (size_t)v * stride;
    for (int t = 1; t < len; ++t) deposit_arc(pv, stride, r[t - 1], r[t], deposit_amount);
  }
}

namespace {

__global__ void k_compat_deposit_interleaved(uint8_t *tau, const int *routes, const int *lens,
                                             float dep, int best_ant, CudaParams p) {
  extern __shared__ int s_off[];
  const PheromoneView pv = compat_pv(tau, p);
  deposit_solution(pv, (size_t)p.n + 1, InterleavedNodes{routes, p.m, best_ant},
                   lens + (size_t)best_ant * p.K, p.K, dep,
                   p.K <= kDepositSmemRoutes ? s_off : nullptr);
}

__global__ void k_compat_deposit_flat(uint8_t *tau, const int *flat, const int *lens, float dep,
                                      CudaParams p) {
  extern __shared__ int s_off[];
  const PheromoneView pv = compat_pv(tau, p);
  deposit_solution(pv, (size_t)p.n + 1, FlatNodes{flat, p.n + 1}, lens, p.K, dep,
                   p.K <= kDepositSmemRoutes ? s_off : nullptr);
}

int sweep_blocks(unsigned long long bytes) {
  unsigned long long b = (bytes / 16 + 511) / 512;
  if (b < 1) b = 1;
  if (b > 148 * 4) b = 148 * 4;
  return (int)b;
}

// Host copy of the weight tables (same construction as the native set-up).
void compat_tables_host(double alpha, double beta, float log_step, CompatTables *t) {
  const double ln2 = 0.69314718055994530942;
  for (int q = 0; q < 256; ++q)
    t->A[q] = (int32_t)std::floor(alpha * (double)q * (double)log_step * kLevelsPerOctave / ln2 + 0.5);
  for (int r = 0; r < kRelMax; ++r)
    t->lut[r] = (uint32_t)std::floor(8388608.0 * std::exp2(-(double)r / kLevelsPerOctave) + 0.5);
  t->lut[kRelMax] = 0u;
  for (int j = 1; j <= kThresholds; ++j) {
    double v = beta > 0.0 ? std::exp2(2.0 * (double)j / (beta * kLevelsPerOctave)) : INFINITY;
    t->thr[j - 1] = (v > 3.0e38) ? INFINITY : (float)v;
  }
  t->ready = 1;
}

}  // namespace

// ---------------------------------------------------------------------------
// launch_* wrappers (reference: aco_cuda_kernels.cu:678-772): default stream,
// no synchronisation, no return code.
// ---------------------------------------------------------------------------

ACO_API void launch_init_tau(uint8_t *d_tau, int n, uint8_t q_tau0) {
  const unsigned long long total = (unsigned long long)(n + 1) * (n + 1);
  kernel_init_tau<<<sweep_blocks(total), 512>>>(d_tau, total, q_tau0);
}

ACO_API void launch_evaporate_tau(uint8_t *d_tau, int n, uint8_t delta, uint8_t q_min) {
  const unsigned long long total = (unsigned long long)(n + 1) * (n + 1);
  kernel_evaporate_tau<<<sweep_blocks(total), 512>>>(d_tau, total, delta, q_min);
}

ACO_API void launch_build_candidate_lists(const float2 *d_coords, int *d_candidate_idx,
                                  float *d_eta_beta, CudaParams params) {
  int blocks = (params.n + 1 + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  kernel_build_candidate_lists<<<blocks, 256>>>(d_coords, d_candidate_idx, d_eta_beta, params);
}

ACO_API void launch_reset_ant_state(int *d_routes, int *d_route_lengths, uint64_t *d_visited_l1,
                            uint64_t *d_visited_l2, unsigned int *d_rng_states,
                            CudaAntSummary *d_ant_summary, CudaParams params,
                            unsigned int seed) {
  const int blocks = (params.m + 127) / 128;
  kernel_reset_ant_state<<<blocks > 0 ? blocks : 1, 128>>>(
      d_routes, d_route_lengths, d_visited_l1, d_visited_l2, d_rng_states, d_ant_summary, params,
      seed);
}

ACO_API void launch_construct_solutions(const float2 *d_coords, const uint8_t *d_tau,
                                const int *d_candidate_idx, const float *d_eta_beta,
                                int *d_routes, int *d_route_lengths, uint64_t *d_visited_l1,
                                uint64_t *d_visited_l2, unsigned int *d_rng_states,
                                CudaAntSummary *d_ant_summary, CudaIterStats *d_iter_stats,
                                CudaParams params) {
  static float last_alpha = NAN, last_beta = NAN, last_step = NAN;
  if (!(params.alpha == last_alpha && params.beta == last_beta && params.log_tau_step == last_step)) {
    static CompatTables host;
    compat_tables_host(params.alpha, params.beta, params.log_tau_step, &host);
    cudaMemcpyToSymbol(g_compat, &host, sizeof(host));
    last_alpha = params.alpha;
    last_beta = params.beta;
    last_step = params.log_tau_step;
  }
  const int warps_per_block = 4;
  const int blocks = (params.m + warps_per_block - 1) / warps_per_block;
  kernel_construct_solutions<<<blocks > 0 ? blocks : 1, 32 * warps_per_block>>>(
      d_coords, d_tau, d_candidate_idx, d_eta_beta, d_routes, d_route_lengths, d_visited_l1,
      d_visited_l2, d_rng_states, d_ant_summary, d_iter_stats, params);
}

ACO_API void launch_deposit_solution(uint8_t *d_tau, const int *d_routes, const int *d_route_lengths,
                             float deposit_amount, int best_ant, CudaParams params) {
  const size_t smem = params.K <= kDepositSmemRoutes ? sizeof(int) * (params.K + 1) : 0;
  k_compat_deposit_interleaved<<<1, 512, smem>>>(d_tau, d_routes, d_route_lengths,
                                                 deposit_amount, best_ant, params);
}

ACO_API void launch_deposit_flat_solution(uint8_t *d_tau, const int *d_flat_routes,
                                  const int *d_flat_lengths, float deposit_amount,
                                  CudaParams params) {
  const size_t smem = params.K <= kDepositSmemRoutes ? sizeof(int) * (params.K + 1) : 0;
  k_compat_deposit_flat<<<1, 512, smem>>>(d_tau, d_flat_routes, d_flat_lengths, deposit_amount,
                                          params);
}
