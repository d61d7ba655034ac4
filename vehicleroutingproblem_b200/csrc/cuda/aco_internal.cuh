// aco_internal.cuh -- structures shared by the host solver and the kernels,
// and the device helpers of the B200 ACO-for-CVRP hot path.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace acob200 {

// ---------------------------------------------------------------------------
// Integer selection weights.  A candidate t of row i gets the level
//   e = A[q] - L,  A[q] = round(alpha q step G / ln 2),  L = #{T_j <= d^2}
// with G = 16 levels per octave, and the weight
//   w = LUT[min(emax_i - e, 255)],  LUT[r] = round(2^23 2^(-r/G)), LUT[255] = 0
// where emax_i is the largest level of the row.  w < 2^24, a row of at most
// 32 weights sums below 2^29, and a 24-bit draw r times that sum is below
// 2^53: the roulette below is exact in integers and in the FP64 arithmetic
// of the reference's select_next_customer (src/seq/aco_sequential.c:505-561).
// ---------------------------------------------------------------------------
constexpr int kLevelsPerOctave = 16;
constexpr int kRelMax = 255;
constexpr int kThresholds = 4095;
constexpr int kMaxCand = 32;
constexpr int kDrawBits = 24;
constexpr uint32_t kDrawKey1 = 0x5EEDC0DEu;
constexpr unsigned kFull = 0xffffffffu;

// Stop-rule bits (DevState::stop_flags).
constexpr int kStopStagnation = 1;
constexpr int kStopFixed = 2;
constexpr int kStopTimeout = 4;
constexpr int kStopRunLimit = 8;

// Depot rules of the construction (InstanceView::depot_rule).
constexpr int kDepotRuleSeq = 0;      // src/seq/aco_sequential.c:616-681
constexpr int kDepotRuleCudaRef = 1;  // stochastic close, aco_cuda_kernels.cu:487-520

// Device error bits (DevState::error).
constexpr int kErrStageTimeout = 1;

// Construct table layouts.
constexpr int kLayoutSmemWeights = 0;  // cand u16 + w u32 staged in smem
constexpr int kLayoutSmemPacked = 1;   // cand u16 + rel u8 + LUT in smem
constexpr int kLayoutGlobal = 2;       // rows read from global memory (L2)

struct EpochRec {
  int epoch;
  int iter_since_best;
  int improved;
  int found;
  double global_best;
  unsigned long long elapsed_ns;
};

constexpr int kLogCap = 1024;

// Run state of one solve, resident on the device.  The epoch loop of the
// reference (src/cuda/aco_cuda.cu:331-429) keeps these on the host; here the
// kernels update them so that whole epochs run without host round trips.
struct DevState {
  int stop_flags;          // kStop* bits; nonzero: the next epoch is skipped
  int skip;                // this epoch is skipped (set by the weights kernel)
  int epoch;               // epochs completed
  int iter_since_best;
  int found;               // this epoch had a feasible ant
  int improved;            // this epoch improved the global best
  int best_ant;
  int error;
  double global_best;
  double iter_best;
  float dep_iter;
  float dep_global;
  unsigned long long total_steps;
  unsigned long long start_ns;
  // configuration
  int stagnation;
  int fixed_epochs;
  int run_limit;
  int log_count;
  double min_rel;
  unsigned long long timeout_ns;
  float Qs;                // Q * 100 (src/cuda/aco_cuda.cu:228)
  uint32_t seed;           // draw seed of the graph-launched epochs
  int tau_sel;             // current pheromone buffer (0: tau, 1: tau_alt)
  int pad1;
};

// Current pheromone buffer.  The graph-launched epochs keep two: while the
// ants are built the evaporated matrix is written into the other buffer,
// the deposits go there, and the buffers switch (only when an iteration
// best exists, as the reference evaporates only then).
__device__ __forceinline__ uint8_t *cur_tau(uint8_t *tau, uint8_t *tau_alt, const DevState *st) {
  return (tau_alt && st && *(volatile const int *)&st->tau_sel) ? tau_alt : tau;
}

// Byte offsets of the construct kernel's dynamic shared memory.
struct SmemPlan {
  uint32_t off_cand, off_w, off_coords, off_dem, off_lut, off_draw, off_vis;
  uint32_t bytes_cand, bytes_w, bytes_coords, bytes_dem;
  uint32_t total;
  int vis_words;           // 32-bit words per ant bitmap
  int vreg;                // bitmap words per lane held in registers (0: smem)
  int wpb;                 // warps (ants) per block
  int layout;
  uint32_t off_route;      // route_smem: each ant's route (route_stride ints) in shared memory
  int route_smem;
};

struct InstanceView {
  int n, K, k, m;
  long long cap;
  long long total_demand;
  int unit;                // 1: every customer has demand 1
  int max_demand;          // largest customer demand
  int route_stride;        // n + 2K
  int ant_base;            // global id of local ant 0 (colony split over devices)
  int depot_rule;          // kDepotRuleSeq or kDepotRuleCudaRef
  int stage_extra_tx;      // test hook: bytes the staging wait expects beyond the copies
  const float2 *coords;    // [n+1]
  const int *demand;       // [n+1]
  const uint16_t *cand;    // [(n+1) k]
  const uint16_t *lvl;     // [(n+1) k]
  // Neighbours of ranks k+1 .. k+64 of every node in the candidates' order
  // ([(n+1) kTierLen], 0 = none), or null: the nearest-customer fallback
  // looks there before it scans every node.
  const uint16_t *tier;
  // Ranks k+65 .. k+64+kTier2Len ([(n+1) kTier2Len], 0 = none), or null:
  // looked at after the tier lists, before the scan (large instances).
  const uint16_t *tier2;
};

constexpr int kTierLen = 64;
// Smallest instance whose construction uses the tier lists.
constexpr int kTierMinCustomers = 512;
constexpr int kTier2Len = 192;
// Smallest instance whose construction uses the second tier lists.
constexpr int kTier2MinCustomers = 1500;

struct AntBuffers {
  int *routes;             // [m][n + 2K] compact routes
  int *lens;               // [m][K]
  double *cost;            // [m]
  int *feasible;           // [m]
  int *steps;              // [m]
  uint32_t *draws;         // [m]
  int *loads;              // [m][K]  per-vehicle load (repair scratch)
  int *rep;                // [m][n]  repair additions (scratch)
  int *repc;               // [m][K]  repair additions per vehicle (scratch)
};

struct EpochTables {
  uint32_t *w;             // [(n+1) k] weights
  uint8_t *rel;            // [(n+1) k] weight levels below the row maximum
  const int32_t *A;        // [256]
  const uint32_t *lut;     // [256]
  // Reference-CUDA depot rule only (else null): per row, the depot-close
  // weight's level below the row maximum, rdep[i] = emax_i - (e_dep - lvl0[i]).
  int32_t *rdep;           // [(n+1)]
  const uint16_t *lvl0;    // [(n+1)] eta level of d(i,0)^2
  int e_dep;               // level of the depot factor 2 / tau_min^alpha
  uint8_t *tau_alt;        // second pheromone buffer (pipelined epochs), or null
};

struct PheromoneView {
  uint8_t *tau;            // [(n+1)^2], row stride n+1
  unsigned long long total;
  float log_min, log_step;
  uint8_t q_min, q_max, delta, pad;
};

// ---------------------------------------------------------------------------
// Launch wrappers (aco_kernels.cu).
// ---------------------------------------------------------------------------
cudaError_t launch_knn_levels(const float2 *coords, int n, int k,
                              const float *thr, int J, uint16_t *cand,
                              uint16_t *lvl, cudaStream_t s);
cudaError_t launch_knn_tier(const float2 *coords, int n, int k, uint16_t *tier, uint16_t *tier2,
                            cudaStream_t s);
cudaError_t launch_knn_tier_multi(const float2 *coords, const long long *seg_off,
                                  const int *seg_n, int count, long long rows, int k,
                                  uint16_t *tier, cudaStream_t s);
// Candidate lists of `count` instances packed one after another: instance s
// has seg_n[s] customers and starts at row seg_off[s] (device arrays).
cudaError_t launch_knn_levels_multi(const float2 *coords, const long long *seg_off,
                                    const int *seg_n, int count, long long rows, int k,
                                    const float *thr, int J, uint16_t *cand, uint16_t *lvl,
                                    cudaStream_t s);
cudaError_t launch_fill_u8(uint8_t *p, unsigned long long count, uint8_t v,
                           cudaStream_t s);
cudaError_t launch_weights(const InstanceView &iv, const PheromoneView &pv,
                           const EpochTables &et, DevState *st, cudaStream_t s);
cudaError_t launch_construct(const InstanceView &iv, const EpochTables &et,
                             const AntBuffers &ab, const SmemPlan &plan,
                             DevState *st, uint32_t seed, uint32_t epoch,
                             uint32_t stream_id, int use_state_epoch,
                             cudaStream_t s, const uint32_t *draw_src = nullptr,
                             uint32_t draw_per_ant = 0);
cudaError_t launch_best(const InstanceView &iv, const AntBuffers &ab,
                        DevState *st, int *gbest_nodes, int *gbest_lens,
                        EpochRec *log, cudaStream_t s);
cudaError_t launch_evap_deposit(const InstanceView &iv, const PheromoneView &pv,
                                const AntBuffers &ab, DevState *st,
                                const int *gbest_nodes, const int *gbest_lens,
                                unsigned int *counter, int grid, uint8_t *tau_alt,
                                cudaStream_t s);
cudaError_t launch_set_run_limit(DevState *st, int limit, cudaStream_t s);
int evap_grid_for(unsigned long long total, int num_sms);
cudaError_t launch_evaporate_to(const PheromoneView &pv, uint8_t *tau_alt, DevState *st,
                                int grid, cudaStream_t s);
cudaError_t launch_best_deposit(const InstanceView &iv, const AntBuffers &ab,
                                const PheromoneView &pv, uint8_t *tau_alt, DevState *st,
                                int *gbest_nodes, int *gbest_lens, EpochRec *log,
                                cudaStream_t s);
cudaError_t launch_depot_levels(const float2 *coords, int n, const float *thr, int J,
                                uint16_t *lvl0, cudaStream_t s);
int shard_packet_size(int n, int K);
cudaError_t launch_shard_pack(const InstanceView &iv, const AntBuffers &ab, DevState *st,
                              int *send, cudaStream_t s);
cudaError_t launch_shard_select(const InstanceView &iv, DevState *st, const int *recv,
                                int world, int *iter_nodes, int *iter_lens,
                                int *gbest_nodes, int *gbest_lens, EpochRec *log,
                                const PheromoneView &pv, uint8_t *tau_alt, cudaStream_t s);
int construct_max_smem();
cudaError_t prepare_construct_kernels();
SmemPlan plan_construct(const InstanceView &iv, int layout, int num_sms,
                        int max_smem);

}  // namespace acob200

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
namespace acob200 {

// Philox4x32-10 (Salmon et al., SC'11).
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1,
                                              uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1,
                                              uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Squared distance in float without contraction: exact for integer
// coordinates whose differences are below 2896.
__device__ __forceinline__ float dist2f(float2 a, float2 b) {
  float dx = __fsub_rn(a.x, b.x);
  float dy = __fsub_rn(a.y, b.y);
  return __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
}

// FP64 Euclidean distance, rounded as sqrt(dx*dx + dy*dy) in double.
__device__ __forceinline__ double dist64(float2 a, float2 b) {
  double dx = __dsub_rn((double)a.x, (double)b.x);
  double dy = __dsub_rn((double)a.y, (double)b.y);
  return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// 1-D bulk copy global -> shared (TMA engine), completing on an mbarrier.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Marks `bytes` of the barrier's expected transaction count as arrived
// without a copy (used to balance an expectation no copy will meet).
__device__ __forceinline__ void mbar_complete_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after max_polls polls (returns false).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar,
                                                  uint32_t parity,
                                                  uint32_t max_polls) {
  for (uint32_t i = 0; i < max_polls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  return false;
}

__device__ __forceinline__ uint8_t ld_cg_u8(const uint8_t *p) {
  unsigned short v;
  asm volatile("ld.global.cg.u8 %0, [%1];" : "=h"(v) : "l"(p));
  return (uint8_t)v;
}

__device__ __forceinline__ void st_cg_u8(uint8_t *p, uint8_t v) {
  unsigned short w = v;
  asm volatile("st.global.cg.u8 [%0], %1;" ::"l"(p), "h"(w) : "memory");
}

// Warp-wide k-nearest selection for node i: the k smallest keys
// (d^2 bits << 32 | j) over j in 1..n, j != i.  Lane t < k ends holding the
// t-th smallest (~0 when fewer than k exist).  Keys are unique, so the order
// is total: ascending d^2, ties to the lower j, as the reference's insertion
// with a strict '<' (aco_cuda_kernels.cu:187-201).
// With `after` given (not ~0), the k smallest keys greater than it: the
// next ranks of the same order.
__device__ inline unsigned long long warp_knn(const float2 *coords, int n, int k,
                                       int i, int lane,
                                       unsigned long long after = ~0ull) {
  const unsigned long long kNone = ~0ull;
  unsigned long long list = kNone;
  unsigned long long kth = kNone;
  const float2 pi = coords[i];
  for (int base = 1; base <= n; base += 32) {
    int j = base + lane;
    unsigned long long key = kNone;
    if (j <= n && j != i) {
      float d2 = dist2f(pi, __ldg(coords + j));
      key = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)j;
      if (after != kNone && key <= after) key = kNone;
    }
    unsigned m = __ballot_sync(kFull, key < kth);
    while (m) {
      int b = __ffs(m) - 1;
      m &= m - 1;
      unsigned long long x = __shfl_sync(kFull, key, b);
      if (x < kth) {
        int pos = __popc(__ballot_sync(kFull, lane < k && list < x));
        unsigned long long up = __shfl_up_sync(kFull, list, 1);
        if (lane > pos) list = up;
        else if (lane == pos) list = x;
        kth = __shfl_sync(kFull, list, k - 1);
      }
    }
  }
  return list;
}

// ---------------------------------------------------------------------------
// Pheromone deposit (shared by the native kernels and the drop-in kernels)
// ---------------------------------------------------------------------------
// Route layouts a deposit can read: node t of route v, whose first node is
// entry off_v of the compact sequence (K segments [0 .. 0] back to back).
struct CompactNodes {  // compact sequence (this library's layout)
  const int *p;
  __device__ __forceinline__ int operator()(int v, int off_v, int t) const {
    return p[off_v + t];
  }
};
struct InterleavedNodes {  // reference: routes[step * m + ant], shared depots
  const int *p;
  int m, ant;
  __device__ __forceinline__ int operator()(int v, int off_v, int t) const {
    return p[(size_t)(off_v - v + t) * m + ant];
  }
};
struct FlatNodes {  // reference global-best buffer: flat[v * (n+1) + t]
  const int *p;
  int stride;
  __device__ __forceinline__ int operator()(int v, int off_v, int t) const {
    return p[(size_t)v * stride + t];
  }
};

// quantize_tau / dequantize_tau of the reference (aco_cuda_kernels.cu:25-45),
// the same expressions so that the device math rounds identically.
__device__ __forceinline__ float dequant(uint8_t q, float log_min, float log_step) {
  return expf((float)q * log_step + log_min);
}

__device__ __forceinline__ uint8_t quant(float tau, float log_min,
                                         float log_step, uint8_t q_min,
                                         uint8_t q_max) {
  if (tau <= 0.0f) return q_min;
  float log_t = logf(tau);
  float q_f = (log_t - log_min) / log_step;
  if (q_f <= (float)q_min) return q_min;
  if (q_f >= (float)q_max) return q_max;
  return (uint8_t)roundf(q_f);
}

// One arc (u, c): new = quantize(dequantize(tau[u][c]) + dep), max-ed into
// tau[u][c] and tau[c][u] (aco_cuda_kernels.cu:614-623).  The caller
// guarantees that no other thread touches these two cells concurrently.
__device__ __forceinline__ void deposit_arc(const PheromoneView &pv,
                                            size_t stride, int u, int c,
                                            float dep) {
  uint8_t *fwd = pv.tau + (size_t)u * stride + c;
  uint8_t *rev = pv.tau + (size_t)c * stride + u;
  const uint8_t old = ld_cg_u8(fwd);
  const uint8_t nq = quant(dequant(old, pv.log_min, pv.log_step) + dep,
                           pv.log_min, pv.log_step, pv.q_min, pv.q_max);
  if (nq > old) st_cg_u8(fwd, nq);
  const uint8_t oldr = ld_cg_u8(rev);
  if (nq > oldr) st_cg_u8(rev, nq);
}

// Deposit of one solution by one block.  Arcs of different routes touch
// different cells, except the depot loop (0,0) of empty routes; inside a
// route of >= 4 nodes all 2(len-1) cells are distinct too.  So: route
// offsets are scanned into shared memory; the arcs of routes of >= 4 nodes
// are dealt over all threads, each thread loading all its cells before it
// stores any; a one-customer route [0 a 0] (whose two arcs share the cells
// {0,a}) is walked by one thread in order, and all empty routes by thread 0
// in vehicle order.  s_off holds K+1 ints, or is null for very large K
// (then every thread walks the length list).
template <class Nodes>
__device__ void deposit_solution(const PheromoneView &pv, size_t stride,
                                 const Nodes &nodes, const int *lens, int K,
                                 float dep, int *s_off, int gtid = 0, int gthreads = 0) {
  // Arcs are shared out over gthreads threads (this thread is gtid) when
  // several blocks deposit one solution, else over the block.
  const int bd = gthreads > 0 ? gthreads : (int)blockDim.x;
  const int tid = gthreads > 0 ? gtid : (int)threadIdx.x;
  const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5;
  if (!s_off) {
    int off = 0, base = 0;
    for (int v = 0; v < K; ++v) {
      const int len = lens[v];
      const int owner = base % bd;
      if (len >= 4) {
        for (int t = (tid - owner + bd) % bd; t < len - 1; t += bd)
          deposit_arc(pv, stride, nodes(v, off, t), nodes(v, off, t + 1), dep);
      } else if (len == 3 && tid == owner) {
        deposit_arc(pv, stride, nodes(v, off, 0), nodes(v, off, 1), dep);
        deposit_arc(pv, stride, nodes(v, off, 1), nodes(v, off, 2), dep);
      } else if (len == 2 && tid == 0) {
        deposit_arc(pv, stride, nodes(v, off, 0), nodes(v, off, 1), dep);
      }
      off += len;
      base += len > 1 ? len - 1 : 0;
    }
    return;
  }
  if (warp == 0) {
    int carry = 0;
    for (int b = 0; b < K; b += 32) {
      const int v = b + lane;
      const int len = v < K ? lens[v] : 0;
      const int inc = (int)warp_incl_scan((uint32_t)len, lane);
      if (v < K) s_off[v + 1] = carry + inc;
      carry += __shfl_sync(kFull, inc, 31);
    }
    if (lane == 0) s_off[0] = 0;
  }
  __syncthreads();
  const int total = s_off[K];
  constexpr int kBatch = 4;
  for (int j0 = tid; j0 < total; j0 += kBatch * bd) {
    int us[kBatch], cs[kBatch];
    bool valid[kBatch];
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      const int j = j0 + q * bd;
      valid[q] = false;
      us[q] = cs[q] = 0;
      if (j < total) {
        int lo = 0, hi = K;  // route v with s_off[v] <= j < s_off[v+1]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= j) lo = mid; else hi = mid;
        }
        const int off = s_off[lo], len = s_off[lo + 1] - off;
        if (len >= 4 && j > off) {
          valid[q] = true;
          us[q] = nodes(lo, off, j - off - 1);
          cs[q] = nodes(lo, off, j - off);
        }
      }
    }
    uint8_t fq[kBatch], rq[kBatch];
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      fq[q] = rq[q] = 0;
      if (valid[q]) {
        fq[q] = ld_cg_u8(pv.tau + (size_t)us[q] * stride + cs[q]);
        rq[q] = ld_cg_u8(pv.tau + (size_t)cs[q] * stride + us[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      if (valid[q]) {
        const uint8_t nq = quant(dequant(fq[q], pv.log_min, pv.log_step) + dep, pv.log_min,
                                 pv.log_step, pv.q_min, pv.q_max);
        if (nq > fq[q]) st_cg_u8(pv.tau + (size_t)us[q] * stride + cs[q], nq);
        if (nq > rq[q]) st_cg_u8(pv.tau + (size_t)cs[q] * stride + us[q], nq);
      }
    }
  }
  for (int v = tid; v < K; v += bd) {
    const int off = s_off[v];
    if (s_off[v + 1] - off == 3) {
      deposit_arc(pv, stride, nodes(v, off, 0), nodes(v, off, 1), dep);
      deposit_arc(pv, stride, nodes(v, off, 1), nodes(v, off, 2), dep);
    }
  }
  if (tid == 0) {
    for (int v = 0; v < K; ++v)
      if (s_off[v + 1] - s_off[v] == 2) deposit_arc(pv, stride, 0, 0, dep);
  }
}

constexpr int kDepositSmemRoutes = 4096;

}  // namespace acob200
#endif
