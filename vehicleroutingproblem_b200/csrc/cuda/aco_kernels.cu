// aco_kernels.cu -- sm_100a kernels of the ACO-for-CVRP hot path.
//
//   k_knn_levels      candidate lists + eta levels, warp per node
//                     (reference: kernel_build_candidate_lists,
//                      src/cuda/aco_cuda_kernels.cu:164-214)
//   k_weights         per-epoch integer weights from the quantized pheromone
//                     (role of seq_shared_update_scores,
//                      src/seq/aco_sequential.c:410-442)
//   k_construct       warp-per-ant route construction with the sequential
//                     path's rules (src/seq/aco_sequential.c:477-681) over
//                     candidate tables staged in shared memory by the TMA
//                     engine (reference kernel: aco_cuda_kernels.cu:447-562)
//   k_best_cluster    iteration best, global best, stop rules and both
//                     deposits of the pipelined epoch over a cluster of 8
//                     blocks; k_best the same without the deposits, on the
//                     device (src/cuda/aco_cuda.cu:83-126, :331-399)
//   k_evap_deposit    128-bit streaming evaporation, then the deposit of the
//                     iteration best and global best by the last block
//                     (aco_cuda_kernels.cu:145-155, :569-668)
#include "aco_internal.cuh"

#include <cooperative_groups.h>

#include <cfloat>
#include <climits>

namespace acob200 {

// ===========================================================================
// Candidate lists and eta levels
// ===========================================================================

__device__ __forceinline__ int level_of(float d2, const float *thr, int J) {
  int lo = 0, hi = J;  // number of thresholds <= d2
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(thr + mid) <= d2) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_knn_levels(
    const float2 *__restrict__ coords, int n, int k,
    const float *__restrict__ thr, int J, uint16_t *__restrict__ cand,
    uint16_t *__restrict__ lvl) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i <= n;
       i += warps) {
    unsigned long long key = warp_knn(coords, n, k, i, lane);
    if (lane < k) {
      int node = (key == ~0ull) ? 0 : (int)(key & 0xffffffffu);
      float d2 = __uint_as_float((unsigned)(key >> 32));
      cand[(size_t)i * k + lane] = (uint16_t)node;
      lvl[(size_t)i * k + lane] = (uint16_t)(node ? level_of(d2, thr, J) : 0);
    }
  }
}

cudaError_t launch_knn_levels(const float2 *coords, int n, int k,
                              const float *thr, int J, uint16_t *cand,
                              uint16_t *lvl, cudaStream_t s) {
  int rows = n + 1;
  int blocks = (rows + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_knn_levels<<<blocks, 256, 0, s>>>(coords, n, k, thr, J, cand, lvl);
  return cudaGetLastError();
}

// Neighbours of ranks k+1 .. k+64 of every node i (warp per node), the ranks
// right after its k candidates: the 32 keys after the candidate list's last,
// then the 32 after those, in the candidates' order (ascending d^2 bits, then
// node).  0 marks an empty slot; an empty last slot means the candidates and
// this row hold every other customer.
__global__ void __launch_bounds__(256) k_knn_tier(const float2 *__restrict__ coords, int n,
                                                  int k, uint16_t *__restrict__ tier,
                                                  uint16_t *__restrict__ tier2) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const unsigned long long kNone = ~0ull;
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i <= n; i += warps) {
    unsigned long long key = warp_knn(coords, n, k, i, lane);
    int last_lane = k - 1;
    uint16_t *row = tier + (size_t)i * kTierLen;
#pragma unroll
    for (int r = 0; r < kTierLen / 32; ++r) {
      const unsigned long long last = __shfl_sync(kFull, key, last_lane);
      key = (last == kNone) ? kNone : warp_knn(coords, n, 32, i, lane, last);
      last_lane = 31;
      row[32 * r + lane] = (uint16_t)(key == kNone ? 0u : (unsigned)(key & 0xffffffffu));
    }
    if (!tier2) continue;
    // The second tier: the next kTier2Len ranks, 32 per pass as above.
    uint16_t *row2 = tier2 + (size_t)i * kTier2Len;
#pragma unroll 1
    for (int r = 0; r < kTier2Len / 32; ++r) {
      const unsigned long long last = __shfl_sync(kFull, key, 31);
      key = (last == kNone) ? kNone : warp_knn(coords, n, 32, i, lane, last);
      row2[32 * r + lane] = (uint16_t)(key == kNone ? 0u : (unsigned)(key & 0xffffffffu));
    }
  }
}

cudaError_t launch_knn_tier(const float2 *coords, int n, int k, uint16_t *tier, uint16_t *tier2,
                            cudaStream_t s) {
  if (k < 1 || k > kMaxCand) return cudaErrorInvalidValue;
  int blocks = (n + 1 + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_knn_tier<<<blocks, 256, 0, s>>>(coords, n, k, tier, tier2);
  return cudaGetLastError();
}

// Tier lists of many instances in one launch (rows as k_knn_levels_multi):
// row r of instance s holds what k_knn_tier gives that instance alone.
__global__ void __launch_bounds__(256) k_knn_tier_multi(
    const float2 *__restrict__ coords, const long long *__restrict__ seg_off,
    const int *__restrict__ seg_n, int count, long long rows, int k,
    uint16_t *__restrict__ tier) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const unsigned long long kNone = ~0ull;
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
       r += warps) {
    int lo = 0, hi = count;  // last s with seg_off[s] <= r
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(seg_off + mid) <= r) lo = mid; else hi = mid;
    }
    const long long off = __ldg(seg_off + lo);
    const int n = __ldg(seg_n + lo);
    const int i = (int)(r - off);
    if (i > n) continue;
    unsigned long long key = warp_knn(coords + off, n, k, i, lane);
    int last_lane = k - 1;
    uint16_t *row = tier + (size_t)r * kTierLen;
#pragma unroll
    for (int q = 0; q < kTierLen / 32; ++q) {
      const unsigned long long last = __shfl_sync(kFull, key, last_lane);
      key = (last == kNone) ? kNone : warp_knn(coords + off, n, 32, i, lane, last);
      last_lane = 31;
      row[32 * q + lane] = (uint16_t)(key == kNone ? 0u : (unsigned)(key & 0xffffffffu));
    }
  }
}

cudaError_t launch_knn_tier_multi(const float2 *coords, const long long *seg_off,
                                  const int *seg_n, int count, long long rows, int k,
                                  uint16_t *tier, cudaStream_t s) {
  if (count < 1 || rows < 1 || k < 1 || k > kMaxCand) return cudaErrorInvalidValue;
  long long blocks = (rows + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_knn_tier_multi<<<(int)blocks, 256, 0, s>>>(coords, seg_off, seg_n, count, rows, k, tier);
  return cudaGetLastError();
}

// Candidate lists of many instances in one launch.  Instance s owns rows
// [seg_off[s], seg_off[s] + seg_n[s] + 1) of the concatenated coordinates
// (seg_off ascending); each warp finds its row's instance by binary search and
// writes the same lists as k_knn_levels on that instance alone.
__global__ void __launch_bounds__(256) k_knn_levels_multi(
    const float2 *__restrict__ coords, const long long *__restrict__ seg_off,
    const int *__restrict__ seg_n, int count, long long rows, int k,
    const float *__restrict__ thr, int J, uint16_t *__restrict__ cand,
    uint16_t *__restrict__ lvl) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
       r += warps) {
    int lo = 0, hi = count;  // last s with seg_off[s] <= r
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(seg_off + mid) <= r) lo = mid; else hi = mid;
    }
    const long long off = __ldg(seg_off + lo);
    const int n = __ldg(seg_n + lo);
    const int i = (int)(r - off);
    if (i > n) continue;  // gap rows (none when the segments are packed)
    const unsigned long long key = warp_knn(coords + off, n, k, i, lane);
    if (lane < k) {
      const int node = (key == ~0ull) ? 0 : (int)(key & 0xffffffffu);
      const float d2 = __uint_as_float((unsigned)(key >> 32));
      cand[(size_t)r * k + lane] = (uint16_t)node;
      lvl[(size_t)r * k + lane] = (uint16_t)(node ? level_of(d2, thr, J) : 0);
    }
  }
}

cudaError_t launch_knn_levels_multi(const float2 *coords, const long long *seg_off,
                                    const int *seg_n, int count, long long rows, int k,
                                    const float *thr, int J, uint16_t *cand, uint16_t *lvl,
                                    cudaStream_t s) {
  if (count < 1 || rows < 1) return cudaErrorInvalidValue;
  long long blocks = (rows + 7) / 8;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_knn_levels_multi<<<(int)blocks, 256, 0, s>>>(coords, seg_off, seg_n, count, rows, k, thr, J,
                                                 cand, lvl);
  return cudaGetLastError();
}

// eta level of d(i,0)^2 for every node (reference-CUDA depot rule).
__global__ void k_depot_levels(const float2 *__restrict__ coords, int n,
                               const float *__restrict__ thr, int J, uint16_t *lvl0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  lvl0[i] = (uint16_t)level_of(dist2f(coords[i], coords[0]), thr, J);
}

cudaError_t launch_depot_levels(const float2 *coords, int n, const float *thr, int J,
                                uint16_t *lvl0, cudaStream_t s) {
  k_depot_levels<<<(n + 1 + 255) / 256, 256, 0, s>>>(coords, n, thr, J, lvl0);
  return cudaGetLastError();
}

// ===========================================================================
// Byte fill (pheromone initialisation, kernel_init_tau :131-136)
// ===========================================================================

__global__ void k_fill_u8(uint8_t *p, unsigned long long count, uint8_t v) {
  const unsigned long long nvec = count / 16;
  const uint32_t w = 0x01010101u * v;
  const uint4 vv = make_uint4(w, w, w, w);
  uint4 *p4 = reinterpret_cast<uint4 *>(p);
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
       i < nvec; i += stride)
    p4[i] = vv;
  if (blockIdx.x == 0) {
    for (unsigned long long i = nvec * 16 + threadIdx.x; i < count; i += blockDim.x) p[i] = v;
  }
}

cudaError_t launch_fill_u8(uint8_t *p, unsigned long long count, uint8_t v,
                           cudaStream_t s) {
  unsigned long long nvec = count / 16;
  unsigned long long blocks = (nvec + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_fill_u8<<<(unsigned)blocks, 256, 0, s>>>(p, count, v);
  return cudaGetLastError();
}

// ===========================================================================
// Per-epoch weights
// ===========================================================================

__global__ void __launch_bounds__(256) k_weights(InstanceView iv,
                                                 PheromoneView pv,
                                                 EpochTables et,
                                                 DevState *st) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int k = iv.k;
  const size_t stride = (size_t)iv.n + 1;
  // This warp's first row's candidates and levels, the buffer selector and
  // the stop flag are all requested before any of them is used, so that
  // their round trips overlap.
  const int i0 = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int c0 = 0, l0 = 0;
  if (i0 <= iv.n && lane < k) {
    c0 = iv.cand[(size_t)i0 * k + lane];
    l0 = iv.lvl[(size_t)i0 * k + lane];
  }
  const uint8_t *tau = cur_tau(pv.tau, et.tau_alt, st);
  if (st) {
    int stop = *(volatile int *)&st->stop_flags;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->skip = stop ? 1 : 0;
      if (!stop && st->start_ns == 0ull) st->start_ns = global_timer_ns();
    }
    if (stop) return;
  }
  for (int i = i0; i <= iv.n; i += warps) {
    int c = 0;
    int e = INT_MIN;
    if (lane < k) {
      int lv;
      if (i == i0) {
        c = c0;
        lv = l0;
      } else {
        c = iv.cand[(size_t)i * k + lane];
        lv = iv.lvl[(size_t)i * k + lane];
      }
      if (c > 0) {
        uint8_t q = tau[(size_t)i * stride + c];
        e = __ldg(et.A + q) - lv;
      }
    }
    int emax = __reduce_max_sync(kFull, e);
    if (et.rdep && lane == 0)
      et.rdep[i] = (emax == INT_MIN) ? 0 : emax - (et.e_dep - (int)et.lvl0[i]);
    if (lane < k) {
      uint32_t w = 0u;
      uint8_t rel = (uint8_t)kRelMax;
      if (c > 0) {
        int r = emax - e;
        if (r > kRelMax) r = kRelMax;
        rel = (uint8_t)r;
        w = __ldg(et.lut + r);
      }
      et.w[(size_t)i * k + lane] = w;
      et.rel[(size_t)i * k + lane] = rel;
    }
  }
}

cudaError_t launch_weights(const InstanceView &iv, const PheromoneView &pv,
                           const EpochTables &et, DevState *st,
                           cudaStream_t s) {
  int rows = iv.n + 1;
  int blocks = (rows + 7) / 8;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_weights<<<blocks, 256, 0, s>>>(iv, pv, et, st);
  return cudaGetLastError();
}

// ===========================================================================
// Construction
// ===========================================================================

// Draws of one ant, 128 at a time in a per-warp shared buffer: draw d is
// word d%4 of Philox({d/4, ant, epoch, stream}, {seed, kDrawKey1}) >> 8;
// lane L computes block 32 b + L of batch b and stores its 4 words.
__device__ __forceinline__ void draw_refill(uint32_t *buf, uint32_t d,
                                            uint32_t seed, uint32_t epoch,
                                            uint32_t ant, uint32_t stream,
                                            int lane) {
  uint32_t r[4];
  philox4x32_10(((d >> 7) << 5) + (uint32_t)lane, ant, epoch, stream, seed,
                kDrawKey1, r);
  __syncwarp();
  uint4 v = make_uint4(r[0] >> (32 - kDrawBits), r[1] >> (32 - kDrawBits),
                       r[2] >> (32 - kDrawBits), r[3] >> (32 - kDrawBits));
  reinterpret_cast<uint4 *>(buf)[lane] = v;
  __syncwarp();
}

template <int L, bool UNIT>
struct Tables {
  const uint16_t *tier;  // global, or null
  const uint16_t *tier2;  // global, or null
  const uint16_t *cand;
  const uint32_t *w;
  const uint8_t *rel;
  const uint32_t *lut;
  const float2 *coords;
  const int *dem;

  __device__ __forceinline__ uint32_t weight(int idx) const {
    if (L == kLayoutSmemPacked) return lut[rel[idx]];
    return w[idx];
  }
  __device__ __forceinline__ float2 coord(int node) const {
    if (L == kLayoutGlobal) return __ldg(coords + node);
    return coords[node];
  }
  __device__ __forceinline__ int demand(int node) const {
    if (UNIT) return 1;
    if (L == kLayoutGlobal) return __ldg(dem + node);
    return dem[node];
  }
};

// Visited set of one ant.  V = 1 or 2 (n < 2048): registers, transposed so
// that lane L holds nodes L, L + 32, L + 64, ... (and from 1024 on in a
// second word): the nodes of any instance spread evenly over the lanes,
// which keeps the nearest-customer scan short on small instances.  V = 0:
// the bitmap is in shared memory, word wi holding nodes 32 wi .. 32 wi + 31.
// The depot and the bits past node n start set.  test/set are collective.
__device__ __forceinline__ uint32_t vis_init_word(int wi, int n) {
  uint32_t word = 0u;
  const int lo = wi << 5;
  if (lo == 0) word |= 1u;
  const int valid = n + 1 - lo;  // nodes lo..n in this word
  if (valid < 32) word |= (valid <= 0) ? 0xffffffffu : (0xffffffffu << valid);
  return word;
}

template <int V>
struct Visited {
  uint32_t w0, w1;
  uint32_t *s;
  int vw;

  __device__ __forceinline__ void init(uint32_t *smem_words, int vw_, int n,
                                       int lane) {
    vw = vw_;
    s = smem_words;
    w0 = w1 = 0xffffffffu;
    // Registers hold the bitmap transposed: bit b of lane L's w0 is node
    // L + 32 b, of its w1 node 1024 + L + 32 b.
    if (V >= 1) w0 = lane_word(lane, n) | (lane == 0 ? 1u : 0u);
    if (V == 2) w1 = lane_word(1024 + lane, n);
    if (V == 0) {
      for (int wi = lane; wi < vw; wi += 32) s[wi] = vis_init_word(wi, n);
      __syncwarp();
    }
  }
  // Nodes first + 32 b (b = 0..31) that are beyond n: their bits start set.
  __device__ __forceinline__ static uint32_t lane_word(int first, int n) {
    const int cnt = n >= first ? (n - first) / 32 + 1 : 0;  // nodes <= n
    return cnt >= 32 ? 0u : (0xffffffffu << cnt);
  }
  __device__ __forceinline__ bool test(int c) const {
    if (V == 0) {
      const uint32_t word = s[c >> 5];
      return (__funnelshift_r(word, word, c) & 1u) != 0u;  // bit c mod 32
    }
    // Lane c mod 32 holds node c (the shuffle takes the source modulo 32),
    // at bit (c / 32) mod 32.
    const uint32_t bit = __funnelshift_l(0u, 1u, c >> 5);  // formed while the shuffle flies
    uint32_t word = __shfl_sync(kFull, w0, c);
    if (V == 2) {
      const uint32_t hi = __shfl_sync(kFull, w1, c);
      word = (c >> 10) ? hi : word;
    }
    return (word & bit) != 0u;
  }
  __device__ __forceinline__ void set(int node, int lane) {
    if (V == 0) {
      const uint32_t bit = __funnelshift_l(0u, 1u, node);  // 1 << (node mod 32)
      if (lane == 0) s[node >> 5] |= bit;
      __syncwarp();
    } else {
      const uint32_t bit = __funnelshift_l(0u, 1u, node >> 5);  // 1 << ((node / 32) mod 32)
      const bool mine = lane == (node & 31);
      if (V == 2 && (node >> 10)) w1 |= mine ? bit : 0u;
      else w0 |= mine ? bit : 0u;
    }
  }
};

// The full scan over a register bitmap of two words per lane (V = 2, the
// transposed layout of Visited<2>: bit b of word j is node 1024 j + lane +
// 32 b), in ascending node order, 8 unvisited nodes at a time with their
// coordinate (and demand) loads issued together; the lane's best node (its
// squared distance's bits in *best_h_out).  Out of line, as scan_words.
// (With one word per lane the plain loop is as fast and shorter.)
template <int L, bool UNIT, int V>
__device__ __noinline__ uint32_t scan_regs(const float2 *coords, const int *dem, uint32_t w0,
                                           uint32_t w1, float2 pc, int room, bool check_dem,
                                           int lane, uint32_t *best_h_out) {
  uint32_t best_h = 0xffffffffu, best_n = 0xffffffffu;
  constexpr int kB = 8;
  int j = 0;
  uint32_t fr = ~w0;
  while (true) {
    int nd[kB];
#pragma unroll
    for (int q = 0; q < kB; ++q) {
      if (V == 2 && fr == 0u && j == 0) { fr = ~w1; j = 1; }
      nd[q] = -1;
      if (fr) {
        nd[q] = 1024 * j + lane + 32 * (__ffs(fr) - 1);
        fr &= fr - 1;
      }
    }
    float2 pq[kB];
    int dq[kB];
#pragma unroll
    for (int q = 0; q < kB; ++q) {
      pq[q] = make_float2(0.f, 0.f);
      dq[q] = 0;
      if (nd[q] >= 0) {
        pq[q] = L == kLayoutGlobal ? __ldg(coords + nd[q]) : coords[nd[q]];
        if (!UNIT && check_dem) dq[q] = L == kLayoutGlobal ? __ldg(dem + nd[q]) : dem[nd[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < kB; ++q) {
      if (nd[q] < 0 || (!UNIT && check_dem && dq[q] > room)) continue;
      const uint32_t h = __float_as_uint(dist2f(pc, pq[q]));
      if (h < best_h) {
        best_h = h;
        best_n = (uint32_t)nd[q];
      }
    }
    if (nd[kB - 1] < 0) break;
  }
  *best_h_out = best_h;
  return best_n;
}

// The full scan over a bitmap in shared memory (word wi holds nodes 32 wi ..
// 32 wi + 31): lane L walks words L, L + 32, ... in ascending node order.
// Its unvisited nodes are taken kScanBatch at a time and their coordinate
// (and demand) loads issued together, so a lane waits once per batch rather
// than once per node; they are still compared in ascending order, so the
// lane's first nearest node wins.  Returns the lane's best node (its
// squared distance's bits in *best_h_out).  Out of line: the batch's
// registers do not weigh on the step loop that calls it (the scan is rare).
template <int L, bool UNIT>
__device__ __noinline__ uint32_t scan_words(const float2 *coords, const int *dem,
                                            const uint32_t *s, int vw, float2 pc, int room,
                                            bool check_dem, int lane, uint32_t *best_h_out) {
  uint32_t best_h = 0xffffffffu, best_n = 0xffffffffu;
  auto visit = [&](int node, float2 p, int dm) {
    if (!UNIT && check_dem && dm > room) return;
    const uint32_t h = __float_as_uint(dist2f(pc, p));
    if (h < best_h) {
      best_h = h;
      best_n = (uint32_t)node;
    }
  };
  constexpr int kScanBatch = 16;
  const int nwords = lane < vw ? (vw - 1 - lane) / 32 + 1 : 0;
  int j = 0;
  uint32_t fr = nwords > 0 ? ~s[lane] : 0u;
  while (true) {
    int nd[kScanBatch];
#pragma unroll
    for (int q = 0; q < kScanBatch; ++q) {
      while (fr == 0u && ++j < nwords) fr = ~s[lane + 32 * j];
      nd[q] = -1;
      if (fr) {
        nd[q] = ((lane + 32 * j) << 5) + __ffs(fr) - 1;
        fr &= fr - 1;
      }
    }
    float2 pq[kScanBatch];
    int dq[kScanBatch];
#pragma unroll
    for (int q = 0; q < kScanBatch; ++q) {
      pq[q] = make_float2(0.f, 0.f);
      dq[q] = 0;
      if (nd[q] >= 0) {
        pq[q] = L == kLayoutGlobal ? __ldg(coords + nd[q]) : coords[nd[q]];
        if (!UNIT && check_dem) dq[q] = L == kLayoutGlobal ? __ldg(dem + nd[q]) : dem[nd[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < kScanBatch; ++q)
      if (nd[q] >= 0) visit(nd[q], pq[q], dq[q]);
    if (nd[kScanBatch - 1] < 0) break;
  }
  *best_h_out = best_h;
  return best_n;
}

// Nearest unvisited customer that fits (find_nearest_unvisited,
// src/seq/aco_sequential.c:477-493: strict '<' over ascending nodes, so the
// lowest index wins ties).  0 if none.
template <int L, bool UNIT, int V>
__device__ __forceinline__ int nearest_unvisited(const Tables<L, UNIT> &tb,
                                                 const Visited<V> &vis,
                                                 float2 pc, int room,
                                                 bool check_dem, int lane) {
  uint32_t best_h = 0xffffffffu, best_n = 0xffffffffu;
  auto visit = [&](int node, float2 p, int dem) {
    if (!UNIT && check_dem && dem > room) return;
    const uint32_t h = __float_as_uint(dist2f(pc, p));
    if (h < best_h) {
      best_h = h;
      best_n = (uint32_t)node;
    }
  };
  if (V == 2) {
    best_n = scan_regs<L, UNIT, V>(tb.coords, tb.dem, vis.w0, vis.w1, pc, room, check_dem, lane,
                                   &best_h);
  } else if (V == 1) {
    // Bit b of w0 is node lane + 32 b (ascending); one node at a time.
    auto scan = [&](uint32_t fr, int first) {
      while (fr) {
        const int b = __ffs(fr) - 1;
        fr &= fr - 1;
        const int node = first + b * 32;
        if (!UNIT && check_dem && tb.demand(node) > room) continue;
        visit(node, tb.coord(node), 0);
      }
    };
    scan(~vis.w0, lane);
  } else {
    best_n = scan_words<L, UNIT>(tb.coords, tb.dem, vis.s, vis.vw, pc, room, check_dem, lane,
                                 &best_h);
  }
  const uint32_t mh = __reduce_min_sync(kFull, best_h);
  const uint32_t mn = __reduce_min_sync(kFull, best_h == mh ? best_n : 0xffffffffu);
  return (mh == 0xffffffffu) ? 0 : (int)mn;
}

// The first eligible node of a second-tier row: the node (> 0); 0 when the
// row lists every remaining customer and none is eligible; -1 when none of
// the row is eligible and the row is full (customers beyond it remain).  The
// visited bitmap is read as Visited<V> holds it: V = 0 in shared memory at s
// (word wi holding nodes 32 wi .. 32 wi + 31), V = 1, 2 in the registers w0,
// w1 of the lanes (transposed).  All of the row and its demands are loaded
// at once.  Out of line: it is rare.
template <int L, bool UNIT, int V>
__device__ __noinline__ int tier2_first(const uint16_t *row, const uint32_t *s, uint32_t w0,
                                        uint32_t w1, const int *dem, int room, bool check_dem,
                                        int lane) {
  constexpr int kParts = kTier2Len / 32;
  int nodes[kParts], dq[kParts];
#pragma unroll
  for (int r = 0; r < kParts; ++r) nodes[r] = (int)__ldg(row + 32 * r + lane);
#pragma unroll
  for (int r = 0; r < kParts; ++r)
    dq[r] = (!UNIT && check_dem) ? (L == kLayoutGlobal ? __ldg(dem + nodes[r]) : dem[nodes[r]]) : 0;
#pragma unroll
  for (int r = 0; r < kParts; ++r) {
    const int node = nodes[r];
    // node 0 (empty slot) reads as visited: the depot's bit is set
    bool ok;
    if (V == 0) {
      const uint32_t word = s[node >> 5];
      ok = (__funnelshift_r(word, word, node) & 1u) == 0u;
    } else {
      const uint32_t bit = __funnelshift_l(0u, 1u, node >> 5);
      uint32_t word = __shfl_sync(kFull, w0, node);
      if (V == 2) {
        const uint32_t hi = __shfl_sync(kFull, w1, node);
        word = (node >> 10) ? hi : word;
      }
      ok = (word & bit) == 0u;
    }
    if (!UNIT && check_dem) ok = ok && dq[r] <= room;
    const unsigned m = __ballot_sync(kFull, ok);
    if (m) return __shfl_sync(kFull, node, __ffs(m) - 1);
  }
  return (__shfl_sync(kFull, nodes[kParts - 1], 31) == 0) ? 0 : -1;
}

// Nearest eligible customer of the fallback, when no candidate of row cur
// has a weight (find_nearest_unvisited's rule, as nearest_unvisited): the
// first eligible candidate (okm: the row's eligible candidates; they come
// first in the order), else the first eligible node of the tier row (the
// next 64 ranks of the same order), else the full scan; 0 when the
// candidates and a complete tier row hold no eligible customer.
template <int L, bool UNIT, int V>
__device__ __forceinline__ int nearest_eligible(const Tables<L, UNIT> &tb, const Visited<V> &vis,
                                                int cur, unsigned okm, int c, int room,
                                                bool check_dem, int lane) {
  if (okm) return __shfl_sync(kFull, c, __ffs(okm) - 1);
  if (tb.tier) {
    const uint16_t *row = tb.tier + (size_t)cur * kTierLen;
    int nodes[kTierLen / 32];
#pragma unroll
    for (int r = 0; r < kTierLen / 32; ++r)  // both halves in flight at once
      nodes[r] = (int)__ldg(row + 32 * r + lane);
#pragma unroll
    for (int r = 0; r < kTierLen / 32; ++r) {
      const int node = nodes[r];
      bool ok = !vis.test(node);  // node 0 (empty slot) reads as visited
      if (!UNIT && check_dem && ok) ok = tb.demand(node) <= room;
      const unsigned m = __ballot_sync(kFull, ok);
      if (m) return __shfl_sync(kFull, node, __ffs(m) - 1);
    }
    // every customer was listed
    if (__shfl_sync(kFull, nodes[kTierLen / 32 - 1], 31) == 0) return 0;
    if (tb.tier2) {
      const int r = tier2_first<L, UNIT, V>(tb.tier2 + (size_t)cur * kTier2Len, vis.s, vis.w0,
                                            vis.w1, tb.dem, room, check_dem, lane);
      if (r >= 0) return r;
    }
  }
  return nearest_unvisited<L, UNIT, V>(tb, vis, tb.coord(cur), room, check_dem, lane);
}

struct ConstructArgs {
  InstanceView iv;
  EpochTables et;
  AntBuffers ab;
  SmemPlan plan;
  DevState *st;
  uint32_t seed;
  uint32_t epoch;
  uint32_t stream;
  int use_state_epoch;  // 1: epoch number = st->epoch (graph replays)
  const uint32_t *draw_src;  // test hook: recorded draws [m][draw_per_ant], or null
  uint32_t draw_per_ant;
};

// Next 128 draws of an ant: Philox, or (test hook) the recorded stream,
// whose draws past its end read as 0.
__device__ __forceinline__ void next_draws(const ConstructArgs &a, uint32_t *buf, uint32_t d,
                                           uint32_t seed, uint32_t epoch, uint32_t gant,
                                           int ant, int lane) {
  if (a.draw_src) {
    __syncwarp();
    const uint32_t *src = a.draw_src + (size_t)ant * a.draw_per_ant;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t idx = (d & ~127u) + 4u * (uint32_t)lane + (uint32_t)q;
      buf[4 * lane + q] = idx < a.draw_per_ant ? (src[idx] & 0xFFFFFFu) : 0u;
    }
    __syncwarp();
    return;
  }
  draw_refill(buf, d, seed, epoch, gant, a.stream, lane);
}

// FP64 cost of a compact route sequence, summed in route order
// (solution_cost, src/common/solution.c:126-137).  Lanes compute the arc
// lengths, the sum runs in order in every lane; the (0,0) pairs between
// consecutive routes add +0.0, which leaves the sum unchanged.
template <int L, bool UNIT>
__device__ __forceinline__ double route_cost(const Tables<L, UNIT> &tb,
                                             const int *route, int entries,
                                             int lane) {
  double acc = 0.0;
  const int arcs = entries - 1;
  // The next 32 arcs' end points are loaded while the current ones are summed.
  int u = 0, v = 0;
  if (lane < arcs) {
    u = route[lane];
    v = route[lane + 1];
  }
  for (int b = 0; b < arcs; b += 32) {
    double dj = 0.0;
    if (b + lane < arcs) dj = dist64(tb.coord(u), tb.coord(v));
    const int j2 = b + 32 + lane;
    if (j2 < arcs) {
      u = route[j2];
      v = route[j2 + 1];
    }
    if (arcs - b >= 32) {
#pragma unroll
      for (int t = 0; t < 32; ++t) acc = __dadd_rn(acc, __shfl_sync(kFull, dj, t));
    } else {
      const int cnt = arcs - b;
      for (int t = 0; t < cnt; ++t) acc = __dadd_rn(acc, __shfl_sync(kFull, dj, t));
    }
  }
  return acc;
}

// Depot-close weight of the reference-CUDA rule on the scale of the row's
// candidate weights: 2^23 2^(-r/16) for r = rdep (may be negative, i.e. above
// the row maximum), exact in FP64 as LUT[r mod 16] 2^(-floor(r/16)); 0 from
// r = 255 on, like the candidate weights.
__device__ __forceinline__ double depot_weight(int r, const uint32_t *lut) {
  if (r >= kRelMax) return 0.0;
  const int q = (r >= 0) ? (r / 16) : -((-r + 15) / 16);
  return ldexp((double)__ldg(lut + (r - 16 * q)), -q);
}

// One ant, one warp.  Rules of build_ant_solution
// (src/seq/aco_sequential.c:616-681) with the demand extension:
//   vehicle v extends while remaining > 0, remaining demand > (K-v-1) Q and
//   load < Q; the next customer is drawn by roulette over the eligible
//   candidates (unvisited, load + d <= Q), else the nearest eligible one;
//   customers left over are added by the backward repair pass.
// CREF (reference-CUDA depot rule, kernel_construct_solutions,
// src/cuda/aco_cuda_kernels.cu:487-520): vehicle v extends while customers
// remain and load < Q; once the remaining demand fits the later vehicles
// (<= (K-v-1) Q) the route may close: at the depot it closes at once (the
// reference's 2 (1/(0+eps))^beta dwarfs every candidate), with no eligible
// candidate it closes, and after a roulette draw a second draw u closes it
// when u (denom + w_depot) >= denom, w_depot = depot_weight(rdep[cur]).
template <int L, bool UNIT, int V, bool CREF>
__device__ void build_ant(const ConstructArgs &a, const Tables<L, UNIT> &tb,
                          Visited<V> &vis, uint32_t *dbuf, int *route_s, int ant,
                          uint32_t epoch, uint32_t seed, int lane) {
  const InstanceView &iv = a.iv;
  const int k = iv.k, K = iv.K, R = iv.route_stride;
  const int cap = (int)iv.cap;
  const int max_dem = iv.max_demand;
  // The route is built in shared memory where the plan has room for it
  // (route_s), and copied out once it is complete.
  int *route = route_s ? route_s : a.ab.routes + (size_t)ant * R;
  int *lens = a.ab.lens + (size_t)ant * K;
  int *loads = a.ab.loads + (size_t)ant * K;

  // Draws are keyed by the ant's global id (ant_base > 0 when the colony is
  // split over several devices).
  const uint32_t gant = (uint32_t)(ant + iv.ant_base);
  uint32_t d = 0;
  next_draws(a, dbuf, d, seed, epoch, gant, ant, lane);
  uint32_t r_next = dbuf[0];

  int remaining = iv.n;
  int rem_dem = (int)iv.total_demand;
  int pos = 0;

  for (int v = 0; v < K; ++v) {
    const int start = pos;
    if (lane == 0) route[pos] = 0;
    ++pos;
    int cur = 0;
    int load = 0;
    const long long fut64 = (long long)(K - v - 1) * iv.cap;
    const int future = fut64 > 0x7fffffffLL ? 0x7fffffff : (int)fut64;
    // room < max_dem  <=>  load > cap - max_dem
    const int tight_load = cap - max_dem;
    bool tight = !UNIT && 0 > tight_load;
    // Row of the current node; the next row's loads are issued as soon as the
    // next node is known, ahead of this step's bookkeeping.
    // cb: this lane's candidate's row offset, formed as soon as the row is
    // loaded, so the selected lane's offset reaches the next row's loads by
    // one shuffle, with no multiply on the chain.
    int c = 0, dc = 0, cb = 0;
    uint32_t w = 0u;
    if (lane < k) {
      c = tb.cand[lane];
      w = tb.weight(lane);
    }
    cb = c * k;
    if (!UNIT) dc = tb.demand(c);
    // Every demand is >= 1, so rem_dem > future >= 0 implies remaining > 0.
    const int limit = CREF ? 0 : future;
    // One step to customer nx (row offset base = nx k) of demand dnx: the
    // next row's loads first, then the bookkeeping.
    auto take_step = [&](int nx, int base, int dnx) {
      c = 0;
      w = 0u;
      if (lane < k) {
        c = tb.cand[base + lane];
        w = tb.weight(base + lane);
      }
      cb = c * k;
      if (!UNIT) dc = tb.demand(c);
      route[pos] = nx;  // every lane stores the same value
      vis.set(nx, lane);
      ++pos;
      --remaining;
      load += dnx;
      rem_dem -= dnx;
      tight = !UNIT && load > tight_load;
      cur = nx;
    };
    // One step per loop trip (unrolling by two was 0.9 % slower at n=1000
    // once the prefix came from independent shuffles).
#pragma unroll 1
    while (rem_dem > limit && load < cap) {
      const bool may_close = CREF && rem_dem <= future;
      if (CREF && may_close && cur == 0) break;
      bool ok = !vis.test(c);
      // Demands only bind when the room left is below the largest demand;
      // until then the speculative demand load stays off the step's chain.
      if (!UNIT && tight) ok = ok && dc + load <= cap;
      const uint32_t wv = ok ? w : 0u;
      const uint32_t denom = __reduce_add_sync(kFull, wv);
      // cum * 2^24 >= r * denom  <=>  cum >= ceil(r * denom / 2^24)
      const uint32_t thr =
          (uint32_t)(((unsigned long long)r_next * denom + 0xFFFFFFull) >> kDrawBits);
      // Sum of the 8 masked weights ending at this lane (lanes 0..7: the
      // inclusive prefix, where most draws land): 7 independent shuffles of
      // the weights and an add tree, the value three scan steps give with
      // three dependent shuffles.  The last two scan steps run only if
      // needed.
      uint32_t u[8];
      u[0] = wv;
#pragma unroll
      for (int o = 1; o < 8; ++o) {
        const uint32_t t = __shfl_up_sync(kFull, wv, o);
        u[o] = lane >= o ? t : 0u;
      }
      uint32_t cum = ((u[0] + u[1]) + (u[2] + u[3])) + ((u[4] + u[5]) + (u[6] + u[7]));
      unsigned msk = __ballot_sync(kFull, lane < 8 && wv != 0u && cum >= thr);
      if (msk == 0u) {
#pragma unroll
        for (int o = 8; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(kFull, cum, o);
          if (lane >= o) cum += t;
        }
        msk = __ballot_sync(kFull, wv != 0u && cum >= thr);
        if (denom == 0u) {
          // No eligible candidate: the reference-CUDA rule closes the route
          // when it may; otherwise the nearest eligible customer, which
          // consumes no draw.
          if (CREF && may_close) break;
          const int nx = nearest_eligible<L, UNIT, V>(tb, vis, cur, __ballot_sync(kFull, ok), c,
                                                      cap - load, tight, lane);
          if (nx <= 0) break;
          take_step(nx, nx * k, tb.demand(nx));
          continue;
        }
      }
      const int src = __ffs(msk) - 1;  // msk != 0 here: denom > 0
      const int nbase = __shfl_sync(kFull, cb, src);
      int next = __shfl_sync(kFull, c, src);
      int dn = UNIT ? 1 : __shfl_sync(kFull, dc, src);
      bool drawn = false;  // draws of this step already accounted
      if (CREF && may_close) {
        d += 1u;  // the roulette draw is spent
        if ((d & 127u) == 0u) next_draws(a, dbuf, d, seed, epoch, gant, ant, lane);
        const uint32_t r2 = dbuf[d & 127u];
        d += 1u;  // and the close draw
        if ((d & 127u) == 0u) next_draws(a, dbuf, d, seed, epoch, gant, ant, lane);
        r_next = dbuf[d & 127u];
        drawn = true;
        const double wd = depot_weight(a.et.rdep[cur], a.et.lut);
        if (__dmul_rn((double)r2, __dadd_rn((double)denom, wd)) >= (double)denom * 16777216.0)
          break;
      }
      take_step(next, nbase, dn);
      // A draw is consumed only by a roulette selection (denom > 0).
      if (!drawn) {
        d += 1u;
        if ((d & 127u) == 0u) next_draws(a, dbuf, d, seed, epoch, gant, ant, lane);
        r_next = dbuf[d & 127u];
      }
    }
    if (lane == 0) {
      route[pos] = 0;
      lens[v] = pos + 1 - start;
      loads[v] = load;
    }
    ++pos;
  }

  if (remaining > 0) {
    // Backward repair (aco_sequential.c:659-680): from the last vehicle down,
    // reopen the route and append the nearest eligible customers.
    __syncwarp();
    int *rep = a.ab.rep + (size_t)ant * iv.n;
    int *repc = a.ab.repc + (size_t)ant * K;
    for (int v = lane; v < K; v += 32) repc[v] = 0;
    __syncwarp();
    int nrep = 0;
    int off_end = pos;
    for (int v = K - 1; v >= 0 && remaining > 0; --v) {
      const int len_v = lens[v];
      off_end -= len_v;
      int cur = route[off_end + len_v - 2];
      int load = loads[v];
      int cnt = 0;
      while (remaining > 0 && load < cap) {
        const int next = nearest_unvisited<L, UNIT, V>(tb, vis, tb.coord(cur), cap - load,
                                                       true, lane);
        if (next <= 0) break;
        if (lane == 0) rep[nrep + cnt] = next;
        vis.set(next, lane);
        ++cnt;
        load += tb.demand(next);
        --remaining;
        cur = next;
      }
      if (lane == 0) repc[v] = cnt;
      nrep += cnt;
    }
    __syncwarp();
    if (lane == 0 && nrep > 0) {
      // Re-lay the compact routes with each vehicle's additions appended
      // before its closing depot; vehicles are moved right, last first.
      int off_total = pos;
      int add_after = 0;  // additions of vehicles > v (stored first)
      int shift = nrep;   // additions of vehicles <= v
      for (int v = K - 1; v >= 0; --v) {
        const int len_v = lens[v];
        off_total -= len_v;
        const int cnt = repc[v];
        shift -= cnt;  // now: additions of vehicles < v
        const int old_off = off_total, new_off = off_total + shift;
        const int main_len = len_v - 1;
        for (int t = main_len - 1; t >= 0; --t) route[new_off + t] = route[old_off + t];
        for (int j = 0; j < cnt; ++j) route[new_off + main_len + j] = rep[add_after + j];
        route[new_off + main_len + cnt] = 0;
        lens[v] = len_v + cnt;
        add_after += cnt;
      }
    }
    pos += nrep;
  }
  __syncwarp();
  const double cost = route_cost<L, UNIT>(tb, route, pos, lane);
  if (route_s) {
    int *g = a.ab.routes + (size_t)ant * R;
    for (int j = lane; j < pos; j += 32) g[j] = route_s[j];
  }
  if (lane == 0) {
    a.ab.cost[ant] = cost;
    a.ab.feasible[ant] = (remaining == 0) ? 1 : 0;
    a.ab.steps[ant] = pos - K;
    a.ab.draws[ant] = d;
  }
}

template <int L, bool UNIT, int V, bool CREF>
__global__ void __launch_bounds__(512, 1) k_construct(ConstructArgs a) {
  if (a.st && *(volatile int *)&a.st->skip) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const SmemPlan &pl = a.plan;
  const InstanceView &iv = a.iv;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem);

  Tables<L, UNIT> tb;
  tb.tier = iv.tier;
  tb.tier2 = iv.tier2;
  if (L == kLayoutGlobal) {
    tb.cand = iv.cand;
    tb.w = a.et.w;
    tb.rel = nullptr;
    tb.lut = nullptr;
    tb.coords = iv.coords;
    tb.dem = iv.demand;
  } else {
    tb.cand = reinterpret_cast<const uint16_t *>(smem + pl.off_cand);
    tb.w = reinterpret_cast<const uint32_t *>(smem + pl.off_w);
    tb.rel = reinterpret_cast<const uint8_t *>(smem + pl.off_w);
    tb.lut = reinterpret_cast<const uint32_t *>(smem + pl.off_lut);
    tb.coords = reinterpret_cast<const float2 *>(smem + pl.off_coords);
    tb.dem = reinterpret_cast<const int *>(smem + pl.off_dem);
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t total = pl.bytes_cand + pl.bytes_w + pl.bytes_coords + (UNIT ? 0u : pl.bytes_dem);
      mbar_arrive_expect_tx(bar, total + (uint32_t)iv.stage_extra_tx);
      const uint32_t kChunk = 32768u;
      auto issue = [&](unsigned char *dst, const void *src, uint32_t bytes) {
        const unsigned char *sp = reinterpret_cast<const unsigned char *>(src);
        for (uint32_t o = 0; o < bytes; o += kChunk) {
          const uint32_t b = bytes - o < kChunk ? bytes - o : kChunk;
          bulk_g2s(dst + o, sp + o, b, bar);
        }
      };
      issue(smem + pl.off_cand, iv.cand, pl.bytes_cand);
      if (L == kLayoutSmemPacked) issue(smem + pl.off_w, a.et.rel, pl.bytes_w);
      else issue(smem + pl.off_w, a.et.w, pl.bytes_w);
      issue(smem + pl.off_coords, iv.coords, pl.bytes_coords);
      if (!UNIT) issue(smem + pl.off_dem, iv.demand, pl.bytes_dem);
    }
    if (L == kLayoutSmemPacked) {
      uint32_t *lut = reinterpret_cast<uint32_t *>(smem + pl.off_lut);
      for (int r = threadIdx.x; r < 256; r += blockDim.x) lut[r] = __ldg(a.et.lut + r);
      __syncthreads();
    }
  }

  uint32_t *dbuf = reinterpret_cast<uint32_t *>(smem + pl.off_draw) + (size_t)warp * 128;
  Visited<V> vis;
  vis.init(reinterpret_cast<uint32_t *>(smem + pl.off_vis) + (size_t)warp * pl.vis_words,
           pl.vis_words, iv.n, lane);

  if (L != kLayoutGlobal) {
    // Bounded wait for the staged tables.  The decision is the block's: it
    // goes on only when every thread saw the tables arrive, so no warp
    // enters the full-mask collectives of build_ant with lanes or warps
    // gone.  On time-out the block flags the error, waits (bounded again)
    // for its copies still in flight and exits.  The injected time-out
    // expects stage_extra_tx bytes that no copy brings; thread 0 marks them
    // arrived, so that second wait ends once the real copies have landed.
    // After a genuine time-out the second wait may run out as well; the
    // block then exits with the error flag set.
    const uint32_t limit = iv.stage_extra_tx ? (1u << 14) : (1u << 22);
    const bool ok = __syncthreads_and(mbar_wait_bounded(bar, 0, limit) ? 1 : 0) != 0;
    if (!ok) {
      if (threadIdx.x == 0) {
        if (a.st) atomicOr(&a.st->error, kErrStageTimeout);
        if (iv.stage_extra_tx) mbar_complete_tx(bar, (uint32_t)iv.stage_extra_tx);
      }
      __syncthreads();
      mbar_wait_bounded(bar, 0, limit << 2);
      __syncthreads();
      return;
    }
  }

  const int ant = blockIdx.x * pl.wpb + warp;
  if (ant >= iv.m) return;
  // Graph replays read the epoch number and the seed from the device state,
  // so one captured graph serves every solve of a context.
  const uint32_t epoch = a.use_state_epoch ? (uint32_t)a.st->epoch : a.epoch;
  const uint32_t seed = a.use_state_epoch ? a.st->seed : a.seed;
  int *route_s = pl.route_smem
                     ? reinterpret_cast<int *>(smem + pl.off_route) + (size_t)warp * iv.route_stride
                     : nullptr;
  build_ant<L, UNIT, V, CREF>(a, tb, vis, dbuf, route_s, ant, epoch, seed, lane);
}

static int g_max_smem = 0;

int construct_max_smem() {
  if (g_max_smem == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    g_max_smem = v;
  }
  return g_max_smem;
}

static uint32_t pad16(size_t b) { return (uint32_t)((b + 15) & ~size_t(15)); }

SmemPlan plan_construct(const InstanceView &iv, int layout, int num_sms,
                        int max_smem) {
  SmemPlan p = {};
  const size_t rows = (size_t)iv.n + 1;
  p.vis_words = (int)((rows + 31) / 32);
  p.vreg = p.vis_words <= 32 ? 1 : (p.vis_words <= 64 ? 2 : 0);
  int wpb = (iv.m + num_sms - 1) / num_sms;
  if (wpb < 1) wpb = 1;
  if (wpb > 16) wpb = 16;
  p.wpb = wpb;
  p.bytes_cand = pad16(rows * iv.k * sizeof(uint16_t));
  p.bytes_coords = pad16(rows * sizeof(float2));
  p.bytes_dem = iv.unit ? 0u : pad16(rows * sizeof(int));
  const uint32_t vis_bytes = p.vreg ? 0u : (uint32_t)wpb * p.vis_words * 4u;
  const uint32_t draw_bytes = (uint32_t)wpb * 512u;
  auto finish = [&](int lay) {
    p.layout = lay;
    uint32_t off = 16;  // mbarrier
    if (lay == kLayoutGlobal) {
      p.bytes_cand = p.bytes_w = p.bytes_coords = p.bytes_dem = 0;
      p.off_cand = p.off_w = p.off_coords = p.off_dem = p.off_lut = off;
    } else {
      p.bytes_w = (lay == kLayoutSmemPacked) ? pad16(rows * iv.k) : pad16(rows * iv.k * 4);
      p.off_cand = off; off += p.bytes_cand;
      p.off_w = off; off += p.bytes_w;
      p.off_coords = off; off += p.bytes_coords;
      p.off_dem = off; off += p.bytes_dem;
      p.off_lut = off; off += (lay == kLayoutSmemPacked) ? 1024u : 0u;
    }
    p.off_draw = off;
    off += draw_bytes;
    p.off_vis = off;
    off += vis_bytes;
    p.total = off;
    // Each ant's route in shared memory too, with the tables in shared
    // memory, where it fits and the launch is one block per SM anyway (so
    // the space costs no residency): n=1000 265.0 -> 260.4 us, n=100 34.1
    // -> 33.4 us.  Not with rows from global memory: the space comes out of
    // the L1 that serves those rows (n=3000 1418 -> 1638 us).
    p.route_smem = 0;
    p.off_route = off;
    const size_t rb = pad16((size_t)wpb * (size_t)iv.route_stride * 4u);
    if (lay != kLayoutGlobal && off + rb <= (size_t)max_smem &&
        (iv.m + wpb - 1) / wpb <= num_sms) {
      p.route_smem = 1;
      p.total = off + (uint32_t)rb;
    }
  };
  if (layout >= 0) {
    finish(layout);
    return p;
  }
  finish(kLayoutSmemWeights);
  if ((int)p.total <= max_smem) return p;
  finish(kLayoutSmemPacked);
  if ((int)p.total <= max_smem) return p;
  finish(kLayoutGlobal);
  return p;
}

template <int L, bool UNIT, int V>
static cudaError_t configure_t() {
  cudaError_t e = cudaFuncSetAttribute(k_construct<L, UNIT, V, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       construct_max_smem());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_construct<L, UNIT, V, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, construct_max_smem());
  return e;
}

template <int L, bool UNIT>
static cudaError_t configure_lu() {
  cudaError_t e = configure_t<L, UNIT, 0>();
  if (e == cudaSuccess) e = configure_t<L, UNIT, 1>();
  if (e == cudaSuccess) e = configure_t<L, UNIT, 2>();
  return e;
}

// Opts every construct instantiation into the full shared-memory carve-out;
// called once per device before any launch or graph capture.
cudaError_t prepare_construct_kernels() {
  cudaError_t e = configure_lu<kLayoutSmemWeights, false>();
  if (e == cudaSuccess) e = configure_lu<kLayoutSmemWeights, true>();
  if (e == cudaSuccess) e = configure_lu<kLayoutSmemPacked, false>();
  if (e == cudaSuccess) e = configure_lu<kLayoutSmemPacked, true>();
  if (e == cudaSuccess) e = configure_lu<kLayoutGlobal, false>();
  if (e == cudaSuccess) e = configure_lu<kLayoutGlobal, true>();
  return e;
}

template <int L, bool UNIT, bool CREF>
static cudaError_t launch_construct_luc(const ConstructArgs &a, cudaStream_t s) {
  const int grid = (a.iv.m + a.plan.wpb - 1) / a.plan.wpb;
  const int threads = a.plan.wpb * 32;
  switch (a.plan.vreg) {
    case 1: k_construct<L, UNIT, 1, CREF><<<grid, threads, a.plan.total, s>>>(a); break;
    case 2: k_construct<L, UNIT, 2, CREF><<<grid, threads, a.plan.total, s>>>(a); break;
    default: k_construct<L, UNIT, 0, CREF><<<grid, threads, a.plan.total, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <int L, bool UNIT>
static cudaError_t launch_construct_lu(const ConstructArgs &a, cudaStream_t s) {
  if (a.iv.depot_rule == kDepotRuleCudaRef) {
    if (!a.et.rdep) return cudaErrorInvalidValue;
    return launch_construct_luc<L, UNIT, true>(a, s);
  }
  return launch_construct_luc<L, UNIT, false>(a, s);
}

cudaError_t launch_construct(const InstanceView &iv, const EpochTables &et,
                             const AntBuffers &ab, const SmemPlan &plan,
                             DevState *st, uint32_t seed, uint32_t epoch,
                             uint32_t stream_id, int use_state_epoch,
                             cudaStream_t s, const uint32_t *draw_src,
                             uint32_t draw_per_ant) {
  ConstructArgs a;
  a.draw_src = draw_src;
  a.draw_per_ant = draw_per_ant;
  a.iv = iv;
  a.et = et;
  a.ab = ab;
  a.plan = plan;
  a.st = st;
  a.seed = seed;
  a.epoch = epoch;
  a.stream = stream_id;
  a.use_state_epoch = use_state_epoch;
  if ((int)plan.total > construct_max_smem()) return cudaErrorInvalidValue;
  switch (plan.layout * 2 + (iv.unit ? 1 : 0)) {
    case 0: return launch_construct_lu<kLayoutSmemWeights, false>(a, s);
    case 1: return launch_construct_lu<kLayoutSmemWeights, true>(a, s);
    case 2: return launch_construct_lu<kLayoutSmemPacked, false>(a, s);
    case 3: return launch_construct_lu<kLayoutSmemPacked, true>(a, s);
    case 4: return launch_construct_lu<kLayoutGlobal, false>(a, s);
    case 5: return launch_construct_lu<kLayoutGlobal, true>(a, s);
  }
  return cudaErrorInvalidValue;
}

// ===========================================================================
// Iteration best, global best and stop rules
// ===========================================================================

// is_significant_improvement, src/cuda/aco_cuda.cu:83-94.
__device__ __forceinline__ bool significant(double prev, double next,
                                            double min_rel) {
  if (prev >= DBL_MAX || next >= DBL_MAX) return next < prev;
  if (next >= __dsub_rn(prev, 1e-9)) return false;
  double gain = __dsub_rn(prev, next);
  double rel = __ddiv_rn(gain, fmax(prev, 1e-9));
  return __dadd_rn(rel, 1e-9) >= min_rel;
}

// Epoch bookkeeping of src/cuda/aco_cuda.cu:349-399 and the stop rules
// checked at the start of the next epoch (:333-339), given the iteration's
// best feasible ant (found, cost bc, ant ba) and its ant-steps.  Returns
// whether the global best improved.
__device__ int epoch_bookkeeping(DevState *st, bool found, double bc, int ba,
                                 unsigned long long steps, EpochRec *log) {
  int improved = 0;
  st->found = found ? 1 : 0;
  st->total_steps += steps;
  if (found) {
    st->iter_best = bc;
    st->best_ant = ba;
    if (bc < st->global_best) {
      improved = 1;
      if (significant(st->global_best, bc, st->min_rel)) st->iter_since_best = 0;
      else st->iter_since_best += 1;
      st->global_best = bc;
    } else {
      st->iter_since_best += 1;
    }
    st->dep_iter = __fdiv_rn(0.3f * st->Qs, (float)bc);
    st->dep_global = __fdiv_rn(0.7f * st->Qs, (float)st->global_best);
  } else {
    st->iter_since_best += 1;
  }
  st->improved = improved;
  st->epoch += 1;
  const unsigned long long now = global_timer_ns();
  const unsigned long long elapsed = now > st->start_ns ? now - st->start_ns : 0ull;
  EpochRec rec;
  rec.epoch = st->epoch;
  rec.iter_since_best = st->iter_since_best;
  rec.improved = improved;
  rec.found = found ? 1 : 0;
  rec.global_best = st->global_best;
  rec.elapsed_ns = elapsed;
  if (log) log[st->log_count % kLogCap] = rec;
  st->log_count += 1;
  int flags = st->stop_flags;
  if (st->stagnation > 0 && st->iter_since_best >= st->stagnation) flags |= kStopStagnation;
  if (st->fixed_epochs > 0 && st->epoch >= st->fixed_epochs) flags |= kStopFixed;
  if (st->timeout_ns > 0ull && elapsed > st->timeout_ns) flags |= kStopTimeout;
  if (st->run_limit > 0 && st->epoch >= st->run_limit) flags |= kStopRunLimit;
  st->stop_flags = flags;
  return improved;
}

// The device state staged in shared memory by one block: one coalesced read,
// the bookkeeping on the copy, one write-back before the block ends.
__device__ __forceinline__ void state_load(DevState *s, const DevState *g) {
  static_assert(sizeof(DevState) % sizeof(int) == 0, "DevState is whole words");
  constexpr int kWords = (int)(sizeof(DevState) / sizeof(int));
  for (int i = threadIdx.x; i < kWords; i += blockDim.x)
    reinterpret_cast<int *>(s)[i] = reinterpret_cast<const volatile int *>(g)[i];
  __syncthreads();
}
__device__ __forceinline__ void state_store(DevState *g, const DevState *s) {
  constexpr int kWords = (int)(sizeof(DevState) / sizeof(int));
  for (int i = threadIdx.x; i < kWords; i += blockDim.x)
    reinterpret_cast<int *>(g)[i] = reinterpret_cast<const int *>(s)[i];
}

__device__ __forceinline__ uint32_t evap4(uint32_t x, uint32_t floor4,
                                          uint32_t delta4) {
  return __vsub4(__vmaxu4(x, floor4), delta4);
}

// Evaporation sweep of pv.total bytes from src to dst (src == dst: in
// place), q > q_min + delta ? q - delta : q_min as max(q, q_min + delta) -
// delta on 16 bytes at a time (kernel_evaporate_tau,
// src/cuda/aco_cuda_kernels.cu:145-155).  Each thread keeps kEvapUnroll
// 16-byte loads in flight before its stores (a block covers
// kEvapUnroll * blockDim.x vectors per trip), and the loads and stores are
// streaming (evict-first), so a matrix larger than L2 passes through without
// displacing the construction's tables.  Block 0 also does the tail past the
// last whole vector.
constexpr int kEvapUnroll = 4;
constexpr int kEvapThreads = 512;

__device__ __forceinline__ void evap_sweep(const uint8_t *src, uint8_t *dst,
                                           unsigned long long total, uint8_t q_min,
                                           uint8_t delta) {
  const int fl = (int)q_min + (int)delta;
  const bool sat_all = fl > 255;
  const uint32_t floor4 = 0x01010101u * (uint32_t)(sat_all ? 0 : fl);
  const uint32_t delta4 = 0x01010101u * (uint32_t)delta;
  const uint32_t qmin4 = 0x01010101u * (uint32_t)q_min;
  const unsigned long long nvec = total / 16;
  const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
  uint4 *d4 = reinterpret_cast<uint4 *>(dst);
  const unsigned long long tile = (unsigned long long)kEvapUnroll * blockDim.x;
  const unsigned long long step = tile * gridDim.x;
  for (unsigned long long base = blockIdx.x * tile + threadIdx.x; base < nvec; base += step) {
    uint4 v[kEvapUnroll];
#pragma unroll
    for (int u = 0; u < kEvapUnroll; ++u) {
      const unsigned long long i = base + (unsigned long long)u * blockDim.x;
      if (i < nvec) v[u] = __ldcs(s4 + i);
    }
#pragma unroll
    for (int u = 0; u < kEvapUnroll; ++u) {
      const unsigned long long i = base + (unsigned long long)u * blockDim.x;
      if (i < nvec) {
        uint4 r = v[u];
        if (sat_all) {
          r = make_uint4(qmin4, qmin4, qmin4, qmin4);
        } else {
          r.x = evap4(r.x, floor4, delta4);
          r.y = evap4(r.y, floor4, delta4);
          r.z = evap4(r.z, floor4, delta4);
          r.w = evap4(r.w, floor4, delta4);
        }
        __stcs(d4 + i, r);
      }
    }
  }
  if (blockIdx.x == 0) {
    for (unsigned long long i = nvec * 16 + threadIdx.x; i < total; i += blockDim.x) {
      const uint8_t q = src[i];
      dst[i] = ((int)q > fl) ? (uint8_t)(q - delta) : q_min;
    }
  }
}

// Folds (oc, oa) into the running best (bc, ba): least cost, then lowest
// ant (the first minimum of select_iter_best_host, src/cuda/aco_cuda.cu:96-126).
__device__ __forceinline__ void best_fold(double &bc, int &ba, double oc, int oa) {
  if (oa != INT_MAX && (ba == INT_MAX || oc < bc || (oc == bc && oa < ba))) {
    bc = oc;
    ba = oa;
  }
}

__device__ __forceinline__ void warp_best(double &bc, int &ba, unsigned long long &steps) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double oc = __shfl_down_sync(kFull, bc, o);
    const int oa = __shfl_down_sync(kFull, ba, o);
    steps += __shfl_down_sync(kFull, steps, o);
    best_fold(bc, ba, oc, oa);
  }
}

// Iteration best of the m ants (INT_MAX: none feasible) and their
// ant-steps, over one block; every thread calls it, lane 0 of warp 0 holds
// the result.  The s_* scratch holds one entry per warp.
__device__ __forceinline__ void block_iter_best(const AntBuffers &ab, int m, double *s_cost,
                                                int *s_ant, unsigned long long *s_steps,
                                                double &bc, int &ba, unsigned long long &steps) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bc = DBL_MAX;
  ba = INT_MAX;
  steps = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    steps += (unsigned long long)ab.steps[i];
    if (ab.feasible[i]) {
      const double c = ab.cost[i];
      if (ba == INT_MAX || c < bc) {  // ascending i: first minimum kept
        bc = c;
        ba = i;
      }
    }
  }
  warp_best(bc, ba, steps);
  if (lane == 0) {
    s_cost[warp] = bc;
    s_ant[warp] = ba;
    s_steps[warp] = steps;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    bc = (lane < nw) ? s_cost[lane] : DBL_MAX;
    ba = (lane < nw) ? s_ant[lane] : INT_MAX;
    steps = (lane < nw) ? s_steps[lane] : 0ull;
    warp_best(bc, ba, steps);
  }
}

// Iteration best, bookkeeping and the global-best copy in one block, for the
// epochs whose pheromone update is a separate k_evap_deposit launch.
__global__ void __launch_bounds__(1024) k_best(InstanceView iv, AntBuffers ab,
                                               DevState *st, int *gbest_nodes,
                                               int *gbest_lens, EpochRec *log) {
  if (*(volatile int *)&st->skip) return;
  __shared__ double s_cost[32];
  __shared__ int s_ant[32];
  __shared__ unsigned long long s_steps[32];
  __shared__ int s_improved, s_best;
  double bc;
  int ba;
  unsigned long long steps;
  block_iter_best(ab, iv.m, s_cost, s_ant, s_steps, bc, ba, steps);
  if (threadIdx.x == 0) {
    s_improved = epoch_bookkeeping(st, ba != INT_MAX, bc, ba, steps, log);
    s_best = ba;
  }
  __syncthreads();
  if (s_improved) {
    // New global best: keep a copy (the reference copies it to the host and
    // uploads a flat buffer, aco_cuda.cu:367-380).
    const int *src = ab.routes + (size_t)s_best * iv.route_stride;
    const int *sl = ab.lens + (size_t)s_best * iv.K;
    int total = 0;
    for (int v = 0; v < iv.K; ++v) total += sl[v];
    for (int t = threadIdx.x; t < total; t += blockDim.x) gbest_nodes[t] = src[t];
    for (int v = threadIdx.x; v < iv.K; v += blockDim.x) gbest_lens[v] = sl[v];
  }
}

// The pipelined epoch's iteration best, bookkeeping and both deposits over a
// cluster of kBestCluster blocks, so that the deposits' scattered pheromone
// reads and writes are issued from as many SMs.  Every block finds the same
// iteration best and, from the same state snapshot, the same deposit
// amounts; block 0 alone keeps the bookkeeping (state, log, global-best
// copy).  The cluster barrier puts the iteration-best deposit before the
// global-best one.
constexpr int kBestCluster = 8;
constexpr int kBestThreads = 256;

// The epoch's two deposits over the cluster, into the buffer evaporated
// beside the construction: the iteration best, a cluster barrier (its stores
// before the next deposit's loads, release / acquire at cluster scope), the
// global best; then block 0 switches the buffer and writes the state back.
__device__ __forceinline__ void cluster_deposits(cooperative_groups::cluster_group &cluster,
                                                 int rank, const InstanceView &iv,
                                                 const PheromoneView &pv, uint8_t *tau_alt,
                                                 DevState *s_st, DevState *st,
                                                 const int *it_nodes, const int *it_lens,
                                                 const int *gb_nodes, const int *gb_lens) {
  const bool sel = s_st->tau_sel != 0;
  PheromoneView pd = pv;
  pd.tau = sel ? pv.tau : tau_alt;  // the evaporated copy
  const size_t stride_n = (size_t)iv.n + 1;
  extern __shared__ int s_off[];
  int *offs = (iv.K <= kDepositSmemRoutes) ? s_off : nullptr;
  const int gt = rank * kBestThreads + (int)threadIdx.x, gn = kBestCluster * kBestThreads;
  deposit_solution(pd, stride_n, CompactNodes{it_nodes}, it_lens, iv.K, s_st->dep_iter, offs, gt,
                   gn);
  cluster.sync();
  deposit_solution(pd, stride_n, CompactNodes{gb_nodes}, gb_lens, iv.K, s_st->dep_global, offs,
                   gt, gn);
  if (rank == 0) {
    __syncthreads();
    if (threadIdx.x == 0) s_st->tau_sel = sel ? 0 : 1;
    __syncthreads();
    state_store(st, s_st);
  }
}

__global__ void __cluster_dims__(kBestCluster, 1, 1) __launch_bounds__(kBestThreads)
    k_best_cluster(InstanceView iv, AntBuffers ab, DevState *st, int *gbest_nodes,
                   int *gbest_lens, EpochRec *log, PheromoneView pv, uint8_t *tau_alt) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  __shared__ DevState s_st;
  __shared__ double s_cost[kBestThreads / 32];
  __shared__ int s_ant[kBestThreads / 32];
  __shared__ unsigned long long s_steps[kBestThreads / 32];
  __shared__ int s_improved, s_best;
  state_load(&s_st, st);
  double bc;
  int ba;
  unsigned long long steps;
  block_iter_best(ab, iv.m, s_cost, s_ant, s_steps, bc, ba, steps);
  if (s_st.skip) return;  // the same in every block: nothing is written
  if (threadIdx.x == 0) {
    // Each block updates its own copy; only block 0's copy and log entry are
    // kept (the others differ at most in the elapsed-time fields).
    s_improved = epoch_bookkeeping(&s_st, ba != INT_MAX, bc, ba, steps, rank == 0 ? log : nullptr);
    s_best = ba;
  }
  __syncthreads();
  const int R = iv.route_stride;
  if (rank == 0 && s_improved) {
    // New global best: keep a copy (aco_cuda.cu:367-380).
    const int *src = ab.routes + (size_t)s_best * R;
    const int *sl = ab.lens + (size_t)s_best * iv.K;
    int total = 0;
    for (int v = 0; v < iv.K; ++v) total += sl[v];
    for (int t = threadIdx.x; t < total; t += blockDim.x) gbest_nodes[t] = src[t];
    for (int v = threadIdx.x; v < iv.K; v += blockDim.x) gbest_lens[v] = sl[v];
  }
  if (s_best == INT_MAX) {
    // No feasible ant: no evaporation, no deposit; every block has read the
    // state before block 0 writes it back.
    cluster.sync();
    if (rank == 0) state_store(st, &s_st);
    return;
  }
  const int *it_nodes = ab.routes + (size_t)s_best * R;
  const int *it_lens = ab.lens + (size_t)s_best * iv.K;
  // The global best is this epoch's iteration best when it improved (the
  // copy block 0 makes holds the same routes).
  cluster_deposits(cluster, rank, iv, pv, tau_alt, &s_st, st, it_nodes, it_lens,
                   s_improved ? it_nodes : gbest_nodes, s_improved ? it_lens : gbest_lens);
}

cudaError_t launch_best(const InstanceView &iv, const AntBuffers &ab,
                        DevState *st, int *gbest_nodes, int *gbest_lens,
                        EpochRec *log, cudaStream_t s) {
  k_best<<<1, 1024, 0, s>>>(iv, ab, st, gbest_nodes, gbest_lens, log);
  return cudaGetLastError();
}

cudaError_t launch_best_deposit(const InstanceView &iv, const AntBuffers &ab,
                                const PheromoneView &pv, uint8_t *tau_alt, DevState *st,
                                int *gbest_nodes, int *gbest_lens, EpochRec *log,
                                cudaStream_t s) {
  const size_t smem = iv.K <= kDepositSmemRoutes ? sizeof(int) * (iv.K + 1) : 0;
  k_best_cluster<<<kBestCluster, kBestThreads, smem, s>>>(iv, ab, st, gbest_nodes, gbest_lens,
                                                          log, pv, tau_alt);
  return cudaGetLastError();
}

// Evaporation of the current pheromone buffer into the other one, run beside
// the construction (which reads only the weights): 16 bytes per thread,
// max(q, q_min + delta) - delta.
__global__ void __launch_bounds__(kEvapThreads) k_evaporate_to(PheromoneView pv,
                                                               uint8_t *tau_alt, DevState *st) {
  if (*(volatile int *)&st->skip) return;
  const bool sel = *(volatile int *)&st->tau_sel != 0;
  const uint8_t *src = sel ? tau_alt : pv.tau;
  uint8_t *dst = sel ? pv.tau : tau_alt;
  evap_sweep(src, dst, pv.total, pv.q_min, pv.delta);
}

// Blocks of an evaporation sweep over `total` bytes: one per kEvapUnroll *
// kEvapThreads vectors, at most one wave (the blocks resident on all SMs at
// once), so that large matrices are swept by a grid-stride loop.
int evap_grid_for(unsigned long long total, int num_sms) {
  static int resident = 0;
  if (resident == 0) {
    int r = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_evaporate_to, kEvapThreads, 0) !=
            cudaSuccess ||
        r < 1)
      r = 1;
    resident = r;
  }
  const unsigned long long per_block = (unsigned long long)kEvapUnroll * kEvapThreads;
  unsigned long long g = (total / 16 + per_block - 1) / per_block;
  const unsigned long long cap =
      (unsigned long long)(num_sms > 0 ? num_sms : 148) * (unsigned long long)resident;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

cudaError_t launch_evaporate_to(const PheromoneView &pv, uint8_t *tau_alt, DevState *st,
                                int grid, cudaStream_t s) {
  k_evaporate_to<<<grid, kEvapThreads, 0, s>>>(pv, tau_alt, st);
  return cudaGetLastError();
}

__global__ void k_set_run_limit(DevState *st, int limit) {
  st->run_limit = limit;
  st->stop_flags &= ~kStopRunLimit;
  if (limit > 0 && st->epoch >= limit) st->stop_flags |= kStopRunLimit;
}

cudaError_t launch_set_run_limit(DevState *st, int limit, cudaStream_t s) {
  k_set_run_limit<<<1, 1, 0, s>>>(st, limit);
  return cudaGetLastError();
}

// ===========================================================================
// Evaporation + deposit
// ===========================================================================

struct EvapArgs {
  InstanceView iv;
  PheromoneView pv;
  AntBuffers ab;
  DevState *st;
  const int *gbest_nodes;
  const int *gbest_lens;
  unsigned int *counter;
  int best_ant;          // used when st == nullptr
  float dep_iter, dep_global;
  uint8_t *tau_alt;      // second pheromone buffer of the context, or null
};

__global__ void __launch_bounds__(kEvapThreads) k_evap_deposit(EvapArgs a) {
  if (a.st) {
    if (*(volatile int *)&a.st->skip || !*(volatile int *)&a.st->found) return;
  }
  PheromoneView pv = a.pv;  // in place, on the current buffer
  pv.tau = cur_tau(a.pv.tau, a.tau_alt, a.st);
  evap_sweep(pv.tau, pv.tau, pv.total, pv.q_min, pv.delta);
  // The last block to finish the sweep deposits (threadfence reduction).
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned ticket = atomicAdd(a.counter, 1u);
    s_last = (ticket == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const size_t stride_n = (size_t)a.iv.n + 1;
  const int best = a.st ? a.st->best_ant : a.best_ant;
  const float dep_i = a.st ? a.st->dep_iter : a.dep_iter;
  const float dep_g = a.st ? a.st->dep_global : a.dep_global;
  extern __shared__ int s_off[];
  int *offs = (a.iv.K <= kDepositSmemRoutes) ? s_off : nullptr;
  deposit_solution(pv, stride_n, CompactNodes{a.ab.routes + (size_t)best * a.iv.route_stride},
                   a.ab.lens + (size_t)best * a.iv.K, a.iv.K, dep_i, offs);
  __syncthreads();
  if (a.gbest_nodes) {
    deposit_solution(pv, stride_n, CompactNodes{a.gbest_nodes}, a.gbest_lens, a.iv.K, dep_g, offs);
  }
  if (threadIdx.x == 0) *a.counter = 0u;
}

cudaError_t launch_evap_deposit(const InstanceView &iv, const PheromoneView &pv,
                                const AntBuffers &ab, DevState *st,
                                const int *gbest_nodes, const int *gbest_lens,
                                unsigned int *counter, int grid, uint8_t *tau_alt,
                                cudaStream_t s) {
  EvapArgs a;
  a.iv = iv;
  a.pv = pv;
  a.ab = ab;
  a.st = st;
  a.gbest_nodes = gbest_nodes;
  a.gbest_lens = gbest_lens;
  a.counter = counter;
  a.best_ant = 0;
  a.dep_iter = a.dep_global = 0.0f;
  a.tau_alt = tau_alt;
  const size_t smem = iv.K <= kDepositSmemRoutes ? sizeof(int) * (iv.K + 1) : 0;
  k_evap_deposit<<<grid, kEvapThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// Test-hook variant with explicit best ant and amounts (no device state).
cudaError_t launch_evap_deposit_explicit(const InstanceView &iv,
                                         const PheromoneView &pv,
                                         const AntBuffers &ab, int best_ant,
                                         float dep_iter,
                                         const int *gbest_nodes,
                                         const int *gbest_lens,
                                         float dep_global,
                                         unsigned int *counter, int grid,
                                         cudaStream_t s) {
  EvapArgs a;
  a.iv = iv;
  a.pv = pv;
  a.ab = ab;
  a.st = nullptr;
  a.gbest_nodes = gbest_nodes;
  a.gbest_lens = gbest_lens;
  a.counter = counter;
  a.best_ant = best_ant;
  a.dep_iter = dep_iter;
  a.dep_global = dep_global;
  a.tau_alt = nullptr;  // the caller passes the current buffer
  const size_t smem = iv.K <= kDepositSmemRoutes ? sizeof(int) * (iv.K + 1) : 0;
  k_evap_deposit<<<grid, kEvapThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// ===========================================================================
// Colony split over several devices: local best packet, exchange, winner
// ===========================================================================

// Packet of one device's iteration best (int32 words):
//   [0,1] cost (FP64 bits; DBL_MAX when no feasible ant)  [2] found
//   [3] global ant id  [4,5] ant-steps of all local ants  [6, 6+K) lengths
//   [6+K, 6+K+n+2K) compact route.
__host__ __device__ inline int shard_packet_ints(int n, int K) {
  return (6 + K + n + 2 * K + 3) & ~3;
}

__global__ void __launch_bounds__(1024) k_shard_pack(InstanceView iv, AntBuffers ab,
                                                     DevState *st, int *send) {
  __shared__ double s_cost[32];
  __shared__ int s_ant[32];
  __shared__ unsigned long long s_steps[32];
  __shared__ int s_best;
  const bool skip = *(volatile int *)&st->skip;
  double bc;
  int ba;
  unsigned long long steps;
  block_iter_best(ab, skip ? 0 : iv.m, s_cost, s_ant, s_steps, bc, ba, steps);
  if (threadIdx.x == 0) {
    const unsigned long long cb = (unsigned long long)__double_as_longlong(bc);
    send[0] = (int)(cb & 0xffffffffu);
    send[1] = (int)(cb >> 32);
    send[2] = (ba != INT_MAX) ? 1 : 0;
    send[3] = (ba != INT_MAX) ? ba + iv.ant_base : INT_MAX;
    send[4] = (int)(steps & 0xffffffffu);
    send[5] = (int)(steps >> 32);
    s_best = ba;
  }
  __syncthreads();
  if (s_best != INT_MAX) {
    const int *src = ab.routes + (size_t)s_best * iv.route_stride;
    const int *sl = ab.lens + (size_t)s_best * iv.K;
    for (int v = threadIdx.x; v < iv.K; v += blockDim.x) send[6 + v] = sl[v];
    int total = 0;
    for (int v = 0; v < iv.K; ++v) total += sl[v];
    for (int t = threadIdx.x; t < total; t += blockDim.x) send[6 + iv.K + t] = src[t];
  }
}

// Winner over the gathered packets (lowest cost, then lowest global ant:
// the first minimum a single device holding every ant would find), then the
// same bookkeeping as k_best; its route goes to iter_nodes/iter_lens and,
// on improvement, to the global best; then both deposits into the
// evaporated pheromone buffer and the buffer switch.
__global__ void __cluster_dims__(kBestCluster, 1, 1) __launch_bounds__(kBestThreads)
    k_shard_select(InstanceView iv, DevState *st, const int *recv, int world, int *iter_nodes,
                   int *iter_lens, int *gbest_nodes, int *gbest_lens, EpochRec *log,
                   PheromoneView pv, uint8_t *tau_alt) {
  // A cluster like k_best_cluster: every block selects the same winner and
  // deposit amounts from the same packets and state snapshot, block 0 keeps
  // the bookkeeping and the copies, the deposits' arcs are shared out over
  // the cluster with a barrier between the two deposits.
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  __shared__ DevState s_st;
  __shared__ int s_src, s_improved;
  state_load(&s_st, st);
  if (s_st.skip) return;  // the same in every block: nothing is written
  const int P = shard_packet_ints(iv.n, iv.K);
  if (threadIdx.x == 0) {
    double bc = DBL_MAX;
    int ba = INT_MAX, src = -1;
    unsigned long long steps = 0;
    for (int r = 0; r < world; ++r) {
      const int *pk = recv + (size_t)r * P;
      steps += (unsigned long long)(unsigned)pk[4] | ((unsigned long long)(unsigned)pk[5] << 32);
      if (!pk[2]) continue;
      const double c = __longlong_as_double(
          (long long)((unsigned long long)(unsigned)pk[0] | ((unsigned long long)(unsigned)pk[1] << 32)));
      const int ga = pk[3];
      if (src < 0 || c < bc || (c == bc && ga < ba)) {
        bc = c;
        ba = ga;
        src = r;
      }
    }
    s_improved = epoch_bookkeeping(&s_st, src >= 0, bc, ba, steps, rank == 0 ? log : nullptr);
    s_src = src;
  }
  __syncthreads();
  if (s_src < 0) {
    // No feasible ant anywhere: no evaporation, no deposit; every block has
    // read the state before block 0 writes it back.
    cluster.sync();
    if (rank == 0) state_store(st, &s_st);
    return;
  }
  const int *pk = recv + (size_t)s_src * P;
  const int *w_lens = pk + 6;
  const int *w_nodes = pk + 6 + iv.K;
  if (rank == 0) {
    int total = 0;
    for (int v = 0; v < iv.K; ++v) total += w_lens[v];
    for (int v = threadIdx.x; v < iv.K; v += blockDim.x) {
      iter_lens[v] = w_lens[v];
      if (s_improved) gbest_lens[v] = w_lens[v];
    }
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      iter_nodes[t] = w_nodes[t];
      if (s_improved) gbest_nodes[t] = w_nodes[t];
    }
  }
  // The deposits read the winner straight from its packet.
  cluster_deposits(cluster, rank, iv, pv, tau_alt, &s_st, st, w_nodes, w_lens,
                   s_improved ? w_nodes : gbest_nodes, s_improved ? w_lens : gbest_lens);
}

int shard_packet_size(int n, int K) { return shard_packet_ints(n, K); }

cudaError_t launch_shard_pack(const InstanceView &iv, const AntBuffers &ab, DevState *st,
                              int *send, cudaStream_t s) {
  k_shard_pack<<<1, 1024, 0, s>>>(iv, ab, st, send);
  return cudaGetLastError();
}

cudaError_t launch_shard_select(const InstanceView &iv, DevState *st, const int *recv,
                                int world, int *iter_nodes, int *iter_lens,
                                int *gbest_nodes, int *gbest_lens, EpochRec *log,
                                const PheromoneView &pv, uint8_t *tau_alt, cudaStream_t s) {
  const size_t smem = iv.K <= kDepositSmemRoutes ? sizeof(int) * (iv.K + 1) : 0;
  k_shard_select<<<kBestCluster, kBestThreads, smem, s>>>(iv, st, recv, world, iter_nodes,
                                                          iter_lens, gbest_nodes, gbest_lens,
                                                          log, pv, tau_alt);
  return cudaGetLastError();
}

}  // namespace acob200
