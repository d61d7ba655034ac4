// aco_batch.cu -- many independent instances in one persistent launch.
//
// Each block pulls instances from a queue and runs every epoch of an
// instance by itself: per-epoch weights into shared memory, the ants'
// construction (one segment of 16 or 32 lanes per ant), iteration/global
// best and stop rules, evaporation and deposit -- phases separated by
// __syncthreads only, so the whole batch is one launch with no grid-wide
// synchronisation and no host round trip.  Instance i is solved exactly as
// the single-instance path solves it with seed + i (same draws, same rules,
// same device math), which the tests check route for route.
#include "aco_internal.cuh"
#include "aco_prior_internal.h"

extern "C" {
#include "aco.h"
#include "aco_b200.h"
}

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

using namespace acob200;

namespace {

struct BatchInst {
  int n, K, cap, total_demand, max_demand;
  int unit;
  long long node_off;   // coords / demand / rows (cand, lvl at node_off * k)
  long long tau_off;    // bytes, 16-aligned
  long long route_off;  // m * (n + 2K) ints
  long long lens_off;   // m * K ints
  long long gbest_off;  // n + 2K ints
  long long gblens_off; // K ints
  long long rep_off;    // m * n ints (repair scratch)
};

struct BatchArgs {
  const BatchInst *inst;
  const int *order;          // queue order of instance ids
  int count;
  int m, k;
  int epochs, stagnation;
  double min_rel;
  float Qs, log_min, log_step;
  uint8_t delta, q_tau0, pad0, pad1;
  uint32_t seed;
  const float2 *coords;
  const int *demand;
  const uint16_t *cand, *lvl;
  const uint16_t *tier;      // [rows][kTierLen]: ranks k+1 .. k+64 (fallback)
  const int32_t *A;
  const uint32_t *lut;
  uint8_t *tau;
  int *routes, *lens, *loads, *rep, *repc;
  double *cost;
  int *feasible, *steps;
  int *gbest_nodes, *gbest_lens;
  double *out_cost;
  int *out_epochs;
  unsigned long long *out_steps;
  unsigned int *queue;       // work counter (scratch, zeroed before launch)
  int max_rows;              // smem sizing: largest n + 1
  int max_K;
};

// Shared-memory layout of a block (bytes).
struct BatchSmem {
  uint32_t off_cand, off_lvl, off_w, off_coords, off_dem, off_A, off_lut, off_draw, off_red, off_off;
  uint32_t total;
};

__host__ __device__ inline uint32_t pad16u(uint32_t b) { return (b + 15u) & ~15u; }

__host__ __device__ inline BatchSmem batch_smem(int max_rows, int k, int ants_per_block,
                                                int threads, int max_K) {
  BatchSmem s;
  uint32_t o = 0;
  s.off_cand = o; o += pad16u((uint32_t)max_rows * k * 2);
  s.off_lvl = o; o += pad16u((uint32_t)max_rows * k * 2);
  s.off_w = o; o += pad16u((uint32_t)max_rows * k * 4);
  s.off_coords = o; o += pad16u((uint32_t)max_rows * 8);
  s.off_dem = o; o += pad16u((uint32_t)max_rows * 4);
  s.off_A = o; o += 1024;
  s.off_lut = o; o += 1024;
  s.off_draw = o; o += (uint32_t)ants_per_block * 512;
  s.off_red = o; o += pad16u((uint32_t)(threads / 32) * 16 + 64);
  s.off_off = o; o += pad16u((uint32_t)(max_K + 1) * 4);
  s.total = o;
  return s;
}

// Segment collectives: a segment is LANES consecutive lanes of a warp
// (LANES = 16: two ants per warp; 32: one).  Masks name the segment only, so
// the two ants of a warp may diverge.
template <int LANES>
struct Seg {
  int lane;       // lane within the segment
  unsigned mask;  // the segment's lanes
  int base;       // first warp lane of the segment
  __device__ __forceinline__ Seg() {
    const int wl = threadIdx.x & 31;
    lane = wl & (LANES - 1);
    base = wl & ~(LANES - 1);
    mask = (LANES == 32) ? 0xffffffffu : (0xffffu << base);
  }
  template <class T>
  __device__ __forceinline__ T shfl(T v, int src) const { return __shfl_sync(mask, v, src, LANES); }
  __device__ __forceinline__ uint32_t shfl_up(uint32_t v, int d) const {
    return __shfl_up_sync(mask, v, d, LANES);
  }
  __device__ __forceinline__ unsigned ballot(bool p) const {
    return (__ballot_sync(mask, p) >> base) & (LANES == 32 ? 0xffffffffu : 0xffffu);
  }
  __device__ __forceinline__ uint32_t sum(uint32_t v) const { return __reduce_add_sync(mask, v); }
  __device__ __forceinline__ int imax(int v) const { return __reduce_max_sync(mask, v); }
  __device__ __forceinline__ uint32_t umin(uint32_t v) const { return __reduce_min_sync(mask, v); }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// Visited bitmap of one ant in the segment's registers, transposed: bit b
// of lane L's w0 is node L + LANES b, of its w1 node 32 LANES + L + LANES b
// (V = 2).  The nodes of any instance spread evenly over the lanes, which
// keeps the nearest-customer scan short.
template <int LANES, int V>
struct SegVisited {
  static constexpr int kShift = (LANES == 16) ? 4 : 5;  // log2(LANES)
  uint32_t w0, w1;
  __device__ __forceinline__ void init(const Seg<LANES> &sg, int n) {
    w0 = lane_word(sg.lane, n) | (sg.lane == 0 ? 1u : 0u);  // the depot starts visited
    w1 = (V == 2) ? lane_word(32 * LANES + sg.lane, n) : 0xffffffffu;
  }
  // Nodes first + LANES b (b = 0..31) beyond n start set.
  __device__ __forceinline__ static uint32_t lane_word(int first, int n) {
    const int cnt = n >= first ? (n - first) / LANES + 1 : 0;  // nodes <= n
    return cnt >= 32 ? 0u : (0xffffffffu << cnt);
  }
  __device__ __forceinline__ bool test(const Seg<LANES> &sg, int c) const {
    // The shuffle takes the source lane modulo the segment width.
    uint32_t word = sg.shfl(w0, c);
    if (V == 2) {
      const uint32_t hi = sg.shfl(w1, c);
      word = (c >= 32 * LANES) ? hi : word;
    }
    return __funnelshift_r(word, word, c >> kShift) & 1u;  // bit (c / LANES) mod 32
  }
  __device__ __forceinline__ void set(const Seg<LANES> &sg, int node) {
    const uint32_t bit = __funnelshift_l(0u, 1u, node >> kShift);
    if (sg.lane == (node & (LANES - 1))) {
      if (V == 2 && node >= 32 * LANES) w1 |= bit; else w0 |= bit;
    }
  }
};
template <int LANES, int V>
__device__ __forceinline__ int seg_nearest(const Seg<LANES> &sg, const SegVisited<LANES, V> &vis,
                                           const float2 *coords, const int *dem, bool unit,
                                           float2 pc, int room, bool check_dem) {
  uint32_t best_h = 0xffffffffu, best_n = 0xffffffffu;
  // Bit b of a word is node first + LANES b: ascending within a lane.
  auto scan = [&](uint32_t fr, int first) {
    while (fr) {
      const int b = __ffs(fr) - 1;
      fr &= fr - 1;
      const int node = first + b * LANES;
      if (!unit && check_dem && dem[node] > room) continue;
      const uint32_t h = __float_as_uint(dist2f(pc, coords[node]));
      if (h < best_h) {
        best_h = h;
        best_n = (uint32_t)node;
      }
    }
  };
  scan(~vis.w0, sg.lane);
  if (V == 2) scan(~vis.w1, 32 * LANES + sg.lane);
  const uint32_t mh = sg.umin(best_h);
  const uint32_t mn = sg.umin(best_h == mh ? best_n : 0xffffffffu);
  return (mh == 0xffffffffu) ? 0 : (int)mn;
}

// Smallest instance whose fallback uses the tier lists (a lane of a 16-lane
// segment walks (n+1)/16 bitmap bits in the full scan).
constexpr int kBatchTierMinCustomers = 256;

// The fallback of a row none of whose candidates has a weight, exactly as
// seg_nearest: the first eligible candidate (okm), else the first eligible
// node of the tier row (the next 64 ranks), else the scan of every node; 0
// when a complete tier row lists no eligible customer.
template <int LANES, int V>
__device__ __forceinline__ int seg_nearest_eligible(const Seg<LANES> &sg,
                                                    const SegVisited<LANES, V> &vis,
                                                    const uint16_t *tier_row, unsigned okm, int c,
                                                    const float2 *coords, const int *dem,
                                                    bool unit, float2 pc, int room,
                                                    bool check_dem) {
  if (okm) return sg.shfl(c, __ffs(okm) - 1);
  int nodes[kTierLen / LANES];
#pragma unroll
  for (int q = 0; q < kTierLen / LANES; ++q)  // every part of the row in flight at once
    nodes[q] = (int)__ldg(tier_row + q * LANES + sg.lane);
#pragma unroll
  for (int q = 0; q < kTierLen / LANES; ++q) {
    const int node = nodes[q];
    bool ok = !vis.test(sg, node);  // node 0 (empty slot) reads as visited
    if (!unit && check_dem && ok) ok = dem[node] <= room;
    const unsigned m = sg.ballot(ok);
    if (m) return sg.shfl(node, __ffs(m) - 1);
  }
  // every customer was listed
  if (sg.shfl(nodes[kTierLen / LANES - 1], LANES - 1) == 0) return 0;
  return seg_nearest<LANES, V>(sg, vis, coords, dem, unit, pc, room, check_dem);
}

__device__ __forceinline__ void seg_draw_refill(uint32_t *buf, uint32_t d, uint32_t seed,
                                                uint32_t epoch, uint32_t ant, int lane,
                                                int lanes, unsigned mask) {
  // 128 draws: lane L of the segment computes Philox blocks L, L + lanes, ...
  __syncwarp(mask);
  for (int b = lane; b < 32; b += lanes) {
    uint32_t r[4];
    philox4x32_10(((d >> 7) << 5) + (uint32_t)b, ant, epoch, 0u, seed, kDrawKey1, r);
    reinterpret_cast<uint4 *>(buf)[b] =
        make_uint4(r[0] >> (32 - kDrawBits), r[1] >> (32 - kDrawBits),
                   r[2] >> (32 - kDrawBits), r[3] >> (32 - kDrawBits));
  }
  __syncwarp(mask);
}

// One ant on one segment: the rules of build_ant in aco_kernels.cu
// (src/seq/aco_sequential.c:616-681 with the demand extension), on the
// block's shared tables.  UNIT: every customer's demand is 1 (instance flag).
template <int LANES, int V, bool UNIT>
__device__ void seg_build_ant(const BatchArgs &a, const BatchInst &I, const Seg<LANES> &sg,
                              const uint16_t *cand, const uint32_t *wt, const float2 *coords,
                              const int *dem, uint32_t *dbuf, uint32_t seed, int ant,
                              uint32_t epoch, long long ai) {
  const int k = a.k, K = I.K, n = I.n, R = n + 2 * K, cap = I.cap;
  constexpr bool unit = UNIT;
  int *route = a.routes + I.route_off + (long long)ant * R;
  int *lens = a.lens + I.lens_off + (long long)ant * K;
  int *loads = a.loads + I.lens_off + (long long)ant * K;
  SegVisited<LANES, V> vis;
  vis.init(sg, n);
  uint32_t d = 0;
  seg_draw_refill(dbuf, d, seed, epoch, (uint32_t)ant, sg.lane, LANES, sg.mask);
  uint32_t r_next = dbuf[0];
  int remaining = n, rem_dem = I.total_demand, pos = 0;
  const int tight_load = cap - I.max_demand;
  for (int v = 0; v < K; ++v) {
    const int start = pos;
    route[pos] = 0;
    ++pos;
    int cur = 0, load = 0;
    const long long fut64 = (long long)(K - v - 1) * cap;
    const int future = fut64 > 0x7fffffffLL ? 0x7fffffff : (int)fut64;
    while (rem_dem > future && load < cap) {
      // room < max demand  <=>  load > cap - max demand
      const bool tight = !unit && load > tight_load;
      int c = 0;
      uint32_t w = 0u;
      if (sg.lane < k) {
        c = cand[cur * k + sg.lane];
        w = wt[cur * k + sg.lane];
      }
      bool ok = !vis.test(sg, c);
      if (tight) ok = ok && dem[c] + load <= cap;
      const uint32_t wv = ok ? w : 0u;
      const uint32_t denom = sg.sum(wv);
      uint32_t cum = wv;
#pragma unroll
      for (int o = 1; o < LANES; o <<= 1) {
        const uint32_t t = sg.shfl_up(cum, o);
        if (sg.lane >= o) cum += t;
      }
      int next;
      if (denom != 0u) {
        const uint32_t thr =
            (uint32_t)(((unsigned long long)r_next * denom + 0xFFFFFFull) >> kDrawBits);
        const unsigned msk = sg.ballot(wv != 0u && cum >= thr);
        next = sg.shfl(c, __ffs(msk) - 1);  // msk != 0 when denom != 0
        ++d;
        if ((d & 127u) == 0u) seg_draw_refill(dbuf, d, seed, epoch, (uint32_t)ant, sg.lane, LANES, sg.mask);
        r_next = dbuf[d & 127u];
      } else {
        next = (n >= kBatchTierMinCustomers)
                   ? seg_nearest_eligible<LANES, V>(
                         sg, vis, a.tier + (size_t)(I.node_off + cur) * kTierLen, sg.ballot(ok),
                         c, coords, dem, unit, coords[cur], cap - load, tight)
                   : seg_nearest<LANES, V>(sg, vis, coords, dem, unit, coords[cur], cap - load,
                                           tight);
        if (next <= 0) break;
      }
      route[pos] = next;
      vis.set(sg, next);
      ++pos;
      --remaining;
      const int dn = unit ? 1 : dem[next];
      load += dn;
      rem_dem -= dn;
      cur = next;
    }
    route[pos] = 0;
    if (sg.lane == 0) {
      lens[v] = pos + 1 - start;
      loads[v] = load;
    }
    ++pos;
  }
  if (remaining > 0) {
    // Backward repair (aco_sequential.c:659-680), as in build_ant.
    sg.sync();
    int *rep = a.rep + I.rep_off + (long long)ant * n;
    int *repc = a.repc + I.lens_off + (long long)ant * K;
    for (int v = sg.lane; v < K; v += LANES) repc[v] = 0;
    sg.sync();
    int nrep = 0, off_end = pos;
    for (int v = K - 1; v >= 0 && remaining > 0; --v) {
      const int len_v = lens[v];
      off_end -= len_v;
      int cur = route[off_end + len_v - 2];
      int load = loads[v], cnt = 0;
      while (remaining > 0 && load < cap) {
        const int next = seg_nearest<LANES, V>(sg, vis, coords, dem, unit, coords[cur],
                                               cap - load, true);
        if (next <= 0) break;
        if (sg.lane == 0) rep[nrep + cnt] = next;
        vis.set(sg, next);
        ++cnt;
        load += unit ? 1 : dem[next];
        --remaining;
        cur = next;
      }
      if (sg.lane == 0) repc[v] = cnt;
      nrep += cnt;
    }
    sg.sync();
    if (sg.lane == 0 && nrep > 0) {
      int off_total = pos, add_after = 0, shift = nrep;
      for (int v = K - 1; v >= 0; --v) {
        const int len_v = lens[v];
        off_total -= len_v;
        const int cnt = repc[v];
        shift -= cnt;
        const int old_off = off_total, new_off = off_total + shift, main_len = len_v - 1;
        for (int t = main_len - 1; t >= 0; --t) route[new_off + t] = route[old_off + t];
        for (int j = 0; j < cnt; ++j) route[new_off + main_len + j] = rep[add_after + j];
        route[new_off + main_len + cnt] = 0;
        lens[v] = len_v + cnt;
        add_after += cnt;
      }
    }
    pos += nrep;
  }
  sg.sync();
  // FP64 cost in route order (boundary (0,0) pairs add +0.0).
  // The next LANES arcs' end points are loaded while the current ones are
  // summed.
  double acc = 0.0;
  const int arcs = pos - 1;
  int ru = 0, rv = 0;
  if (sg.lane < arcs) {
    ru = route[sg.lane];
    rv = route[sg.lane + 1];
  }
  for (int b = 0; b < arcs; b += LANES) {
    double dj = 0.0;
    if (b + sg.lane < arcs) dj = dist64(coords[ru], coords[rv]);
    const int j2 = b + LANES + sg.lane;
    if (j2 < arcs) {
      ru = route[j2];
      rv = route[j2 + 1];
    }
    if (arcs - b >= LANES) {
#pragma unroll
      for (int t = 0; t < LANES; ++t) acc = __dadd_rn(acc, sg.shfl(dj, t));
    } else {
      const int cnt = arcs - b;
      for (int t = 0; t < cnt; ++t) acc = __dadd_rn(acc, sg.shfl(dj, t));
    }
  }
  if (sg.lane == 0) {
    a.cost[ai] = acc;
    a.feasible[ai] = remaining == 0 ? 1 : 0;
    a.steps[ai] = pos - K;
  }
}

// is_significant_improvement, src/cuda/aco_cuda.cu:83-94.
__device__ __forceinline__ bool b_significant(double prev, double next, double min_rel) {
  if (prev >= DBL_MAX || next >= DBL_MAX) return next < prev;
  if (next >= __dsub_rn(prev, 1e-9)) return false;
  const double rel = __ddiv_rn(__dsub_rn(prev, next), fmax(prev, 1e-9));
  return __dadd_rn(rel, 1e-9) >= min_rel;
}

template <int LANES, int V>
__global__ void __launch_bounds__(1024) k_batch_solve(BatchArgs a, BatchSmem ly,
                                                      int ants_per_block) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t *s_cand = reinterpret_cast<uint16_t *>(smem + ly.off_cand);
  uint16_t *s_lvl = reinterpret_cast<uint16_t *>(smem + ly.off_lvl);
  uint32_t *s_w = reinterpret_cast<uint32_t *>(smem + ly.off_w);
  float2 *s_coords = reinterpret_cast<float2 *>(smem + ly.off_coords);
  int *s_dem = reinterpret_cast<int *>(smem + ly.off_dem);
  int32_t *s_A = reinterpret_cast<int32_t *>(smem + ly.off_A);
  uint32_t *s_lut = reinterpret_cast<uint32_t *>(smem + ly.off_lut);
  double *s_redc = reinterpret_cast<double *>(smem + ly.off_red);
  int *s_reda = reinterpret_cast<int *>(smem + ly.off_red + (blockDim.x / 32) * 8);
  int *s_off = reinterpret_cast<int *>(smem + ly.off_off);
  __shared__ int s_inst, s_best, s_found, s_improved, s_stop;
  __shared__ double s_gbest;
  __shared__ int s_since;
  __shared__ float s_dep_i, s_dep_g;
  __shared__ unsigned long long s_steps;

  const int tid = threadIdx.x, nthr = blockDim.x;
  const int warp = tid >> 5, nwarps = nthr >> 5;
  const Seg<LANES> sg;
  const int seg = tid / LANES;  // ant slot of this segment
  for (int i = tid; i < 256; i += nthr) {
    s_A[i] = a.A[i];
    s_lut[i] = a.lut[i];
  }
  while (true) {
    __syncthreads();
    if (tid == 0) {
      const unsigned q = atomicAdd(a.queue, 1u);
      s_inst = (q < (unsigned)a.count) ? a.order[q] : -1;
    }
    __syncthreads();
    const int ii = s_inst;
    if (ii < 0) return;
    const BatchInst I = a.inst[ii];
    const int n = I.n, k = a.k, rows = n + 1, K = I.K;
    const size_t stride = (size_t)n + 1;
    const uint32_t seed = a.seed + (uint32_t)ii;
    uint8_t *tau = a.tau + I.tau_off;
    // Stage the instance.
    for (int e = tid; e < rows * k; e += nthr) {
      s_cand[e] = a.cand[I.node_off * k + e];
      s_lvl[e] = a.lvl[I.node_off * k + e];
    }
    for (int e = tid; e < rows; e += nthr) {
      s_coords[e] = a.coords[I.node_off + e];
      s_dem[e] = a.demand[I.node_off + e];
    }
    {
      const unsigned long long total = (unsigned long long)rows * rows;
      const uint32_t w4 = 0x01010101u * a.q_tau0;
      uint4 *t4 = reinterpret_cast<uint4 *>(tau);
      for (unsigned long long e = tid; e < total / 16; e += nthr) __stcg(t4 + e, make_uint4(w4, w4, w4, w4));
      for (unsigned long long e = total / 16 * 16 + tid; e < total; e += nthr) st_cg_u8(tau + e, a.q_tau0);
    }
    if (tid == 0) {
      s_gbest = DBL_MAX;
      s_since = 0;
      s_stop = 0;
      s_steps = 0ull;
    }
    __syncthreads();
    int epoch = 0;
    for (; epoch < a.epochs && !s_stop; ++epoch) {
      // Weights (k_weights): segment per row.
      for (int r = seg; r < rows; r += nthr / LANES) {
        int c = 0, e = INT_MIN;
        if (sg.lane < k) {
          c = s_cand[r * k + sg.lane];
          if (c > 0) e = s_A[ld_cg_u8(tau + (size_t)r * stride + c)] - (int)s_lvl[r * k + sg.lane];
        }
        const int emax = sg.imax(e);
        if (sg.lane < k) {
          uint32_t w = 0u;
          if (c > 0) {
            const int rr = emax - e;
            w = s_lut[rr > kRelMax ? kRelMax : rr];
          }
          s_w[r * k + sg.lane] = w;
        }
      }
      __syncthreads();
      // Construction, ants_per_block ants at a time.
      uint32_t *dbuf = reinterpret_cast<uint32_t *>(smem + ly.off_draw) + seg * 128;
      for (int a0 = 0; a0 < a.m; a0 += ants_per_block) {
        const int ant = a0 + seg;
        if (seg < ants_per_block && ant < a.m) {
          const long long ai = (long long)ii * a.m + ant;
          if (I.unit) {
            if (V == 1) seg_build_ant<LANES, 1, true>(a, I, sg, s_cand, s_w, s_coords, s_dem, dbuf, seed, ant, (uint32_t)epoch, ai);
            else seg_build_ant<LANES, 2, true>(a, I, sg, s_cand, s_w, s_coords, s_dem, dbuf, seed, ant, (uint32_t)epoch, ai);
          } else {
            if (V == 1) seg_build_ant<LANES, 1, false>(a, I, sg, s_cand, s_w, s_coords, s_dem, dbuf, seed, ant, (uint32_t)epoch, ai);
            else seg_build_ant<LANES, 2, false>(a, I, sg, s_cand, s_w, s_coords, s_dem, dbuf, seed, ant, (uint32_t)epoch, ai);
          }
        }
      }
      __syncthreads();
      // Iteration best: first minimum among feasible ants (k_best).
      {
        double bc = DBL_MAX;
        int ba = INT_MAX;
        unsigned long long st = 0;
        for (int i = tid; i < a.m; i += nthr) {
          const long long ai = (long long)ii * a.m + i;
          st += (unsigned long long)a.steps[ai];
          if (a.feasible[ai]) {
            const double c = a.cost[ai];
            if (ba == INT_MAX || c < bc) {
              bc = c;
              ba = i;
            }
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double oc = __shfl_down_sync(kFull, bc, o);
          const int oa = __shfl_down_sync(kFull, ba, o);
          st += __shfl_down_sync(kFull, st, o);
          if (oa != INT_MAX && (ba == INT_MAX || oc < bc || (oc == bc && oa < ba))) {
            bc = oc;
            ba = oa;
          }
        }
        if ((tid & 31) == 0) {
          s_redc[warp] = bc;
          s_reda[warp] = ba;
          atomicAdd(&s_steps, st);
        }
        __syncthreads();
        if (tid == 0) {
          bc = DBL_MAX;
          ba = INT_MAX;
          for (int w = 0; w < nwarps; ++w) {
            const double oc = s_redc[w];
            const int oa = s_reda[w];
            if (oa != INT_MAX && (ba == INT_MAX || oc < bc || (oc == bc && oa < ba))) {
              bc = oc;
              ba = oa;
            }
          }
          const bool found = ba != INT_MAX;
          s_found = found;
          s_improved = 0;
          s_best = ba;
          if (found) {
            if (bc < s_gbest) {
              s_improved = 1;
              if (b_significant(s_gbest, bc, a.min_rel)) s_since = 0; else s_since += 1;
              s_gbest = bc;
            } else {
              s_since += 1;
            }
            s_dep_i = __fdiv_rn(0.3f * a.Qs, (float)bc);
            s_dep_g = __fdiv_rn(0.7f * a.Qs, (float)s_gbest);
          } else {
            s_since += 1;
          }
          if (a.stagnation > 0 && s_since >= a.stagnation) s_stop = 1;
        }
        __syncthreads();
      }
      const int R = n + 2 * K;
      if (s_improved) {
        const int *src = a.routes + I.route_off + (long long)s_best * R;
        const int *sl = a.lens + I.lens_off + (long long)s_best * K;
        int total = 0;
        for (int v = 0; v < K; ++v) total += sl[v];
        for (int t = tid; t < total; t += nthr) a.gbest_nodes[I.gbest_off + t] = src[t];
        for (int v = tid; v < K; v += nthr) a.gbest_lens[I.gblens_off + v] = sl[v];
      }
      __syncthreads();
      if (s_found) {
        // Evaporation (k_evap_deposit's sweep), then both deposits.
        PheromoneView pv;
        pv.tau = tau;
        pv.total = (unsigned long long)rows * rows;
        pv.log_min = a.log_min;
        pv.log_step = a.log_step;
        pv.q_min = 0;
        pv.q_max = 255;
        pv.delta = a.delta;
        pv.pad = 0;
        const int fl = (int)a.delta;
        const uint32_t floor4 = 0x01010101u * (uint32_t)fl, delta4 = 0x01010101u * a.delta;
        uint4 *t4 = reinterpret_cast<uint4 *>(tau);
        const unsigned long long nvec = pv.total / 16;
        for (unsigned long long e = tid; e < nvec; e += nthr) {
          uint4 x = __ldcg(t4 + e);
          x.x = __vsub4(__vmaxu4(x.x, floor4), delta4);
          x.y = __vsub4(__vmaxu4(x.y, floor4), delta4);
          x.z = __vsub4(__vmaxu4(x.z, floor4), delta4);
          x.w = __vsub4(__vmaxu4(x.w, floor4), delta4);
          __stcg(t4 + e, x);
        }
        for (unsigned long long e = nvec * 16 + tid; e < pv.total; e += nthr) {
          const uint8_t q = ld_cg_u8(tau + e);
          st_cg_u8(tau + e, ((int)q > fl) ? (uint8_t)(q - a.delta) : (uint8_t)0);
        }
        __syncthreads();
        deposit_solution(pv, stride,
                         CompactNodes{a.routes + I.route_off + (long long)s_best * R},
                         a.lens + I.lens_off + (long long)s_best * K, K, s_dep_i,
                         K <= a.max_K ? s_off : nullptr);
        __syncthreads();
        deposit_solution(pv, stride, CompactNodes{a.gbest_nodes + I.gbest_off},
                         a.gbest_lens + I.gblens_off, K, s_dep_g,
                         K <= a.max_K ? s_off : nullptr);
        __syncthreads();
      }
    }
    if (tid == 0) {
      a.out_cost[ii] = s_gbest;
      a.out_epochs[ii] = epoch;
      a.out_steps[ii] = s_steps;
    }
  }
}

template <int LANES>
cudaError_t launch_batch_lanes(const BatchArgs &a, const BatchSmem &ly, int grid, int threads,
                               int apb, int v, cudaStream_t s) {
  if (v == 1) k_batch_solve<LANES, 1><<<grid, threads, ly.total, s>>>(a, ly, apb);
  else k_batch_solve<LANES, 2><<<grid, threads, ly.total, s>>>(a, ly, apb);
  return cudaGetLastError();
}

// Opts the kernel into the largest dynamic shared memory its static shared
// variables leave free.
template <int LANES, int V>
cudaError_t configure_batch() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, k_batch_solve<LANES, V>);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_batch_solve<LANES, V>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              construct_max_smem() - (int)fa.sharedSizeBytes);
}

template <int LANES, int V>
int batch_static_smem() {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_batch_solve<LANES, V>) != cudaSuccess) return 1 << 20;
  return (int)fa.sharedSizeBytes;
}

template <int LANES, int V>
int occupancy_batch(int threads, size_t smem) {
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_batch_solve<LANES, V>, threads, smem);
  return blocks;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct aco_b200_batch {
  int device = 0, num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  bool ready = false;
  int count = 0, m = 0, k = 0, epochs = 0, max_rows = 0, max_K = 0, max_n = 0;
  BatchArgs args = {};
  std::vector<BatchInst> inst;
  std::vector<int> sizes;  // work estimate per instance
  // Every device buffer is a 256-byte aligned slice of one allocation; a
  // set-up reuses it while the new batch fits, so solving a stream of
  // batches allocates once.
  unsigned char *arena = nullptr;
  size_t arena_cap = 0, arena_used = 0;
  bool sizing = false;
  aco_b200_batch_tuning tuning = {32, 16, 1};
  // The solve (queue reset + persistent launch) as a CUDA graph, kept while
  // the launch's arguments are unchanged.
  cudaGraphExec_t graph = nullptr;
  std::vector<unsigned char> graph_key;
  const float *d_thr = nullptr;  // eta thresholds (plain levels)
  const long long *d_seg_off = nullptr;  // first row of every instance
  const int *d_seg_n = nullptr;          // customers of every instance
  long long rows = 0;                    // sum of n + 1
  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_key.clear();
  }
  void free_all() {
    drop_graph();
    if (arena) cudaFree(arena);
    arena = nullptr;
    arena_cap = arena_used = 0;
    ready = false;
  }
  template <typename T>
  void carve(T **p, size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    *p = sizing ? nullptr : reinterpret_cast<T *>(arena + arena_used);
    arena_used += bytes;
  }
};

#define BTRY(call)                                                                     \
  do {                                                                                 \
    cudaError_t err__ = (call);                                                        \
    if (err__ != cudaSuccess) {                                                        \
      fprintf(stderr, "aco_b200_batch: CUDA error %s at %s:%d\n",                      \
              cudaGetErrorString(err__), __FILE__, __LINE__);                          \
      return err__ == cudaErrorMemoryAllocation ? ACO_ERR_ALLOCATION : ACO_ERR_BACKEND; \
    }                                                                                  \
  } while (0)

static int batch_v_for(int lanes, int max_rows) {
  const int words = (max_rows + 31) / 32;
  if (words <= lanes) return 1;
  if (words <= 2 * lanes) return 2;
  return 0;
}

extern "C" {

int aco_b200_batch_create(aco_b200_batch **out, int device) {
  if (!out) return ACO_ERR_INVALID_INPUT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    return ACO_ERR_BACKEND;
  aco_b200_batch *b = new aco_b200_batch();
  b->device = device;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = configure_batch<16, 1>();
  if (e == cudaSuccess) e = configure_batch<16, 2>();
  if (e == cudaSuccess) e = configure_batch<32, 1>();
  if (e == cudaSuccess) e = configure_batch<32, 2>();
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_batch_create: %s\n", cudaGetErrorString(e));
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return ACO_ERR_BACKEND;
  }
  *out = b;
  return ACO_OK;
}

int aco_b200_batch_destroy(aco_b200_batch *b) {
  if (!b) return ACO_OK;
  cudaSetDevice(b->device);
  b->free_all();
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return ACO_OK;
}

int aco_b200_batch_set_stream(aco_b200_batch *b, void *cuda_stream) {
  if (!b) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  b->drop_graph();
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  if (cuda_stream) {
    b->stream = (cudaStream_t)cuda_stream;
    b->own_stream = false;
  } else {
    BTRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  return ACO_OK;
}

int aco_b200_batch_setup(aco_b200_batch *b, const aco_b200_batch_problem *p) {
  if (!b || !p || p->count <= 0 || !p->n || !p->K || !p->capacity || !p->x || !p->y)
    return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  b->ready = false;
  const int count = p->count;
  int k = p->cand_k > 0 ? p->cand_k : 32;
  if (k > kMaxCand) k = kMaxCand;
  const int m = p->ants > 0 ? p->ants : 64;
  b->inst.assign(count, BatchInst{});
  b->sizes.assign(count, 0);
  long long node = 0, taub = 0, route = 0, lensn = 0, gb = 0, gbl = 0, rep = 0;
  int max_rows = 0, max_K = 0, max_n = 0;
  std::vector<float2> xy;
  std::vector<int> dem;
  std::vector<long long> seg_off(count);
  std::vector<int> seg_n(count);
  for (int i = 0; i < count; ++i) {
    const int n = p->n[i], K = p->K[i];
    const long long cap = p->capacity[i];
    if (n < 1 || K < 1 || cap < 1 || cap > 0x7fffffffLL || n < k) {
      fprintf(stderr, "aco_b200_batch: instance %d invalid (n=%d K=%d cap=%lld, k=%d)\n", i, n,
              K, cap, k);
      return ACO_ERR_INVALID_INPUT;
    }
    BatchInst &I = b->inst[i];
    I.n = n;
    I.K = K;
    I.cap = (int)cap;
    long long tot = 0;
    int mx = 1;
    bool unit = true;
    for (int j = 0; j <= n; ++j) {
      const int d = p->demand ? p->demand[node + j] : (j ? 1 : 0);
      if ((j == 0 && d != 0) || (j > 0 && d < 1)) return ACO_ERR_INVALID_INPUT;
      if (j > 0) {
        tot += d;
        mx = d > mx ? d : mx;
        unit = unit && d == 1;
      }
      xy.push_back(make_float2(p->x[node + j], p->y[node + j]));
      dem.push_back(d);
    }
    if (tot > 0x7fffffffLL) return ACO_ERR_INVALID_INPUT;
    I.total_demand = (int)tot;
    I.max_demand = mx;
    I.unit = unit ? 1 : 0;
    I.node_off = node;
    seg_off[i] = node;
    seg_n[i] = n;
    I.tau_off = taub;
    I.route_off = route;
    I.lens_off = lensn;
    I.gbest_off = gb;
    I.gblens_off = gbl;
    I.rep_off = rep;
    node += n + 1;
    taub += (((long long)(n + 1) * (n + 1)) + 15) & ~15LL;
    route += (long long)m * (n + 2 * K);
    lensn += (long long)m * K;
    gb += n + 2 * K;
    gbl += K;
    rep += (long long)m * n;
    max_rows = std::max(max_rows, n + 1);
    max_K = std::max(max_K, K);
    max_n = std::max(max_n, n);
    b->sizes[i] = (n + K) * m;
  }
  if (batch_v_for(16, max_rows) == 0 && batch_v_for(32, max_rows) == 0) {
    fprintf(stderr, "aco_b200_batch: n <= 2046 per instance\n");
    return ACO_ERR_INVALID_INPUT;
  }
  b->count = count;
  b->m = m;
  b->k = k;
  b->epochs = p->epochs;
  b->max_rows = max_rows;
  b->max_K = max_K;
  b->max_n = max_n;

  float lmin = logf(0.0001f), lmax = logf(100.0f);
  float step = (lmax - lmin) / 255.0f;
  const float log_rho = logf(1.0f - (float)p->rho);
  uint8_t delta = (uint8_t)fmaxf(1.0f, roundf(-log_rho / step));
  uint8_t q0 = (uint8_t)fmaxf(0.0f, fminf(255.0f, roundf((logf((float)p->tau0) - lmin) / step)));
  // Tables as in the single-instance set-up.
  std::vector<int32_t> A(256);
  std::vector<uint32_t> lut(256);
  std::vector<float> thr(kThresholds, INFINITY);
  const double ln2 = 0.69314718055994530942;
  for (int q = 0; q < 256; ++q)
    A[q] = (int32_t)std::floor(p->alpha * (double)q * (double)step * kLevelsPerOctave / ln2 + 0.5);
  for (int r = 0; r < kRelMax; ++r)
    lut[r] = (uint32_t)std::floor(8388608.0 * std::exp2(-(double)r / kLevelsPerOctave) + 0.5);
  lut[kRelMax] = 0u;
  if (p->beta > 0.0)
    for (int j = 1; j <= kThresholds; ++j) {
      const double t = std::exp2(2.0 * (double)j / (p->beta * kLevelsPerOctave));
      thr[j - 1] = (t > 3.0e38) ? INFINITY : (float)t;
    }

  BatchArgs &a = b->args;
  a = BatchArgs{};
  a.count = count;
  a.m = m;
  a.k = k;
  a.epochs = p->epochs;
  a.stagnation = p->stagnation_epochs > 0 ? p->stagnation_epochs : 0;
  a.min_rel = p->min_rel_improvement > 0.0 ? p->min_rel_improvement : 1e-3;
  a.Qs = (float)p->Q * 100.0f;
  a.log_min = lmin;
  a.log_step = step;
  a.delta = delta;
  a.q_tau0 = q0;
  a.seed = p->seed;
  a.max_rows = max_rows;
  a.max_K = max_K;
  BatchInst *d_inst;
  int *d_order;
  float2 *d_coords;
  int *d_dem;
  uint16_t *d_cand, *d_lvl, *d_tier;
  int32_t *d_A;
  uint32_t *d_lut;
  float *d_thr;
  long long *d_soff;
  int *d_sn;
  auto layout = [&]() {
    b->arena_used = 0;
    b->carve(&d_inst, count);
    b->carve(&d_order, count);
    b->carve(&d_coords, node);
    b->carve(&d_dem, node);
    // Candidate tables sized for the longest list, so that
    // aco_b200_batch_set_cand_k can rebuild them with any length in place.
    b->carve(&d_cand, node * kMaxCand);
    b->carve(&d_lvl, node * kMaxCand);
    b->carve(&d_tier, node * kTierLen);
    b->carve(&d_A, 256);
    b->carve(&d_lut, 256);
    b->carve(&d_thr, kThresholds);
    b->carve(&d_soff, count);
    b->carve(&d_sn, count);
    b->carve(&a.tau, taub);
    b->carve(&a.routes, route);
    b->carve(&a.lens, lensn);
    b->carve(&a.loads, lensn);
    b->carve(&a.repc, lensn);
    b->carve(&a.rep, rep);
    b->carve(&a.cost, (long long)count * m);
    b->carve(&a.feasible, (long long)count * m);
    b->carve(&a.steps, (long long)count * m);
    b->carve(&a.gbest_nodes, gb);
    b->carve(&a.gbest_lens, gbl);
    b->carve(&a.out_cost, count);
    b->carve(&a.out_epochs, count);
    b->carve(&a.out_steps, count);
    b->carve(&a.queue, 1);
  };
  b->sizing = true;
  layout();
  b->sizing = false;
  const size_t need = b->arena_used;
  if (need > b->arena_cap) {
    b->free_all();
    BTRY(cudaMalloc((void **)&b->arena, need));
    b->arena_cap = need;
  }
  layout();
  cudaStream_t s = b->stream;
  BTRY(cudaMemsetAsync(b->arena, 0, need, s));
  BTRY(cudaMemcpyAsync(d_inst, b->inst.data(), sizeof(BatchInst) * count, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_coords, xy.data(), sizeof(float2) * node, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_dem, dem.data(), sizeof(int) * node, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_A, A.data(), 1024, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_lut, lut.data(), 1024, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_thr, thr.data(), sizeof(float) * kThresholds, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_soff, seg_off.data(), sizeof(long long) * count, cudaMemcpyHostToDevice, s));
  BTRY(cudaMemcpyAsync(d_sn, seg_n.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
  BTRY(launch_knn_levels_multi(d_coords, d_soff, d_sn, count, node, k, d_thr, kThresholds, d_cand,
                               d_lvl, s));
  BTRY(launch_knn_tier_multi(d_coords, d_soff, d_sn, count, node, k, d_tier, s));
  b->d_seg_off = d_soff;
  b->d_seg_n = d_sn;
  b->rows = node;
  b->d_thr = d_thr;
  a.inst = d_inst;
  a.order = d_order;
  a.coords = d_coords;
  a.demand = d_dem;
  a.cand = d_cand;
  a.lvl = d_lvl;
  a.tier = d_tier;
  a.A = d_A;
  a.lut = d_lut;
  BTRY(cudaStreamSynchronize(s));
  b->ready = true;
  aco_b200_batch_tuning t = {32, 16, 1};
  return aco_b200_batch_set_tuning(b, &t);
}

int aco_b200_batch_set_tuning(aco_b200_batch *b, const aco_b200_batch_tuning *t) {
  if (!b || !b->ready || !t) return ACO_ERR_INVALID_INPUT;
  if (t->lanes_per_ant != 16 && t->lanes_per_ant != 32) return ACO_ERR_INVALID_INPUT;
  if (t->lanes_per_ant < b->k) return ACO_ERR_INVALID_INPUT;
  if (t->ants_per_block < 1 || t->ants_per_block * t->lanes_per_ant > 1024) return ACO_ERR_INVALID_INPUT;
  if ((t->ants_per_block * t->lanes_per_ant) % 32) return ACO_ERR_INVALID_INPUT;
  if (batch_v_for(t->lanes_per_ant, b->max_rows) == 0) return ACO_ERR_INVALID_INPUT;
  const int threads = t->ants_per_block * t->lanes_per_ant;
  const BatchSmem ly = batch_smem(b->max_rows, b->k, t->ants_per_block, threads, b->max_K);
  if ((int)ly.total + batch_static_smem<32, 2>() > construct_max_smem()) return ACO_ERR_INVALID_INPUT;
  // Queue order: 0 = as given, 1 = largest work first.
  std::vector<int> order(b->count);
  std::iota(order.begin(), order.end(), 0);
  if (t->order == 1)
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b->sizes[x] > b->sizes[y]; });
  cudaSetDevice(b->device);
  // Stream-ordered after any solve in flight; a pageable source is staged
  // before the call returns.
  BTRY(cudaMemcpyAsync(const_cast<int *>(b->args.order), order.data(), sizeof(int) * b->count,
                       cudaMemcpyHostToDevice, b->stream));
  b->tuning = *t;
  return ACO_OK;
}

int aco_b200_batch_get_tuning(aco_b200_batch *b, aco_b200_batch_tuning *t) {
  if (!b || !b->ready || !t) return ACO_ERR_INVALID_INPUT;
  *t = b->tuning;
  return ACO_OK;
}

int aco_b200_batch_enqueue(aco_b200_batch *b) {
  if (!b || !b->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  const aco_b200_batch_tuning &t = b->tuning;
  const int threads = t.ants_per_block * t.lanes_per_ant;
  const BatchSmem ly = batch_smem(b->max_rows, b->k, t.ants_per_block, threads, b->max_K);
  const int v = batch_v_for(t.lanes_per_ant, b->max_rows);
  int per_sm = 0;
  if (t.lanes_per_ant == 16) per_sm = v == 1 ? occupancy_batch<16, 1>(threads, ly.total) : occupancy_batch<16, 2>(threads, ly.total);
  else per_sm = v == 1 ? occupancy_batch<32, 1>(threads, ly.total) : occupancy_batch<32, 2>(threads, ly.total);
  if (per_sm < 1) return ACO_ERR_INVALID_INPUT;
  int grid = per_sm * b->num_sms;
  if (grid > b->count) grid = b->count;
  auto record = [&](cudaStream_t s) -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(b->args.queue, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    return (t.lanes_per_ant == 16)
               ? launch_batch_lanes<16>(b->args, ly, grid, threads, t.ants_per_block, v, s)
               : launch_batch_lanes<32>(b->args, ly, grid, threads, t.ants_per_block, v, s);
  };
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BTRY(cudaStreamIsCapturing(b->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    // The caller is capturing this stream into a graph of its own: record
    // the solve there.
    BTRY(record(b->stream));
    return ACO_OK;
  }
  // The key: every argument of the two graph nodes.
  std::vector<unsigned char> key(sizeof(BatchArgs) + sizeof(BatchSmem) + 4 * sizeof(int));
  const int shape[4] = {grid, threads, t.ants_per_block, v * 64 + t.lanes_per_ant};
  memcpy(key.data(), &b->args, sizeof(BatchArgs));
  memcpy(key.data() + sizeof(BatchArgs), &ly, sizeof(BatchSmem));
  memcpy(key.data() + sizeof(BatchArgs) + sizeof(BatchSmem), shape, sizeof(shape));
  if (!b->graph || key != b->graph_key) {
    b->drop_graph();
    cudaGraph_t g = nullptr;
    BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t err = record(b->stream);
    const cudaError_t end = cudaStreamEndCapture(b->stream, &g);
    if (err != cudaSuccess || end != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      BTRY(err != cudaSuccess ? err : end);
    }
    const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) b->graph = nullptr;
    BTRY(ie);
    b->graph_key = key;
  }
  BTRY(cudaGraphLaunch(b->graph, b->stream));
  return ACO_OK;
}

int aco_b200_batch_solve(aco_b200_batch *b) {
  int rc = aco_b200_batch_enqueue(b);
  if (rc) return rc;
  BTRY(cudaStreamSynchronize(b->stream));
  return ACO_OK;
}

int aco_b200_batch_synchronize(aco_b200_batch *b) {
  if (!b) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  BTRY(cudaStreamSynchronize(b->stream));
  return ACO_OK;
}

int aco_b200_batch_autotune(aco_b200_batch *b, int trial_epochs, aco_b200_batch_tuning *chosen,
                            float *trial_ms, int max_trials, int *n_trials) {
  if (!b || !b->ready || trial_epochs < 1) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  const int saved_epochs = b->args.epochs;
  b->args.epochs = trial_epochs;
  const aco_b200_batch_tuning cands[] = {
      {32, 8, 1}, {32, 16, 1}, {32, 32, 1}, {16, 16, 1}, {16, 32, 1}, {16, 64, 1},
      {32, 16, 0}, {16, 32, 0}};
  float best_ms = 1e30f;
  aco_b200_batch_tuning best = b->tuning;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int nt = 0;
  for (const auto &c : cands) {
    if (aco_b200_batch_set_tuning(b, &c) != ACO_OK) continue;
    float ms = -1.f;
    cudaEventRecord(e0, b->stream);
    int rc = aco_b200_batch_enqueue(b);
    cudaEventRecord(e1, b->stream);
    if (rc == ACO_OK && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (trial_ms && nt < max_trials) trial_ms[nt] = ms;
    ++nt;
    if (ms > 0.f && ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->args.epochs = saved_epochs;
  if (n_trials) *n_trials = nt;
  int rc = aco_b200_batch_set_tuning(b, &best);
  if (chosen) *chosen = best;
  return rc;
}

int aco_b200_batch_set_cand_k(aco_b200_batch *b, int k) {
  if (!b || !b->ready || k < 1 || k > kMaxCand) return ACO_ERR_INVALID_INPUT;
  for (const BatchInst &I : b->inst)
    if (I.n < k) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  BatchArgs &a = b->args;
  BTRY(launch_knn_levels_multi(a.coords, b->d_seg_off, b->d_seg_n, b->count, b->rows, k,
                               b->d_thr, kThresholds, const_cast<uint16_t *>(a.cand),
                               const_cast<uint16_t *>(a.lvl), b->stream));
  BTRY(launch_knn_tier_multi(a.coords, b->d_seg_off, b->d_seg_n, b->count, b->rows, k,
                             const_cast<uint16_t *>(a.tier), b->stream));
  b->k = k;
  a.k = k;
  // The launch shape must hold the new list: keep it when it does, else the
  // default shape (32 lanes per ant).
  aco_b200_batch_tuning t = b->tuning;
  if (aco_b200_batch_set_tuning(b, &t) != ACO_OK) {
    t = aco_b200_batch_tuning{32, 16, 1};
    const int rc = aco_b200_batch_set_tuning(b, &t);
    if (rc) return rc;
  }
  BTRY(cudaStreamSynchronize(b->stream));
  return ACO_OK;
}

int aco_b200_batch_get_cand_k(aco_b200_batch *b, int *k) {
  if (!b || !b->ready || !k) return ACO_ERR_INVALID_INPUT;
  *k = b->k;
  return ACO_OK;
}

int aco_b200_batch_autotune_k(aco_b200_batch *b, int trial_epochs, const int *ks, int nks,
                              double quality_tol, aco_b200_batch_tuning *chosen, int *chosen_k,
                              double *k_solve_ms, double *k_mean_cost, int *k_feasible,
                              float *trial_ms, int max_trials, int *n_trials) {
  if (!b || !b->ready || !ks || nks < 1 || nks > 16 || !(quality_tol >= 0.0))
    return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  const int count = b->count;
  std::vector<std::vector<double>> costs(nks);
  std::vector<double> ms(nks, -1.0);
  std::vector<int> valid(nks, 0);
  cudaEvent_t e0, e1;
  BTRY(cudaEventCreate(&e0));
  BTRY(cudaEventCreate(&e1));
  // Stage 1: one whole solve per candidate-list length, on the default
  // launch shape (the shape does not change results, the length does).
  for (int i = 0; i < nks; ++i) {
    if (aco_b200_batch_set_cand_k(b, ks[i]) != ACO_OK) continue;
    aco_b200_batch_tuning t = {32, 16, 1};
    if (aco_b200_batch_set_tuning(b, &t) != ACO_OK) continue;
    cudaEventRecord(e0, b->stream);
    const int rc = aco_b200_batch_enqueue(b);
    cudaEventRecord(e1, b->stream);
    float t_ms = -1.f;
    if (rc != ACO_OK || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&t_ms, e0, e1) != cudaSuccess)
      continue;
    costs[i].resize(count);
    if (aco_b200_batch_get_costs(b, costs[i].data(), nullptr, nullptr) != ACO_OK) continue;
    ms[i] = t_ms;
    valid[i] = 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // Quality: the mean final cost over the instances every length solved;
  // a length that leaves more instances without a solution is worse.
  std::vector<int> infeasible(nks, 0);
  std::vector<char> common(count, 1);
  for (int i = 0; i < nks; ++i) {
    if (!valid[i]) continue;
    for (int j = 0; j < count; ++j) {
      if (costs[i][j] >= DBL_MAX) {
        infeasible[i] += 1;
        common[j] = 0;
      }
    }
  }
  int min_inf = count + 1;
  for (int i = 0; i < nks; ++i)
    if (valid[i] && infeasible[i] < min_inf) min_inf = infeasible[i];
  std::vector<double> mean(nks, DBL_MAX);
  double best_mean = DBL_MAX;
  for (int i = 0; i < nks; ++i) {
    if (!valid[i]) continue;
    double sum = 0.0;
    int cnt = 0;
    for (int j = 0; j < count; ++j)
      if (common[j]) {
        sum += costs[i][j];
        ++cnt;
      }
    mean[i] = cnt ? sum / cnt : DBL_MAX;
    if (infeasible[i] == min_inf && mean[i] < best_mean) best_mean = mean[i];
  }
  // The fastest length within quality_tol of the best quality.
  int pick = -1;
  for (int i = 0; i < nks; ++i) {
    if (!valid[i] || infeasible[i] != min_inf) continue;
    if (mean[i] > best_mean * (1.0 + quality_tol)) continue;
    if (pick < 0 || ms[i] < ms[pick]) pick = i;
  }
  for (int i = 0; i < nks; ++i) {
    if (k_solve_ms) k_solve_ms[i] = ms[i];
    if (k_mean_cost) k_mean_cost[i] = valid[i] ? mean[i] : -1.0;
    if (k_feasible) k_feasible[i] = valid[i] ? count - infeasible[i] : -1;
  }
  if (pick < 0) return ACO_ERR_INVALID_INPUT;
  int rc = aco_b200_batch_set_cand_k(b, ks[pick]);
  if (rc) return rc;
  if (chosen_k) *chosen_k = ks[pick];
  // Stage 2: the launch shape for that length.
  return aco_b200_batch_autotune(b, trial_epochs, chosen, trial_ms, max_trials, n_trials);
}

int aco_b200_batch_get(aco_b200_batch *b, int instance, int *nodes, int *lens, double *cost,
                       int *epochs) {
  if (!b || !b->ready || instance < 0 || instance >= b->count) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  const BatchInst &I = b->inst[instance];
  cudaStream_t s = b->stream;
  BTRY(cudaMemcpyAsync(cost, b->args.out_cost + instance, sizeof(double), cudaMemcpyDeviceToHost, s));
  if (epochs)
    BTRY(cudaMemcpyAsync(epochs, b->args.out_epochs + instance, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (lens)
    BTRY(cudaMemcpyAsync(lens, b->args.gbest_lens + I.gblens_off, sizeof(int) * I.K,
                         cudaMemcpyDeviceToHost, s));
  if (nodes)
    BTRY(cudaMemcpyAsync(nodes, b->args.gbest_nodes + I.gbest_off, sizeof(int) * (I.n + 2 * I.K),
                         cudaMemcpyDeviceToHost, s));
  BTRY(cudaStreamSynchronize(s));
  return *cost < DBL_MAX ? ACO_OK : ACO_ERR_NO_SOLUTION;
}

int aco_b200_batch_get_costs(aco_b200_batch *b, double *costs, int *epochs,
                             unsigned long long *steps) {
  if (!b || !b->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  cudaStream_t s = b->stream;
  if (costs)
    BTRY(cudaMemcpyAsync(costs, b->args.out_cost, sizeof(double) * b->count, cudaMemcpyDeviceToHost, s));
  if (epochs)
    BTRY(cudaMemcpyAsync(epochs, b->args.out_epochs, sizeof(int) * b->count, cudaMemcpyDeviceToHost, s));
  if (steps)
    BTRY(cudaMemcpyAsync(steps, b->args.out_steps, sizeof(unsigned long long) * b->count,
                         cudaMemcpyDeviceToHost, s));
  BTRY(cudaStreamSynchronize(s));
  return ACO_OK;
}

int aco_b200_batch_get_all(aco_b200_batch *b, int *nodes, int *lens, double *costs) {
  if (!b || !b->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  cudaStream_t s = b->stream;
  const BatchInst &last = b->inst[b->count - 1];
  if (nodes)
    BTRY(cudaMemcpyAsync(nodes, b->args.gbest_nodes,
                         sizeof(int) * (last.gbest_off + last.n + 2 * last.K),
                         cudaMemcpyDeviceToHost, s));
  if (lens)
    BTRY(cudaMemcpyAsync(lens, b->args.gbest_lens, sizeof(int) * (last.gblens_off + last.K),
                         cudaMemcpyDeviceToHost, s));
  if (costs)
    BTRY(cudaMemcpyAsync(costs, b->args.out_cost, sizeof(double) * b->count, cudaMemcpyDeviceToHost, s));
  BTRY(cudaStreamSynchronize(s));
  return ACO_OK;
}

}  // extern "C"

extern "C" int aco_b200_batch_apply_prior(aco_b200_batch *b, aco_b200_prior *prior, float gamma) {
  if (!b || !b->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(b->device);
  cudaStream_t s = b->stream;
  const BatchArgs &a = b->args;
  uint16_t *lvl = const_cast<uint16_t *>(a.lvl);
  if (prior && gamma > 0.f) {
    for (int i = 0; i < b->count; ++i) {
      const BatchInst &I = b->inst[i];
      int rc = acob200::prior::learned_levels(prior, a.coords + I.node_off, a.demand + I.node_off,
                                              I.cap, I.n, b->k, a.cand + I.node_off * b->k,
                                              lvl + I.node_off * b->k, gamma, 0, s);
      if (rc) return rc;
    }
  } else {
    BTRY(launch_knn_levels_multi(a.coords, b->d_seg_off, b->d_seg_n, b->count, b->rows, b->k,
                                 b->d_thr, kThresholds, const_cast<uint16_t *>(a.cand), lvl, s));
  }
  BTRY(cudaStreamSynchronize(s));
  return ACO_OK;
}
