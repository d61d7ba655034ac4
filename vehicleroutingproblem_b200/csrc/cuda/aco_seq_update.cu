// aco_seq_update.cu -- the sequential path's FP64 pheromone update on the
// device (src/seq/aco_sequential.c:829-886), bit-exact.
//
// The reference runs, per epoch with an iteration best:
//   1. tau[i][j] *= (1 - rho)                    for every i != j
//   2. tau[u][v] += d_it, tau[v][u] += d_it       every arc of the iteration best
//   3. the same with d_best for the global best
//   4. tau[i][j] = clamp(tau[i][j], tau_min, tau_max)   (MMAS), i != j
//   5. on a stagnation trigger: tau[i][j] = 0.5 tau[i][j] + 0.5 tau0, i != j
// i.e. three passes over the (n+1)^2 matrix.  Here a bitmap of the cells the
// deposits touch lets one sweep do 1, 4 and 5 on every other cell (16 bytes
// of traffic per cell instead of 32-48), and a small kernel does 2-5 on the
// touched cells only:
//   k_seq_mark     sets the bit of every deposit cell (i != j)
//   k_seq_sweep    the matrix two cells (16 bytes) at a time, four pairs per
//                  thread in flight: evaporate; unmarked cells also clamp
//                  and reset
//   k_seq_add      the adds of one solution, one launch for the iteration
//                  best, then one for the global best (double atomics: the
//                  adds to one cell within one deposit are of the same
//                  amount, so their order does not change the sum; the
//                  launch boundary orders the two deposits)
//   k_seq_clamp    every marked cell clamped and reset by the thread that
//                  clears its bit -- which leaves the bitmap zeroed for the
//                  next call.
// The arc kernels deal a solution's arcs over all their threads, one arc
// per thread at the sizes of interest (n + K arcs).
// Every operation is an IEEE FP64 multiply, add or compare in the
// reference's order, written with __dmul_rn/__dadd_rn so that nothing is
// contracted into a fused multiply-add.
#include "aco_internal.cuh"

extern "C" {
#include "aco.h"
#include "aco_b200.h"
}

#include <cstdio>

using namespace acob200;

namespace {

constexpr int kSeqMaxRoutes = 8192;
constexpr int kSweepThreads = 256;
constexpr int kSweepUnroll = 4;

struct SeqArgs {
  double *tau;
  int n, K;
  const int *it_nodes, *it_lens;
  const int *gb_nodes, *gb_lens;  // null: no global best
  double d_it, d_gb;
  double keep;                    // 1 - rho
  double tau_min, tau_max;
  int reset;
  double tau0;
  unsigned int *marks;            // (n+1)^2 bits, zero between calls
};

__device__ __forceinline__ double clamp_reset(double x, const SeqArgs &a) {
  // if (x < tau_min) x = tau_min; else if (x > tau_max) x = tau_max;
  x = (x < a.tau_min) ? a.tau_min : ((x > a.tau_max) ? a.tau_max : x);
  if (a.reset) x = __dadd_rn(__dmul_rn(0.5, x), __dmul_rn(0.5, a.tau0));
  return x;
}

// Arc offsets of one solution in shared memory: route v's arcs are
// [off[v], off[v+1]) in the solution's arc order, its first entry is at
// off[v] + v.  Returns the number of arcs.
__device__ int load_arc_offsets(const int *lens, int K, int *off) {
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int v = 0; v < K; ++v) {
      off[v] = acc;
      acc += lens[v] - 1;
    }
    off[K] = acc;
  }
  __syncthreads();
  const int total = off[K];
  __syncthreads();
  return total;
}

// Arc j of a solution: (u, v) = (nodes[e], nodes[e+1]).
__device__ __forceinline__ void arc_of(const int *nodes, const int *off, int K, int j, int *u,
                                       int *v) {
  int lo = 0, hi = K;  // route r with off[r] <= j < off[r+1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= j) lo = mid; else hi = mid;
  }
  const int e = j + lo;  // entries before route lo: off[lo] + lo
  *u = nodes[e];
  *v = nodes[e + 1];
}

__device__ __forceinline__ unsigned long long cell(int n, int u, int v) {
  return (unsigned long long)u * (unsigned long long)(n + 1) + (unsigned long long)v;
}

constexpr int kArcThreads = 256;

__global__ void __launch_bounds__(kArcThreads) k_seq_mark(SeqArgs a) {
  extern __shared__ int s_off[];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  for (int which = 0; which < 2; ++which) {
    const int *nodes = which ? a.gb_nodes : a.it_nodes;
    const int *lens = which ? a.gb_lens : a.it_lens;
    if (!nodes) break;
    const int total = load_arc_offsets(lens, a.K, s_off);
    for (int j = gt; j < total; j += gn) {
      int u, v;
      arc_of(nodes, s_off, a.K, j, &u, &v);
      if (u == v) continue;  // the diagonal is never swept
      const unsigned long long c1 = cell(a.n, u, v), c2 = cell(a.n, v, u);
      atomicOr(a.marks + (c1 >> 5), 1u << (c1 & 31));
      atomicOr(a.marks + (c2 >> 5), 1u << (c2 & 31));
    }
    __syncthreads();
  }
}

// The matrix as a flat array of (n+1)^2 cells taken two at a time (16-byte
// loads and stores; the matrix starts 16-byte aligned): cell e is on the
// diagonal exactly when e mod (n+2) == 0, and its mark is bit e mod 32 of
// word e / 32 (both cells of a pair share the word).
__device__ __forceinline__ bool on_diagonal(unsigned long long e, unsigned long long n2,
                                            double inv_n2) {
  // e / n2 from the FP64 reciprocal, corrected to the exact quotient
  long long q = (long long)((double)e * inv_n2);
  long long r = (long long)e - q * (long long)n2;
  if (r < 0) r += (long long)n2;
  if (r >= (long long)n2) r -= (long long)n2;
  return r == 0;
}

__device__ __forceinline__ double sweep_cell(double x, unsigned long long e, unsigned int word,
                                             unsigned long long n2, double inv_n2,
                                             const SeqArgs &a) {
  if (on_diagonal(e, n2, inv_n2)) return x;
  double y = __dmul_rn(x, a.keep);
  if (!((word >> (e & 31)) & 1u)) y = clamp_reset(y, a);
  return y;
}

__global__ void __launch_bounds__(kSweepThreads) k_seq_sweep(SeqArgs a) {
  const unsigned long long cells = (unsigned long long)(a.n + 1) * (unsigned long long)(a.n + 1);
  const unsigned long long n2 = (unsigned long long)a.n + 2;
  const double inv_n2 = 1.0 / (double)n2;
  const unsigned long long nvec = cells / 2;
  double2 *t2 = reinterpret_cast<double2 *>(a.tau);
  const unsigned long long tile = (unsigned long long)kSweepUnroll * blockDim.x;
  const unsigned long long step = tile * gridDim.x;
  for (unsigned long long base = blockIdx.x * tile + threadIdx.x; base < nvec; base += step) {
    double2 v[kSweepUnroll];
    unsigned int m[kSweepUnroll];
#pragma unroll
    for (int q = 0; q < kSweepUnroll; ++q) {
      const unsigned long long i = base + (unsigned long long)q * blockDim.x;
      v[q] = make_double2(0.0, 0.0);
      m[q] = 0u;
      if (i < nvec) {
        v[q] = __ldcs(t2 + i);
        m[q] = __ldg(a.marks + ((2 * i) >> 5));
      }
    }
#pragma unroll
    for (int q = 0; q < kSweepUnroll; ++q) {
      const unsigned long long i = base + (unsigned long long)q * blockDim.x;
      if (i < nvec) {
        const unsigned long long e = 2 * i;
        double2 r;
        r.x = sweep_cell(v[q].x, e, m[q], n2, inv_n2, a);
        r.y = sweep_cell(v[q].y, e + 1, m[q], n2, inv_n2, a);
        __stcs(t2 + i, r);
      }
    }
  }
  // An odd cell count leaves the last cell, (n, n), out of the pairs: it is
  // on the diagonal, which the update never changes.
}

// The adds of one solution (which = 0: the iteration best, 1: the global
// best) into the evaporated matrix.
__global__ void __launch_bounds__(kArcThreads) k_seq_add(SeqArgs a, int which) {
  extern __shared__ int s_off[];
  const int *nodes = which ? a.gb_nodes : a.it_nodes;
  const int *lens = which ? a.gb_lens : a.it_lens;
  const double d = which ? a.d_gb : a.d_it;
  const int total = load_arc_offsets(lens, a.K, s_off);
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  for (int j = gt; j < total; j += gn) {
    int u, v;
    arc_of(nodes, s_off, a.K, j, &u, &v);
    atomicAdd(a.tau + cell(a.n, u, v), d);
    atomicAdd(a.tau + cell(a.n, v, u), d);
  }
}

// Clamp and reset each marked cell once: the thread that clears its bit.
__global__ void __launch_bounds__(kArcThreads) k_seq_clamp(SeqArgs a) {
  extern __shared__ int s_off[];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
  for (int which = 0; which < 2; ++which) {
    const int *nodes = which ? a.gb_nodes : a.it_nodes;
    const int *lens = which ? a.gb_lens : a.it_lens;
    if (!nodes) break;
    const int total = load_arc_offsets(lens, a.K, s_off);
    for (int j = gt; j < total; j += gn) {
      int u, v;
      arc_of(nodes, s_off, a.K, j, &u, &v);
      if (u == v) continue;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const unsigned long long c = side ? cell(a.n, v, u) : cell(a.n, u, v);
        const unsigned int bit = 1u << (c & 31);
        if (atomicAnd(a.marks + (c >> 5), ~bit) & bit) {
          double *p = a.tau + c;
          p[0] = clamp_reset(__ldcg(p), a);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" ACO_API size_t aco_b200_seq_update_scratch_bytes(int n) {
  if (n < 1) return 0;
  const unsigned long long cells = (unsigned long long)(n + 1) * (unsigned long long)(n + 1);
  return (size_t)(((cells + 31) / 32) * 4 + 15) & ~(size_t)15;
}

extern "C" ACO_API int aco_b200_seq_pheromone_update(
    double *d_tau, int n, int K, const int *d_iter_nodes, const int *d_iter_lens,
    double iter_deposit, const int *d_best_nodes, const int *d_best_lens, double best_deposit,
    double rho, double tau_min, double tau_max, int reset, double tau0, void *d_scratch,
    void *stream) {
  if (!d_tau || !d_iter_nodes || !d_iter_lens || !d_scratch || n < 1 || K < 1 ||
      K > kSeqMaxRoutes || (d_best_nodes == nullptr) != (d_best_lens == nullptr) ||
      !(rho >= 0.0 && rho <= 1.0) || !(tau_min <= tau_max)) {
    fprintf(stderr, "aco_b200_seq_pheromone_update: invalid arguments\n");
    return ACO_ERR_INVALID_INPUT;
  }
  if (((uintptr_t)d_tau & 15u) != 0u) {
    fprintf(stderr, "aco_b200_seq_pheromone_update: d_tau must be 16-byte aligned\n");
    return ACO_ERR_INVALID_INPUT;
  }
  SeqArgs a;
  a.tau = d_tau;
  a.n = n;
  a.K = K;
  a.it_nodes = d_iter_nodes;
  a.it_lens = d_iter_lens;
  a.gb_nodes = d_best_nodes;
  a.gb_lens = d_best_lens;
  a.d_it = iter_deposit;
  a.d_gb = best_deposit;
  a.keep = 1.0 - rho;  // (1.0 - rho), as the reference computes it
  a.tau_min = tau_min;
  a.tau_max = tau_max;
  a.reset = reset ? 1 : 0;
  a.tau0 = tau0;
  a.marks = static_cast<unsigned int *>(d_scratch);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = sizeof(int) * (size_t)(K + 1);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned long long pairs = (unsigned long long)(n + 1) * (unsigned long long)(n + 1) / 2;
  const unsigned long long per_block = (unsigned long long)kSweepUnroll * kSweepThreads;
  unsigned long long g = (pairs + per_block - 1) / per_block;
  if (g > (unsigned long long)sms * 8) g = (unsigned long long)sms * 8;
  if (g < 1) g = 1;
  const int grid = (int)g;
  // The arc kernels: enough blocks for one arc per thread (a solution has
  // n + K arcs at most), at most 4 per SM.
  unsigned long long ga = ((unsigned long long)n + K + kArcThreads - 1) / kArcThreads;
  if (ga > (unsigned long long)sms * 4) ga = (unsigned long long)sms * 4;
  const int arc_grid = (int)ga;
  k_seq_mark<<<arc_grid, kArcThreads, smem, s>>>(a);
  k_seq_sweep<<<grid, kSweepThreads, 0, s>>>(a);
  k_seq_add<<<arc_grid, kArcThreads, smem, s>>>(a, 0);
  if (a.gb_nodes) k_seq_add<<<arc_grid, kArcThreads, smem, s>>>(a, 1);
  k_seq_clamp<<<arc_grid, kArcThreads, smem, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_seq_pheromone_update: %s\n", cudaGetErrorString(e));
    return ACO_ERR_BACKEND;
  }
  return ACO_OK;
}
