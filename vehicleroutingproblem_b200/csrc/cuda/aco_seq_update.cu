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
//   k_seq_sweep    rows of the matrix, 4 cells per thread in flight: evaporate;
//                  unmarked cells also clamp and reset
//   k_seq_deposit  one block: the iteration-best adds, then the global-best
//                  adds (double atomics: the adds to one cell within one
//                  deposit are of the same amount, so their order does not
//                  change the sum), then every marked cell is clamped and
//                  reset by the thread that clears its bit -- which leaves the
//                  bitmap zeroed for the next call.
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

__global__ void __launch_bounds__(1024) k_seq_mark(SeqArgs a) {
  extern __shared__ int s_off[];
  for (int which = 0; which < 2; ++which) {
    const int *nodes = which ? a.gb_nodes : a.it_nodes;
    const int *lens = which ? a.gb_lens : a.it_lens;
    if (!nodes) break;
    const int total = load_arc_offsets(lens, a.K, s_off);
    for (int j = threadIdx.x; j < total; j += blockDim.x) {
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

__global__ void __launch_bounds__(kSweepThreads) k_seq_sweep(SeqArgs a) {
  const int rows = a.n + 1;
  const int span = kSweepUnroll * blockDim.x;
  for (int i = blockIdx.x; i < rows; i += gridDim.x) {
    double *row = a.tau + (size_t)i * rows;
    const unsigned long long row0 = (unsigned long long)i * rows;
    for (int j0 = threadIdx.x; j0 < rows; j0 += span) {
      double x[kSweepUnroll];
      unsigned int m[kSweepUnroll];
#pragma unroll
      for (int q = 0; q < kSweepUnroll; ++q) {
        const int j = j0 + q * blockDim.x;
        x[q] = 0.0;
        m[q] = 0u;
        if (j < rows) {
          x[q] = __ldcs(row + j);
          const unsigned long long c = row0 + j;
          m[q] = (__ldg(a.marks + (c >> 5)) >> (c & 31)) & 1u;
        }
      }
#pragma unroll
      for (int q = 0; q < kSweepUnroll; ++q) {
        const int j = j0 + q * blockDim.x;
        if (j < rows && j != i) {
          double y = __dmul_rn(x[q], a.keep);
          if (!m[q]) y = clamp_reset(y, a);
          __stcs(row + j, y);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(1024) k_seq_deposit(SeqArgs a) {
  extern __shared__ int s_off[];
  for (int which = 0; which < 2; ++which) {
    const int *nodes = which ? a.gb_nodes : a.it_nodes;
    const int *lens = which ? a.gb_lens : a.it_lens;
    if (!nodes) break;
    const double d = which ? a.d_gb : a.d_it;
    const int total = load_arc_offsets(lens, a.K, s_off);
    for (int j = threadIdx.x; j < total; j += blockDim.x) {
      int u, v;
      arc_of(nodes, s_off, a.K, j, &u, &v);
      atomicAdd(a.tau + cell(a.n, u, v), d);
      atomicAdd(a.tau + cell(a.n, v, u), d);
    }
    // every add of this deposit before any of the next (or the clamps)
    __threadfence();
    __syncthreads();
  }
  // Clamp and reset each marked cell once: the thread that clears its bit.
  for (int which = 0; which < 2; ++which) {
    const int *nodes = which ? a.gb_nodes : a.it_nodes;
    const int *lens = which ? a.gb_lens : a.it_lens;
    if (!nodes) break;
    const int total = load_arc_offsets(lens, a.K, s_off);
    for (int j = threadIdx.x; j < total; j += blockDim.x) {
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
  int grid = sms * 8;
  if (grid > n + 1) grid = n + 1;
  k_seq_mark<<<1, 1024, smem, s>>>(a);
  k_seq_sweep<<<grid, kSweepThreads, 0, s>>>(a);
  k_seq_deposit<<<1, 1024, smem, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "aco_b200_seq_pheromone_update: %s\n", cudaGetErrorString(e));
    return ACO_ERR_BACKEND;
  }
  return ACO_OK;
}
