#ifndef ACO_CUDA_KERNELS_H
#define ACO_CUDA_KERNELS_H

/*
 * Drop-in for the reference's include/aco_cuda_kernels.h: the same constants,
 * parameter/summary structs (same field order), the 7 kernels and the 7
 * launch_* host functions with C++ linkage, default stream, no return codes
 * and no internal synchronisation (reference :10-181).  Code written against
 * that header compiles and links against libaco_b200.so unchanged.
 *
 * Semantics, kernel by kernel:
 *   kernel_init_tau, kernel_evaporate_tau      byte-identical to the reference
 *   kernel_build_candidate_lists               identical lists and eta^beta for
 *                                              integer coordinates
 *   kernel_deposit_solution / _flat_solution   byte-identical, except that the
 *                                              depot loop cell [0][0], which the
 *                                              reference updates racily when two
 *                                              or more routes are empty, is
 *                                              updated in vehicle order
 *   kernel_reset_ant_state                     the reference's buffer state
 *   kernel_construct_solutions                 the sequential path's rules
 *                                              (src/seq/aco_sequential.c:616-681)
 *                                              with the exact integer roulette,
 *                                              in place of the reference's
 *                                              stochastic depot rule; draws are
 *                                              Philox4x32-10 keyed by the ant's
 *                                              d_rng_states word
 * The native API (aco_b200.h) is the fast path; these entry points serve
 * callers of the reference's kernel-level interface.
 */

#include <cuda_runtime.h>
#include <stdint.h>

#include "aco_api.h"

#define CUDA_THREADS_PER_BLOCK 128
#define CUDA_WARP_SIZE 32
#define CUDA_CACHE_LINE_SIZE 128
#define CUDA_MAX_CANDIDATES 32
#define CUDA_EPS 1e-9f

typedef struct {
  int n;
  int K;
  int m;
  int cap;
  int cand_k;
  int route_max_len;

  float alpha;
  float beta;
  float rho;
  float tau0;
  float Q;
  float tau_min;
  float tau_max;

  float log_tau_min;
  float log_tau_step;
  uint8_t q_tau_min;
  uint8_t q_tau_max;
  uint8_t q_evap_delta;

  int visited_l1_words;
  int visited_l2_words;
  size_t visited_row_stride;

  float depot_close_weight;
} CudaParams;

typedef struct {
  int feasible;
  int unvisited_count;
  float cost;
} CudaAntSummary;

typedef struct {
  unsigned long long candidate_calls;
  unsigned long long candidate_moves;
  unsigned long long fallback_calls;
  unsigned long long fallback_moves;
  unsigned long long depot_offer_calls;
  unsigned long long depot_close_moves;
  unsigned long long customer_moves;
  unsigned long long nonempty_routes;
  unsigned long long fallback_word_groups_scanned;
  unsigned long long fallback_nodes_scored;
} CudaIterStats;

__global__ void kernel_init_tau(uint8_t *d_tau, uint64_t total_elements, uint8_t q_tau0);

__global__ void kernel_build_candidate_lists(const float2 *d_coords,
                                             int *d_candidate_idx,
                                             float *d_eta_beta,
                                             CudaParams params);

__global__ void kernel_reset_ant_state(int *d_routes,
                                       int *d_route_lengths,
                                       uint64_t *d_visited_l1,
                                       uint64_t *d_visited_l2,
                                       unsigned int *d_rng_states,
                                       CudaAntSummary *d_ant_summary,
                                       CudaParams params,
                                       unsigned int seed);

__global__ void kernel_construct_solutions(const float2 *d_coords,
                                           const uint8_t *d_tau,
                                           const int *d_candidate_idx,
                                           const float *d_eta_beta,
                                           int *d_routes,
                                           int *d_route_lengths,
                                           uint64_t *d_visited_l1,
                                           uint64_t *d_visited_l2,
                                           unsigned int *d_rng_states,
                                           CudaAntSummary *d_ant_summary,
                                           CudaIterStats *d_iter_stats,
                                           CudaParams params);

__global__ void kernel_evaporate_tau(uint8_t *d_tau, uint64_t total_elements, uint8_t delta, uint8_t q_min);

__global__ void kernel_deposit_solution(uint8_t *d_tau,
                                        const int *d_routes,
                                        const int *d_route_lengths,
                                        float deposit_amount,
                                        int best_ant,
                                        CudaParams params);

__global__ void kernel_deposit_flat_solution(uint8_t *d_tau,
                                             const int *d_flat_routes,
                                             const int *d_flat_lengths,
                                             float deposit_amount,
                                             CudaParams params);

ACO_API void launch_init_tau(uint8_t *d_tau, int n, uint8_t q_tau0);
ACO_API void launch_build_candidate_lists(const float2 *d_coords, int *d_candidate_idx, float *d_eta_beta, CudaParams params);
ACO_API void launch_reset_ant_state(int *d_routes, int *d_route_lengths, uint64_t *d_visited_l1, uint64_t *d_visited_l2, unsigned int *d_rng_states, CudaAntSummary *d_ant_summary, CudaParams params, unsigned int seed);
ACO_API void launch_construct_solutions(const float2 *d_coords, const uint8_t *d_tau, const int *d_candidate_idx, const float *d_eta_beta, int *d_routes, int *d_route_lengths, uint64_t *d_visited_l1, uint64_t *d_visited_l2, unsigned int *d_rng_states, CudaAntSummary *d_ant_summary, CudaIterStats *d_iter_stats, CudaParams params);
ACO_API void launch_evaporate_tau(uint8_t *d_tau, int n, uint8_t delta, uint8_t q_min);
ACO_API void launch_deposit_solution(uint8_t *d_tau, const int *d_routes, const int *d_route_lengths, float deposit_amount, int best_ant, CudaParams params);
ACO_API void launch_deposit_flat_solution(uint8_t *d_tau, const int *d_flat_routes, const int *d_flat_lengths, float deposit_amount, CudaParams params);

#endif
