#ifndef ACO_H
#define ACO_H

#include "aco_api.h"

/*
 * Status codes and solver entry points of the B200 ACO-for-CVRP library.
 *
 * Same status values and meanings as the reference (include/aco.h:82-88) so
 * that callers written against it keep their error handling.
 */

#include "solution.h"

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACO_EPS 1e-9

typedef enum {
  ACO_OK = 0,
  ACO_ERR_INVALID_INPUT = 1,
  ACO_ERR_ALLOCATION = 2,
  ACO_ERR_NO_SOLUTION = 3,
  ACO_ERR_BACKEND = 4
} AcoStatus;

/* Human-readable name of a status (reference: src/common/aco_shared.c:8). */
ACO_API const char *aco_status_string(AcoStatus status);

/*
 * Runs the GPU solver with a per-vehicle capacity in customers (every
 * customer has demand 1).  Same signature and behaviour as the reference's
 * aco_vrp_cuda_with_capacity (src/cuda/aco_cuda.cu:188-192, prototype in
 * src/cuda/main_vrp.cu:29-35): coords_x/coords_y hold n+1 points (depot
 * first); m = 0 selects 256 ants; reads the ACO_SOLVER_* environment; prints
 * the "CUDA Solver starting..." and "[progress][cuda]" lines; fills
 * best_solution (created by solution_create(K, n)) and *best_cost.
 */
ACO_API AcoStatus aco_vrp_cuda_with_capacity(int n, int K,
                                     int vehicle_capacity_customers, int m,
                                     float *coords_x, float *coords_y,
                                     double alpha, double beta, double rho,
                                     double tau0, double Q, unsigned int seed,
                                     Solution *best_solution,
                                     double *best_cost);

/*
 * Demand-weighted variant (no reference counterpart: the reference accepts
 * unit demand only).  demand[0] must be 0; demand[j] >= 1; capacity is in
 * demand units.  With every demand 1 it is identical to
 * aco_vrp_cuda_with_capacity.
 */
ACO_API AcoStatus aco_vrp_cuda_with_demands(int n, int K, int capacity, int m,
                                    const float *coords_x,
                                    const float *coords_y, const int *demand,
                                    double alpha, double beta, double rho,
                                    double tau0, double Q, unsigned int seed,
                                    Solution *best_solution,
                                    double *best_cost);

#ifdef __cplusplus
}
#endif

#endif
