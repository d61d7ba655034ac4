// aco_prior_internal.h -- entry of the learned prior used by the solver and
// the batched solver (not part of the C ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

struct aco_b200_prior;

namespace acob200 {
namespace prior {

// Learned eta levels of one instance: features of its (n+1) x k candidate
// edges, the MLP's scores and L = min(4095, round(gamma (s_max - s) 16/ln 2))
// written to lvl[(n+1) k] -- or, residual != 0, added to the plain levels
// lvl holds.  Enqueued on s; 0 or an AcoStatus code.
int learned_levels(aco_b200_prior *p, const float2 *coords, const int *demand, long long cap,
                   int n, int k, const uint16_t *cand, uint16_t *lvl, float gamma,
                   int residual, cudaStream_t s);

}  // namespace prior
}  // namespace acob200
