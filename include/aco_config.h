#ifndef ACO_CONFIG_H
#define ACO_CONFIG_H

#include "aco_api.h"

/*
 * Runtime configuration from the environment.  Same fields and variables as
 * the reference (include/aco_config.h, src/common/aco_config.c:33-73):
 *   ACO_SOLVER_TIMEOUT_SECONDS            wall-clock limit (0 = none)
 *   ACO_SOLVER_STAGNATION_EPOCHS          stop after N epochs without a
 *                                         significant improvement (0 = none)
 *   ACO_SOLVER_MIN_REL_IMPROVEMENT        in PERCENT (default 0.1%)
 *   ACO_SOLVER_FIXED_EPOCHS               run exactly N epochs (the reference
 *                                         honours it in OpenMP only; here the
 *                                         GPU path honours it too)
 *   ACO_SOLVER_PROGRESS_INTERVAL_SECONDS  stderr progress period (default 10)
 * and, new here:
 *   ACO_CUDA_CANDIDATE_K                  candidate list length (fills the
 *                                         reference's unused candidate_k)
 */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double timeout_seconds;
  int stagnation_epochs;
  double min_rel_improvement;
  int fixed_epochs;
  int candidate_k;
  int ants;
  unsigned int seed;
  double progress_interval_seconds;
} AcoRuntimeConfig;

ACO_API void aco_runtime_config_defaults(AcoRuntimeConfig *config);
ACO_API void aco_runtime_config_load_env(AcoRuntimeConfig *config);
ACO_API double aco_parse_min_rel_improvement_percent(const char *s,
                                             double default_fraction);

#ifdef __cplusplus
}
#endif

#endif
