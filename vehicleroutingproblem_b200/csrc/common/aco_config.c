/*
 * Environment configuration (reference: src/common/aco_config.c:5-73).
 * Defaults: no timeout, no stagnation stop, 0.1% minimum relative gain,
 * progress every 10 s.  ACO_SOLVER_MIN_REL_IMPROVEMENT is a percentage;
 * non-positive or empty values keep the default.  ACO_CUDA_CANDIDATE_K fills
 * candidate_k (the reference declares the field but never loads it).
 */
#include "aco_config.h"

#include <stdlib.h>

static const char *env(const char *name) {
  const char *v = getenv(name);
  return (v && *v) ? v : NULL;
}

double aco_parse_min_rel_improvement_percent(const char *s,
                                             double default_fraction) {
  if (!s || !*s) return default_fraction;
  double pct = atof(s);
  return (pct > 0.0) ? pct / 100.0 : default_fraction;
}

void aco_runtime_config_defaults(AcoRuntimeConfig *c) {
  if (!c) return;
  c->timeout_seconds = 0.0;
  c->stagnation_epochs = 0;
  c->min_rel_improvement = 1e-3;
  c->fixed_epochs = 0;
  c->candidate_k = 0;
  c->ants = 0;
  c->seed = 1234u;
  c->progress_interval_seconds = 10.0;
}

void aco_runtime_config_load_env(AcoRuntimeConfig *c) {
  if (!c) return;
  aco_runtime_config_defaults(c);
  const char *s;
  if ((s = env("ACO_SOLVER_TIMEOUT_SECONDS"))) c->timeout_seconds = atof(s);
  if ((s = env("ACO_SOLVER_STAGNATION_EPOCHS"))) c->stagnation_epochs = atoi(s);
  c->min_rel_improvement =
      aco_parse_min_rel_improvement_percent(env("ACO_SOLVER_MIN_REL_IMPROVEMENT"), 1e-3);
  if ((s = env("ACO_SOLVER_FIXED_EPOCHS"))) c->fixed_epochs = atoi(s);
  if ((s = env("ACO_SOLVER_PROGRESS_INTERVAL_SECONDS"))) c->progress_interval_seconds = atof(s);
  if ((s = env("ACO_CUDA_CANDIDATE_K"))) c->candidate_k = atoi(s);
  if (c->stagnation_epochs < 0) c->stagnation_epochs = 0;
  if (c->min_rel_improvement <= 0.0) c->min_rel_improvement = 1e-3;
  if (c->fixed_epochs < 0) c->fixed_epochs = 0;
  if (c->candidate_k < 0) c->candidate_k = 0;
  if (c->progress_interval_seconds < 0.0) c->progress_interval_seconds = 0.0;
}
