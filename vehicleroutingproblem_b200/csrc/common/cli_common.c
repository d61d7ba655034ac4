/*
 * CLI helpers with the reference's contract (src/common/cli_common.c:8-85)
 * and the status strings of src/common/aco_shared.c:8-23.
 */
#include "cli_common.h"
#include "aco.h"

#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

int cli_parse_int_arg(const char *s, int *out) {
  if (!s || !out) return 0;
  char *end = NULL;
  errno = 0;
  long v = strtol(s, &end, 10);
  if (errno || end == s || *end != '\0' || v < 0 || v > 100000000L) return 0;
  *out = (int)v;
  return 1;
}

unsigned int cli_parse_uint_arg(const char *s, int *ok) {
  if (!ok) return 0u;
  if (!s) {
    *ok = 0;
    return 0u;
  }
  char *end = NULL;
  errno = 0;
  unsigned long v = strtoul(s, &end, 10);
  if (errno || end == s || *end != '\0' || v > 0xFFFFFFFFUL) {
    *ok = 0;
    return 0u;
  }
  *ok = 1;
  return (unsigned int)v;
}

void cli_print_solution_routes(const Solution *best, int K) {
  for (int v = 0; v < K; ++v) {
    const Route *r = &best->routes[v];
    printf("Route %d:", v + 1);
    for (int t = 0; t < r->len; ++t) {
      if (r->nodes[t] != 0) printf(" %d", r->nodes[t]);
    }
    printf("\n");
  }
}

void cli_print_solution_cost(double best_cost) {
  printf("Cost: %.3f\n", best_cost);
  printf("best cost: %.3f\n", best_cost);
}

int cli_validate_solution_or_report(const Solution *best, int n, int K,
                                    double best_cost) {
  if (!isfinite(best_cost) || best_cost <= 0.0) {
    fprintf(stderr, "invalid solution cost: %.12g\n", best_cost);
    return 0;
  }
  char err[160];
  if (!solution_validate(best, n, K, err, sizeof(err))) {
    fprintf(stderr, "invalid solution: %s\n", err);
    return 0;
  }
  return 1;
}

const char *aco_status_string(AcoStatus status) {
  switch (status) {
    case ACO_OK: return "ok";
    case ACO_ERR_INVALID_INPUT: return "invalid input";
    case ACO_ERR_ALLOCATION: return "allocation failure";
    case ACO_ERR_NO_SOLUTION: return "no solution";
    case ACO_ERR_BACKEND: return "backend failure";
  }
  return "unknown status";
}
