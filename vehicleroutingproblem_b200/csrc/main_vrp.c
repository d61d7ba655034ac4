/*
 * aco_vrp_cuda.out <instance.vrp> <K> <m> [seed]
 *
 * Drop-in for the reference CLI (src/cuda/main_vrp.cu:43-124): same
 * arguments, same checks (K must equal the file's VEHICLES), alpha=1, beta=2,
 * rho=0.5, tau0=1, Q=1, default seed 1234, same stdout and exit codes.
 * Extension: instances with customer demands other than 1 are accepted and
 * solved with demand-weighted capacity (the reference rejects them); their
 * routes are additionally checked against CAPACITY.
 */
#include "aco.h"
#include "cli_common.h"
#include "instance_parser.h"
#include "solution.h"

#include <stdio.h>
#include <stdlib.h>

static int check_loads(const Solution *s, const int *demand, int capacity) {
  for (int v = 0; v < s->K; ++v) {
    long long load = 0;
    for (int t = 0; t < s->routes[v].len; ++t) load += demand[s->routes[v].nodes[t]];
    if (load > capacity) {
      fprintf(stderr, "invalid solution: route %d load %lld exceeds capacity %d\n",
              v + 1, load, capacity);
      return 0;
    }
  }
  return 1;
}

int main(int argc, char **argv) {
  int K = 0, m = 0, ok = 1, n = 0;
  unsigned int seed = 1234u;
  VrpInstanceMeta meta = {0, 0};
  float *x = NULL, *y = NULL;
  int *demand = NULL;
  const double alpha = 1.0, beta = 2.0, rho = 0.5, tau0 = 1.0, Q = 1.0;

  if (argc < 4 || argc > 5) {
    fprintf(stderr, "usage: %s <instance.vrp> <K> <m> [seed]\n", argv[0]);
    fprintf(stderr, "example: %s instances/generated_benchmark/n500_k8_s19000.vrp 8 0 1234\n", argv[0]);
    return 1;
  }
  ok = ok && cli_parse_int_arg(argv[2], &K);
  ok = ok && cli_parse_int_arg(argv[3], &m);
  if (argc == 5) seed = cli_parse_uint_arg(argv[4], &ok);
  if (!ok || K <= 0 || m < 0) {
    fprintf(stderr, "usage: %s <instance.vrp> <K> <m> [seed]\n", argv[0]);
    return 1;
  }
  if (vrp_load_tsplib_euc2d_coords_demands(argv[1], &n, &x, &y, &demand, &meta) != 0) return 1;
  if (meta.vehicles > 0 && meta.vehicles != K) {
    fprintf(stderr, "instance VEHICLES mismatch: CLI K=%d, file VEHICLES=%d\n", K, meta.vehicles);
    free(x);
    free(y);
    free(demand);
    return 1;
  }
  int unit = 1;
  for (int j = 1; j <= n; ++j) unit = unit && demand[j] == 1;

  Solution *best = solution_create(K, n);
  if (!best) {
    fprintf(stderr, "failed to allocate solution\n");
    free(x);
    free(y);
    free(demand);
    return 1;
  }
  double best_cost = 0.0;
  AcoStatus st = unit
      ? aco_vrp_cuda_with_capacity(n, K, meta.capacity, m, x, y, alpha, beta, rho, tau0, Q, seed, best, &best_cost)
      : aco_vrp_cuda_with_demands(n, K, meta.capacity, m, x, y, demand, alpha, beta, rho, tau0, Q, seed, best, &best_cost);
  int rc = 0;
  if (st != ACO_OK) {
    fprintf(stderr, "CUDA solver failed: %s\n", aco_status_string(st));
    rc = 1;
  } else if (!cli_validate_solution_or_report(best, n, K, best_cost) ||
             (!unit && !check_loads(best, demand, meta.capacity))) {
    rc = 1;
  } else {
    cli_print_solution_routes(best, K);
    cli_print_solution_cost(best_cost);
  }
  solution_free(best);
  free(x);
  free(y);
  free(demand);
  return rc;
}
