#ifndef SOLUTION_H
#define SOLUTION_H

#include "aco_api.h"

/*
 * Route/Solution containers.  Same layout and functions as the reference's
 * include/solution.h (src/common/solution.c) so that code which creates,
 * reads or validates solutions keeps working unchanged.
 */

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One vehicle route: nodes[0..len) with capacity cap (= n + 2). */
typedef struct {
  int *nodes;
  int len;
  int cap;
} Route;

/* K routes backed by one contiguous node store. */
typedef struct {
  Route *routes;
  int K;
  int route_cap;
  int *nodes_storage;
} Solution;

ACO_API Solution *solution_create(int K, int n);
ACO_API void solution_free(Solution *s);
ACO_API void solution_reset(Solution *s);
ACO_API void solution_copy(Solution *dst, const Solution *src);
/* FP64 cost over a dense (n+1)x(n+1) matrix given as row pointers. */
ACO_API double solution_cost(const Solution *s, double **c);
ACO_API void route_append(Route *r, int node);
/* Structural check: K routes, depot at both ends only, every customer once. */
ACO_API bool solution_validate(const Solution *s, int n, int K, char *err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif
