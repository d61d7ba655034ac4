/*
 * Route/Solution containers with the reference's API
 * (src/common/solution.c:31-234): K routes of capacity n+2 carved from one
 * 64-byte aligned node store; FP64 cost over a dense matrix; structural
 * validation with the same error strings.
 */
#include "solution.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void route_append(Route *r, int node) {
  if (r->len < r->cap) r->nodes[r->len++] = node;
}

Solution *solution_create(int K, int n) {
  if (K <= 0 || n < 0) return NULL;
  Solution *s = (Solution *)calloc(1, sizeof(Solution));
  if (!s) return NULL;
  s->K = K;
  s->route_cap = n + 2;
  s->routes = (Route *)calloc((size_t)K, sizeof(Route));
  size_t bytes = round_up((size_t)K * (size_t)s->route_cap * sizeof(int), 64);
  s->nodes_storage = s->routes ? (int *)aligned_alloc(64, bytes) : NULL;
  if (!s->routes || !s->nodes_storage) {
    free(s->routes);
    free(s);
    return NULL;
  }
  memset(s->nodes_storage, 0, bytes);
  for (int v = 0; v < K; ++v) {
    s->routes[v].nodes = s->nodes_storage + (size_t)v * (size_t)s->route_cap;
    s->routes[v].cap = s->route_cap;
    s->routes[v].len = 0;
  }
  return s;
}

void solution_reset(Solution *s) {
  for (int v = 0; v < s->K; ++v) s->routes[v].len = 0;
}

void solution_free(Solution *s) {
  if (!s) return;
  free(s->nodes_storage);
  free(s->routes);
  free(s);
}

void solution_copy(Solution *dst, const Solution *src) {
  for (int v = 0; v < src->K; ++v) {
    dst->routes[v].len = src->routes[v].len;
    memcpy(dst->routes[v].nodes, src->routes[v].nodes,
           (size_t)src->routes[v].len * sizeof(int));
  }
}

double solution_cost(const Solution *s, double **c) {
  double total = 0.0;
  for (int v = 0; v < s->K; ++v) {
    const Route *r = &s->routes[v];
    for (int t = 1; t < r->len; ++t) total += c[r->nodes[t - 1]][r->nodes[t]];
  }
  return total;
}

static bool fail(char *err, size_t err_len, const char *msg) {
  if (err && err_len) snprintf(err, err_len, "%s", msg);
  return false;
}

bool solution_validate(const Solution *s, int n, int K, char *err,
                       size_t err_len) {
  if (!s) return fail(err, err_len, "solution is NULL");
  if (s->K != K) return fail(err, err_len, "solution K does not match expected K");
  if (!s->routes) return fail(err, err_len, "solution routes are NULL");
  if (n < 0 || K < 0) return fail(err, err_len, "invalid n or K");
  unsigned char *seen = (unsigned char *)calloc((size_t)n + 1, 1);
  if (!seen) return fail(err, err_len, "allocation failure in solution_validate");
  const char *msg = NULL;
  for (int v = 0; v < s->K && !msg; ++v) {
    const Route *r = &s->routes[v];
    if (r->len < 2) { msg = "route length < 2"; break; }
    if (r->nodes[0] != 0 || r->nodes[r->len - 1] != 0) {
      msg = "route must start/end at depot 0";
      break;
    }
    for (int t = 0; t < r->len; ++t) {
      int node = r->nodes[t];
      if (node < 0 || node > n) { msg = "route contains out-of-range node"; break; }
      if (node == 0) {
        if (t != 0 && t != r->len - 1) { msg = "route contains depot inside the path"; break; }
        continue;
      }
      if (seen[node]) { msg = "customer visited more than once"; break; }
      seen[node] = 1;
    }
  }
  for (int node = 1; node <= n && !msg; ++node) {
    if (!seen[node]) msg = "customer not visited";
  }
  free(seen);
  if (msg) return fail(err, err_len, msg);
  if (err && err_len) err[0] = '\0';
  return true;
}
