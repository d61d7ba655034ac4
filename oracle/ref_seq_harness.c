/*
 * ref_seq_harness.c -- drives the reference's own sequential construct path.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
 * the reference sources where they lie (never copied into this repository):
 * this file #includes src/seq/aco_sequential.c so that its static
 * build_ant_solution (:616-681), select_next_customer (:505-561) and
 * find_nearest_unvisited (:477-493) can be called directly.
 *
 * Interposition: aco_rand01_state (declared in include/aco.h:138, defined in
 * src/common/aco_shared.c:294, which the Makefile compiles with that symbol
 * renamed) is replaced by a function that pops the next value of a recorded
 * stream of 24-bit draws r and returns r / 2^24.  The candidate lists and the
 * integer weights (as float scores, exact below 2^24) are supplied by the
 * caller, exactly as the GPU uses them.
 */
#include "aco_sequential.c"

#include <stdint.h>

static const uint32_t *g_draws = NULL;
static int g_n_draws = 0;
static int g_next_draw = 0;
static int g_overflow = 0;

double aco_rand01_state(unsigned int *state) {
  (void)state;
  if (g_next_draw >= g_n_draws) {
    g_overflow = 1;
    return 0.0;
  }
  return (double)g_draws[g_next_draw++] / 16777216.0;
}

/* Distance matrix as the reference builds it from EUC_2D coordinates
 * (src/common/instance_parser.c:17-19, :186-190). */
static double **harness_matrix(int n, const float *x, const float *y) {
  double **c = matrix_alloc(n);
  if (!c) return NULL;
  for (int i = 0; i <= n; ++i) {
    for (int j = 0; j <= n; ++j) {
      double dx = (double)x[i] - (double)x[j];
      double dy = (double)y[i] - (double)y[j];
      c[i][j] = sqrt(pow(dx, 2) + pow(dy, 2));
    }
  }
  return c;
}

/*
 * Builds m ants with the reference code over one distance matrix (built once
 * per call; at n=8000 it is 512 MB).  Ant a pops the recorded stream
 * draws[a * n_draws .. (a+1) * n_draws).  Returns 0, -1 on allocation
 * failure, -2 if a recorded stream ran out.  Ant a's routes are written in
 * compact form (K segments [0 ... 0] back to back) at nodes_out + a (n + 2K),
 * its K lengths at lens_out + a K, the reference's solution_cost at
 * cost_out[a] and the number of draws it used at used_out[a].
 */
__attribute__((visibility("default")))
int seqref_construct_ants(int n, int K, int cap, int k, const float *x,
                          const float *y, const int32_t *cand,
                          const uint32_t *w, int m, const uint32_t *draws,
                          int n_draws, int32_t *nodes_out, int32_t *lens_out,
                          double *cost_out, int32_t *used_out) {
  SeqShared shared;
  memset(&shared, 0, sizeof(shared));
  shared.n = n;
  shared.candidate_k = k;
  shared.stride = k;
  shared.visited_words = (n / 64) + 1;
  size_t elems = (size_t)(n + 1) * (size_t)k;
  shared.candidate_idx = (int *)calloc(elems, sizeof(int));
  shared.eta_beta = (float *)calloc(elems, sizeof(float));
  shared.score = (float *)calloc(elems, sizeof(float));
  double **c = harness_matrix(n, x, y);
  if (!shared.candidate_idx || !shared.eta_beta || !shared.score || !c) {
    free(shared.candidate_idx);
    free(shared.eta_beta);
    free(shared.score);
    matrix_free(c);
    return -1;
  }
  for (size_t e = 0; e < elems; ++e) {
    shared.candidate_idx[e] = cand[e];
    shared.score[e] = (float)w[e];
  }
  int rc = 0;
  for (int a = 0; a < m && rc == 0; ++a) {
    SeqWorkspace ws;
    if (!seq_workspace_init(&ws, K, n, shared.visited_words)) {
      rc = -1;
      break;
    }
    g_draws = draws + (size_t)a * (size_t)n_draws;
    g_n_draws = n_draws;
    g_next_draw = 0;
    g_overflow = 0;
    build_ant_solution(&ws, &shared, K, cap < 1 ? 1 : cap, c);
    cost_out[a] = solution_cost(ws.sol, c);
    int32_t *nodes = nodes_out + (size_t)a * (size_t)(n + 2 * K);
    int off = 0;
    for (int v = 0; v < K; ++v) {
      const Route *r = &ws.sol->routes[v];
      for (int t = 0; t < r->len; ++t) nodes[off + t] = r->nodes[t];
      lens_out[(size_t)a * K + v] = r->len;
      off += r->len;
    }
    used_out[a] = g_next_draw;
    if (g_overflow) rc = -2;
    seq_workspace_free(&ws);
  }
  free(shared.candidate_idx);
  free(shared.eta_beta);
  free(shared.score);
  matrix_free(c);
  return rc;
}

/* One ant (seqref_construct_ants with m = 1).  Returns the number of draws
 * used, or -1 on allocation failure, -2 if the recorded stream ran out;
 * cost_out is the reference's solution_cost. */
__attribute__((visibility("default")))
int seqref_construct_ant(int n, int K, int cap, int k, const float *x,
                         const float *y, const int32_t *cand,
                         const uint32_t *w, const uint32_t *draws,
                         int n_draws, int32_t *nodes_out, int32_t *lens_out,
                         double *cost_out) {
  int32_t used = 0;
  const int rc = seqref_construct_ants(n, K, cap, k, x, y, cand, w, 1, draws, n_draws,
                                       nodes_out, lens_out, cost_out, &used);
  return rc < 0 ? rc : used;
}

/* The reference's FP64 cost of a route set in compact form
 * (src/common/solution.c:126-137 over the matrix above). */
__attribute__((visibility("default")))
double seqref_solution_cost(int n, int K, const float *x, const float *y,
                            const int32_t *nodes, const int32_t *lens) {
  double **c = harness_matrix(n, x, y);
  Solution *s = solution_create(K, n);
  if (!c || !s) {
    matrix_free(c);
    solution_free(s);
    return -1.0;
  }
  int off = 0;
  for (int v = 0; v < K; ++v) {
    for (int t = 0; t < lens[v]; ++t) route_append(&s->routes[v], nodes[off + t]);
    off += lens[v];
  }
  double cost = solution_cost(s, c);
  solution_free(s);
  matrix_free(c);
  return cost;
}

/* The reference's structural validator (src/common/solution.c:161-234). */
__attribute__((visibility("default")))
int seqref_validate(int n, int K, const int32_t *nodes, const int32_t *lens) {
  Solution *s = solution_create(K, n);
  if (!s) return 0;
  int off = 0;
  for (int v = 0; v < K; ++v) {
    for (int t = 0; t < lens[v]; ++t) route_append(&s->routes[v], nodes[off + t]);
    off += lens[v];
  }
  char err[160];
  int ok = solution_validate(s, n, K, err, sizeof(err)) ? 1 : 0;
  solution_free(s);
  return ok;
}
