/*
 * aco_oracle.c -- CPU restatement of the ACO-for-CVRP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py compare the CUDA path
 * against.  The product (vehicleroutingproblem_b200) never links, loads or
 * calls it.
 *
 * Parity is pinned two ways (see tests/test_oracle_*.py):
 *   - against the reference's own sequential construct path compiled from its
 *     sources into oracle/_ref (ref_seq_harness.c), fed the same candidate
 *     lists, integer weights and draws, on unit-demand instances;
 *   - against golden vectors in tests/golden/ produced by that harness.
 *
 * Every function cites the reference file:line it restates.  Where the
 * reference has no counterpart (integer weights, counter-based draws, demand
 * weighted capacity) the comment says so and gives the rule.
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off; no FMA contraction
 * so that float/double expressions round exactly as written).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Counter-based draws: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel  */
/* random numbers: as easy as 1, 2, 3", SC'11).  The reference uses a         */
/* stateful xorshift32 per ant (src/common/aco_shared.c:294-310); the counter */
/* form lets every draw be addressed by (seed, epoch, ant, stream, index).    */
/* ------------------------------------------------------------------------ */

ORC_EXPORT void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                                  uint32_t out[4]) {
  uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)0xD2511F53u * x0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0;
    uint32_t y1 = (uint32_t)p1;
    uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
    uint32_t y3 = (uint32_t)p0;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

/* Second key word of every draw stream. */
#define ORC_DRAW_KEY1 0x5EEDC0DEu

/* Draw number d of (seed, epoch, ant, stream): the top 24 bits of word d%4 of
 * Philox(ctr = {d/4, ant, epoch, stream}, key = {seed, ORC_DRAW_KEY1}).
 * u = r / 2^24 is the uniform the roulette uses. */
ORC_EXPORT uint32_t orc_draw24(uint32_t seed, uint32_t epoch, uint32_t ant,
                               uint32_t stream, uint32_t d) {
  uint32_t ctr[4] = {d >> 2, ant, epoch, stream};
  uint32_t key[2] = {seed, ORC_DRAW_KEY1};
  uint32_t out[4];
  orc_philox4x32_10(ctr, key, out);
  return out[d & 3u] >> 8;
}

/* ------------------------------------------------------------------------ */
/* Parameter derivation, restating src/cuda/aco_cuda.cu:209-242.             */
/* ------------------------------------------------------------------------ */

ORC_EXPORT void orc_params(double rho, double tau0, float *log_tau_min,
                           float *log_tau_step, uint8_t *q_evap_delta,
                           uint8_t *q_tau0) {
  float lmin = logf(0.0001f);
  float lmax = logf(100.0f);
  float step = (lmax - lmin) / (float)(255 - 0);
  float log_rho = logf(1.0f - (float)rho);
  *log_tau_min = lmin;
  *log_tau_step = step;
  *q_evap_delta = (uint8_t)fmaxf(1.0f, roundf(-log_rho / step));
  *q_tau0 = (uint8_t)fmaxf(0.0f,
                           fminf(255.0f, roundf((logf((float)tau0) - lmin) / step)));
}

/* ------------------------------------------------------------------------ */
/* Integer selection weights (no reference counterpart: the reference scores */
/* a candidate with float tau^alpha * eta^beta, aco_cuda_kernels.cu:284-296, */
/* seq aco_sequential.c:346-442).  Rule:                                     */
/*   weight level  e = A[q] - L(d^2),   G = 16 levels per octave             */
/*   A[q]  = floor(alpha * q * step * G / ln 2 + 1/2)       (tau^alpha)      */
/*   L(d2) = #{ j in 1..J : d2 >= T_j },  T_j = (float) 2^(2 j / (beta G))   */
/*           (eta^beta = d^-beta, so L counts 1/G-octave steps of d^beta)    */
/*   w = LUT[min(emax_row - e, 255)],  LUT[r] = floor(2^23 2^(-r/G) + 1/2),  */
/*       LUT[255] = 0, emax_row = max of e over the row's real candidates.   */
/* Every weight is < 2^24 (exact as a float score) and a row of k <= 32      */
/* sums to < 2^29, so u * denom with u = r / 2^24 is exact in double.        */
/* ------------------------------------------------------------------------ */

#define ORC_G 16
#define ORC_REL_MAX 255

ORC_EXPORT void orc_tables(double alpha, double beta, float log_tau_step,
                           int32_t A[256], uint32_t lut[256], float *thr,
                           int J) {
  const double ln2 = 0.69314718055994530942;
  for (int q = 0; q < 256; ++q) {
    double v = alpha * (double)q * (double)log_tau_step * (double)ORC_G / ln2;
    A[q] = (int32_t)floor(v + 0.5);
  }
  for (int r = 0; r < ORC_REL_MAX; ++r) {
    lut[r] = (uint32_t)floor(8388608.0 * exp2(-(double)r / (double)ORC_G) + 0.5);
  }
  lut[ORC_REL_MAX] = 0u;
  for (int j = 1; j <= J; ++j) {
    if (beta > 0.0) {
      double t = exp2(2.0 * (double)j / (beta * (double)ORC_G));
      thr[j - 1] = (t > 3.0e38) ? INFINITY : (float)t;
    } else {
      thr[j - 1] = INFINITY;
    }
  }
}

/* Squared distance in float, no contraction: exact for integer coordinates
 * up to 2896 in magnitude difference. */
static inline float d2f(const float *x, const float *y, int a, int b) {
  float dx = x[a] - x[b];
  float dy = y[a] - y[b];
  float xx = dx * dx;
  float yy = dy * dy;
  return xx + yy;
}

ORC_EXPORT uint16_t orc_level(float d2, const float *thr, int J) {
  int lo = 0, hi = J; /* count of thr[j] <= d2 */
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (thr[mid] <= d2) lo = mid + 1; else hi = mid;
  }
  return (uint16_t)lo;
}

/* k-nearest candidate lists, restating kernel_build_candidate_lists
 * (src/cuda/aco_cuda_kernels.cu:164-214): for every node i in 0..n the k
 * nearest nodes j in 1..n, j != i, ascending, ties to the lower j (the
 * reference's insertion with strict '<' at :189 keeps the earlier j first).
 * Ordered by float d^2, which orders exactly as the reference's sqrtf(d^2)
 * for integer coordinates (sqrtf is strictly increasing on integers < 2^24).
 * Slots past the n-1 (customer rows) or n (depot row) real nodes hold 0. */
ORC_EXPORT void orc_knn(int n, int k, const float *x, const float *y,
                        int32_t *cand) {
  float *bd = (float *)malloc(sizeof(float) * (size_t)k);
  int32_t *bj = (int32_t *)malloc(sizeof(int32_t) * (size_t)k);
  for (int i = 0; i <= n; ++i) {
    int cnt = 0;
    for (int j = 1; j <= n; ++j) {
      if (j == i) continue;
      float d = d2f(x, y, i, j);
      if (cnt == k && !(d < bd[k - 1])) continue;
      int pos = (cnt < k) ? cnt : k - 1;
      while (pos > 0 && d < bd[pos - 1]) {
        bd[pos] = bd[pos - 1];
        bj[pos] = bj[pos - 1];
        --pos;
      }
      bd[pos] = d;
      bj[pos] = j;
      if (cnt < k) ++cnt;
    }
    for (int t = 0; t < k; ++t) cand[(size_t)i * k + t] = (t < cnt) ? bj[t] : 0;
  }
  free(bd);
  free(bj);
}

ORC_EXPORT void orc_levels(int n, int k, const float *x, const float *y,
                           const int32_t *cand, const float *thr, int J,
                           uint16_t *lvl) {
  for (int i = 0; i <= n; ++i) {
    for (int t = 0; t < k; ++t) {
      int c = cand[(size_t)i * k + t];
      lvl[(size_t)i * k + t] = (c > 0) ? orc_level(d2f(x, y, i, c), thr, J) : 0;
    }
  }
}

/* Per-epoch weight table (the role of seq_shared_update_scores,
 * src/seq/aco_sequential.c:410-442, recomputed from the quantized tau). */
ORC_EXPORT void orc_weights(int n, int k, const int32_t *cand,
                            const uint16_t *lvl, const uint8_t *tau,
                            const int32_t *A, const uint32_t *lut,
                            uint32_t *w) {
  size_t stride = (size_t)n + 1;
  for (int i = 0; i <= n; ++i) {
    int have = 0;
    int32_t emax = 0;
    for (int t = 0; t < k; ++t) {
      int c = cand[(size_t)i * k + t];
      if (c <= 0) continue;
      int32_t e = A[tau[(size_t)i * stride + c]] - (int32_t)lvl[(size_t)i * k + t];
      if (!have || e > emax) emax = e;
      have = 1;
    }
    for (int t = 0; t < k; ++t) {
      int c = cand[(size_t)i * k + t];
      uint32_t v = 0;
      if (c > 0) {
        int32_t e = A[tau[(size_t)i * stride + c]] - (int32_t)lvl[(size_t)i * k + t];
        int32_t rel = emax - e;
        if (rel > ORC_REL_MAX) rel = ORC_REL_MAX;
        v = lut[rel];
      }
      w[(size_t)i * k + t] = v;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Route construction, restating src/seq/aco_sequential.c:477-681.           */
/* Demand extension (no reference counterpart; the reference's capacity is a */
/* customer count): a customer j is eligible only if load + d_j <= Q; the    */
/* vehicle loop runs while remaining > 0, remaining_demand > (K-v-1) Q and   */
/* load < Q; the repair pass fills from the last vehicle backwards with the  */
/* nearest eligible customer.  With every d_j = 1 this is the reference.     */
/* ------------------------------------------------------------------------ */

typedef struct {
  int n, K, k;
  int64_t cap;
  const float *x, *y;
  const int32_t *demand;   /* NULL => unit demand */
  const int32_t *cand;     /* [(n+1) * k] */
  const uint32_t *w;       /* [(n+1) * k] */
  uint32_t seed, epoch, ant, stream;
  uint32_t draws;          /* draws consumed so far */
  uint64_t *visited;
} OrcAnt;

static inline int vis_get(const uint64_t *v, int node) {
  return (int)((v[(unsigned)node >> 6] >> ((unsigned)node & 63u)) & 1u);
}
static inline void vis_set(uint64_t *v, int node) {
  v[(unsigned)node >> 6] |= (uint64_t)1u << ((unsigned)node & 63u);
}
static inline int64_t dem(const OrcAnt *a, int node) {
  return a->demand ? (int64_t)a->demand[node] : 1;
}

/* find_nearest_unvisited, aco_sequential.c:477-493 (strict '<', so the
 * lowest index wins ties), restricted to customers that fit. */
static int nearest_unvisited(const OrcAnt *a, int cur, int64_t load) {
  int best = 0;
  float best_d = INFINITY;
  for (int node = 1; node <= a->n; ++node) {
    if (vis_get(a->visited, node)) continue;
    if (load + dem(a, node) > a->cap) continue;
    float d = d2f(a->x, a->y, cur, node);
    if (d < best_d) {
      best_d = d;
      best = node;
    }
  }
  return best;
}

/* select_next_customer, aco_sequential.c:505-561, in exact integers:
 * denom = sum of eligible weights; if denom > 0 one draw r is consumed and
 * the first eligible t with cum_t * 2^24 >= r * denom is taken (the
 * reference's 'cumulative >= u * denom' with u = r / 2^24); else nearest. */
static int select_next(OrcAnt *a, int cur, int64_t load) {
  const int32_t *crow = a->cand + (size_t)cur * a->k;
  const uint32_t *wrow = a->w + (size_t)cur * a->k;
  uint64_t denom = 0;
  for (int t = 0; t < a->k; ++t) {
    int c = crow[t];
    if (c <= 0 || vis_get(a->visited, c) || load + dem(a, c) > a->cap) continue;
    denom += wrow[t];
  }
  if (denom > 0) {
    uint64_t r = orc_draw24(a->seed, a->epoch, a->ant, a->stream, a->draws++);
    uint64_t thr = r * denom;
    uint64_t cum = 0;
    int last_valid = 0;
    for (int t = 0; t < a->k; ++t) {
      int c = crow[t];
      if (c <= 0 || vis_get(a->visited, c) || load + dem(a, c) > a->cap) continue;
      if (wrow[t] == 0) continue;
      cum += wrow[t];
      last_valid = c;
      if ((cum << 24) >= thr) return c;
    }
    if (last_valid > 0) return last_valid;
  }
  return nearest_unvisited(a, cur, load);
}

static double dist64(const float *x, const float *y, int a, int b) {
  double dx = (double)x[a] - (double)x[b];
  double dy = (double)y[a] - (double)y[b];
  double xx = dx * dx;
  double yy = dy * dy;
  return sqrt(xx + yy);
}

/* solution_cost, src/common/solution.c:126-137: FP64 sum over the routes in
 * order.  Routes are in compact form: K segments [0 ... 0] back to back. */
ORC_EXPORT double orc_route_cost(const float *x, const float *y,
                                 const int32_t *nodes, const int32_t *lens,
                                 int K) {
  double cost = 0.0;
  int off = 0;
  for (int v = 0; v < K; ++v) {
    for (int t = 0; t + 1 < lens[v]; ++t) {
      cost += dist64(x, y, nodes[off + t], nodes[off + t + 1]);
    }
    off += lens[v];
  }
  return cost;
}

/* Reference-CUDA depot rule (kernel_construct_solutions,
 * src/cuda/aco_cuda_kernels.cu:487-520), restated on the integer weights.
 * The reference weighs closing the route against the candidates by
 * 2 (1/(d0+eps))^beta versus tau^alpha eta^beta; in 1/16-octave levels the
 * close level of row i is e_dep - lvl0[i] (e_dep = 16 (1 - alpha log2 tau_min),
 * lvl0 = eta level of d(i,0)^2) and, on the row's weight scale,
 * rdep[i] = emax_i - (e_dep - lvl0[i]) levels below the row maximum. */
ORC_EXPORT void orc_depot_rel(int n, int k, const int32_t *cand, const uint16_t *lvl,
                              const uint8_t *tau, const int32_t *A, const uint16_t *lvl0,
                              int32_t e_dep, int32_t *rdep) {
  size_t stride = (size_t)n + 1;
  for (int i = 0; i <= n; ++i) {
    int have = 0;
    int32_t emax = 0;
    for (int t = 0; t < k; ++t) {
      int c = cand[(size_t)i * k + t];
      if (c <= 0) continue;
      int32_t e = A[tau[(size_t)i * stride + c]] - (int32_t)lvl[(size_t)i * k + t];
      if (!have || e > emax) emax = e;
      have = 1;
    }
    rdep[i] = have ? emax - (e_dep - (int32_t)lvl0[i]) : 0;
  }
}

/* Close weight 2^23 2^(-r/16) on the row's weight scale, exact in FP64:
 * LUT[r mod 16] 2^(-floor(r/16)); 0 from r = 255 on. */
static double depot_weight(int32_t r, const uint32_t *lut) {
  if (r >= ORC_REL_MAX) return 0.0;
  int32_t q = (r >= 0) ? (r / 16) : -((-r + 15) / 16);
  return ldexp((double)lut[r - 16 * q], -q);
}

typedef struct {
  int rule;              /* 0 sequential path, 1 reference CUDA kernel */
  const int32_t *rdep;   /* rule 1: [(n+1)] */
  const uint32_t *lut;   /* rule 1: [256] */
} OrcRule;

static int construct_ant(int n, int K, int k, int64_t cap, const float *x, const float *y,
                         const int32_t *demand, const int32_t *cand, const uint32_t *w,
                         uint32_t seed, uint32_t epoch, uint32_t ant, uint32_t stream,
                         const OrcRule *rule, int32_t *nodes_out, int32_t *lens_out,
                         double *cost_out, int32_t *steps_out, uint32_t *draws_out);

/* build_ant_solution, aco_sequential.c:616-681.  Writes the compact route
 * (capacity n + 2K), the K lengths, the FP64 cost and the number of moves
 * (customers plus depot returns).  Returns 1 if every customer is served. */
ORC_EXPORT int orc_construct_ant(int n, int K, int k, int64_t cap,
                                 const float *x, const float *y,
                                 const int32_t *demand, const int32_t *cand,
                                 const uint32_t *w, uint32_t seed,
                                 uint32_t epoch, uint32_t ant, uint32_t stream,
                                 int32_t *nodes_out, int32_t *lens_out,
                                 double *cost_out, int32_t *steps_out,
                                 uint32_t *draws_out) {
  OrcRule r = {0, NULL, NULL};
  return construct_ant(n, K, k, cap, x, y, demand, cand, w, seed, epoch, ant, stream, &r,
                       nodes_out, lens_out, cost_out, steps_out, draws_out);
}

/* The same with the reference-CUDA depot rule (rule 1): vehicle v extends
 * while customers remain and load < Q; once the remaining demand fits the
 * later vehicles the route may close -- at the depot at once, with no
 * eligible candidate at once, and after a roulette draw when a second draw
 * u satisfies u (denom + w_depot) >= denom (FP64, u = r / 2^24). */
ORC_EXPORT int orc_construct_ant_rule(int n, int K, int k, int64_t cap,
                                      const float *x, const float *y,
                                      const int32_t *demand, const int32_t *cand,
                                      const uint32_t *w, uint32_t seed,
                                      uint32_t epoch, uint32_t ant, uint32_t stream,
                                      int rule, const int32_t *rdep, const uint32_t *lut,
                                      int32_t *nodes_out, int32_t *lens_out,
                                      double *cost_out, int32_t *steps_out,
                                      uint32_t *draws_out) {
  OrcRule r = {rule, rdep, lut};
  return construct_ant(n, K, k, cap, x, y, demand, cand, w, seed, epoch, ant, stream, &r,
                       nodes_out, lens_out, cost_out, steps_out, draws_out);
}

/* A step of the reference-CUDA rule where the route may close: no eligible
 * candidate closes it; otherwise the roulette draw picks a candidate and a
 * second draw decides whether the route closes instead (returns 0). */
static int select_close(OrcAnt *a, int cur, int64_t load, const OrcRule *rule) {
  const int32_t *crow = a->cand + (size_t)cur * a->k;
  const uint32_t *wrow = a->w + (size_t)cur * a->k;
  uint64_t denom = 0;
  for (int t = 0; t < a->k; ++t) {
    int c = crow[t];
    if (c <= 0 || vis_get(a->visited, c) || load + dem(a, c) > a->cap) continue;
    denom += wrow[t];
  }
  if (denom == 0) return 0;
  int next = select_next(a, cur, load);  /* consumes the roulette draw */
  uint64_t r2 = orc_draw24(a->seed, a->epoch, a->ant, a->stream, a->draws++);
  double wd = depot_weight(rule->rdep[cur], rule->lut);
  if ((double)r2 * ((double)denom + wd) >= (double)denom * 16777216.0) return 0;
  return next;
}

static int construct_ant(int n, int K, int k, int64_t cap, const float *x, const float *y,
                         const int32_t *demand, const int32_t *cand, const uint32_t *w,
                         uint32_t seed, uint32_t epoch, uint32_t ant, uint32_t stream,
                         const OrcRule *rule, int32_t *nodes_out, int32_t *lens_out,
                         double *cost_out, int32_t *steps_out, uint32_t *draws_out) {
  int words = n / 64 + 1;
  uint64_t *visited = (uint64_t *)calloc((size_t)words, sizeof(uint64_t));
  int32_t *routes = (int32_t *)malloc(sizeof(int32_t) * (size_t)K * (size_t)(n + 2));
  int32_t *rlen = (int32_t *)calloc((size_t)K, sizeof(int32_t));
  int64_t *loads = (int64_t *)calloc((size_t)K, sizeof(int64_t));
  OrcAnt a = {n, K, k, cap < 1 ? 1 : cap, x, y, demand, cand, w,
              seed, epoch, ant, stream, 0u, visited};
  int64_t remaining = n;
  int64_t rem_dem = 0;
  for (int j = 1; j <= n; ++j) rem_dem += dem(&a, j);

  for (int v = 0; v < K; ++v) {
    int32_t *r = routes + (size_t)v * (n + 2);
    r[rlen[v]++] = 0;
    int cur = 0;
    int64_t future = (int64_t)(K - v - 1) * a.cap;
    int64_t limit = rule->rule == 1 ? 0 : future;
    while (remaining > 0 && rem_dem > limit && loads[v] < a.cap) {
      int next;
      if (rule->rule == 1 && rem_dem <= future) {
        if (cur == 0) break;
        next = select_close(&a, cur, loads[v], rule);
      } else {
        next = select_next(&a, cur, loads[v]);
      }
      if (next <= 0 || vis_get(visited, next)) break;
      r[rlen[v]++] = next;
      vis_set(visited, next);
      loads[v] += dem(&a, next);
      --remaining;
      rem_dem -= dem(&a, next);
      cur = next;
    }
    r[rlen[v]++] = 0;
  }

  if (remaining > 0) {
    for (int v = K - 1; v >= 0 && remaining > 0; --v) {
      int32_t *r = routes + (size_t)v * (n + 2);
      if (rlen[v] > 0 && r[rlen[v] - 1] == 0) --rlen[v];
      while (remaining > 0 && loads[v] < a.cap) {
        int cur = (rlen[v] > 0) ? r[rlen[v] - 1] : 0;
        int next = nearest_unvisited(&a, cur, loads[v]);
        if (next <= 0 || vis_get(visited, next)) break;
        r[rlen[v]++] = next;
        vis_set(visited, next);
        loads[v] += dem(&a, next);
        --remaining;
      }
      r[rlen[v]++] = 0;
    }
  }

  int off = 0, steps = 0;
  for (int v = 0; v < K; ++v) {
    memcpy(nodes_out + off, routes + (size_t)v * (n + 2), sizeof(int32_t) * (size_t)rlen[v]);
    lens_out[v] = rlen[v];
    off += rlen[v];
    steps += rlen[v] - 1;
  }
  *cost_out = orc_route_cost(x, y, nodes_out, lens_out, K);
  *steps_out = steps;
  if (draws_out) *draws_out = a.draws;
  free(visited);
  free(routes);
  free(rlen);
  free(loads);
  return remaining == 0;
}

/* ------------------------------------------------------------------------ */
/* Pheromone update on the quantized matrix.                                 */
/* ------------------------------------------------------------------------ */

/* kernel_evaporate_tau, src/cuda/aco_cuda_kernels.cu:145-155 (exact). */
ORC_EXPORT void orc_evaporate(uint8_t *tau, uint64_t total, uint8_t delta,
                              uint8_t q_min) {
  for (uint64_t i = 0; i < total; ++i) {
    uint8_t q = tau[i];
    tau[i] = ((int)q > (int)q_min + (int)delta) ? (uint8_t)(q - delta) : q_min;
  }
}

/* quantize_tau / dequantize_tau, aco_cuda_kernels.cu:25-45, with the host
 * libm's expf/logf.  The device functions can differ from these by an ulp,
 * so a deposited cell may differ by one level from the GPU; the GPU deposit
 * is checked bit-exactly against the reference's own kernel instead. */
ORC_EXPORT uint8_t orc_deposit_level(uint8_t q, float dep, float log_min,
                                     float log_step, uint8_t q_min,
                                     uint8_t q_max) {
  float old_tau = expf(fmaf((float)q, log_step, log_min));
  float tau = old_tau + dep;
  if (tau <= 0.0f) return q_min;
  float log_t = logf(tau);
  float q_f = (log_t - log_min) / log_step;
  if (q_f <= (float)q_min) return q_min;
  if (q_f >= (float)q_max) return q_max;
  return (uint8_t)roundf(q_f);
}

/* kernel_deposit_solution / kernel_deposit_flat_solution,
 * aco_cuda_kernels.cu:592-668: for every arc (u,v) of every route, in route
 * order, new = quantize(dequantize(tau[u][v]) + dep) is max-ed into
 * tau[u][v] and tau[v][u].  Routes in compact form. */
ORC_EXPORT void orc_deposit(uint8_t *tau, int n, const int32_t *nodes,
                            const int32_t *lens, int K, float dep,
                            float log_min, float log_step, uint8_t q_min,
                            uint8_t q_max) {
  size_t stride = (size_t)n + 1;
  int off = 0;
  for (int v = 0; v < K; ++v) {
    for (int t = 1; t < lens[v]; ++t) {
      int u = nodes[off + t - 1], c = nodes[off + t];
      size_t fwd = (size_t)u * stride + c, rev = (size_t)c * stride + u;
      uint8_t nq = orc_deposit_level(tau[fwd], dep, log_min, log_step, q_min, q_max);
      if (nq > tau[fwd]) tau[fwd] = nq;
      if (nq > tau[rev]) tau[rev] = nq;
    }
    off += lens[v];
  }
}
