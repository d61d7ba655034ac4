// aco_solver.cu -- host side of the B200 ACO-for-CVRP library: the context
// behind the C ABI (include/aco_b200.h), the device-resident epoch loop in
// CUDA-graph chunks, and the reference-facing aco_vrp_cuda_with_capacity
// (src/cuda/aco_cuda.cu:188-454) with its progress output.
#include "aco_internal.cuh"
#include "aco_prior_internal.h"

extern "C" {
#include "aco.h"
#include "aco_b200.h"
#include "aco_config.h"
#include "solution.h"
}

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

namespace acob200 {
cudaError_t launch_evap_deposit_explicit(const InstanceView &iv,
                                         const PheromoneView &pv,
                                         const AntBuffers &ab, int best_ant,
                                         float dep_iter,
                                         const int *gbest_nodes,
                                         const int *gbest_lens,
                                         float dep_global,
                                         unsigned int *counter, int grid,
                                         cudaStream_t s);
}

using namespace acob200;

namespace {

constexpr int kChunkEpochs = 16;

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  size_t bytes = (count * sizeof(T) + 15) & ~size_t(15);
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
  return e;
}

}  // namespace

struct aco_b200_ctx {
  int device = 0;
  int num_sms = 148;
  int max_smem = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t side = nullptr;       // evaporation beside the construction
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool ready = false;

  // problem
  int n = 0, K = 0, k = 0, m = 0;
  long long cap = 0, total_demand = 0;
  bool unit = true;
  uint32_t seed = 0;
  float log_min = 0.f, log_step = 0.f, Qs = 0.f;
  uint8_t delta = 0, q_tau0 = 0;

  // host tables
  int32_t A[256];
  uint32_t lut[256];
  std::vector<float> thr;

  // device buffers
  float2 *d_coords = nullptr;
  int *d_demand = nullptr;
  uint16_t *d_cand = nullptr, *d_lvl = nullptr;
  uint16_t *d_tier = nullptr;  // neighbours of ranks k+1 .. k+64 (fallback)
  uint16_t *d_tier2 = nullptr;  // ranks k+65 .. k+256 (fallback, n >= kTier2MinCustomers)
  float *d_thr = nullptr;
  int32_t *d_A = nullptr;
  uint32_t *d_lut = nullptr;
  uint8_t *d_tau = nullptr;
  uint8_t *d_tau2 = nullptr;  // second pheromone buffer of the pipelined epochs
  uint32_t *d_w = nullptr;
  uint8_t *d_rel = nullptr;
  AntBuffers ab = {};
  DevState *d_state = nullptr;
  EpochRec *d_log = nullptr;
  int *d_gbest_nodes = nullptr, *d_gbest_lens = nullptr;
  int *d_tmp_nodes = nullptr, *d_tmp_lens = nullptr;
  int *d_iter_nodes = nullptr, *d_iter_lens = nullptr;  // exchanged iteration best
  int32_t *d_rdep = nullptr;  // depot rule 1: depot-close levels per row
  uint16_t *d_lvl0 = nullptr; // depot rule 1: eta level of d(i,0)^2
  unsigned int *d_counter = nullptr;

  // host mirrors
  DevState *h_state = nullptr;  // pinned
  int log_read = 0;

  InstanceView iv = {};
  PheromoneView pv = {};
  EpochTables et = {};
  SmemPlan plan = {};
  int evap_grid = 1;

  cudaGraphExec_t graph_chunk = nullptr;
  cudaGraphExec_t graph_one = nullptr;
  int graph_gen = 1;  // changes whenever the captured launch arguments may have
  bool run_limit_off = false;  // device run limit known to be disabled
  int depot_rule = 0;
  int inject_alloc = 0;  // test hook: the n-th device allocation of a set-up fails
  // Kernel arguments the graphs were captured with: a set-up that leaves
  // them unchanged (same sizes, parameters and buffers) keeps the graphs.
  unsigned char graph_key[sizeof(InstanceView) + sizeof(PheromoneView) + sizeof(EpochTables) +
                          sizeof(AntBuffers) + sizeof(SmemPlan) + 8 * sizeof(void *)] = {};
  void make_graph_key(unsigned char *key) const;

  void free_buffers();
  ~aco_b200_ctx();
};

void aco_b200_ctx::make_graph_key(unsigned char *key) const {
  size_t o = 0;
  auto put = [&](const void *p, size_t b) {
    memcpy(key + o, p, b);
    o += b;
  };
  put(&iv, sizeof(iv));
  put(&pv, sizeof(pv));
  put(&et, sizeof(et));
  put(&ab, sizeof(ab));
  put(&plan, sizeof(plan));
  const void *ptrs[8] = {d_state, d_log, d_gbest_nodes, d_gbest_lens, d_counter, nullptr,
                         nullptr, nullptr};
  const long long grid = evap_grid;
  memcpy((void *)&ptrs[5], &grid, sizeof(grid));
  put(ptrs, sizeof(ptrs));
}

void aco_b200_ctx::free_buffers() {
  if (graph_chunk) cudaGraphExecDestroy(graph_chunk);
  if (graph_one) cudaGraphExecDestroy(graph_one);
  graph_chunk = graph_one = nullptr;
  ++graph_gen;
  void *ptrs[] = {d_coords, d_demand, d_cand, d_lvl, d_thr, d_A, d_lut, d_tau, d_tau2,
                  d_w, d_rel, ab.routes, ab.lens, ab.cost, ab.feasible, ab.steps,
                  ab.draws, ab.loads, ab.rep, ab.repc, d_state, d_log,
                  d_gbest_nodes, d_gbest_lens, d_tmp_nodes, d_tmp_lens, d_iter_nodes,
                  d_iter_lens, d_counter, d_rdep, d_lvl0, d_tier, d_tier2};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d_coords = nullptr; d_demand = nullptr; d_cand = d_lvl = nullptr; d_thr = nullptr;
  d_A = nullptr; d_lut = nullptr; d_tau = nullptr; d_tau2 = nullptr; d_w = nullptr;
  d_rel = nullptr;
  ab = AntBuffers{};
  d_state = nullptr; d_log = nullptr; d_gbest_nodes = d_gbest_lens = nullptr;
  d_tmp_nodes = d_tmp_lens = nullptr; d_iter_nodes = d_iter_lens = nullptr;
  d_rdep = nullptr; d_lvl0 = nullptr; d_tier = nullptr; d_tier2 = nullptr;
  d_counter = nullptr;
  ready = false;
}

aco_b200_ctx::~aco_b200_ctx() {
  cudaSetDevice(device);
  free_buffers();
  if (h_state) cudaFreeHost(h_state);
  if (own_stream && stream) cudaStreamDestroy(stream);
  if (side) cudaStreamDestroy(side);
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
}

#define TRY(call)                                                        \
  do {                                                                   \
    cudaError_t err__ = (call);                                          \
    if (err__ != cudaSuccess) {                                          \
      fprintf(stderr, "aco_b200: CUDA error %s at %s:%d\n",              \
              cudaGetErrorString(err__), __FILE__, __LINE__);            \
      return ACO_ERR_BACKEND;                                            \
    }                                                                    \
  } while (0)

#define TRY_ALLOC(call)                                                  \
  do {                                                                   \
    cudaError_t err__ = (ctx->inject_alloc > 0 && --ctx->inject_alloc == 0) \
                            ? cudaErrorMemoryAllocation                  \
                            : (call);                                    \
    if (err__ != cudaSuccess) {                                          \
      fprintf(stderr, "aco_b200: device allocation failed: %s\n",       \
              cudaGetErrorString(err__));                                \
      ctx->free_buffers();                                               \
      return err__ == cudaErrorMemoryAllocation ? ACO_ERR_ALLOCATION     \
                                                : ACO_ERR_BACKEND;       \
    }                                                                    \
  } while (0)

// Quantization constants and deposit scale (src/cuda/aco_cuda.cu:198-242).
static void derive_params(double rho, double tau0, float *log_min,
                          float *log_step, uint8_t *delta, uint8_t *q_tau0) {
  const float lmin = logf(0.0001f);
  const float lmax = logf(100.0f);
  const float step = (lmax - lmin) / (float)(255 - 0);
  const float log_rho = logf(1.0f - (float)rho);
  *log_min = lmin;
  *log_step = step;
  *delta = (uint8_t)fmaxf(1.0f, roundf(-log_rho / step));
  *q_tau0 = (uint8_t)fmaxf(0.0f, fminf(255.0f, roundf((logf((float)tau0) - lmin) / step)));
}

// Weight tables: A[q] (tau^alpha in 1/16-octave levels), LUT (2^23 2^(-r/16)),
// and the d^2 thresholds of the eta^beta levels.
static void build_tables(double alpha, double beta, float log_step, int32_t *A,
                         uint32_t *lut, std::vector<float> &thr) {
  const double ln2 = 0.69314718055994530942;
  for (int q = 0; q < 256; ++q)
    A[q] = (int32_t)std::floor(alpha * (double)q * (double)log_step * kLevelsPerOctave / ln2 + 0.5);
  for (int r = 0; r < kRelMax; ++r)
    lut[r] = (uint32_t)std::floor(8388608.0 * std::exp2(-(double)r / kLevelsPerOctave) + 0.5);
  lut[kRelMax] = 0u;
  thr.assign(kThresholds, INFINITY);
  if (beta > 0.0) {
    for (int j = 1; j <= kThresholds; ++j) {
      double t = std::exp2(2.0 * (double)j / (beta * kLevelsPerOctave));
      thr[j - 1] = (t > 3.0e38) ? INFINITY : (float)t;
    }
  }
}

static int build_graph(aco_b200_ctx *ctx, int epochs, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  // One epoch: weights, then the construction and (on the side stream) the
  // evaporation into the other pheromone buffer, then iteration best, global
  // best, stop rules and the deposits, which switch the buffers.
  for (int e = 0; e < epochs && err == cudaSuccess; ++e) {
    err = launch_weights(ctx->iv, ctx->pv, ctx->et, ctx->d_state, ctx->stream);
    if (err == cudaSuccess) err = cudaEventRecord(ctx->ev_fork, ctx->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
    if (err == cudaSuccess)
      err = launch_evaporate_to(ctx->pv, ctx->d_tau2, ctx->d_state, ctx->evap_grid, ctx->side);
    if (err == cudaSuccess)
      err = launch_construct(ctx->iv, ctx->et, ctx->ab, ctx->plan, ctx->d_state,
                             ctx->seed, 0, 0, 1, ctx->stream);
    if (err == cudaSuccess) err = cudaEventRecord(ctx->ev_join, ctx->side);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
    if (err == cudaSuccess)
      err = launch_best_deposit(ctx->iv, ctx->ab, ctx->pv, ctx->d_tau2, ctx->d_state,
                                ctx->d_gbest_nodes, ctx->d_gbest_lens, ctx->d_log,
                                ctx->stream);
  }
  cudaError_t end = cudaStreamEndCapture(ctx->stream, &g);
  if (err != cudaSuccess || end != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    fprintf(stderr, "aco_b200: graph capture failed: %s\n",
            cudaGetErrorString(err != cudaSuccess ? err : end));
    return ACO_ERR_BACKEND;
  }
  err = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  TRY(err);
  return ACO_OK;
}

static void fill_state(aco_b200_state *o, const DevState &s) {
  o->epochs = s.epoch;
  o->iter_since_best = s.iter_since_best;
  o->stopped = (s.stop_flags & ~kStopRunLimit) != 0;
  o->stop_reason = s.stop_flags & ~kStopRunLimit;
  o->found = s.found;
  o->improved = s.improved;
  o->best_ant = s.best_ant;
  o->error = s.error;
  o->global_best = s.global_best;
  o->iter_best = s.iter_best;
  o->dep_iter = s.dep_iter;
  o->dep_global = s.dep_global;
  o->total_steps = s.total_steps;
}

extern "C" {

int aco_b200_create(aco_b200_ctx **out, int device) {
  if (!out) return ACO_ERR_INVALID_INPUT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    fprintf(stderr, "aco_b200: no CUDA device %d\n", device);
    return ACO_ERR_BACKEND;
  }
  aco_b200_ctx *ctx = new aco_b200_ctx();
  ctx->device = device;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  ctx->max_smem = construct_max_smem();
  if (prepare_construct_kernels() != cudaSuccess) {
    fprintf(stderr, "aco_b200: cannot configure the construct kernels\n");
    delete ctx;
    return ACO_ERR_BACKEND;
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_state, sizeof(DevState)) != cudaSuccess) {
    delete ctx;
    return ACO_ERR_BACKEND;
  }
  ctx->own_stream = true;
  *out = ctx;
  return ACO_OK;
}

int aco_b200_destroy(aco_b200_ctx *ctx) {
  delete ctx;
  return ACO_OK;
}

int aco_b200_set_stream(aco_b200_ctx *ctx, void *cuda_stream) {
  if (!ctx) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  if (ctx->graph_chunk) cudaGraphExecDestroy(ctx->graph_chunk);
  if (ctx->graph_one) cudaGraphExecDestroy(ctx->graph_one);
  ctx->graph_chunk = ctx->graph_one = nullptr;
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (cuda_stream) {
    ctx->stream = (cudaStream_t)cuda_stream;
    ctx->own_stream = false;
  } else {
    TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return ACO_OK;
}

int aco_b200_setup(aco_b200_ctx *ctx, const aco_b200_problem *p) {
  if (!ctx || !p || !p->x || !p->y) return ACO_ERR_INVALID_INPUT;
  if (p->n <= 0 || p->K <= 0 || p->n > 65534 || p->capacity <= 0) {
    fprintf(stderr, "aco_b200: invalid n=%d K=%d capacity=%lld (n in 1..65534)\n",
            p->n, p->K, p->capacity);
    return ACO_ERR_INVALID_INPUT;
  }
  const int n = p->n;
  long long total_demand = n;
  int max_demand = 1;
  bool unit = true;
  if (p->demand) {
    if (p->demand[0] != 0) return ACO_ERR_INVALID_INPUT;
    total_demand = 0;
    for (int j = 1; j <= n; ++j) {
      if (p->demand[j] < 1) return ACO_ERR_INVALID_INPUT;
      if (p->demand[j] != 1) unit = false;
      if (p->demand[j] > max_demand) max_demand = p->demand[j];
      total_demand += p->demand[j];
    }
  }
  // Loads and remaining demand are 32-bit on the device.
  if (total_demand > 0x7fffffffLL || p->capacity > 0x7fffffffLL) {
    fprintf(stderr, "aco_b200: total demand and capacity must be below 2^31\n");
    return ACO_ERR_INVALID_INPUT;
  }
  int k = p->cand_k > 0 ? p->cand_k : 32;
  if (k > kMaxCand) k = kMaxCand;
  if (k > n) k = n;
  int m = p->ants > 0 ? p->ants : 256;
  if ((long long)m * (n + 2LL * p->K) > (1LL << 31)) return ACO_ERR_INVALID_INPUT;
  if (p->depot_rule != kDepotRuleSeq && p->depot_rule != kDepotRuleCudaRef) {
    fprintf(stderr, "aco_b200: invalid depot_rule=%d (0 or 1)\n", p->depot_rule);
    return ACO_ERR_INVALID_INPUT;
  }
  if (p->ant_base < 0 || (long long)p->ant_base + m > 0x7fffffffLL) {
    fprintf(stderr, "aco_b200: invalid ant_base=%d\n", p->ant_base);
    return ACO_ERR_INVALID_INPUT;
  }

  cudaSetDevice(ctx->device);
  // Same sizes as the last set-up: the device buffers are reused (no
  // allocation), and the graphs too when their captured arguments match.
  const bool reuse = ctx->ready && ctx->n == n && ctx->K == p->K && ctx->k == k &&
                     ctx->m == m && ctx->depot_rule == p->depot_rule;
  if (!reuse) ctx->free_buffers();
  ctx->ready = false;
  ctx->depot_rule = p->depot_rule;
  ctx->n = n;
  ctx->K = p->K;
  ctx->k = k;
  ctx->m = m;
  ctx->cap = p->capacity;
  ctx->total_demand = total_demand;
  ctx->unit = unit;
  ctx->seed = p->seed;
  derive_params(p->rho, p->tau0, &ctx->log_min, &ctx->log_step, &ctx->delta, &ctx->q_tau0);
  ctx->Qs = (float)p->Q * 100.0f;
  build_tables(p->alpha, p->beta, ctx->log_step, ctx->A, ctx->lut, ctx->thr);

  const size_t rows = (size_t)n + 1;
  const int R = n + 2 * p->K;
  const unsigned long long tau_total = (unsigned long long)rows * rows;
  if (!reuse) {
    TRY_ALLOC(dalloc(&ctx->d_coords, rows));
    TRY_ALLOC(dalloc(&ctx->d_demand, rows));
    TRY_ALLOC(dalloc(&ctx->d_cand, rows * k));
    TRY_ALLOC(dalloc(&ctx->d_lvl, rows * k));
    TRY_ALLOC(dalloc(&ctx->d_tier, rows * kTierLen));
    if (n >= kTier2MinCustomers) TRY_ALLOC(dalloc(&ctx->d_tier2, rows * kTier2Len));
    TRY_ALLOC(dalloc(&ctx->d_thr, (size_t)kThresholds));
    TRY_ALLOC(dalloc(&ctx->d_A, 256));
    TRY_ALLOC(dalloc(&ctx->d_lut, 256));
    TRY_ALLOC(dalloc(&ctx->d_tau, (size_t)tau_total));
    TRY_ALLOC(dalloc(&ctx->d_tau2, (size_t)tau_total));
    TRY_ALLOC(dalloc(&ctx->d_w, rows * k));
    TRY_ALLOC(dalloc(&ctx->d_rel, rows * k));
    TRY_ALLOC(dalloc(&ctx->ab.routes, (size_t)m * R));
    TRY_ALLOC(dalloc(&ctx->ab.lens, (size_t)m * p->K));
    TRY_ALLOC(dalloc(&ctx->ab.cost, (size_t)m));
    TRY_ALLOC(dalloc(&ctx->ab.feasible, (size_t)m));
    TRY_ALLOC(dalloc(&ctx->ab.steps, (size_t)m));
    TRY_ALLOC(dalloc(&ctx->ab.draws, (size_t)m));
    TRY_ALLOC(dalloc(&ctx->ab.loads, (size_t)m * p->K));
    TRY_ALLOC(dalloc(&ctx->ab.rep, (size_t)m * n));
    TRY_ALLOC(dalloc(&ctx->ab.repc, (size_t)m * p->K));
    TRY_ALLOC(dalloc(&ctx->d_state, 1));
    TRY_ALLOC(dalloc(&ctx->d_log, (size_t)kLogCap));
    TRY_ALLOC(dalloc(&ctx->d_gbest_nodes, (size_t)R));
    TRY_ALLOC(dalloc(&ctx->d_gbest_lens, (size_t)p->K));
    TRY_ALLOC(dalloc(&ctx->d_tmp_nodes, (size_t)R));
    TRY_ALLOC(dalloc(&ctx->d_tmp_lens, (size_t)p->K));
    TRY_ALLOC(dalloc(&ctx->d_iter_nodes, (size_t)R));
    TRY_ALLOC(dalloc(&ctx->d_iter_lens, (size_t)p->K));
    if (p->depot_rule == kDepotRuleCudaRef) {
      TRY_ALLOC(dalloc(&ctx->d_rdep, rows));
      TRY_ALLOC(dalloc(&ctx->d_lvl0, rows));
    }
    TRY_ALLOC(dalloc(&ctx->d_counter, 1));
  }

  std::vector<float2> xy(rows);
  std::vector<int> dem(rows, 1);
  dem[0] = 0;
  for (size_t i = 0; i < rows; ++i) xy[i] = make_float2(p->x[i], p->y[i]);
  if (p->demand) for (size_t i = 0; i < rows; ++i) dem[i] = p->demand[i];
  cudaStream_t s = ctx->stream;
  if (reuse) TRY(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned int), s));
  TRY(cudaMemcpyAsync(ctx->d_coords, xy.data(), rows * sizeof(float2), cudaMemcpyHostToDevice, s));
  TRY(cudaMemcpyAsync(ctx->d_demand, dem.data(), rows * sizeof(int), cudaMemcpyHostToDevice, s));
  TRY(cudaMemcpyAsync(ctx->d_thr, ctx->thr.data(), kThresholds * sizeof(float), cudaMemcpyHostToDevice, s));
  TRY(cudaMemcpyAsync(ctx->d_A, ctx->A, sizeof(ctx->A), cudaMemcpyHostToDevice, s));
  TRY(cudaMemcpyAsync(ctx->d_lut, ctx->lut, sizeof(ctx->lut), cudaMemcpyHostToDevice, s));

  InstanceView &iv = ctx->iv;
  iv.n = n;
  iv.K = p->K;
  iv.k = k;
  iv.m = m;
  iv.cap = p->capacity;
  iv.total_demand = total_demand;
  iv.unit = unit ? 1 : 0;
  iv.max_demand = max_demand;
  iv.route_stride = R;
  iv.ant_base = p->ant_base;
  iv.stage_extra_tx = 0;
  iv.depot_rule = p->depot_rule;
  iv.coords = ctx->d_coords;
  iv.demand = ctx->d_demand;
  iv.cand = ctx->d_cand;
  iv.lvl = ctx->d_lvl;
  // The fallback's tier lists pay for their two L2 round trips only where
  // the full scan is long (each lane walks (n+1)/32 bitmap bits): at n=1000
  // the construction takes 279 -> 268 us with them, at n=100 34.2 -> 36.0.
  iv.tier = (n >= kTierMinCustomers) ? ctx->d_tier : nullptr;
  // The second tier (ranks k+65 .. k+256) from n = 1500 on, where the full
  // scan walks two or more bitmap words per lane: clustered n=2000 756 ->
  // 706 us with it, n=3000 1544 -> 1420 us; at n=1000 (one word per lane)
  // its L2 loads cost more than the scans they replace.
  iv.tier2 = (n >= kTier2MinCustomers) ? ctx->d_tier2 : nullptr;
  PheromoneView &pv = ctx->pv;
  pv.tau = ctx->d_tau;
  pv.total = tau_total;
  pv.log_min = ctx->log_min;
  pv.log_step = ctx->log_step;
  pv.q_min = 0;
  pv.q_max = 255;
  pv.delta = ctx->delta;
  ctx->et.w = ctx->d_w;
  ctx->et.rel = ctx->d_rel;
  ctx->et.A = ctx->d_A;
  ctx->et.lut = ctx->d_lut;
  ctx->et.rdep = ctx->d_rdep;
  ctx->et.tau_alt = ctx->d_tau2;
  ctx->et.lvl0 = ctx->d_lvl0;
  // Level of the reference's depot factor 2 relative to the candidates'
  // tau_min^alpha scale: 16 (1 - alpha log2 tau_min).
  ctx->et.e_dep = (int)llround(16.0 * (1.0 - p->alpha * (double)ctx->log_min / log(2.0)));
  ctx->plan = plan_construct(iv, -1, ctx->num_sms, ctx->max_smem);
  ctx->evap_grid = evap_grid_for(tau_total, ctx->num_sms);

  TRY(launch_knn_levels(ctx->d_coords, n, k, ctx->d_thr, kThresholds, ctx->d_cand, ctx->d_lvl, s));
  TRY(launch_knn_tier(ctx->d_coords, n, k, ctx->d_tier, iv.tier2 ? ctx->d_tier2 : nullptr, s));
  TRY(launch_fill_u8(ctx->d_tau, tau_total, ctx->q_tau0, s));
  if (ctx->d_lvl0) TRY(launch_depot_levels(ctx->d_coords, n, ctx->d_thr, kThresholds, ctx->d_lvl0, s));

  DevState st = {};
  st.global_best = DBL_MAX;
  st.iter_best = DBL_MAX;
  st.best_ant = -1;
  st.stagnation = p->stagnation_epochs > 0 ? p->stagnation_epochs : 0;
  st.fixed_epochs = p->fixed_epochs > 0 ? p->fixed_epochs : 0;
  st.min_rel = p->min_rel_improvement > 0.0 ? p->min_rel_improvement : 1e-3;
  st.timeout_ns = p->timeout_seconds > 0.0
                      ? (unsigned long long)(p->timeout_seconds * 1e9)
                      : 0ull;
  st.Qs = ctx->Qs;
  st.seed = ctx->seed;
  *ctx->h_state = st;
  TRY(cudaMemcpyAsync(ctx->d_state, ctx->h_state, sizeof(DevState), cudaMemcpyHostToDevice, s));
  TRY(cudaStreamSynchronize(s));
  ctx->log_read = 0;
  ctx->run_limit_off = true;  // fresh state: run_limit = 0
  unsigned char key[sizeof(ctx->graph_key)];
  memset(key, 0, sizeof(key));
  ctx->make_graph_key(key);
  if (memcmp(key, ctx->graph_key, sizeof(key)) != 0) {
    if (ctx->graph_chunk) cudaGraphExecDestroy(ctx->graph_chunk);
    if (ctx->graph_one) cudaGraphExecDestroy(ctx->graph_one);
    ctx->graph_chunk = ctx->graph_one = nullptr;
    memcpy(ctx->graph_key, key, sizeof(key));
    ++ctx->graph_gen;
  }
  ctx->ready = true;
  return ACO_OK;
}

static int ensure_graphs(aco_b200_ctx *ctx) {
  if (!ctx->graph_one) {
    int rc = build_graph(ctx, 1, &ctx->graph_one);
    if (rc) return rc;
  }
  if (!ctx->graph_chunk) {
    int rc = build_graph(ctx, kChunkEpochs, &ctx->graph_chunk);
    if (rc) return rc;
  }
  return ACO_OK;
}

int aco_b200_run(aco_b200_ctx *ctx, int max_epochs, aco_b200_state *state,
                 aco_b200_epoch_record *records, int max_records,
                 int *n_records) {
  if (!ctx || !ctx->ready || max_epochs < 0) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  int rc = ensure_graphs(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  TRY(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  TRY(cudaStreamSynchronize(s));
  const int limit = ctx->h_state->epoch + max_epochs;
  TRY(launch_set_run_limit(ctx->d_state, limit, s));
  ctx->run_limit_off = false;
  int nrec = 0;
  std::vector<EpochRec> recs;
  // Every pass either stops or advances the device epoch; the guard only
  // bounds the loop should a device-side rule misbehave.
  long long guard = (long long)max_epochs + 8;
  while (guard-- > 0) {
    TRY(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    TRY(cudaStreamSynchronize(s));
    const DevState &hs = *ctx->h_state;
    // Epoch records written since the last read.
    int avail = hs.log_count - ctx->log_read;
    if (avail > kLogCap) {
      ctx->log_read = hs.log_count - kLogCap;
      avail = kLogCap;
    }
    if (avail > 0 && records && nrec < max_records) {
      recs.resize(kLogCap);
      TRY(cudaMemcpy(recs.data(), ctx->d_log, sizeof(EpochRec) * kLogCap, cudaMemcpyDeviceToHost));
      for (int i = 0; i < avail && nrec < max_records; ++i) {
        const EpochRec &r = recs[(ctx->log_read + i) % kLogCap];
        aco_b200_epoch_record &o = records[nrec++];
        o.epoch = r.epoch;
        o.iter_since_best = r.iter_since_best;
        o.improved = r.improved;
        o.found = r.found;
        o.global_best = r.global_best;
        o.elapsed_ns = r.elapsed_ns;
      }
    }
    ctx->log_read = hs.log_count;
    if (hs.error) {
      fprintf(stderr, "aco_b200: device error flag 0x%x\n", hs.error);
      if (state) fill_state(state, hs);
      if (n_records) *n_records = nrec;
      return ACO_ERR_BACKEND;
    }
    if (hs.stop_flags || hs.epoch >= limit) break;
    const int left = limit - hs.epoch;
    if (left >= kChunkEpochs) {
      TRY(cudaGraphLaunch(ctx->graph_chunk, s));
    } else {
      for (int i = 0; i < left; ++i) TRY(cudaGraphLaunch(ctx->graph_one, s));
    }
  }
  if (state) fill_state(state, *ctx->h_state);
  if (n_records) *n_records = nrec;
  return ACO_OK;
}

int aco_b200_enqueue_epochs(aco_b200_ctx *ctx, int epochs) {
  if (!ctx || !ctx->ready || epochs < 0) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  int rc = ensure_graphs(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  if (!ctx->run_limit_off) {
    TRY(launch_set_run_limit(ctx->d_state, 0, s));
    ctx->run_limit_off = true;
  }
  int left = epochs;
  while (left >= kChunkEpochs) {
    TRY(cudaGraphLaunch(ctx->graph_chunk, s));
    left -= kChunkEpochs;
  }
  for (int i = 0; i < left; ++i) TRY(cudaGraphLaunch(ctx->graph_one, s));
  return ACO_OK;
}

int aco_b200_debug_inject(aco_b200_ctx *ctx, int what, int value) {
  if (!ctx || value < 0) return ACO_ERR_INVALID_INPUT;
  if (what == 1) {
    ctx->inject_alloc = value;
    return ACO_OK;
  }
  if (what == 2) {
    cudaSetDevice(ctx->device);
    ctx->iv.stage_extra_tx = value ? 16 : 0;
    if (ctx->graph_chunk) cudaGraphExecDestroy(ctx->graph_chunk);
    if (ctx->graph_one) cudaGraphExecDestroy(ctx->graph_one);
    ctx->graph_chunk = ctx->graph_one = nullptr;
    memset(ctx->graph_key, 0, sizeof(ctx->graph_key));
    ++ctx->graph_gen;
    return ACO_OK;
  }
  return ACO_ERR_INVALID_INPUT;
}

int aco_b200_get_depot_tables(aco_b200_ctx *ctx, uint16_t *lvl0, int32_t *rdep, int *e_dep) {
  if (!ctx || !ctx->ready || !ctx->d_rdep) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  TRY(cudaStreamSynchronize(ctx->stream));
  const size_t rows = (size_t)ctx->n + 1;
  if (lvl0) TRY(cudaMemcpy(lvl0, ctx->d_lvl0, rows * sizeof(uint16_t), cudaMemcpyDeviceToHost));
  if (rdep) TRY(cudaMemcpy(rdep, ctx->d_rdep, rows * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (e_dep) *e_dep = ctx->et.e_dep;
  return ACO_OK;
}

int aco_b200_apply_prior_mode(aco_b200_ctx *ctx, aco_b200_prior *prior, float gamma,
                              int mode) {
  if (!ctx || !ctx->ready || mode < 0 || mode > 1) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  // Plain levels first: they are the result without a prior and the base of
  // the residual mode.
  TRY(launch_knn_levels(ctx->d_coords, ctx->n, ctx->k, ctx->d_thr, kThresholds, ctx->d_cand,
                        ctx->d_lvl, s));
  if (prior && gamma > 0.f) {
    int rc = acob200::prior::learned_levels(prior, ctx->d_coords, ctx->d_demand, ctx->cap, ctx->n,
                                            ctx->k, ctx->d_cand, ctx->d_lvl, gamma, mode, s);
    if (rc) return rc;
  }
  TRY(cudaStreamSynchronize(s));
  return ACO_OK;
}

int aco_b200_apply_prior(aco_b200_ctx *ctx, aco_b200_prior *prior, float gamma) {
  return aco_b200_apply_prior_mode(ctx, prior, gamma, 0);
}

int aco_b200_graph_generation(aco_b200_ctx *ctx) {
  if (!ctx || !ctx->ready) return -1;
  return ctx->graph_gen & 0x7fffffff;
}

int aco_b200_shard_packet_ints(aco_b200_ctx *ctx) {
  if (!ctx || !ctx->ready) return -1;
  return shard_packet_size(ctx->n, ctx->K);
}

int aco_b200_shard_construct(aco_b200_ctx *ctx, int32_t *d_send) {
  if (!ctx || !ctx->ready || !d_send) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  if (!ctx->run_limit_off) {
    TRY(launch_set_run_limit(ctx->d_state, 0, s));
    ctx->run_limit_off = true;
  }
  // As in the epoch graph: the evaporation into the other pheromone buffer
  // runs on the side stream beside the construction.
  TRY(launch_weights(ctx->iv, ctx->pv, ctx->et, ctx->d_state, s));
  TRY(cudaEventRecord(ctx->ev_fork, s));
  TRY(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
  TRY(launch_evaporate_to(ctx->pv, ctx->d_tau2, ctx->d_state, ctx->evap_grid, ctx->side));
  TRY(launch_construct(ctx->iv, ctx->et, ctx->ab, ctx->plan, ctx->d_state, ctx->seed, 0, 0, 1, s));
  TRY(launch_shard_pack(ctx->iv, ctx->ab, ctx->d_state, d_send, s));
  TRY(cudaEventRecord(ctx->ev_join, ctx->side));
  TRY(cudaStreamWaitEvent(s, ctx->ev_join, 0));
  return ACO_OK;
}

int aco_b200_shard_update(aco_b200_ctx *ctx, const int32_t *d_recv, int world) {
  if (!ctx || !ctx->ready || !d_recv || world < 1) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  TRY(launch_shard_select(ctx->iv, ctx->d_state, d_recv, world, ctx->d_iter_nodes,
                          ctx->d_iter_lens, ctx->d_gbest_nodes, ctx->d_gbest_lens, ctx->d_log,
                          ctx->pv, ctx->d_tau2, s));
  return ACO_OK;
}

int aco_b200_profile_epochs(aco_b200_ctx *ctx, int epochs, float *kernel_ms) {
  if (!ctx || !ctx->ready || epochs < 0 || !kernel_ms) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev[5];
  for (int i = 0; i < 5; ++i) TRY(cudaEventCreate(&ev[i]));
  int rc = ACO_OK;
  if (launch_set_run_limit(ctx->d_state, 0, s) != cudaSuccess) rc = ACO_ERR_BACKEND;
  ctx->run_limit_off = true;
  for (int e = 0; e < epochs && rc == ACO_OK; ++e) {
    cudaError_t err = cudaEventRecord(ev[0], s);
    if (err == cudaSuccess) err = launch_weights(ctx->iv, ctx->pv, ctx->et, ctx->d_state, s);
    if (err == cudaSuccess) err = cudaEventRecord(ev[1], s);
    if (err == cudaSuccess)
      err = launch_construct(ctx->iv, ctx->et, ctx->ab, ctx->plan, ctx->d_state, ctx->seed, 0, 0, 1, s);
    if (err == cudaSuccess) err = cudaEventRecord(ev[2], s);
    if (err == cudaSuccess)
      err = launch_evaporate_to(ctx->pv, ctx->d_tau2, ctx->d_state, ctx->evap_grid, s);
    if (err == cudaSuccess) err = cudaEventRecord(ev[3], s);
    if (err == cudaSuccess)
      err = launch_best_deposit(ctx->iv, ctx->ab, ctx->pv, ctx->d_tau2, ctx->d_state,
                                ctx->d_gbest_nodes, ctx->d_gbest_lens, ctx->d_log, s);
    if (err == cudaSuccess) err = cudaEventRecord(ev[4], s);
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[4]);
    for (int i = 0; i < 4 && err == cudaSuccess; ++i) {
      float ms = 0.f;
      err = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      kernel_ms[i] += ms;
    }
    if (err != cudaSuccess) {
      fprintf(stderr, "aco_b200: profile failed: %s\n", cudaGetErrorString(err));
      rc = ACO_ERR_BACKEND;
    }
  }
  for (int i = 0; i < 5; ++i) cudaEventDestroy(ev[i]);
  return rc;
}

int aco_b200_profile_update(aco_b200_ctx *ctx, int launches, float *ms_per_launch) {
  if (!ctx || !ctx->ready || launches < 1 || !ms_per_launch) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int rc = ACO_OK;
  cudaError_t err = cudaEventCreate(&ev[0]);
  if (err == cudaSuccess) err = cudaEventCreate(&ev[1]);
  // The sweep reads the skip flag: make sure this epoch is not marked skipped.
  if (err == cudaSuccess) err = launch_set_run_limit(ctx->d_state, 0, s);
  ctx->run_limit_off = true;
  if (err == cudaSuccess) err = cudaMemsetAsync(&ctx->d_state->skip, 0, sizeof(int), s);
  // One untimed launch, then `launches` back to back between two events.
  if (err == cudaSuccess)
    err = launch_evaporate_to(ctx->pv, ctx->d_tau2, ctx->d_state, ctx->evap_grid, s);
  if (err == cudaSuccess) err = cudaEventRecord(ev[0], s);
  for (int i = 0; i < launches && err == cudaSuccess; ++i)
    err = launch_evaporate_to(ctx->pv, ctx->d_tau2, ctx->d_state, ctx->evap_grid, s);
  if (err == cudaSuccess) err = cudaEventRecord(ev[1], s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, ev[0], ev[1]);
  if (err != cudaSuccess) {
    fprintf(stderr, "aco_b200: profile_update failed: %s\n", cudaGetErrorString(err));
    rc = ACO_ERR_BACKEND;
  } else {
    *ms_per_launch = ms / (float)launches;
  }
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

int aco_b200_synchronize(aco_b200_ctx *ctx) {
  if (!ctx) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_get_state(aco_b200_ctx *ctx, aco_b200_state *state) {
  if (!ctx || !ctx->ready || !state) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  TRY(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  fill_state(state, *ctx->h_state);
  return ACO_OK;
}

int aco_b200_get_dims(aco_b200_ctx *ctx, int *n, int *K, int *k, int *m) {
  if (!ctx || !ctx->ready) return ACO_ERR_INVALID_INPUT;
  if (n) *n = ctx->n;
  if (K) *K = ctx->K;
  if (k) *k = ctx->k;
  if (m) *m = ctx->m;
  return ACO_OK;
}

int aco_b200_get_plan(aco_b200_ctx *ctx, int out[4]) {
  if (!ctx || !ctx->ready || !out) return ACO_ERR_INVALID_INPUT;
  out[0] = ctx->plan.wpb;
  out[1] = ctx->plan.layout;
  out[2] = ctx->plan.vreg;
  out[3] = (int)ctx->plan.total;
  return ACO_OK;
}

int aco_b200_get_best(aco_b200_ctx *ctx, int *nodes, int *lens, double *cost) {
  if (!ctx || !ctx->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  TRY(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  if (lens) TRY(cudaMemcpyAsync(lens, ctx->d_gbest_lens, sizeof(int) * ctx->K, cudaMemcpyDeviceToHost, s));
  if (nodes)
    TRY(cudaMemcpyAsync(nodes, ctx->d_gbest_nodes, sizeof(int) * (ctx->n + 2 * ctx->K),
                        cudaMemcpyDeviceToHost, s));
  TRY(cudaStreamSynchronize(s));
  if (cost) *cost = ctx->h_state->global_best;
  return ctx->h_state->global_best < DBL_MAX ? ACO_OK : ACO_ERR_NO_SOLUTION;
}

// The context's current pheromone buffer (read from the device state).
static int current_tau(aco_b200_ctx *ctx, uint8_t **out) {
  TRY(cudaMemcpyAsync(ctx->h_state, ctx->d_state, sizeof(DevState), cudaMemcpyDeviceToHost,
                      ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  *out = ctx->h_state->tau_sel ? ctx->d_tau2 : ctx->d_tau;
  return ACO_OK;
}

int aco_b200_get_tau(aco_b200_ctx *ctx, uint8_t *tau) {
  if (!ctx || !ctx->ready || !tau) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  uint8_t *cur = nullptr;
  int rc = current_tau(ctx, &cur);
  if (rc) return rc;
  TRY(cudaMemcpyAsync(tau, cur, ctx->pv.total, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_set_tau(aco_b200_ctx *ctx, const uint8_t *tau) {
  if (!ctx || !ctx->ready || !tau) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  uint8_t *cur = nullptr;
  int rc = current_tau(ctx, &cur);
  if (rc) return rc;
  TRY(cudaMemcpyAsync(cur, tau, ctx->pv.total, cudaMemcpyHostToDevice, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_get_candidates(aco_b200_ctx *ctx, int *cand, uint16_t *levels) {
  if (!ctx || !ctx->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  const size_t cnt = ((size_t)ctx->n + 1) * ctx->k;
  std::vector<uint16_t> c16(cnt);
  TRY(cudaMemcpyAsync(c16.data(), ctx->d_cand, cnt * 2, cudaMemcpyDeviceToHost, ctx->stream));
  if (levels) TRY(cudaMemcpyAsync(levels, ctx->d_lvl, cnt * 2, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  if (cand)
    for (size_t i = 0; i < cnt; ++i) cand[i] = c16[i];
  return ACO_OK;
}

int aco_b200_get_tier(aco_b200_ctx *ctx, uint16_t *tier) {
  if (!ctx || !ctx->ready || !tier) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  const size_t cnt = ((size_t)ctx->n + 1) * kTierLen;
  TRY(cudaMemcpyAsync(tier, ctx->d_tier, cnt * 2, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_get_tier2(aco_b200_ctx *ctx, uint16_t *tier2) {
  if (!ctx || !ctx->ready || !tier2 || !ctx->iv.tier2) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  const size_t cnt = ((size_t)ctx->n + 1) * kTier2Len;
  TRY(cudaMemcpyAsync(tier2, ctx->d_tier2, cnt * 2, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_get_tables(aco_b200_ctx *ctx, int32_t *A, uint32_t *lut,
                        float *thresholds, int n_thresholds) {
  if (!ctx || !ctx->ready) return ACO_ERR_INVALID_INPUT;
  if (A) memcpy(A, ctx->A, sizeof(ctx->A));
  if (lut) memcpy(lut, ctx->lut, sizeof(ctx->lut));
  if (thresholds)
    for (int j = 0; j < n_thresholds && j < kThresholds; ++j) thresholds[j] = ctx->thr[j];
  return ACO_OK;
}

int aco_b200_get_weights(aco_b200_ctx *ctx, uint32_t *w) {
  if (!ctx || !ctx->ready || !w) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  PheromoneView pv = ctx->pv;
  EpochTables et = ctx->et;
  int rc = current_tau(ctx, &pv.tau);
  if (rc) return rc;
  et.tau_alt = nullptr;
  TRY(launch_weights(ctx->iv, pv, et, nullptr, ctx->stream));
  const size_t cnt = ((size_t)ctx->n + 1) * ctx->k;
  TRY(cudaMemcpyAsync(w, ctx->d_w, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_construct(aco_b200_ctx *ctx, int epoch, int layout) {
  if (!ctx || !ctx->ready || epoch < 0 || layout < -1 || layout > 2)
    return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  SmemPlan plan = (layout < 0) ? ctx->plan
                               : plan_construct(ctx->iv, layout, ctx->num_sms, ctx->max_smem);
  if ((int)plan.total > ctx->max_smem) return ACO_ERR_INVALID_INPUT;
  PheromoneView pv = ctx->pv;
  EpochTables et = ctx->et;
  int rc = current_tau(ctx, &pv.tau);
  if (rc) return rc;
  et.tau_alt = nullptr;
  TRY(launch_weights(ctx->iv, pv, et, nullptr, ctx->stream));
  TRY(launch_construct(ctx->iv, ctx->et, ctx->ab, plan, nullptr, ctx->seed,
                       (uint32_t)epoch, 0, 0, ctx->stream));
  TRY(cudaStreamSynchronize(ctx->stream));
  return ACO_OK;
}

int aco_b200_construct_with_draws(aco_b200_ctx *ctx, const uint32_t *draws, int per_ant) {
  if (!ctx || !ctx->ready || !draws || per_ant < 1) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  PheromoneView pv = ctx->pv;
  EpochTables et = ctx->et;
  int rc = current_tau(ctx, &pv.tau);
  if (rc) return rc;
  et.tau_alt = nullptr;
  const size_t bytes = (size_t)ctx->m * (size_t)per_ant * sizeof(uint32_t);
  uint32_t *d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return ACO_ERR_ALLOCATION;
  cudaError_t e = cudaMemcpyAsync(d, draws, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_weights(ctx->iv, pv, et, nullptr, ctx->stream);
  if (e == cudaSuccess)
    e = launch_construct(ctx->iv, ctx->et, ctx->ab, ctx->plan, nullptr, ctx->seed, 0, 0, 0,
                         ctx->stream, d, (uint32_t)per_ant);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  TRY(e);
  return ACO_OK;
}

int aco_b200_get_ants(aco_b200_ctx *ctx, int *nodes, int *lens, double *cost,
                      int *feasible, int *steps, uint32_t *draws) {
  if (!ctx || !ctx->ready) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t m = ctx->m;
  if (nodes)
    TRY(cudaMemcpyAsync(nodes, ctx->ab.routes, sizeof(int) * m * (ctx->n + 2 * ctx->K),
                        cudaMemcpyDeviceToHost, s));
  if (lens) TRY(cudaMemcpyAsync(lens, ctx->ab.lens, sizeof(int) * m * ctx->K, cudaMemcpyDeviceToHost, s));
  if (cost) TRY(cudaMemcpyAsync(cost, ctx->ab.cost, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
  if (feasible) TRY(cudaMemcpyAsync(feasible, ctx->ab.feasible, sizeof(int) * m, cudaMemcpyDeviceToHost, s));
  if (steps) TRY(cudaMemcpyAsync(steps, ctx->ab.steps, sizeof(int) * m, cudaMemcpyDeviceToHost, s));
  if (draws) TRY(cudaMemcpyAsync(draws, ctx->ab.draws, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost, s));
  TRY(cudaStreamSynchronize(s));
  return ACO_OK;
}

int aco_b200_evaporate_deposit(aco_b200_ctx *ctx, int best_ant, float dep_iter,
                               const int *gbest_nodes, const int *gbest_lens,
                               float dep_global) {
  if (!ctx || !ctx->ready || best_ant < 0 || best_ant >= ctx->m)
    return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int *dn = nullptr, *dl = nullptr;
  if (gbest_nodes && gbest_lens) {
    int total = 0;
    for (int v = 0; v < ctx->K; ++v) {
      if (gbest_lens[v] < 2) return ACO_ERR_INVALID_INPUT;
      total += gbest_lens[v];
    }
    if (total > ctx->n + 2 * ctx->K) return ACO_ERR_INVALID_INPUT;
    for (int t = 0; t < total; ++t)
      if (gbest_nodes[t] < 0 || gbest_nodes[t] > ctx->n) return ACO_ERR_INVALID_INPUT;
    TRY(cudaMemcpyAsync(ctx->d_tmp_nodes, gbest_nodes, sizeof(int) * total, cudaMemcpyHostToDevice, s));
    TRY(cudaMemcpyAsync(ctx->d_tmp_lens, gbest_lens, sizeof(int) * ctx->K, cudaMemcpyHostToDevice, s));
    dn = ctx->d_tmp_nodes;
    dl = ctx->d_tmp_lens;
  }
  PheromoneView pv = ctx->pv;
  int rc = current_tau(ctx, &pv.tau);
  if (rc) return rc;
  TRY(launch_evap_deposit_explicit(ctx->iv, pv, ctx->ab, best_ant, dep_iter, dn, dl,
                                   dep_global, ctx->d_counter, ctx->evap_grid, s));
  TRY(cudaStreamSynchronize(s));
  return ACO_OK;
}

const char *aco_b200_build_info(void) {
  return "aco_b200 sm_100a: warp-per-ant construct (TMA-staged tables), "
         "integer roulette, Philox4x32-10 draws, 128-bit evaporation";
}

// ---------------------------------------------------------------------------
// Reference-facing solver (src/cuda/aco_cuda.cu:188-454).
// ---------------------------------------------------------------------------

static double wall_seconds(void) {
  struct timespec ts;
  timespec_get(&ts, TIME_UTC);
  return (double)ts.tv_sec + (double)ts.tv_nsec * 1e-9;
}

// print_cuda_progress, src/cuda/aco_cuda.cu:39-74 (same text).
static void print_progress(int epoch, double elapsed_s, double max_runtime_s,
                           int since, int max_stag, double best) {
  char t_rem[32], e_rem[32], best_txt[64];
  if (max_runtime_s > 0.0) snprintf(t_rem, sizeof(t_rem), "%.1fs", fmax(0.0, max_runtime_s - elapsed_s));
  else snprintf(t_rem, sizeof(t_rem), "senza limite");
  if (max_stag > 0) {
    int left = max_stag - since;
    snprintf(e_rem, sizeof(e_rem), "%d", left > 0 ? left : 0);
    if (left <= 0) snprintf(t_rem, sizeof(t_rem), "0.0s");
  } else {
    snprintf(e_rem, sizeof(e_rem), "senza limite");
  }
  if (best < DBL_MAX) snprintf(best_txt, sizeof(best_txt), "%.3f", best);
  else snprintf(best_txt, sizeof(best_txt), "non disponibile");
  printf("[progress][cuda] epoca=%d | epoche_rimanenti_prima_stop=%s | "
         "tempo_trascorso=%.1fs | tempo_rimanente=%s | best_cost=%s\n",
         epoch, e_rem, elapsed_s, t_rem, best_txt);
  fflush(stdout);
}

// ACO_CUDA_PRIOR=learned with ACO_CUDA_PRIOR_FILE (ACO_B200_PRIOR_PARAMS raw
// float32 values) and ACO_CUDA_PRIOR_GAMMA (default 2): learned eta levels.
// Any failure keeps the plain levels, with a note on stderr.
static void apply_prior_from_env(aco_b200_ctx *ctx) {
  const char *mode = getenv("ACO_CUDA_PRIOR");
  if (!mode || !*mode || strcmp(mode, "plain") == 0) return;
  if (strcmp(mode, "learned") != 0) {
    fprintf(stderr, "[cuda] ACO_CUDA_PRIOR=%s not recognised (plain|learned): plain eta\n", mode);
    return;
  }
  const char *file = getenv("ACO_CUDA_PRIOR_FILE");
  float gamma = 2.0f;
  const char *g = getenv("ACO_CUDA_PRIOR_GAMMA");
  if (g && *g) {
    char *end = nullptr;
    const double v = strtod(g, &end);
    if (end && *end == '\0' && v > 0.0 && v < 1e6) gamma = (float)v;
    else fprintf(stderr, "[cuda] ACO_CUDA_PRIOR_GAMMA=%s ignored\n", g);
  }
  aco_b200_prior *prior = nullptr;
  int rc = file && *file ? aco_b200_prior_create(&prior, ctx->device) : ACO_ERR_INVALID_INPUT;
  if (rc == ACO_OK) rc = aco_b200_prior_load(prior, file);
  if (rc == ACO_OK) rc = aco_b200_apply_prior(ctx, prior, gamma);
  if (rc != ACO_OK) {
    fprintf(stderr, "[cuda] learned prior unavailable (%s, file %s): plain eta\n",
            aco_status_string((AcoStatus)rc), file ? file : "not set");
    aco_b200_apply_prior(ctx, nullptr, 0.f);
  }
  if (prior) aco_b200_prior_destroy(prior);
}

static AcoStatus solve_impl(int n, int K, long long capacity, int m,
                            const float *x, const float *y, const int *demand,
                            double alpha, double beta, double rho, double tau0,
                            double Q, unsigned int seed, Solution *best,
                            double *best_cost) {
  if (n <= 0 || K <= 0 || !x || !y || !best || !best_cost) return ACO_ERR_INVALID_INPUT;
  AcoRuntimeConfig cfg;
  aco_runtime_config_load_env(&cfg);
  if (m == 0) m = 256;
  aco_b200_problem prob;
  memset(&prob, 0, sizeof(prob));
  prob.n = n;
  prob.K = K;
  prob.capacity = capacity;
  prob.ants = m;
  prob.cand_k = cfg.candidate_k;
  prob.x = x;
  prob.y = y;
  prob.demand = demand;
  prob.alpha = alpha;
  prob.beta = beta;
  prob.rho = rho;
  prob.tau0 = tau0;
  prob.Q = Q;
  prob.seed = seed;
  prob.stagnation_epochs = cfg.stagnation_epochs;
  prob.fixed_epochs = cfg.fixed_epochs;
  prob.min_rel_improvement = cfg.min_rel_improvement;
  prob.timeout_seconds = cfg.timeout_seconds;
  // ACO_CUDA_DEPOT_RULE: seq (default) or cuda_ref.
  const char *rule = getenv("ACO_CUDA_DEPOT_RULE");
  if (rule && strcmp(rule, "cuda_ref") == 0) prob.depot_rule = kDepotRuleCudaRef;
  else if (rule && *rule && strcmp(rule, "seq") != 0)
    fprintf(stderr, "[cuda] ACO_CUDA_DEPOT_RULE=%s not recognised (seq|cuda_ref): seq\n", rule);

  aco_b200_ctx *ctx = nullptr;
  int rc = aco_b200_create(&ctx, 0);
  if (rc) return (AcoStatus)rc;
  rc = aco_b200_setup(ctx, &prob);
  if (rc) {
    aco_b200_destroy(ctx);
    return (AcoStatus)rc;
  }
  apply_prior_from_env(ctx);
  printf("CUDA Solver starting... (N=%d, K=%d, M=%d)\n", n, K, m);
  const double start = wall_seconds();
  double next_report = cfg.progress_interval_seconds > 0.0 ? start + cfg.progress_interval_seconds : 0.0;
  std::vector<aco_b200_epoch_record> recs(kChunkEpochs);
  aco_b200_state st;
  memset(&st, 0, sizeof(st));
  while (true) {
    int nrec = 0;
    rc = aco_b200_run(ctx, kChunkEpochs, &st, recs.data(), (int)recs.size(), &nrec);
    if (rc) break;
    for (int i = 0; i < nrec; ++i) {
      const aco_b200_epoch_record &r = recs[i];
      const double elapsed = (double)r.elapsed_ns * 1e-9;
      const bool t_lim = cfg.timeout_seconds > 0.0 && elapsed >= cfg.timeout_seconds;
      const bool e_lim = cfg.stagnation_epochs > 0 && r.iter_since_best >= cfg.stagnation_epochs;
      if (r.epoch == 1 || r.epoch % 10 == 0 || r.improved || t_lim || e_lim)
        print_progress(r.epoch, elapsed, cfg.timeout_seconds, r.iter_since_best,
                       cfg.stagnation_epochs, r.global_best);
    }
    const double now = wall_seconds();
    if (cfg.progress_interval_seconds > 0.0 && now >= next_report) {
      const double el = now - start;
      if (cfg.timeout_seconds > 0.0)
        fprintf(stderr, "[cuda] elapsed %.1fs, remaining %.1fs, iter %d, best %.3f\n", el,
                fmax(0.0, cfg.timeout_seconds - el), st.epochs, st.global_best);
      else
        fprintf(stderr, "[cuda] elapsed %.1fs, iter %d, best %.3f\n", el, st.epochs, st.global_best);
      next_report = now + cfg.progress_interval_seconds;
    }
    if (st.stopped) break;
  }
  if (rc) {
    aco_b200_destroy(ctx);
    return (AcoStatus)rc;
  }
  std::vector<int> nodes((size_t)n + 2 * K), lens((size_t)K);
  double cost = DBL_MAX;
  rc = aco_b200_get_best(ctx, nodes.data(), lens.data(), &cost);
  aco_b200_destroy(ctx);
  *best_cost = cost;
  if (rc == ACO_ERR_NO_SOLUTION) return ACO_ERR_NO_SOLUTION;
  if (rc) return (AcoStatus)rc;
  solution_reset(best);
  int off = 0;
  for (int v = 0; v < K; ++v) {
    Route *r = &best->routes[v];
    if (lens[v] > r->cap) return ACO_ERR_BACKEND;
    for (int t = 0; t < lens[v]; ++t) r->nodes[t] = nodes[off + t];
    r->len = lens[v];
    off += lens[v];
  }
  return ACO_OK;
}

AcoStatus aco_vrp_cuda_with_capacity(int n, int K, int vehicle_capacity_customers,
                                     int m, float *coords_x, float *coords_y,
                                     double alpha, double beta, double rho,
                                     double tau0, double Q, unsigned int seed,
                                     Solution *best_solution, double *best_cost) {
  return solve_impl(n, K, vehicle_capacity_customers, m, coords_x, coords_y, nullptr,
                    alpha, beta, rho, tau0, Q, seed, best_solution, best_cost);
}

AcoStatus aco_vrp_cuda_with_demands(int n, int K, int capacity, int m,
                                    const float *coords_x, const float *coords_y,
                                    const int *demand, double alpha, double beta,
                                    double rho, double tau0, double Q,
                                    unsigned int seed, Solution *best_solution,
                                    double *best_cost) {
  return solve_impl(n, K, capacity, m, coords_x, coords_y, demand, alpha, beta, rho,
                    tau0, Q, seed, best_solution, best_cost);
}

}  // extern "C"
