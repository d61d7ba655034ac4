#ifndef ACO_B200_H
#define ACO_B200_H

#include "aco_api.h"

/*
 * aco_b200.h -- the thin C ABI of the B200 ACO-for-CVRP hot path.
 *
 * Plain C types only.  Host buffers are owned by the caller; device buffers
 * are owned by the context.  One context drives one instance on one GPU
 * through one CUDA stream; a context is used by one host thread at a time.
 * Every function returns an int status: 0 (ACO_OK) or an AcoStatus code
 * (include/aco.h).
 *
 * What each entry point replaces in the reference:
 *   aco_b200_setup        the set-up half of aco_vrp_cuda_with_capacity
 *                         (src/cuda/aco_cuda.cu:198-292: parameters, device
 *                         buffers, launch_init_tau, launch_build_candidate_lists)
 *   aco_b200_run          the epoch loop (aco_cuda.cu:331-429), run on the
 *                         device in CUDA-graph chunks with device-side stop
 *                         rules instead of 7 host synchronisations per epoch
 *   aco_b200_get_best     copy_ant_to_solution + the final D2H
 *                         (aco_cuda.cu:138-168, :367-380)
 *   aco_b200_construct    one launch of kernel_construct_solutions
 *                         (include/aco_cuda_kernels.h:104-115) on the current
 *                         pheromone, for parity checks
 *   aco_b200_evaporate_deposit  kernel_evaporate_tau + kernel_deposit_solution
 *                         + kernel_deposit_flat_solution (aco_cuda.cu:385-396)
 *   aco_b200_get_tau / set_tau / get_candidates / get_weights / get_ants /
 *   get_state             read-outs of the device state for the tests (the
 *                         reference has none; its tests are end-to-end only)
 */

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aco_b200_ctx aco_b200_ctx;

/* Problem and run parameters (the reference's solver arguments plus the
 * ACO_SOLVER_* configuration, src/common/aco_config.c:33-73). */
typedef struct {
  int n;                      /* customers; nodes are 0 (depot) .. n      */
  int K;                      /* vehicles                                  */
  long long capacity;         /* per vehicle, in demand units              */
  int ants;                   /* m; 0 selects 256 (aco_cuda.cu:206)        */
  int cand_k;                 /* 0 selects 32, or n when n <= 32 (:198-199) */
  const float *x;             /* [n+1] host                                */
  const float *y;             /* [n+1] host                                */
  const int *demand;          /* [n+1] host, NULL = unit demand            */
  double alpha, beta, rho, tau0, Q;
  unsigned int seed;
  int stagnation_epochs;      /* 0 = no stagnation stop                    */
  int fixed_epochs;           /* 0 = no epoch limit                        */
  double min_rel_improvement; /* fraction (the env variable is percent)    */
  double timeout_seconds;     /* 0 = none                                  */
  int ant_base;               /* global id of ant 0 (colony split over
                                 devices); 0 for a whole colony            */
  int depot_rule;             /* 0 = sequential path's rule (default);
                                 1 = reference CUDA kernel's stochastic
                                 depot close, aco_cuda_kernels.cu:487-520 */
} aco_b200_problem;

/* Device-side solver state after a run. */
typedef struct {
  int epochs;                 /* epochs completed                          */
  int iter_since_best;        /* epochs since the last significant gain    */
  int stopped;                /* nonzero: a stop rule fired                */
  int stop_reason;            /* bit 1 stagnation, 2 fixed, 4 timeout      */
  int found;                  /* last epoch had a feasible ant             */
  int improved;               /* last epoch improved the global best       */
  int best_ant;               /* last epoch's iteration-best ant           */
  int error;                  /* device error flag (0 = none)              */
  double global_best;         /* DBL_MAX while no feasible solution        */
  double iter_best;           /* last epoch's iteration-best cost          */
  float dep_iter, dep_global; /* last epoch's deposit amounts              */
  unsigned long long total_steps; /* ant-steps (moves) since set-up        */
} aco_b200_state;

/* One record per epoch, for the progress lines (aco_cuda.cu:39-74). */
typedef struct {
  int epoch;                  /* 1-based, as printed by the reference      */
  int iter_since_best;
  int improved;
  int found;
  double global_best;
  unsigned long long elapsed_ns;
} aco_b200_epoch_record;

ACO_API int aco_b200_create(aco_b200_ctx **out, int device);
ACO_API int aco_b200_destroy(aco_b200_ctx *ctx);
/* Use an external stream (e.g. a framework's current stream); NULL = own. */
ACO_API int aco_b200_set_stream(aco_b200_ctx *ctx, void *cuda_stream);

/* Uploads the instance, builds candidate lists and eta levels on the device,
 * initialises the pheromone matrix and the run state. */
ACO_API int aco_b200_setup(aco_b200_ctx *ctx, const aco_b200_problem *problem);

/* Runs up to max_epochs more epochs (stops earlier on a stop rule); fills
 * *state.  Epoch records since the last call are returned through
 * records/n_records when records is not NULL (capacity max_records). */
ACO_API int aco_b200_run(aco_b200_ctx *ctx, int max_epochs, aco_b200_state *state,
                 aco_b200_epoch_record *records, int max_records,
                 int *n_records);

/* Enqueues max_epochs epochs on the context stream without synchronising
 * (for timing with events on that stream). */
ACO_API int aco_b200_enqueue_epochs(aco_b200_ctx *ctx, int epochs);
ACO_API int aco_b200_synchronize(aco_b200_ctx *ctx);

/* Runs `epochs` epochs, their kernels one after another with a CUDA event
 * between consecutive kernels on the context stream (the epoch graph runs
 * the evaporation beside the construction), and adds each kernel's device
 * time (ms) into kernel_ms[4]: weights, construct, evaporate, best+deposit. */
ACO_API int aco_b200_profile_epochs(aco_b200_ctx *ctx, int epochs, float *kernel_ms);

/* Times the pheromone evaporation sweep alone: `launches` launches of the
 * kernel and grid the epoch graph uses (current buffer into the other one,
 * which the next epoch overwrites; the current buffer and the solve's
 * progress are left unchanged, and the run limit is cleared as by
 * aco_b200_enqueue_epochs): one untimed launch, then `launches` launches
 * back to back between two CUDA events on the context stream.
 * *ms_per_launch is the events' interval over `launches`.  The sweep
 * moves 2 (n+1)^2 bytes (read + write); the reference's counterpart is
 * kernel_evaporate_tau (src/cuda/aco_cuda_kernels.cu:145-155). */
ACO_API int aco_b200_profile_update(aco_b200_ctx *ctx, int launches, float *ms_per_launch);

/* Best solution so far in compact form: K segments [0 c.. 0] back to back
 * (nodes capacity n + 2K), the K segment lengths and the FP64 cost. */
ACO_API int aco_b200_get_best(aco_b200_ctx *ctx, int *nodes, int *lens, double *cost);

ACO_API int aco_b200_get_state(aco_b200_ctx *ctx, aco_b200_state *state);
ACO_API int aco_b200_get_dims(aco_b200_ctx *ctx, int *n, int *K, int *k, int *m);
/* Launch shape of the construction chosen at set-up: out[0] ants (warps)
 * per block, out[1] table layout (0 weights staged in shared memory, 1
 * packed levels staged, 2 rows read from global memory), out[2] visited
 * bitmap words per lane held in registers (0: bitmap in shared memory),
 * out[3] dynamic shared memory per block in bytes. */
ACO_API int aco_b200_get_plan(aco_b200_ctx *ctx, int out[4]);

/* Test hooks (parity checks against the oracle). */
ACO_API int aco_b200_get_tau(aco_b200_ctx *ctx, uint8_t *tau);       /* (n+1)^2 */
ACO_API int aco_b200_set_tau(aco_b200_ctx *ctx, const uint8_t *tau); /* (n+1)^2 */
ACO_API int aco_b200_get_candidates(aco_b200_ctx *ctx, int *cand, uint16_t *levels);
/* Neighbours of ranks k+1 .. k+64 of every node, in the candidates' order
 * ([(n+1) 64], 0 = empty slot): where the construction's nearest-customer
 * fallback looks before it scans every node. */
ACO_API int aco_b200_get_tier(aco_b200_ctx *ctx, uint16_t *tier);
/* Ranks k+65 .. k+256 of every node ([(n+1) 192], 0 = empty slot), where the
 * fallback looks after the ranks above, for instances of n >= 1500;
 * ACO_ERR_INVALID_INPUT for smaller ones. */
ACO_API int aco_b200_get_tier2(aco_b200_ctx *ctx, uint16_t *tier2);
ACO_API int aco_b200_get_tables(aco_b200_ctx *ctx, int32_t *A, uint32_t *lut,
                        float *thresholds, int n_thresholds);
/* Weights recomputed from the current pheromone ((n+1) k values). */
ACO_API int aco_b200_get_weights(aco_b200_ctx *ctx, uint32_t *w);
/* Fault-injection test hooks (host-made failures; no GPU fault):
 *   what 1: the value-th device allocation of the following set-up fails as
 *           out of memory (0 = off) -- set-up must return ACO_ERR_ALLOCATION
 *           and free what it allocated;
 *   what 2: value 1 makes the construct kernel's bounded wait for its staged
 *           tables run out (the wait expects 16 bytes more than it copies):
 *           the kernel flags the error and returns, and aco_b200_run returns
 *           ACO_ERR_BACKEND; value 0 restores it (a set-up clears the flag). */
ACO_API int aco_b200_debug_inject(aco_b200_ctx *ctx, int what, int value);
/* Depot rule 1 only: eta level of d(i,0)^2 per node, the last weights
 * pass's depot-close levels rdep[n+1] and the depot factor's level e_dep. */
ACO_API int aco_b200_get_depot_tables(aco_b200_ctx *ctx, uint16_t *lvl0, int32_t *rdep,
                                      int *e_dep);
/* One construct pass for epoch number `epoch` on the current pheromone;
 * per-ant results through aco_b200_get_ants.  layout: -1 = automatic,
 * 0 = shared-memory weights, 1 = shared-memory packed levels, 2 = global. */
ACO_API int aco_b200_construct(aco_b200_ctx *ctx, int epoch, int layout);
/* One construct pass that takes its random draws from a recorded stream
 * (draws[ant * per_ant + d], the low 24 bits used; draws past per_ant read as
 * 0) instead of Philox -- for parity against the reference's own
 * construction fed the same stream.  Results through aco_b200_get_ants. */
ACO_API int aco_b200_construct_with_draws(aco_b200_ctx *ctx, const uint32_t *draws,
                                          int per_ant);
ACO_API int aco_b200_get_ants(aco_b200_ctx *ctx, int *nodes /* m (n+2K) */,
                      int *lens /* m K */, double *cost, int *feasible,
                      int *steps, uint32_t *draws);
/* Evaporation then deposit of the given iteration-best ant and of the
 * given global-best solution (compact form), with the given amounts. */
ACO_API int aco_b200_evaporate_deposit(aco_b200_ctx *ctx, int best_ant,
                               float dep_iter, const int *gbest_nodes,
                               const int *gbest_lens, float dep_global);

/*
 * One colony split over several devices (one context per device, same
 * instance and parameters, ants m each, ant_base = rank * m).  The pheromone
 * matrix is replicated; per epoch each device
 *   1. aco_b200_shard_construct: weights, construction of its m ants (random
 *      draws keyed by the global ant id) and a packet with its best ant
 *      (aco_b200_shard_packet_ints int32 words) written to d_send;
 *   2. the caller all-gathers the packets of all devices (rank order) into
 *      d_recv (e.g. ncclAllGather on the context stream);
 *   3. aco_b200_shard_update: the winner over the packets (lowest cost, then
 *      lowest global ant), the epoch bookkeeping and stop rules, evaporation
 *      and the deposits, identical on every device.
 * N devices with m ants each then run exactly the epochs of one device with
 * N m ants.  Calls only enqueue work on the context stream.  The device
 * timeout rule reads each device's own clock, so split colonies leave
 * timeout_seconds at 0 and stop on the host.  Packet layout: [0,1] cost
 * (FP64 bits), [2] found, [3] global ant, [4,5] ant-steps (64-bit), then K
 * lengths and the compact route.
 */
ACO_API int aco_b200_shard_packet_ints(aco_b200_ctx *ctx);
ACO_API int aco_b200_shard_construct(aco_b200_ctx *ctx, int32_t *d_send);
ACO_API int aco_b200_shard_update(aco_b200_ctx *ctx, const int32_t *d_recv, int world);
/* A number that changes whenever a set-up changes the arguments the
 * context's launches are recorded with (sizes, parameters, buffers; -1 if
 * not set up).  The shard calls above only enqueue launches, so a caller may
 * record steps 1-3 of whole epochs in a CUDA graph of its own (stream
 * capture on the context stream, its all-gather included); it re-records
 * when this number changes.  Graph replays read the epoch number from the
 * device state. */
ACO_API int aco_b200_graph_generation(aco_b200_ctx *ctx);

/*
 * Learned heuristic prior.  A small MLP (8 candidate-edge features -> 64 ->
 * 64 -> 1, ReLU; BF16 operands, FP32 accumulation on the tensor cores)
 * scores every candidate edge; aco_b200_apply_prior turns the scores s of
 * row i into eta levels L = min(4095, round(gamma (max s - s) 16 / ln 2)),
 * i.e. selection weights proportional to tau^alpha exp(gamma s), in place
 * of the plain eta^beta = d^-beta levels.  gamma <= 0 (or prior NULL)
 * restores the plain levels.  Training: softmax cross-entropy of each row's
 * candidate slots against the successor an elite route takes (depot -> first
 * customer, and both directions of every customer arc), Adam.
 * Parameters: ACO_B200_PRIOR_PARAMS floats, W1[64][8], b1[64], W2[64][64],
 * b2[64], w3[64], b3.  No counterpart in the reference.
 */
#define ACO_B200_PRIOR_PARAMS 4801
typedef struct aco_b200_prior aco_b200_prior;

/* Training set: instances packed like the batched problem (instance i
 * occupies n[i]+1 entries of x, y, demand), plus one elite solution per
 * instance in compact form (K[i] lengths, routes back to back). */
typedef struct {
  int count;
  const int *n;
  const int *K;
  const long long *capacity;
  const float *x, *y;
  const int *demand;          /* NULL = unit demand */
  const int *nodes;
  const int *lens;
  int cand_k;                 /* candidate list length, <= 32; 0 = 32 */
} aco_b200_prior_dataset;

ACO_API int aco_b200_prior_create(aco_b200_prior **out, int device);
ACO_API int aco_b200_prior_destroy(aco_b200_prior *prior);
ACO_API int aco_b200_prior_set_stream(aco_b200_prior *prior, void *cuda_stream);
ACO_API int aco_b200_prior_init(aco_b200_prior *prior, unsigned int seed);
ACO_API int aco_b200_prior_set_params(aco_b200_prior *prior, const float *params, int count);
ACO_API int aco_b200_prior_get_params(aco_b200_prior *prior, float *params, int count);
ACO_API int aco_b200_prior_load(aco_b200_prior *prior, const char *path);  /* raw float32 */
ACO_API int aco_b200_prior_save(aco_b200_prior *prior, const char *path);
ACO_API int aco_b200_prior_set_dataset(aco_b200_prior *prior,
                                       const aco_b200_prior_dataset *data,
                                       long long *n_examples);
/* epochs over the training set in shuffled minibatches of `batch`
 * examples; epoch_loss[epochs] (mean cross-entropy) may be NULL. */
ACO_API int aco_b200_prior_train(aco_b200_prior *prior, int epochs, int batch, float lr,
                                 unsigned int seed, float *epoch_loss);
/* Test hooks: gradient (ACO_B200_PRIOR_PARAMS floats) and mean loss of the
 * given examples; the examples as (feature row, target slot) pairs; feature
 * rows (32 slots x 8 BF16 bit patterns each), their non-empty slot counts
 * and (scores != NULL) the forward pass on them. */
ACO_API int aco_b200_prior_gradient(aco_b200_prior *prior, const int *examples, int count,
                                    float *grad, float *loss);
ACO_API long long aco_b200_prior_num_examples(aco_b200_prior *prior);
ACO_API int aco_b200_prior_get_examples(aco_b200_prior *prior, int *rows_slots, long long count);
ACO_API int aco_b200_prior_get_rows(aco_b200_prior *prior, long long first, int count,
                                    uint16_t *features, uint8_t *kv, float *scores);
ACO_API int aco_b200_apply_prior(aco_b200_ctx *ctx, aco_b200_prior *prior, float gamma);
/* mode 0: as aco_b200_apply_prior (learned levels replace the plain ones);
 * mode 1: residual, learned levels added to the plain eta^beta levels
 * (weights proportional to tau^alpha eta^beta exp(gamma s)). */
ACO_API int aco_b200_apply_prior_mode(aco_b200_ctx *ctx, aco_b200_prior *prior, float gamma,
                                      int mode);

/*
 * Batched solving: many independent instances in one persistent launch.
 * Each block takes instances from a queue and runs all their epochs itself
 * (weights, construction, best, evaporation, deposit), so instances of
 * uneven size share the GPU without any host round trip.  Instance i is
 * solved exactly as aco_b200_setup/aco_b200_run solve it with seed + i, the
 * same ants, candidate length, parameters and epoch rules.  Coordinates and
 * demands are packed: instance i occupies n[i] + 1 consecutive entries.
 * No counterpart in the reference (it solves one instance per process).
 */
typedef struct aco_b200_batch aco_b200_batch;

typedef struct {
  int count;                  /* instances                                 */
  const int *n;               /* [count] customers (k <= n <= 2046)        */
  const int *K;               /* [count] vehicles                          */
  const long long *capacity;  /* [count] in demand units                   */
  const float *x, *y;         /* packed [sum(n[i] + 1)] host               */
  const int *demand;          /* packed, NULL = unit demand                */
  int ants;                   /* per instance; 0 selects 64                */
  int cand_k;                 /* 0 selects 32                              */
  double alpha, beta, rho, tau0, Q;
  unsigned int seed;          /* instance i uses seed + i                  */
  int epochs;                 /* epochs per instance                       */
  int stagnation_epochs;      /* 0 = none                                  */
  double min_rel_improvement;
} aco_b200_batch_problem;

/* Launch shape: lanes per ant (16: two ants per warp, needs cand_k <= 16;
 * 32: one), ants per block, queue order (0: as given, 1: largest first). */
typedef struct {
  int lanes_per_ant;
  int ants_per_block;
  int order;
} aco_b200_batch_tuning;

ACO_API int aco_b200_batch_create(aco_b200_batch **out, int device);
ACO_API int aco_b200_batch_destroy(aco_b200_batch *batch);
/* Use an external stream; NULL = own. */
ACO_API int aco_b200_batch_set_stream(aco_b200_batch *batch, void *cuda_stream);
ACO_API int aco_b200_batch_setup(aco_b200_batch *batch, const aco_b200_batch_problem *problem);
ACO_API int aco_b200_batch_set_tuning(aco_b200_batch *batch, const aco_b200_batch_tuning *tuning);
ACO_API int aco_b200_batch_get_tuning(aco_b200_batch *batch, aco_b200_batch_tuning *tuning);
/* Times every candidate launch shape on `trial_epochs` epochs of the whole
 * batch and keeps the fastest; per-trial ms through trial_ms. */
ACO_API int aco_b200_batch_autotune(aco_b200_batch *batch, int trial_epochs,
                                    aco_b200_batch_tuning *chosen, float *trial_ms,
                                    int max_trials, int *n_trials);
/* Rebuilds every instance's candidate lists and plain eta levels with
 * length k (1 <= k <= 32, k <= every n; the lists are the first k of the
 * nearest-neighbour order, as aco_b200_setup builds them).  A launch shape
 * that cannot hold k (16 lanes per ant with k > 16) becomes the default
 * {32, 16, 1}.  Learned levels applied before are replaced. */
ACO_API int aco_b200_batch_set_cand_k(aco_b200_batch *batch, int k);
ACO_API int aco_b200_batch_get_cand_k(aco_b200_batch *batch, int *k);
/* Chooses the candidate-list length, then the launch shape.  Stage 1 solves
 * the whole batch once per length ks[0..nks) (nks <= 16) on the default
 * shape and records its device time (k_solve_ms), the mean final cost over
 * the instances every length solved (k_mean_cost) and the instances solved
 * (k_feasible).  The length kept is the fastest among those that solve the
 * most instances and whose mean cost is within quality_tol (a fraction) of
 * the best such mean: a shorter list cannot win on speed at the price of
 * quality.  Stage 2 is aco_b200_batch_autotune at that length.  Any output
 * pointer may be NULL. */
ACO_API int aco_b200_batch_autotune_k(aco_b200_batch *batch, int trial_epochs, const int *ks,
                                      int nks, double quality_tol,
                                      aco_b200_batch_tuning *chosen, int *chosen_k,
                                      double *k_solve_ms, double *k_mean_cost, int *k_feasible,
                                      float *trial_ms, int max_trials, int *n_trials);
/* One launch solving every instance (run as a CUDA graph that is kept while
 * the launch's arguments stay the same); _enqueue does not synchronise. */
ACO_API int aco_b200_batch_solve(aco_b200_batch *batch);
ACO_API int aco_b200_batch_enqueue(aco_b200_batch *batch);
ACO_API int aco_b200_batch_synchronize(aco_b200_batch *batch);
/* Results are read after the batch's stream (the solve included): every
 * getter below copies on that stream and waits for it.
 * Best solution of one instance (compact form, as aco_b200_get_best). */
ACO_API int aco_b200_batch_get(aco_b200_batch *batch, int instance, int *nodes, int *lens,
                               double *cost, int *epochs);
ACO_API int aco_b200_batch_get_costs(aco_b200_batch *batch, double *costs, int *epochs,
                                     unsigned long long *steps);
/* Best solutions of every instance in three copies.  nodes: sum of
 * n_i + 2 K_i ints, instance i's compact sequence at offset
 * sum_{j<i} (n_j + 2 K_j) (its first sum(lens) entries are used);
 * lens: sum of K_i ints, instance i's at sum_{j<i} K_j; costs: count doubles
 * (DBL_MAX where no ant was feasible).  Any pointer may be NULL. */
ACO_API int aco_b200_batch_get_all(aco_b200_batch *batch, int *nodes, int *lens, double *costs);
/* Learned eta levels for every instance of the batch (after setup). */
ACO_API int aco_b200_batch_apply_prior(aco_b200_batch *batch, aco_b200_prior *prior, float gamma);

/*
 * Evaporation then deposit without any device allocation, for callers that
 * cannot allocate device memory while they run: applications that reserve
 * all device memory up front and give plugins only buffers they own (a
 * framework's caching allocator, a service with a fixed memory budget), or
 * real-time loops where cudaMalloc/cudaFree are off limits because they can
 * synchronise the device and can fail under memory pressure.  No counterpart
 * in the reference (its pheromone update allocates through its solver).
 *
 * Every argument is caller-owned device memory or a scalar: d_tau is the
 * (n+1)^2 log-quantized matrix (row stride n+1, 16-byte aligned), updated
 * in place; the
 * iteration-best and (optional, both NULL to skip) global-best solutions are
 * in compact form (K segments [0 c.. 0] back to back, K lengths); rho gives
 * the evaporation step as in the reference (src/cuda/aco_cuda.cu:214-215).
 * Same result as aco_b200_evaporate_deposit.
 *
 * The kernel's scratch is a fixed array in the library's device memory
 * (16.6 KB per GPU), so K may be at most 4096 routes; larger K is rejected
 * with ACO_ERR_INVALID_INPUT and a message on stderr.  Every call on a GPU
 * shares that array: calls whose kernels overlap on the GPU race, so issue
 * them on one stream or otherwise order them.  The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before capturing a stream into a CUDA graph.  The address
 * is kept for the life of the process: it does not survive a device reset
 * (cudaDeviceReset, or the primary context destroyed and made again), after
 * which this entry point must not be called in the same process.
 */
ACO_API int aco_b200_evaporate_deposit_noalloc(uint8_t *d_tau, int n, int K,
                                               const int *d_iter_nodes,
                                               const int *d_iter_lens,
                                               float dep_iter,
                                               const int *d_gbest_nodes,
                                               const int *d_gbest_lens,
                                               float dep_global, double rho,
                                               void *cuda_stream);

/*
 * The sequential path's FP64 pheromone update (src/seq/aco_sequential.c:
 * 829-886, run there when an iteration best exists), bit-exact on a device
 * matrix: tau[i][j] *= (1 - rho) for i != j; tau[u][v] += iter_deposit and
 * tau[v][u] += iter_deposit over every arc of the iteration best, then the
 * same with best_deposit over the global best (d_best_* NULL to skip, as
 * the reference skips it while it has no best); every off-diagonal cell
 * clamped to [tau_min, tau_max] (MMAS); then, when `reset` is nonzero (the
 * reference's stagnation trigger), tau[i][j] = 0.5 tau[i][j] + 0.5 tau0 for
 * i != j.  iter_deposit and best_deposit are the reference's
 * (weight * Q) / cost values.
 *
 * d_tau: (n+1)^2 doubles, row-major, row stride n+1, 16-byte aligned (as
 * cudaMalloc returns it; rejected otherwise).  Solutions in compact
 * form (K segments [0 c.. 0] back to back, K lengths), K <= 8192, device
 * memory.  d_scratch: aco_b200_seq_update_scratch_bytes(n) bytes of device
 * memory, zeroed by the caller before the first call; every call leaves it
 * zeroed again.  The update runs on `cuda_stream` (NULL: the default
 * stream) in three launches: one sweep of the matrix (evaporation, and
 * clamp/reset of every cell no deposit touches) and two small kernels over
 * the solutions' arcs.
 */
ACO_API size_t aco_b200_seq_update_scratch_bytes(int n);
ACO_API int aco_b200_seq_pheromone_update(double *d_tau, int n, int K,
                                          const int *d_iter_nodes, const int *d_iter_lens,
                                          double iter_deposit, const int *d_best_nodes,
                                          const int *d_best_lens, double best_deposit,
                                          double rho, double tau_min, double tau_max,
                                          int reset, double tau0, void *d_scratch,
                                          void *cuda_stream);

/* Library build information. */
ACO_API const char *aco_b200_build_info(void);

#ifdef __cplusplus
}
#endif

#endif
