/*
 * brkga_b200.h -- C ABI of the B200 BRKGA generation engine (libbrkga_b200.so).
 *
 * Plain pointers and sizes only.  Every call returns a brkga_status (0 = OK, negative =
 * error) and records a message readable with brkga_last_error() on the calling thread.
 * Device pointers are CUDA global-memory pointers on the engine's device; `stream` may
 * be 0 (legacy default stream) or any cudaStream_t of that device, passed as void*.
 *
 * Each entry point names the reference interface it replaces (paths relative to the
 * hsaseendran/llm-brkga tree).
 */
#ifndef BRKGA_B200_H
#define BRKGA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BRKGA_B200_ABI_VERSION 1

typedef enum {
    BRKGA_OK = 0,
    BRKGA_ERR_INVALID = -1,      /* bad argument (reference: BRKGAConfig::is_valid, core/config.hpp:159-179) */
    BRKGA_ERR_OOM = -2,          /* device allocation failed                                              */
    BRKGA_ERR_CUDA = -3,         /* a CUDA call failed                                                    */
    BRKGA_ERR_TIMEOUT = -4,      /* a bounded device wait ran out                                         */
    BRKGA_ERR_CANCELLED = -5,    /* request cancelled                                                     */
    BRKGA_ERR_UNSUPPORTED = -6,  /* size or mode outside what this build handles                          */
    BRKGA_ERR_BUSY = -7,         /* admission refused (not enough free device memory / slots)             */
    BRKGA_ERR_NOT_READY = -8     /* result not available yet                                              */
} brkga_status;

/* problem kinds: the reference's problem configs (brkga/configs/) */
typedef enum {
    BRKGA_TSP_COORDS = 1,        /* TSPConfig, Euclidean from coordinates (configs/tsp_config.hpp:301-380)   */
    BRKGA_TSP_MATRIX = 2,        /* TSPConfig(dist, name) with an explicit [n][n] matrix (tsp_config.hpp:38)  */
    BRKGA_KNAP_THRESHOLD = 3,    /* KnapsackConfig: gene > 0.5 selects, penalty x1000 (knapsack_config.hpp:43) */
    BRKGA_KNAP_GREEDY = 4,       /* key-order first-fit greedy knapsack (no reference counterpart)          */
    BRKGA_BITSP_COORDS = 5,      /* MultiTSPConfig with two coordinate sets, depot = point 0                */
    BRKGA_BITSP_MATRIX = 6,      /* MultiTSPConfig(dist, time, name) (configs/multi_tsp_config.hpp:25-52)   */
    BRKGA_TSPJ = 7,              /* TSPJConfig(travel, jobs, name): tour + job assignment, makespan
                                    (configs/tspj_config.hpp:40-66, 555-626)                                */
    BRKGA_JOBSCHED = 8,          /* JobSchedulingGPUConfig(job_times, machines): gene i puts job i on
                                    machine floor(key * machines); makespan = largest machine load
                                    (configs/job_scheduling_gpu_config.hpp:30-52, 132-148)                  */
    BRKGA_CONTINUOUS = 9,        /* ContinuousOptGPUConfig(n, lower, upper, function): x = key *
                                    (upper - lower) + lower; sphere / Rastrigin / Rosenbrock
                                    (configs/continuous_opt_gpu_config.hpp:37-57, 114-173)                  */
    BRKGA_MOVRP = 10,            /* MultiObjectiveVRPConfig: capacitated routes from one biased argsort;
                                    objectives total distance and longest route, with the reference's
                                    overload and fleet penalties (configs/multi_objective_vrp_config.hpp:
                                    214-313); two objectives, so runs take the NSGA-II path            */
    BRKGA_EXTERNAL = 11          /* a config that brings its own fitness (BRKGAConfig::fitness_function /
                                    objective_functions, or its own evaluate_population_gpu kernel;
                                    core/config.hpp:33-53): n keys per row; one objective (BRKGA,
                                    direction from `maximize`) or two (NSGA-II, minimised).  The engine
                                    builds rows and ranks them; the caller evaluates them between
                                    brkga_external_begin and brkga_external_commit.  Engines only (one
                                    island); the evaluation entry points, batches and the server
                                    reject it                                                           */
} brkga_problem_kind;

/* functions of BRKGA_CONTINUOUS (the reference's OptimizationFunction) */
typedef enum { BRKGA_FN_SPHERE = 0, BRKGA_FN_RASTRIGIN = 1, BRKGA_FN_ROSENBROCK = 2 } brkga_function;

/* Instance data (HOST pointers; copied to the device at creation).
 *   TSP:      n cities; coords [n][2] or matrix [n][n]
 *   bi-TSP:   n genes, n+1 points with point 0 the depot; coords/coords2 [n+1][2] or
 *             matrix/matrix2 [n+1][n+1]
 *   knapsack: n items; weights, values [n] (integers); capacity
 *   TSPJ:     n cities besides the depot (node 0) and n job types; matrix = travel times
 *             [n+1][n+1], matrix2 = job durations [n+1][n+1] (row = city, column = job
 *             type); chromosomes hold 2n keys, the n city keys then the n job keys
 *   job scheduling: n jobs; job_times [n]; machines >= 1
 *   continuous: n variables; function (brkga_function); lower < upper
 *   MO-VRP:   n customers; coords [n+1][2] with point 0 the depot; demands [n+1] (>= 0,
 *             the depot's unused); vehicle_capacity >= 1; vehicles >= 1 (the fleet size the
 *             reference reads from the instance name "-k<V>")                           */
typedef struct {
    int32_t kind;
    int32_t n;
    const float* coords;
    const float* coords2;
    const float* matrix;
    const float* matrix2;
    const int32_t* weights;
    const int32_t* values;
    float capacity;
    const float* job_times;      /* job scheduling                                            */
    int32_t machines;
    int32_t function;            /* continuous                                                */
    float lower;
    float upper;
    const int32_t* demands;      /* MO-VRP                                                    */
    int32_t vehicle_capacity;
    int32_t vehicles;
    int32_t maximize;            /* BRKGA_EXTERNAL: 1 = larger fitness is better (the
                                    reference's comparator, core/config.hpp:36); other kinds
                                    fix their own direction and ignore it                     */
    int32_t num_objectives;      /* BRKGA_EXTERNAL: 1 (0 reads as 1) or 2                     */
} brkga_problem_desc;

/* GA parameters (BRKGAConfig fields, core/config.hpp:17-30, plus the engine's own). */
typedef struct {
    int32_t population_size;     /* P                                                         */
    int32_t elite_size;          /* E (absolute, like the reference)                          */
    int32_t mutant_size;         /* M; for NSGA-II: fresh random offspring per generation     */
    double elite_prob;           /* rho                                                       */
    int32_t max_generations;     /* generation budget used by brkga_run                       */
    uint64_t seed;               /* Philox key: the whole run is a function of the seed       */
    int32_t num_islands;         /* >= 1; islands split P evenly (core/solver.hpp:378-476)    */
    int32_t migration_interval;  /* generations between ring migrations (0 = never)          */
    int32_t num_migrants;        /* rows sent to the next island per migration                */
    int32_t device;              /* CUDA device ordinal                                       */
    int32_t diversity_interval;  /* NSGA-II ensure_minimum_diversity period (0 = off)         */
    double mutation_rate;        /* NSGA-II per-gene reset rate (<= 0: the reference's 5/n)   */
    int32_t local_search_interval;     /* TSPJ random 2-opt local search after generation g when
                                          g - 1 > 0 and (g - 1) % interval == 0; 0 = off
                                          (core/solver.hpp:459-461, 562-615)                   */
    int32_t local_search_individuals;  /* top ranks searched per island (at most its elite size) */
    int32_t local_search_moves;        /* random segment reversals per individual              */
} brkga_params;

typedef struct brkga_problem brkga_problem;
typedef struct brkga_engine brkga_engine;

/* ---- library ------------------------------------------------------------------------- */
int32_t brkga_abi_version(void);
/* copy the calling thread's last error message (NUL-terminated, truncated to cap) */
int32_t brkga_last_error(char* buf, size_t cap);
/* fill p with the reference's defaults (core/config.hpp:78-84: P=100, E=20, M=10,
 * rho=0.7, 1000 generations) and the engine's (seed 1, 1 island, device 0) */
void brkga_params_default(brkga_params* p);

/* ---- problem instances (TSPConfig / KnapsackConfig / MultiTSPConfig device data) ------- */
/* Uploads the instance to `device`.  Replaces the per-device data map and its lazy upload
 * in TSPConfig::ensure_gpu_memory (configs/tsp_config.hpp:125-165) and
 * KnapsackGPUConfig::allocate_gpu_memory (configs/knapsack_gpu_config.hpp:104-140). */
int32_t brkga_problem_create(const brkga_problem_desc* desc, int32_t device, brkga_problem** out);
int32_t brkga_problem_destroy(brkga_problem* pb);
int32_t brkga_problem_num_objectives(const brkga_problem* pb);
int32_t brkga_problem_maximize(const brkga_problem* pb);

/* Drop-in for BRKGAConfig::evaluate_population_gpu(T* d_population, T* d_fitness,
 * int pop_size, int chrom_len) (core/config.hpp:50-53; TSP: configs/tsp_config.hpp:70-111,
 * knapsack: configs/knapsack_gpu_config.hpp:66-88).  d_population is [pop_size][ld] float
 * keys on the device (the reference's dense layout is ld == chrom_len); d_fitness is
 * [pop_size][num_objectives].  d_perm (optional, may be NULL) receives the decoded
 * permutation [pop_size][chrom_len] (configs/tsp_config.hpp:206-225).  Asynchronous on
 * `stream`; the reference's call is synchronous -- brkga_evaluate_population_sync waits. */
int32_t brkga_evaluate_population(brkga_problem* pb, const float* d_population, float* d_fitness,
                                  int32_t pop_size, int32_t chrom_len, int32_t ld, int32_t* d_perm,
                                  void* stream);
int32_t brkga_evaluate_population_sync(brkga_problem* pb, const float* d_population, float* d_fitness,
                                       int32_t pop_size, int32_t chrom_len);

/* ---- operators on device buffers (the hot path, one call each) ------------------------- */
/* Elite partition: sorted[r] = row of rank r by (fitness, row) ascending, or fitness
 * descending with ties by row when maximize.  Replaces thrust::sequence +
 * thrust::sort_by_key (core/solver.hpp:329-338) and Population::sort
 * (core/population.hpp:660-682).  `segments` populations of `P` rows each, back to back. */
int32_t brkga_sort_fitness(const float* d_fitness, int32_t P, int32_t segments, int32_t maximize,
                           int32_t* d_sorted, void* stream);

/* Fused generation step for one population: elite copy, biased crossover, mutant fill,
 * decode and fitness of rows [E, P) written to d_next / d_next_fitness.  Replaces
 * brkga_generation_kernel (core/cuda_kernels.cuh:88-138) and the host path
 * evolve_generation_brkga (core/solver.hpp:234-273, 1109-1135, 1244-1258).  Draws come
 * from Philox keyed by (seed, generation, row, gene). */
int32_t brkga_generation_step(brkga_problem* pb, const float* d_pop, const float* d_fitness,
                              const int32_t* d_sorted, float* d_next, float* d_next_fitness,
                              int32_t P, int32_t E, int32_t M, double elite_prob, int32_t ld,
                              uint64_t seed, uint32_t generation, int32_t island, void* stream);

/* Initial population (Population::initialize, core/population.hpp:107-124): Philox keys
 * for generation 0 and their fitness. */
int32_t brkga_init_population(brkga_problem* pb, float* d_pop, float* d_fitness, int32_t P, int32_t ld,
                              uint64_t seed, int32_t island, void* stream);

/* Random 2-opt local search on rows [0, num_to_improve) of d_pop (the elites, in rank
 * order, as the reference's island loop leaves them): replaces
 * TSPJConfig::apply_local_search_gpu (configs/tspj_config.hpp:72-136), i.e.
 * random_2opt_kernel + evaluation + restore_if_worse_kernel (core/cuda_kernels.cuh:166-246).
 * Each row's city keys get num_moves reversals of a random segment [i, j] (skipped when
 * j - i < 2); the row and d_fitness[row] change only if the new makespan is lower.  Draws
 * come from Philox keyed by seed at (move, row, generation, island).  TSPJ problems only;
 * rows must fit the shared-memory row kernel.  ld = 0 means round_up(chrom_len, 4);
 * d_pop must be 16-byte aligned with ld a multiple of 4. */
int32_t brkga_local_search(brkga_problem* pb, float* d_pop, float* d_fitness, int32_t num_to_improve,
                           int32_t chrom_len, int32_t ld, int32_t num_moves, uint64_t seed, uint32_t generation,
                           int32_t island, void* stream);

/* Pareto ranks of N points with m objectives (minimisation), d_obj [N][m].  Replaces
 * Population::fast_non_dominated_sort (core/population.hpp:409-440). */
int32_t brkga_pareto_rank(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream);
/* The same ranks through the bit-packed dominance matrix for any m: bit j of row i set when
 * point i dominates point j, built 32 columns per __ballot_sync; fronts peeled by
 * bit-sliced column sums of the front's rows (for N <= 4096 on a cluster of eight CTAs,
 * the front exchanged through distributed shared memory).  Uses an internal device scratch
 * of about N*ceil(N/32)*4 bytes and returns after the ranks are written. */
int32_t brkga_pareto_rank_bitmatrix(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream);
/* Pareto ranks exactly like brkga_pareto_rank, but the call allocates no device memory:
 * for callers that cannot call cudaMalloc -- code running under a framework whose
 * allocator owns all device memory, or a serving loop that must not allocate once
 * started (cudaMalloc can synchronise the device).  No counterpart in the reference.
 * The dominance rows and counts live in a fixed device array inside the library (532 KiB
 * on every GPU that loads it, held until the process exits), so N is limited to 2048
 * points (larger N returns BRKGA_ERR_UNSUPPORTED); 1 <= m <= 4.  The first call on a
 * device looks up that array's address and raises a kernel's shared-memory limit; make
 * that first call before any stream capture.  The address is kept for the life of the
 * process, so do not use this entry point on a device after cudaDeviceReset.  Asynchronous
 * on `stream`.  Every call uses the same array: calls whose work overlaps on the GPU
 * (different streams, or another thread) race and must be ordered by the caller. */
int32_t brkga_pareto_rank_noalloc(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream);
/* Crowding distance per front (core/population.hpp:453-489), fronts from d_rank; two
 * objectives, N <= 4096.  Asynchronous on `stream`; its scratch comes from the library's
 * stream-ordered pool. */
int32_t brkga_crowding(const float* d_obj, const int32_t* d_rank, int32_t N, int32_t m, float* d_cd,
                       void* stream);

/* ---- solver (Solver<T>, core/solver.hpp:44-1726) ---------------------------------------- */
/* Creates the device-resident population for problem `pb` (the engine keeps its own
 * reference to the instance; pb may be destroyed afterwards).  Single-objective problems
 * run BRKGA; bi-objective ones run NSGA-II (core/solver.hpp:213-231). */
int32_t brkga_create(brkga_problem* pb, const brkga_params* params, brkga_engine** out);
int32_t brkga_destroy(brkga_engine* e);
/* Solver::initialize (core/solver.hpp:190-211) */
int32_t brkga_initialize(brkga_engine* e);
/* `generations` calls of Solver::evolve_generation (core/solver.hpp:213-231), enqueued on
 * the engine's stream (captured once as a CUDA graph); returns after enqueueing. */
int32_t brkga_evolve(brkga_engine* e, int32_t generations);
/* wait for the engine's queued work */
int32_t brkga_synchronize(brkga_engine* e);
/* Solver::run (core/solver.hpp:1517-1556): initialize + max_generations + wait */
int32_t brkga_run(brkga_engine* e);
int32_t brkga_generation(const brkga_engine* e);
/* the engine's CUDA stream (cudaStream_t as void*), for callers that order their own
 * work or timing events after the engine's queued generations */
int32_t brkga_get_stream(brkga_engine* e, void** stream);
/* launch shape the engine chose (autotuned per size): info[0] threads per row CTA,
 * info[1] float4 groups per thread, info[2] grid size, info[3] coordinates staged in
 * shared memory (1/0); cap >= 4 */
int32_t brkga_engine_info(brkga_engine* e, int32_t* info, int32_t cap);
/* Solver::get_best_individual (core/solver.hpp:1625): keys [n], decoded permutation [n]
 * (may be NULL), objective values [num_objectives]; host buffers, waits for the engine. */
int32_t brkga_get_best(brkga_engine* e, float* keys, int32_t* perm, float* fitness);
/* Solver::get_fitness_history (core/solver.hpp:1633): best fitness per generation,
 * history[0] = initial population; *len receives the number written (<= cap). */
int32_t brkga_get_fitness_history(brkga_engine* e, float* history, int32_t cap, int32_t* len);
/* whole population in rank order (host buffers): keys [P][n], fitness [P][m] (either may
 * be NULL).  Islands are returned one after another. */
int32_t brkga_get_population(brkga_engine* e, float* keys, float* fitness);
/* replace the population (host buffers, keys [P][n]) and re-evaluate it; the next
 * generation number stays where it is. */
int32_t brkga_set_population(brkga_engine* e, const float* keys);
/* Solver::get_pareto_front (core/solver.hpp:1629): rank-0 members; objectives [cap][m],
 * keys [cap][n] (may be NULL); *count receives the front size (may exceed cap). */
int32_t brkga_get_pareto_front(brkga_engine* e, float* objectives, float* keys, int32_t cap, int32_t* count);

/* ---- external fitness (BRKGA_EXTERNAL engines) -------------------------------------------
 * One generation of Solver::evolve_generation (core/solver.hpp:234-273, 751-817) with the
 * fitness from the caller, as the reference evaluates a config's fitness_function /
 * objective_functions or its own evaluate_population_gpu (core/population.hpp:523-527,
 * 567-595, 626-652; core/config.hpp:50-53):
 *   brkga_external_begin   builds the rows that need a fitness on the device and waits
 *                          for them: the initial population on the first call (and on the
 *                          first call after brkga_initialize), then each generation's new
 *                          rows -- the non-elite rows of a BRKGA generation (elite rows
 *                          keep theirs, as the reference's evaluated flag does), the P
 *                          offspring of an NSGA-II generation.  *d_keys points at the first
 *                          of *count pending rows, *ld floats apart; *d_fitness at their
 *                          fitness, num_objectives floats per row; *first is the first
 *                          row's index in the engine's buffer.  With dense = 1 the keys are
 *                          a packed [count][n] copy (*ld = n), the layout
 *                          evaluate_population_gpu expects.
 *   brkga_external_get_rows  the pending rows into host keys [count][n].
 *   brkga_external_set_fitness  host fitness [count][num_objectives] for them.
 *   brkga_external_commit  waits for the device (so fitness that the caller's kernels
 *                          wrote on any stream is in place: a cudaDeviceSynchronize, which
 *                          also waits for every other engine's and thread's work on that
 *                          device, so engines driven from several host threads serialise
 *                          at each commit), then ranks the population on
 *                          the engine's stream, completing the generation (calls that read
 *                          the population wait for it).  NSGA-II: when the generation's
 *                          diversity pass (ensure_minimum_diversity, core/population.hpp:
 *                          130-182) replaced rows with fresh keys, it returns
 *                          BRKGA_ERR_NOT_READY instead: the next brkga_external_begin
 *                          returns those rows, and the commit after them completes the
 *                          generation.
 * On these engines brkga_initialize only restarts (the next begin builds a new initial
 * population); brkga_evolve, brkga_run and brkga_set_population return
 * BRKGA_ERR_UNSUPPORTED; brkga_get_best gives keys and fitness, not a permutation (the
 * engine does not decode an external problem). */
int32_t brkga_external_begin(brkga_engine* e, int32_t dense, float** d_keys, float** d_fitness, int32_t* ld,
                             int32_t* first, int32_t* count);
int32_t brkga_external_get_rows(brkga_engine* e, float* keys);
int32_t brkga_external_set_fitness(brkga_engine* e, const float* fitness);
int32_t brkga_external_commit(brkga_engine* e);

/* ---- batched solving (many independent instances advanced together) --------------------- */
typedef struct brkga_batch brkga_batch;
/* `count` problems with their own parameters; all on params[0].device. */
int32_t brkga_batch_create(brkga_problem* const* problems, const brkga_params* params, int32_t count,
                           brkga_batch** out);
int32_t brkga_batch_destroy(brkga_batch* b);
int32_t brkga_batch_evolve(brkga_batch* b, int32_t generations);
int32_t brkga_batch_synchronize(brkga_batch* b);
/* best objective of every instance (host [count][2], second entry unused for
 * single-objective); waits for the batch */
int32_t brkga_batch_get_best(brkga_batch* b, float* best);
int32_t brkga_batch_get_best_keys(brkga_batch* b, int32_t index, float* keys, float* fitness);

/* ---- serving: continuous batching of solve requests ------------------------------------- */
typedef struct brkga_server brkga_server;
typedef struct {
    int32_t device;
    int32_t max_active;          /* slots on the device                                       */
    int64_t memory_budget;       /* bytes of device memory the server may hold (0 = free HBM) */
    int32_t generations_per_tick;/* generations advanced per scheduling round                 */
} brkga_server_config;

int32_t brkga_server_create(const brkga_server_config* cfg, brkga_server** out);
int32_t brkga_server_destroy(brkga_server* s);
/* queue a request; the problem data is copied, so desc's buffers may be freed after the
 * call.  params->max_generations is the request's generation budget; stall_generations
 * (0 = off) retires it early after that many generations without improvement. */
int32_t brkga_server_submit(brkga_server* s, const brkga_problem_desc* desc, const brkga_params* params,
                            int32_t stall_generations, int64_t* request_id);
/* run one scheduling round: admit queued requests, advance active ones, retire finished */
int32_t brkga_server_step(brkga_server* s);
/* result of a finished request: best objectives [2], generations run, and its latency
 * (submit -> retire) in seconds; BRKGA_ERR_NOT_READY while pending. */
int32_t brkga_server_poll(brkga_server* s, int64_t request_id, float* best, int32_t* generations,
                          double* latency_s);
int32_t brkga_server_cancel(brkga_server* s, int64_t request_id);
/* queued, active, finished counts */
int32_t brkga_server_stats(brkga_server* s, int32_t* queued, int32_t* active, int32_t* finished);

#ifdef __cplusplus
}
#endif
#endif
