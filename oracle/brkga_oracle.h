/*
 * brkga_oracle.h -- CPU restatement of the reference BRKGA hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  The
 * product library (llm-brkga_b200/lib/libbrkga_b200.so) never links or calls it.
 *
 * Every function states the reference code it restates (paths relative to the
 * hsaseendran/llm-brkga tree).  Where the reference leaves something unspecified
 * (non-stable std::sort tie order, clock-seeded RNG) this file fixes one definition
 * and the CUDA engine implements the same one, so the two can be compared bit for bit.
 *
 * Parity pin: oracle/ref_harness.cu compiles the reference's own headers and the
 * tests compare this file against it (decode, tour length, knapsack fitness,
 * bi-objective TSP, Pareto ranks, crowding, crossover and mutant fill with replayed
 * draws, whole generations).  Golden vectors from that harness live in tests/golden/.
 */
#ifndef BRKGA_ORACLE_H
#define BRKGA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random stream ------------------------------------------------------------ */
/* Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel Random
 * Numbers: As Easy as 1, 2, 3" (SC'11).  Replaces the reference's clock-seeded
 * mt19937 (core/solver.hpp:167) and cuRAND XORWOW (core/cuda_kernels.cuh:10-15). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Stream tags: counter word 3 = (island << 8) | tag. */
enum {
    ORC_TAG_INIT = 1,     /* initial keys, core/population.hpp:107-110            */
    ORC_TAG_MUTANT = 2,   /* mutant rows, core/solver.hpp:1244-1258                */
    ORC_TAG_COIN = 3,     /* crossover coins, core/solver.hpp:1125-1131            */
    ORC_TAG_PARENT = 4,   /* elite / non-elite parent picks, core/solver.hpp:1117-1118 */
    ORC_TAG_NSGA_TOUR = 5,  /* tournament picks, core/solver.hpp:1042-1056         */
    ORC_TAG_NSGA_COIN = 6,  /* uniform crossover coins, core/solver.hpp:1058-1074   */
    ORC_TAG_NSGA_MUTP = 7,  /* per-gene mutation test, core/solver.hpp:1077-1091    */
    ORC_TAG_NSGA_MUTK = 8,  /* replacement key for a mutated gene                   */
    ORC_TAG_NSGA_REFILL = 9, /* random refill of ensure_minimum_diversity           */
    ORC_TAG_LS = 10          /* TSPJ local search segments, core/cuda_kernels.cuh:188-195 */
};

/* draw word `lane` (0..3) of Philox block (word, row, gen, (island<<8)|tag) keyed by seed */
uint32_t orc_draw(uint64_t seed, uint32_t word, uint32_t row, uint32_t gen, uint32_t stream, int lane);
/* top 24 bits as a float in [0,1): the range of the reference's host keys
 * (std::uniform_real_distribution<float>(0,1), core/individual.hpp:79-87) */
float orc_u24(uint32_t x);
/* threshold T with (x>>8) < T  <=>  u24(x) < p  (p in [0,1]) */
uint32_t orc_prob_threshold(double p);
/* unbiased-enough range map: floor(x * k / 2^32) */
uint32_t orc_pick(uint32_t x, uint32_t k);

/* ---- keys and decode ------------------------------------------------------------ */
/* order-preserving map of a float key to uint32 (-0 folded onto +0, NaN last) */
uint32_t orc_okey(float f);
/* stable argsort of one key row: std::sort over pair<key,index>,
 * configs/tsp_config.hpp:206-225 (ties go to the lower index). */
void orc_decode(const float* keys, int n, int32_t* perm);
void orc_decode_rows(const float* keys, int rows, int n, int ld, int32_t* perm);

/* ---- problems ------------------------------------------------------------------- */
enum {
    ORC_TSP_COORDS = 1,       /* Euclidean from [n][2] coordinates                      */
    ORC_TSP_MATRIX = 2,       /* [n][n] matrix, configs/tsp_config.hpp:180-193          */
    ORC_KNAP_THRESHOLD = 3,   /* key > 0.5, configs/knapsack_config.hpp:43-62           */
    ORC_KNAP_GREEDY = 4,      /* key-order first-fit greedy (no reference counterpart)  */
    ORC_BITSP_COORDS = 5,     /* depot tour, two coordinate sets [n+1][2]               */
    ORC_BITSP_MATRIX = 6,     /* depot tour, two [n+1][n+1] matrices, configs/multi_tsp_config.hpp:54-103 */
    ORC_TSPJ = 7,             /* n = 2c genes; mat = travel [c+1][c+1], mat2 = job durations [c+1][c+1],
                                 configs/tspj_config.hpp:555-626                                       */
    ORC_JOBSCHED = 8,         /* jt [n], machines: makespan, configs/job_scheduling_gpu_config.hpp:132-148 */
    ORC_CONTINUOUS = 9,       /* function 0 sphere / 1 Rastrigin / 2 Rosenbrock over [lo, hi],
                                 configs/continuous_opt_gpu_config.hpp:114-173                        */
    ORC_MOVRP = 10            /* n customers; xy [n+1][2] (node 0 = depot), w = demands [n+1],
                                 vcap = vehicle capacity, machines = vehicles; objectives (total
                                 distance + penalties, longest route + penalty),
                                 configs/multi_objective_vrp_config.hpp:214-313                       */
};

typedef struct {
    int32_t kind;
    int32_t n;             /* chromosome length (genes)                           */
    const float* xy;       /* TSP: [n][2]; bi-TSP: [n+1][2] (node 0 = depot)       */
    const float* xy2;      /* bi-TSP second coordinate set                         */
    const float* mat;      /* TSP: [n][n]; bi-TSP: [n+1][n+1]                      */
    const float* mat2;
    const int32_t* w;      /* knapsack weights [n]                                 */
    const int32_t* v;      /* knapsack values  [n]                                 */
    float cap;             /* knapsack capacity                                    */
    const float* jt;       /* job scheduling: job times [n]                        */
    int32_t machines;
    int32_t function;      /* continuous: function and bounds                      */
    float lo, hi;
    int32_t vcap;          /* MO-VRP vehicle capacity                              */
} orc_problem;

int orc_num_objectives(const orc_problem* pb);
int orc_maximize(const orc_problem* pb);

/* Euclidean edge in the reference's float arithmetic: sqrtf(dx*dx + dy*dy) with no
 * contraction, exactly as the matrix of configs/tsp_config.hpp:361-370 is built. */
float orc_edge(const float* xy, int a, int b);

/* FP32 closed-tour length in the engine's canonical summation order:
 * 256 virtual lanes sum edges e = l, l+256, ... in order; each group of 32 lanes is
 * reduced by an xor butterfly (16,8,4,2,1); the 8 group totals are added as
 * ((g0+g1)+(g2+g3))+((g4+g5)+(g6+g7)). */
float orc_canon_sum(const float* d, int nedges);
/* evaluate one decoded row; out has num_objectives entries (canonical FP32) */
void orc_eval_perm(const orc_problem* pb, const int32_t* perm, const float* keys, float* out);
/* Random 2-opt local search (TSPJConfig::apply_local_search_gpu, configs/tspj_config.hpp:72-136,
 * with random_2opt_kernel / restore_if_worse_kernel, core/cuda_kernels.cuh:166-246) on
 * rows[0, count), the best ranks: `moves` reversals of a city-key segment [i, j] (i, j
 * drawn over the c = n/2 cities at (move, q, gen, island<<8 | ORC_TAG_LS), ordered,
 * skipped when j - i < 2); the row and fit[row] change only if the makespan improved. */
void orc_local_search(const orc_problem* pb, float* pop, float* fit, const int32_t* rows, int count, int ld,
                      int moves, uint64_t seed, uint32_t gen, int island);
/* continuous objective in double precision (the tolerance reference for Rastrigin) */
double orc_continuous_f64(const orc_problem* pb, const float* keys);
/* the problem's decode of one chromosome (two argsorts for TSPJ, see orc_evaluate; for
 * MO-VRP the argsort of the biased values of orc_movrp_values) */
void orc_decode_problem(const orc_problem* pb, const float* keys, int32_t* perm);
/* MultiObjectiveVRPConfig::decode_routes sort values (configs/multi_objective_vrp_config.hpp:
 * 219-230): h = sequential float sum of key[i] * (i + 1); value[i] = key[i] + (i * 1e-5f +
 * h * 1e-5f), all in float without contraction */
void orc_movrp_values(const float* keys, int n, float* val);
/* MO-VRP routes of a decoded row: route index per sorted position (route_of[j] for
 * customer perm[j] + 1); returns the route count */
int orc_movrp_routes(const orc_problem* pb, const int32_t* perm, int32_t* route_of);
/* FP64 restatement of the same objective (tour lengths only), for error bounds */
void orc_eval_perm_f64(const orc_problem* pb, const int32_t* perm, double* out);
/* sequential FP32 tour sum in the reference's order (configs/tsp_config.hpp:186-190) */
float orc_tsp_len_seq(const orc_problem* pb, const int32_t* perm);
/* evaluate rows [r0, r1) of a key matrix; fit is [rows][num_objectives] */
void orc_evaluate(const orc_problem* pb, const float* keys, int rows, int ld, float* fit);

/* ---- BRKGA generation ----------------------------------------------------------- */
typedef struct {
    int32_t P, E, M;       /* population, elite, mutant counts (core/config.hpp:22-24) */
    double rho;            /* elite_prob, core/config.hpp:25                            */
    uint64_t seed;
    int32_t island;
} orc_params;

/* elite partition: order rows by (fitness, row) ascending, or by fitness descending
 * with ties by row ascending when maximize (core/population.hpp:660-682, with the
 * index tie-break of thrust::sort_by_key, core/solver.hpp:333-338). NaN sorts last. */
void orc_sort_fitness(const float* fit, int P, int maximize, int32_t* sorted);

/* Generation core with injected draws (core/solver.hpp:234-273, 1109-1135, 1244-1258):
 *   rows [0,E)      <- pop[sorted[r]]            (elite copy, fitness kept)
 *   rows [E,P-M)    <- child of elite sorted[ep[i]] and non-elite sorted[E+np[i]];
 *                      gene j from the elite parent iff coin[i*n+j] != 0
 *   rows [P-M,P)    <- mutant keys mut[(i)*n + j]
 * newfit is written for elite rows only. */
void orc_generation_core(int P, int E, int M, int n, int ld,
                         const float* pop, const float* fit, const int32_t* sorted,
                         const int32_t* ep, const int32_t* np, const uint8_t* coin,
                         const float* mut, float* newpop, float* newfit);

/* Philox-driven generation g >= 1: draws from the stream, then the core, then
 * evaluation of rows [E,P). newpop/newfit are [P][ld] / [P]. */
void orc_brkga_generation(const orc_problem* pb, const orc_params* pr, uint32_t g,
                          const float* pop, const float* fit, const int32_t* sorted, int ld,
                          float* newpop, float* newfit);
/* initial population (generation 0) + evaluation */
void orc_brkga_init(const orc_problem* pb, const orc_params* pr, int ld, float* pop, float* fit);
/* ring migration among k islands of equal size Pi stored back to back:
 * island i's best m rows (by its sorted order) replace island (i+1)%k's worst m rows
 * (sorted positions Pi-m .. Pi-1), keys and fitness; then every island is re-sorted. */
void orc_migrate(int k, int Pi, int m, int n, int ld, int maximize,
                 float* pop, float* fit, int32_t* sorted);
/* run: init + G generations; writes best-of-generation history [G+1] and the final
 * population / fitness / sorted order. */
void orc_brkga_run(const orc_problem* pb, const orc_params* pr, int G, int ld,
                   float* pop, float* fit, int32_t* sorted, float* history);

/* ---- NSGA-II -------------------------------------------------------------------- */
/* Pareto ranks of N points with m objectives (minimisation) exactly as the reference
 * computes them: domination counts, then front peeling in which every member of the first
 * front decrements the points it dominates TWICE (it is pushed into fronts[0] by
 * fast_non_dominated_sort, core/population.hpp:431-434, and again by
 * build_fronts_from_domination, :335-340); a point takes rank k+1 when its count first
 * drops to <= 0 while front k is processed.  Dominance: core/individual.hpp:99-114. */
void orc_pareto_ranks(const float* obj, int N, int m, int32_t* rank);
/* textbook non-dominated sorting ranks (first front weighted once) */
void orc_pareto_ranks_strict(const float* obj, int N, int m, int32_t* rank);
/* crowding distance per front (core/population.hpp:453-489) over the reference's front
 * lists, in which every rank-0 point is listed twice (the same double push as in the
 * ranks); lists are sorted by (objective, index, copy) and a point listed twice takes
 * both entries' contributions.  FP32 in the reference's accumulation order; FP64 for
 * error bounds.  The _strict variant lists every point once. */
void orc_crowding_f32(const float* obj, const int32_t* rank, int N, int m, float* cd);
void orc_crowding_f64(const float* obj, const int32_t* rank, int N, int m, double* cd);
void orc_crowding_strict_f32(const float* obj, const int32_t* rank, int N, int m, float* cd);
/* survivors (core/population.hpp:491-517) over the same lists: whole fronts while they
 * fit (rank-0 points twice), ordered by (last objective, index); the first front that
 * does not fit sorted by crowding descending, ties by index, and truncated.  Writes P pool
 * indices (a rank-0 index may appear twice); returns the count written. */
int orc_nsga2_select(const int32_t* rank, const float* cd, const float* obj, int N, int m, int P,
                     int32_t* sel);

typedef struct {
    int32_t P;             /* population size (pool is 2P)                         */
    int32_t Mn;            /* fresh random offspring per generation (0 = reference) */
    double rho;            /* uniform-crossover bias toward parent 1               */
    double mut_rate;       /* per-gene reset rate; reference 5/len                  */
    uint64_t seed;
    int32_t diversity_interval; /* ensure_minimum_diversity period (25), 0 = off   */
} orc_nsga2_params;

/* offspring core with injected draws (core/solver.hpp:1019-1091): child i takes
 * tournament(picks[4i],picks[4i+1]) as parent 1 and tournament(picks[4i+2],picks[4i+3])
 * as parent 2; gene j from parent 1 iff coin, then replaced by mkey iff mflag. */
void orc_nsga2_offspring_core(int P, int n, int ld, const float* pop, const int32_t* rank,
                              const float* cd, const int32_t* picks, const uint8_t* coin,
                              const uint8_t* mflag, const float* mkey, float* off);
/* offspring of generation g from the stream: P children into off[P][ld]; the last Mn
 * children are fresh random keys (an option; the reference has none) */
void orc_nsga2_offspring(const orc_nsga2_params* pr, uint32_t g, int n, int ld,
                         const float* pop, const int32_t* rank, const float* cd,
                         float* off);
/* one NSGA-II generation (core/solver.hpp:751-817): pop/obj/rank/cd are [P]
 * in, replaced by the survivors.  Scratch is allocated internally. */
void orc_nsga2_generation(const orc_problem* pb, const orc_nsga2_params* pr, uint32_t g, int ld,
                          float* pop, float* obj, int32_t* rank, float* cd);
void orc_nsga2_init(const orc_problem* pb, const orc_nsga2_params* pr, int ld,
                    float* pop, float* obj, int32_t* rank, float* cd);
/* ensure_minimum_diversity (core/population.hpp:130-182) with refill keys drawn from
 * the stream; returns 1 when the population was rebuilt. */
int orc_nsga2_diversity(const orc_problem* pb, const orc_nsga2_params* pr, uint32_t g, int ld,
                        float* pop, float* obj, int32_t* rank, float* cd);

#ifdef __cplusplus
}
#endif
#endif
