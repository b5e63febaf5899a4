// capi.cu -- the C ABI (include/brkga_b200.h): problem instances, operators on device
// buffers, and the device-resident solver engine.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/brkga_b200.h"
#include "engine.h"
#include "kernels.h"

namespace bk {

// ---------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------
static thread_local std::string g_err;

int32_t fail(int32_t code, const std::string& msg) {
    g_err = msg;
    return code;
}

int32_t cuda_fail(cudaError_t e, const char* what) {
    return fail(BRKGA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceGuard::DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    ok_ = cudaSetDevice(dev) == cudaSuccess;
}
DeviceGuard::~DeviceGuard() { cudaSetDevice(prev_); }

// ---------------------------------------------------------------------------------------
// problem data
// ---------------------------------------------------------------------------------------
ProblemData::~ProblemData() {
    DeviceGuard g(device);
    for (void* p : allocs) dev_free(p, nullptr);
}

static int32_t upload(ProblemData& pd, const void* host, size_t bytes, void** dev) {
    if (!host) return fail(BRKGA_ERR_INVALID, "missing instance array");
    int32_t st = dev_alloc(dev, bytes ? bytes : 4, nullptr);
    if (st != BRKGA_OK) return st;
    pd.allocs.push_back(*dev);
    cudaError_t e = cudaMemcpy(*dev, host, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy instance");
    pd.bytes += bytes;
    return BRKGA_OK;
}

int32_t make_problem(const brkga_problem_desc* d, int device, std::shared_ptr<ProblemData>* out) {
    if (!d) return fail(BRKGA_ERR_INVALID, "null problem description");
    const int n = d->n;
    if (n < 1) return fail(BRKGA_ERR_INVALID, "chromosome length must be >= 1");
    const long long genes = (d->kind == BRKGA_TSPJ) ? 2ll * n : (long long)n;
    if (genes > row_max_n_global())
        return fail(BRKGA_ERR_UNSUPPORTED, "chromosome length " + std::to_string(genes) + " exceeds " +
                                               std::to_string(row_max_n_global()));
    auto pd = std::make_shared<ProblemData>();
    pd->device = device;
    pd->kind = d->kind;
    pd->n = n;
    DeviceGuard g(device);
    if (!g.ok()) return fail(BRKGA_ERR_CUDA, "cannot select device " + std::to_string(device));
    int32_t st = BRKGA_OK;
    void* p = nullptr;
    switch (d->kind) {
    case BRKGA_TSP_COORDS:
        pd->m = 1;
        st = upload(*pd, d->coords, (size_t)n * 8, &p);
        pd->xy = (float*)p;
        break;
    case BRKGA_TSP_MATRIX:
        pd->m = 1;
        st = upload(*pd, d->matrix, (size_t)n * n * 4, &p);
        pd->mat = (float*)p;
        break;
    case BRKGA_BITSP_COORDS:
        pd->m = 2;
        st = upload(*pd, d->coords, (size_t)(n + 1) * 8, &p);
        pd->xy = (float*)p;
        if (st == BRKGA_OK) st = upload(*pd, d->coords2, (size_t)(n + 1) * 8, &p);
        pd->xy2 = (float*)p;
        break;
    case BRKGA_BITSP_MATRIX:
        pd->m = 2;
        st = upload(*pd, d->matrix, (size_t)(n + 1) * (n + 1) * 4, &p);
        pd->mat = (float*)p;
        if (st == BRKGA_OK) st = upload(*pd, d->matrix2, (size_t)(n + 1) * (n + 1) * 4, &p);
        pd->mat2 = (float*)p;
        break;
    case BRKGA_KNAP_THRESHOLD:
    case BRKGA_KNAP_GREEDY: {
        pd->m = 1;
        pd->maximize = 1;
        if (!d->weights || !d->values) return fail(BRKGA_ERR_INVALID, "knapsack needs weights and values");
        for (int i = 0; i < n; ++i)
            if (d->weights[i] < 0) return fail(BRKGA_ERR_INVALID, "knapsack weights must be >= 0");
        if (!std::isfinite(d->capacity) || d->capacity < 0.0f)
            return fail(BRKGA_ERR_INVALID, "knapsack capacity must be finite and >= 0");
        pd->cap = d->capacity;
        pd->capi = (long long)std::floor((double)d->capacity);
        st = upload(*pd, d->weights, (size_t)n * 4, &p);
        pd->w = (int32_t*)p;
        if (st == BRKGA_OK) st = upload(*pd, d->values, (size_t)n * 4, &p);
        pd->v = (int32_t*)p;
        if (st == BRKGA_OK) {
            std::vector<int2> wv(n);
            for (int i = 0; i < n; ++i) wv[i] = make_int2(d->weights[i], d->values[i]);
            st = upload(*pd, wv.data(), (size_t)n * sizeof(int2), &p);
            pd->wv = (int2*)p;
        }
        break;
    }
    case BRKGA_TSPJ: {
        // TSPJConfig (configs/tspj_config.hpp:40-66): travel times and job durations over the
        // depot and n cities; the chromosome is the n city keys followed by the n job keys
        pd->m = 1;
        if (!d->matrix || !d->matrix2) return fail(BRKGA_ERR_INVALID, "TSPJ needs travel and job matrices");
        const size_t D = (size_t)n + 1;
        st = upload(*pd, d->matrix, D * D * 4, &p);
        pd->mat = (float*)p;
        if (st == BRKGA_OK) st = upload(*pd, d->matrix2, D * D * 4, &p);
        pd->mat2 = (float*)p;
        pd->n = 2 * n;
        break;
    }
    case BRKGA_JOBSCHED:
        // JobSchedulingGPUConfig (configs/job_scheduling_gpu_config.hpp:30-52): minimise the makespan
        pd->m = 1;
        if (!d->job_times) return fail(BRKGA_ERR_INVALID, "job scheduling needs job_times");
        if (d->machines < 1) return fail(BRKGA_ERR_INVALID, "machines must be >= 1");
        pd->machines = d->machines;
        st = upload(*pd, d->job_times, (size_t)n * 4, &p);
        pd->jt = (float*)p;
        break;
    case BRKGA_CONTINUOUS:
        // ContinuousOptGPUConfig (configs/continuous_opt_gpu_config.hpp:37-57): minimise
        pd->m = 1;
        if (d->function < BRKGA_FN_SPHERE || d->function > BRKGA_FN_ROSENBROCK)
            return fail(BRKGA_ERR_INVALID, "unknown continuous function " + std::to_string(d->function));
        if (!std::isfinite(d->lower) || !std::isfinite(d->upper) || !(d->lower < d->upper))
            return fail(BRKGA_ERR_INVALID, "need finite bounds with lower < upper");
        pd->function = d->function;
        pd->lo = d->lower;
        pd->hi = d->upper;
        break;
    case BRKGA_EXTERNAL:
        // a config with its own fitness (core/config.hpp:33-53): no instance data on the device
        if (d->num_objectives < 0 || d->num_objectives > 2)
            return fail(BRKGA_ERR_UNSUPPORTED, "external problems have one or two objectives");
        pd->m = d->num_objectives == 2 ? 2 : 1;
        if (pd->m == 2 && d->maximize)
            return fail(BRKGA_ERR_INVALID, "two objectives are minimised (Individual::dominates)");
        pd->maximize = d->maximize ? 1 : 0;
        break;
    case BRKGA_MOVRP: {
        // MultiObjectiveVRPConfig (configs/multi_objective_vrp_config.hpp:78-165): the depot and n
        // customers; integer demands and capacity; two objectives
        pd->m = 2;
        if (!d->coords || !d->demands) return fail(BRKGA_ERR_INVALID, "MO-VRP needs coords and demands");
        if (d->vehicle_capacity < 1 || d->vehicle_capacity > (1 << 30) || d->vehicles < 1)
            return fail(BRKGA_ERR_INVALID, "MO-VRP needs 1 <= vehicle_capacity <= 2^30 and vehicles >= 1");
        for (int i = 0; i <= n; ++i)
            if (d->demands[i] < 0 || d->demands[i] > (1 << 30))
                return fail(BRKGA_ERR_INVALID, "MO-VRP demands must lie in [0, 2^30]");
        if (row_needs_global(n, n + 1, BRKGA_MOVRP))
            return fail(BRKGA_ERR_UNSUPPORTED, "MO-VRP with " + std::to_string(n) +
                                                   " customers: rows must fit the shared-memory row kernel");
        pd->capi = d->vehicle_capacity;
        pd->machines = d->vehicles;
        st = upload(*pd, d->coords, (size_t)(n + 1) * 8, &p);
        pd->xy = (float*)p;
        if (st == BRKGA_OK) st = upload(*pd, d->demands, (size_t)(n + 1) * 4, &p);
        pd->w = (int32_t*)p;
        break;
    }
    default:
        return fail(BRKGA_ERR_INVALID, "unknown problem kind " + std::to_string(d->kind));
    }
    if (st != BRKGA_OK) return st;
    *out = pd;
    return BRKGA_OK;
}

void fill_instance(PopDesc& d, const ProblemData& pd) {
    std::memset(&d, 0, sizeof(d));
    d.kind = pd.kind;
    d.n = pd.n;
    d.ld = round_up(pd.n, 4);
    d.m = pd.m;
    d.xy = pd.xy;
    d.xy2 = pd.xy2;
    d.mat = pd.mat;
    d.mat2 = pd.mat2;
    d.w = pd.w;
    d.wv = pd.wv;
    d.cap = pd.cap;
    d.capi = pd.capi;
    d.jt = pd.jt;
    d.machines = pd.machines;
    d.function = pd.function;
    d.lo = pd.lo;
    d.hi = pd.hi;
    d.maximize = pd.maximize;
}

int points_of(const ProblemData& pd) {
    return (pd.kind == BRKGA_BITSP_COORDS || pd.kind == BRKGA_MOVRP) ? pd.n + 1 : pd.n;
}

bool stage_fits(const RowTile& t, int n, int pts, int kind) {
    return row_smem_bytes(t, n, pts, kind, true) <= kMaxSmem;
}

// ---------------------------------------------------------------------------------------
// tile choice cache
// ---------------------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int>, RowTile> g_tune;  // (device, kind, n, rows)
static bool g_tune_loaded = false;

static int cur_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

static void tune_load_file() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("BRKGA_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    int kind, n, rows, b, g;
    while (std::fscanf(f, "%d %d %d %d %d", &kind, &n, &rows, &b, &g) == 5)
        g_tune[{cur_device(), kind, n, rows}] = RowTile{b, g};
    std::fclose(f);
}

int32_t tune_lookup(int kind, int n, int rows, RowTile* t) {
    if (const char* forced = std::getenv("BRKGA_TILE")) {
        int b = 0, g = 0;
        if (std::sscanf(forced, "%d,%d", &b, &g) == 2 && 4 * b * g >= n) {
            *t = RowTile{b, g};
            return BRKGA_OK;
        }
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_file();
    auto it = g_tune.find({cur_device(), kind, n, rows});
    if (it == g_tune.end()) return BRKGA_ERR_NOT_READY;
    *t = it->second;
    return BRKGA_OK;
}

void tune_store(int kind, int n, int rows, const RowTile& t) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{cur_device(), kind, n, rows}] = t;
    if (const char* path = std::getenv("BRKGA_TUNE_CACHE")) {
        if (FILE* f = std::fopen(path, "a")) {
            std::fprintf(f, "%d %d %d %d %d\n", kind, n, rows, t.block, t.groups);
            std::fclose(f);
        }
    }
}

int32_t tile_setup(const RowTile& t, int kind, int n, int pts, TunedTile* out) {
    TunedTile tt;
    tt.tile = t;
    tt.stage = stage_fits(t, n, pts, kind);
    const size_t smem = row_smem_bytes(t, n, pts, kind, tt.stage);
    if (smem > kMaxSmem) return fail(BRKGA_ERR_UNSUPPORTED, "tile needs too much shared memory");
    int per_sm = 0;
    cudaError_t e = prepare_rows(t, smem, &per_sm);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "tile set-up");
    }
    if (per_sm <= 0) return fail(BRKGA_ERR_UNSUPPORTED, "tile does not fit on an SM");
    tt.grid = per_sm * device_sm_count();
    *out = tt;
    return BRKGA_OK;
}

uint32_t prob_threshold(double p) {
    if (!(p > 0.0)) return 0u;
    if (p >= 1.0) return 1u << 24;
    double t = std::ceil(p * 16777216.0);
    if (t > 16777216.0) t = 16777216.0;
    return (uint32_t)t;
}

}  // namespace bk

using namespace bk;

struct brkga_problem {
    std::shared_ptr<ProblemData> d;
};

extern "C" {

int32_t brkga_abi_version(void) { return BRKGA_B200_ABI_VERSION; }

int32_t brkga_last_error(char* buf, size_t cap) {
    if (!buf || cap == 0) return BRKGA_ERR_INVALID;
    const size_t n = std::min(cap - 1, g_err.size());
    std::memcpy(buf, g_err.data(), n);
    buf[n] = '\0';
    return BRKGA_OK;
}

void brkga_params_default(brkga_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->population_size = 100;
    p->elite_size = 20;
    p->mutant_size = 10;
    p->elite_prob = 0.7;
    p->max_generations = 1000;
    p->seed = 1;
    p->num_islands = 1;
    p->migration_interval = 0;
    p->num_migrants = 0;
    p->device = 0;
    p->diversity_interval = 25;
    p->mutation_rate = 0.0;
    p->local_search_interval = 0;  // off; the reference's island loop uses 2, 100, 5 (core/solver.hpp:166)
    p->local_search_individuals = 100;
    p->local_search_moves = 5;
}

int32_t brkga_problem_create(const brkga_problem_desc* desc, int32_t device, brkga_problem** out) {
    if (!out) return fail(BRKGA_ERR_INVALID, "null output handle");
    *out = nullptr;
    std::shared_ptr<ProblemData> pd;
    int32_t st = make_problem(desc, device, &pd);
    if (st != BRKGA_OK) return st;
    *out = new brkga_problem{pd};
    return BRKGA_OK;
}

int32_t brkga_problem_destroy(brkga_problem* pb) {
    delete pb;
    return BRKGA_OK;
}

int32_t brkga_problem_num_objectives(const brkga_problem* pb) { return pb ? pb->d->m : BRKGA_ERR_INVALID; }
int32_t brkga_problem_maximize(const brkga_problem* pb) { return pb ? pb->d->maximize : BRKGA_ERR_INVALID; }

}  // extern "C"

namespace bk {
// One row launch for an operator entry point: the in-shared-memory kernel, or, for rows
// whose sort does not fit there, the global-scratch kernel with scratch taken from the
// stream-ordered pool and returned to it behind the launch.
static cudaError_t launch_op_rows(RowLaunch& L, const ProblemData& pd, cudaStream_t st) {
    if (!row_needs_global(pd.n, points_of(pd), pd.kind)) {
        const RowTile tile = pick_tile(pd.n);
        L.stage_xy = stage_fits(tile, pd.n, L.max_points, pd.kind) ? 1 : 0;
        return launch_rows_auto(L, pd.kind, tile, st);
    }
    const int grid = row_global_grid(L.ntasks, pd.n);
    L.gstride = row_global_stride(pd.n);
    void* p = nullptr;
    if (dev_alloc(&p, L.gstride * grid, st) != BRKGA_OK) return cudaErrorMemoryAllocation;
    L.gscratch = p;
    const cudaError_t e = launch_rows(L, pd.kind, kGlobalTile, grid, st);
    dev_free(p, st);
    return e;
}
}  // namespace bk

extern "C" {

int32_t brkga_evaluate_population(brkga_problem* pb, const float* d_population, float* d_fitness,
                                  int32_t pop_size, int32_t chrom_len, int32_t ld, int32_t* d_perm,
                                  void* stream) {
    if (!pb || !d_population || !d_fitness) return fail(BRKGA_ERR_INVALID, "null argument");
    const ProblemData& pd = *pb->d;
    if (pd.kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "an external-fitness problem is evaluated by its caller");
    if (chrom_len != pd.n)
        return fail(BRKGA_ERR_INVALID, "chrom_len " + std::to_string(chrom_len) + " != problem size " +
                                           std::to_string(pd.n));
    if (pop_size < 0) return fail(BRKGA_ERR_INVALID, "negative pop_size");
    if (ld <= 0) ld = chrom_len;
    if (ld < chrom_len) return fail(BRKGA_ERR_INVALID, "ld < chrom_len");
    if (pop_size == 0) return BRKGA_OK;
    DeviceGuard g(pd.device);
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    fill_instance(L.single, pd);
    L.single.ld = ld;
    L.single.keys[0] = const_cast<float*>(d_population);
    L.single.fit[0] = d_fitness;
    L.single.P = pop_size;
    L.ntasks = pop_size;
    L.mode = MODE_EVAL;
    L.perm_out = d_perm;
    L.max_n = pd.n;
    L.max_points = points_of(pd);
    cudaError_t e = launch_op_rows(L, pd, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "evaluate launch");
    return BRKGA_OK;
}

int32_t brkga_evaluate_population_sync(brkga_problem* pb, const float* d_population, float* d_fitness,
                                       int32_t pop_size, int32_t chrom_len) {
    int32_t st = brkga_evaluate_population(pb, d_population, d_fitness, pop_size, chrom_len, chrom_len,
                                           nullptr, nullptr);
    if (st != BRKGA_OK) return st;
    DeviceGuard g(pb->d->device);
    cudaError_t e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "evaluate");
    return BRKGA_OK;
}

int32_t brkga_sort_fitness(const float* d_fitness, int32_t P, int32_t segments, int32_t maximize,
                           int32_t* d_sorted, void* stream) {
    if (!d_fitness || !d_sorted) return fail(BRKGA_ERR_INVALID, "null argument");
    if (P < 0 || segments < 0) return fail(BRKGA_ERR_INVALID, "negative size");
    if (P > kMaxPop) return fail(BRKGA_ERR_UNSUPPORTED, "population above " + std::to_string(kMaxPop));
    if (P == 0 || segments == 0) return BRKGA_OK;
    cudaError_t e = prepare_sort(P);
    if (e != cudaSuccess) return cuda_fail(e, "sort setup");
    e = launch_sort_raw(d_fitness, P, segments, maximize ? 1 : 0, d_sorted, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "sort launch");
    return BRKGA_OK;
}

int32_t brkga_generation_step(brkga_problem* pb, const float* d_pop, const float* d_fitness,
                              const int32_t* d_sorted, float* d_next, float* d_next_fitness, int32_t P,
                              int32_t E, int32_t M, double elite_prob, int32_t ld, uint64_t seed,
                              uint32_t generation, int32_t island, void* stream) {
    if (!pb || !d_pop || !d_fitness || !d_sorted || !d_next || !d_next_fitness)
        return fail(BRKGA_ERR_INVALID, "null argument");
    const ProblemData& pd = *pb->d;
    if (pd.kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "an external-fitness problem is evaluated by its caller");
    if (pd.m != 1) return fail(BRKGA_ERR_INVALID, "generation step is single-objective");
    if (P <= 0 || E <= 0 || M < 0 || E + M > P) return fail(BRKGA_ERR_INVALID, "need P > 0, E > 0, E + M <= P");
    if (!(elite_prob >= 0.0 && elite_prob <= 1.0)) return fail(BRKGA_ERR_INVALID, "elite_prob outside [0,1]");
    if (generation < 1) return fail(BRKGA_ERR_INVALID, "generation must be >= 1");
    if (ld <= 0) ld = round_up(pd.n, 4);
    if (ld % 4 != 0 || ld < pd.n) return fail(BRKGA_ERR_INVALID, "ld must be a multiple of 4 and >= n");
    if (((uintptr_t)d_pop | (uintptr_t)d_next) & 15) return fail(BRKGA_ERR_INVALID, "buffers must be 16-byte aligned");
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    fill_instance(L.single, pd);
    L.single.ld = ld;
    L.single.keys[0] = const_cast<float*>(d_pop);
    L.single.keys[1] = d_next;
    L.single.fit[0] = const_cast<float*>(d_fitness);
    L.single.fit[1] = d_next_fitness;
    L.single.sorted = const_cast<int32_t*>(d_sorted);
    L.single.P = P;
    L.single.E = E;
    L.single.M = M;
    L.single.rhoT = prob_threshold(elite_prob);
    L.single.seed = seed;
    L.single.island = (uint32_t)island;
    L.single.gen = generation - 1;
    L.ntasks = P;
    L.mode = MODE_GEN;
    L.max_n = pd.n;
    L.max_points = points_of(pd);
    DeviceGuard g(pd.device);
    cudaError_t e = launch_op_rows(L, pd, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "generation launch");
    return BRKGA_OK;
}

int32_t brkga_local_search(brkga_problem* pb, float* d_pop, float* d_fitness, int32_t num_to_improve,
                           int32_t chrom_len, int32_t ld, int32_t num_moves, uint64_t seed, uint32_t generation,
                           int32_t island, void* stream) {
    if (!pb || !d_pop || !d_fitness) return fail(BRKGA_ERR_INVALID, "null argument");
    const ProblemData& pd = *pb->d;
    if (pd.kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "an external-fitness problem is evaluated by its caller");
    if (pd.kind != BRKGA_TSPJ) return fail(BRKGA_ERR_UNSUPPORTED, "local search is defined for TSPJ problems");
    if (chrom_len != pd.n)
        return fail(BRKGA_ERR_INVALID, "chrom_len " + std::to_string(chrom_len) + " != problem size " +
                                           std::to_string(pd.n));
    if (num_to_improve < 0 || num_moves < 0) return fail(BRKGA_ERR_INVALID, "negative count");
    if (ld <= 0) ld = round_up(pd.n, 4);
    if (ld % 4 != 0 || ld < pd.n) return fail(BRKGA_ERR_INVALID, "ld must be a multiple of 4 and >= chrom_len");
    if ((uintptr_t)d_pop & 15) return fail(BRKGA_ERR_INVALID, "buffer must be 16-byte aligned");
    if (row_needs_global(pd.n, points_of(pd), pd.kind))
        return fail(BRKGA_ERR_UNSUPPORTED, "local search needs rows that fit the shared-memory row kernel");
    if (num_to_improve == 0 || num_moves == 0) return BRKGA_OK;
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    fill_instance(L.single, pd);
    L.single.ld = ld;
    L.single.keys[0] = d_pop;
    L.single.fit[0] = d_fitness;
    L.single.P = num_to_improve;
    L.single.seed = seed;
    L.single.island = (uint32_t)island;
    L.single.gen = generation;
    L.ntasks = num_to_improve;
    L.mode = MODE_LSEARCH;
    L.ls_moves = num_moves;
    L.ls_force = 1;
    L.max_n = pd.n;
    L.max_points = points_of(pd);
    DeviceGuard g(pd.device);
    cudaError_t e = launch_op_rows(L, pd, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "local search launch");
    return BRKGA_OK;
}

int32_t brkga_init_population(brkga_problem* pb, float* d_pop, float* d_fitness, int32_t P, int32_t ld,
                              uint64_t seed, int32_t island, void* stream) {
    if (!pb || !d_pop || !d_fitness) return fail(BRKGA_ERR_INVALID, "null argument");
    const ProblemData& pd = *pb->d;
    if (pd.kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "an external-fitness problem is evaluated by its caller");
    if (P <= 0) return fail(BRKGA_ERR_INVALID, "P must be > 0");
    if (ld <= 0) ld = round_up(pd.n, 4);
    if (ld % 4 != 0 || ld < pd.n) return fail(BRKGA_ERR_INVALID, "ld must be a multiple of 4 and >= n");
    if ((uintptr_t)d_pop & 15) return fail(BRKGA_ERR_INVALID, "buffer must be 16-byte aligned");
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    fill_instance(L.single, pd);
    L.single.ld = ld;
    L.single.keys[0] = d_pop;
    L.single.fit[0] = d_fitness;
    L.single.P = P;
    L.single.seed = seed;
    L.single.island = (uint32_t)island;
    L.ntasks = P;
    L.mode = MODE_INIT;
    L.max_n = pd.n;
    L.max_points = points_of(pd);
    DeviceGuard g(pd.device);
    cudaError_t e = launch_op_rows(L, pd, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "init launch");
    return BRKGA_OK;
}

}  // extern "C"

// problem handle accessor for the other translation units
namespace bk {
std::shared_ptr<ProblemData> problem_data(brkga_problem* pb) { return pb ? pb->d : nullptr; }
}  // namespace bk
