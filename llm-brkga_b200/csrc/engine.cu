// engine.cu -- the device-resident solver (Solver<T>, core/solver.hpp), the drop-in for
// the reference's run / evolve_generation / get_best_individual surface.
//
// The population, its fitness, the rank order and the best-fitness history stay in HBM
// for the whole run; one generation is two launches (the fused row kernel and the
// elite-partition sort) that read their state from device-resident descriptors, so the
// sequence is captured once as a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "engine.h"
#include "nsga2.h"

namespace bk {

int32_t make_shape(const ProblemData& pd, const brkga_params& p, Shape* s) {
    Shape sh;
    sh.n = pd.n;
    sh.ld = round_up(pd.n, 4);
    sh.m = pd.m;
    sh.mo = pd.m > 1;
    const int P = p.population_size;
    if (P <= 0) return fail(BRKGA_ERR_INVALID, "population_size must be > 0");
    if (!(p.elite_prob >= 0.0 && p.elite_prob <= 1.0)) return fail(BRKGA_ERR_INVALID, "elite_prob outside [0,1]");
    if (p.max_generations <= 0) return fail(BRKGA_ERR_INVALID, "max_generations must be > 0");
    sh.k = p.num_islands > 0 ? p.num_islands : 1;
    if (sh.mo) {
        // NSGA-II: elite/mutant sizes are not used by the reference (core/config.hpp:170-178);
        // mutant_size here is the optional count of fresh random offspring
        if (sh.k != 1) return fail(BRKGA_ERR_UNSUPPORTED, "islands are single-objective only");
        if (P < 2) return fail(BRKGA_ERR_INVALID, "NSGA-II needs population_size >= 2");
        if (P > nsga_max_population())
            return fail(BRKGA_ERR_UNSUPPORTED, "NSGA-II population above " + std::to_string(nsga_max_population()));
        sh.Pi = P;
        sh.Mn = std::max(0, std::min(P, p.mutant_size));
    } else {
        sh.Pi = P / sh.k;
        sh.Ei = p.elite_size / sh.k;
        sh.Mi = p.mutant_size / sh.k;
        if (sh.Pi <= 0) return fail(BRKGA_ERR_INVALID, "fewer individuals than islands");
        if (sh.Ei <= 0 || p.mutant_size < 0 || sh.Ei + sh.Mi > sh.Pi)
            return fail(BRKGA_ERR_INVALID, "need elite_size > 0, mutant_size >= 0, elite + mutant <= population");
        if (sh.Pi > kMaxPop) return fail(BRKGA_ERR_UNSUPPORTED, "population above " + std::to_string(kMaxPop));
        if (sh.k > 1 && p.migration_interval > 0 && 2 * p.num_migrants > sh.Pi)
            return fail(BRKGA_ERR_INVALID, "num_migrants must be <= half an island");
    }
    *s = sh;
    return BRKGA_OK;
}

static int32_t dalloc(Population& p, void** ptr, size_t bytes) {
    int32_t st = dev_alloc(ptr, bytes ? bytes : 16, p.stream);
    if (st != BRKGA_OK) return st;
    p.allocs.push_back(*ptr);
    p.bytes += bytes;
    return BRKGA_OK;
}

int32_t Population::allocate(int device) {
    DeviceGuard g(device);
    rows = sh.mo ? 2 * sh.Pi : sh.k * sh.Pi;
    hist_cap = std::max(prm.max_generations, 1) + 1;
    void* p = nullptr;
    int32_t st;
    for (int b = 0; b < 2; ++b) {
        if ((st = dalloc(*this, &p, (size_t)rows * sh.ld * 4)) != BRKGA_OK) return st;
        keys[b] = (float*)p;
        cudaMemsetAsync(p, 0, (size_t)rows * sh.ld * 4, stream);
        if ((st = dalloc(*this, &p, (size_t)rows * sh.m * 4)) != BRKGA_OK) return st;
        fit[b] = (float*)p;
    }
    if ((st = dalloc(*this, &p, (size_t)rows * 4)) != BRKGA_OK) return st;
    sorted = (int32_t*)p;
    if ((st = dalloc(*this, &p, (size_t)rows * 8)) != BRKGA_OK) return st;
    parents = (int2*)p;
    if ((st = dalloc(*this, &p, (size_t)sh.k * 4)) != BRKGA_OK) return st;
    done = (int32_t*)p;
    cudaMemsetAsync(done, 0, (size_t)sh.k * 4, stream);
    if ((st = dalloc(*this, &p, (size_t)sh.k * hist_cap * 4)) != BRKGA_OK) return st;
    history = (float*)p;
    return BRKGA_OK;
}

void Population::release(int device) {
    DeviceGuard g(device);
    for (void* a : allocs) dev_free(a, stream);
    allocs.clear();
}

}  // namespace bk

using namespace bk;

// the longest captured run of plain generations is 2^kMaxRunLog
constexpr int kMaxRunLog = 4;

struct brkga_engine {
    std::mutex mu;
    int device = 0;
    cudaStream_t stream = nullptr;
    Population pop;
    std::vector<PopDesc> hd;
    PopDesc* dd = nullptr;
    Task* d_tasks_gen = nullptr;
    Task* d_tasks_all = nullptr;
    int nt_gen = 0, nt_all = 0;
    RowTile tile{};
    int grid = 0;
    bool stage = false;
    uint32_t gen = 0;
    bool initialized = false;
    // captured runs of 2^k plain generations (k <= kMaxRunLog), and one special generation
    // (a migration for islands, the diversity pass for NSGA-II)
    cudaGraphExec_t gx_run[kMaxRunLog + 1] = {};
    cudaGraphExec_t gx_special = nullptr;
    // external fitness (BRKGA_EXTERNAL): rows pending the caller's fitness (0 none, 1 the
    // initial population, 2 a generation's new rows, 3 NSGA-II refill rows after a
    // diversity rebuild), where they are, the buffer holding the ranked population
    // (BRKGA), and the packed [P][n] copy of the keys for callers that want dense rows
    bool external = false;
    int ext_state = 0;
    int ext_cur = 0;
    float* ext_keys = nullptr;
    float* ext_fit = nullptr;
    int ext_first = 0, ext_count = 0;
    float* ext_dense = nullptr;
    int32_t* d_perm = nullptr;
    float* d_tmpfit = nullptr;
    NsgaState nsga;
    void* gscratch = nullptr;  // sort scratch of the global-memory row kernel (rows beyond shared memory)
    size_t gstride = 0;
    int ls_count = 0;          // TSPJ local search: top ranks searched per island (0 = off)
    Task* d_tasks_ls = nullptr;
};

static RowLaunch base_launch(brkga_engine* e, int mode) {
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.descs = e->dd;
    L.mode = mode;
    L.max_n = e->pop.sh.n;
    L.max_points = points_of(*e->pop.pd);
    L.stage_xy = e->stage ? 1 : 0;
    L.gscratch = e->gscratch;
    L.gstride = e->gstride;
    return L;
}

// the next generation after the current one (counted from 1) that runs the special graph,
// 0 when none does: islands migrate after generations g % interval == 0; NSGA-II runs its
// diversity pass after generations (g - 1) % interval == 0.  Engines set no generation
// limit, so the device's generation counter equals e->gen.
static uint32_t next_special(const brkga_engine* e) {
    const uint32_t g = e->gen;
    if (e->pop.sh.mo) {
        const int iv = e->nsga.div_interval;
        if (iv <= 0) return 0;
        return (g + (uint32_t)iv - 1u) / (uint32_t)iv * (uint32_t)iv + 1u;
    }
    const auto& p = e->pop.prm;
    if (e->pop.sh.k > 1 && p.migration_interval > 0 && p.num_migrants > 0) {
        const uint32_t iv = (uint32_t)p.migration_interval;
        return (g / iv + 1u) * iv;
    }
    return 0;
}

// one single-objective generation: fused rows + elite partition (+ migration, re-sort)
static cudaError_t enqueue_brkga_gen(brkga_engine* e, bool mig) {
    const Shape& sh = e->pop.sh;
    RowLaunch L = base_launch(e, MODE_GEN);
    L.tasks = (sh.k > 1) ? e->d_tasks_gen : nullptr;
    L.ntasks = e->nt_gen;
    cudaError_t err = launch_rows(L, e->pop.pd->kind, e->tile, e->grid, e->stream);
    if (err != cudaSuccess) return err;
    err = launch_sort_pops(e->dd, sh.k, sh.Pi, 1, e->stream);
    if (err != cudaSuccess) return err;
    if (e->ls_count > 0) {
        // random 2-opt on the best ranks when due (decided on the device from the generation
        // counter, so captured graphs stay valid), then re-rank (core/solver.hpp:459-461)
        RowLaunch Ls = base_launch(e, MODE_LSEARCH);
        Ls.tasks = (sh.k > 1) ? e->d_tasks_ls : nullptr;
        Ls.ntasks = sh.k * e->ls_count;
        Ls.ls_moves = e->pop.prm.local_search_moves;
        err = launch_rows(Ls, e->pop.pd->kind, e->tile, e->grid, e->stream);
        if (err != cudaSuccess) return err;
        err = launch_sort_pops_after_ls(e->dd, sh.k, sh.Pi, e->stream);
        if (err != cudaSuccess) return err;
    }
    if (mig) {
        err = launch_migrate(e->dd, 1, sh.k, e->pop.prm.num_migrants, sh.n, e->stream);
        if (err != cudaSuccess) return err;
        err = launch_sort_pops(e->dd, sh.k, sh.Pi, 0, e->stream);
    }
    return err;
}

static cudaError_t enqueue_gen(brkga_engine* e, bool special) {
    if (e->pop.sh.mo) return nsga_enqueue_generation(e->nsga, e->stream, special);
    return enqueue_brkga_gen(e, special);
}

static cudaError_t capture(brkga_engine* e, int gens, bool special, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return err;
    for (int i = 0; i < gens && err == cudaSuccess; ++i) err = enqueue_gen(e, special && i == gens - 1);
    cudaError_t end = cudaStreamEndCapture(e->stream, &g);
    if (err != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return err;
    }
    if (end != cudaSuccess) return end;
    err = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return err;
}

static int32_t sync_descs_to_host(brkga_engine* e) {
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_fail(err, "engine stream");
    err = cudaMemcpy(e->hd.data(), e->dd, sizeof(PopDesc) * e->hd.size(), cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "descriptor read-back");
    return BRKGA_OK;
}

static int32_t grow_history(brkga_engine* e, int need) {
    Population& p = e->pop;
    if (need <= p.hist_cap) return BRKGA_OK;
    int32_t st = sync_descs_to_host(e);
    if (st != BRKGA_OK) return st;
    int cap = p.hist_cap;
    while (cap < need) cap *= 2;
    void* nh = nullptr;
    if ((st = dalloc(p, &nh, (size_t)p.sh.k * cap * 4)) != BRKGA_OK) return st;
    cudaStreamSynchronize(e->stream);
    for (int i = 0; i < p.sh.k; ++i) {
        cudaError_t err = cudaMemcpy((float*)nh + (size_t)i * cap, p.history + (size_t)i * p.hist_cap,
                                     (size_t)p.hist_cap * 4, cudaMemcpyDeviceToDevice);
        if (err != cudaSuccess) return cuda_fail(err, "history copy");
        e->hd[i].history = (float*)nh + (size_t)i * cap;
        e->hd[i].hist_cap = cap;
    }
    p.history = (float*)nh;
    p.hist_cap = cap;
    if (p.sh.mo) nsga_set_history(e->nsga, p.history, cap);
    cudaError_t err = cudaMemcpy(e->dd, e->hd.data(), sizeof(PopDesc) * e->hd.size(), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_fail(err, "descriptor upload");
    return BRKGA_OK;
}

static void destroy_engine(brkga_engine* e) {
    DeviceGuard g(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (cudaGraphExec_t x : e->gx_run)
        if (x) cudaGraphExecDestroy(x);
    if (e->gx_special) cudaGraphExecDestroy(e->gx_special);
    nsga_release(e->nsga);
    e->pop.release(e->device);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

extern "C" {

int32_t brkga_create(brkga_problem* pbh, const brkga_params* params, brkga_engine** out) {
    if (!pbh || !params || !out) return fail(BRKGA_ERR_INVALID, "null argument");
    *out = nullptr;
    auto pd = problem_data(pbh);
    if (params->device != pd->device)
        return fail(BRKGA_ERR_INVALID, "params.device differs from the problem's device");
    Shape sh;
    int32_t st = make_shape(*pd, *params, &sh);
    if (st != BRKGA_OK) return st;
    if (pd->kind == BRKGA_EXTERNAL && sh.k > 1)
        return fail(BRKGA_ERR_UNSUPPORTED, "external-fitness engines run one population (no islands)");
    DeviceGuard g(pd->device);
    if (!g.ok()) return fail(BRKGA_ERR_CUDA, "cannot select device");
    auto* e = new brkga_engine;
    e->device = pd->device;
    e->external = pd->kind == BRKGA_EXTERNAL;
    e->pop.pd = pd;
    e->pop.prm = *params;
    e->pop.sh = sh;
    cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete e;
        return cuda_fail(err, "stream");
    }
    e->pop.stream = e->stream;
    if ((st = e->pop.allocate(e->device)) != BRKGA_OK) {
        destroy_engine(e);
        return st;
    }
    void* p = nullptr;
    if ((st = dalloc(e->pop, &p, sizeof(PopDesc) * sh.k)) != BRKGA_OK) {
        destroy_engine(e);
        return st;
    }
    e->dd = (PopDesc*)p;
    if ((st = dalloc(e->pop, &p, (size_t)sh.n * 4)) != BRKGA_OK || (st = dalloc(e->pop, &p, 8)) != BRKGA_OK) {
        destroy_engine(e);
        return st;
    }
    e->d_perm = (int32_t*)e->pop.allocs[e->pop.allocs.size() - 2];
    e->d_tmpfit = (float*)p;
    // island descriptors
    e->hd.resize(sh.k);
    for (int i = 0; i < sh.k; ++i) {
        PopDesc& d = e->hd[i];
        fill_instance(d, *pd);
        d.P = sh.Pi;
        d.E = sh.Ei;
        d.M = sh.Mi;
        d.rhoT = prob_threshold(params->elite_prob);
        d.seed = params->seed;
        d.island = (uint32_t)i;
        d.row0 = i * sh.Pi;
        for (int b = 0; b < 2; ++b) {
            d.keys[b] = e->pop.keys[b] + (size_t)i * sh.Pi * sh.ld;
            d.fit[b] = e->pop.fit[b] + (size_t)i * sh.Pi * sh.m;
        }
        d.sorted = e->pop.sorted + (size_t)i * sh.Pi;
        d.parents = sh.mo ? nullptr : e->pop.parents + (size_t)i * sh.Pi;
        d.done = e->pop.done + i;
        d.history = e->pop.history + (size_t)i * e->pop.hist_cap;
        d.hist_cap = e->pop.hist_cap;
        d.cur = 0;
        d.gen = 0;
    }
    // TSPJ random 2-opt local search (the reference runs it in its island loop on
    // problems whose config has one: TSPJConfig, configs/tspj_config.hpp:69-136)
    if (!sh.mo && pd->kind == BRKGA_TSPJ && params->local_search_interval > 0 &&
        params->local_search_individuals > 0 && params->local_search_moves > 0) {
        if (row_needs_global(sh.n, points_of(*pd), pd->kind)) {
            destroy_engine(e);
            return fail(BRKGA_ERR_UNSUPPORTED, "local search needs rows that fit the shared-memory row kernel");
        }
        e->ls_count = std::min(params->local_search_individuals, sh.Ei);
        for (auto& d : e->hd) d.ls_interval = params->local_search_interval;
    }
    // pool allocations and clears are ordered on the engine stream: complete them before
    // the synchronous uploads below touch the memory
    err = cudaStreamSynchronize(e->stream);
    if (err == cudaSuccess) err = cudaMemcpy(e->dd, e->hd.data(), sizeof(PopDesc) * sh.k, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        destroy_engine(e);
        return cuda_fail(err, "descriptor upload");
    }
    // work lists: costly rows (children, mutants) of every island first, elite copies last
    if (sh.k > 1) {
        std::vector<Task> tg, ta;
        for (int i = 0; i < sh.k; ++i)
            for (int r = sh.Ei; r < sh.Pi; ++r) tg.push_back({i, r});
        for (int i = 0; i < sh.k; ++i)
            for (int r = 0; r < sh.Ei; ++r) tg.push_back({i, r});
        for (int i = 0; i < sh.k; ++i)
            for (int r = 0; r < sh.Pi; ++r) ta.push_back({i, r});
        if ((st = dalloc(e->pop, &p, tg.size() * sizeof(Task))) != BRKGA_OK) {
            destroy_engine(e);
            return st;
        }
        e->d_tasks_gen = (Task*)p;
        cudaMemcpy(p, tg.data(), tg.size() * sizeof(Task), cudaMemcpyHostToDevice);
        if ((st = dalloc(e->pop, &p, ta.size() * sizeof(Task))) != BRKGA_OK) {
            destroy_engine(e);
            return st;
        }
        e->d_tasks_all = (Task*)p;
        cudaMemcpy(p, ta.data(), ta.size() * sizeof(Task), cudaMemcpyHostToDevice);
        e->nt_gen = (int)tg.size();
        e->nt_all = (int)ta.size();
        if (e->ls_count > 0) {
            std::vector<Task> tl;
            for (int i = 0; i < sh.k; ++i)
                for (int q = 0; q < e->ls_count; ++q) tl.push_back({i, q});
            if ((st = dalloc(e->pop, &p, tl.size() * sizeof(Task))) != BRKGA_OK) {
                destroy_engine(e);
                return st;
            }
            e->d_tasks_ls = (Task*)p;
            cudaMemcpy(p, tl.data(), tl.size() * sizeof(Task), cudaMemcpyHostToDevice);
        }
    } else {
        e->nt_gen = sh.Pi;
        e->nt_all = sh.Pi;
    }
    // tile, staging and grid: autotuned on this engine's own rows (initialisation launches)
    {
        const int pts = points_of(*pd);
        auto launch = [&](const TunedTile& tt) -> cudaError_t {
            RowLaunch L;
            std::memset(&L, 0, sizeof(L));
            L.descs = e->dd;
            L.mode = MODE_INIT;
            L.tasks = (sh.k > 1) ? e->d_tasks_all : nullptr;
            L.ntasks = sh.mo ? sh.Pi : e->nt_all;
            L.max_n = sh.n;
            L.max_points = pts;
            L.stage_xy = tt.stage ? 1 : 0;
            return launch_rows(L, pd->kind, tt.tile, tt.grid, e->stream);
        };
        const int rows = sh.mo ? sh.Pi : e->nt_all;
        if (row_needs_global(sh.n, pts, pd->kind)) {
            // the row's sort does not fit in shared memory: global-scratch kernel
            e->tile = kGlobalTile;
            e->grid = row_global_grid(rows, sh.n);
            e->stage = false;
            e->gstride = row_global_stride(sh.n);
            if ((st = dalloc(e->pop, &e->gscratch, e->gstride * e->grid)) != BRKGA_OK) {
                destroy_engine(e);
                return st;
            }
        } else {
            TunedTile tt;
            st = autotune_tile(pd->kind, sh.n, pts, rows, e->stream, launch, &tt);
            if (st != BRKGA_OK) {
                destroy_engine(e);
                return st;
            }
            e->tile = tt.tile;
            e->grid = tt.grid;
            e->stage = tt.stage;
        }
    }
    err = prepare_sort(sh.mo ? 2 * sh.Pi : sh.Pi);
    if (err != cudaSuccess) {
        destroy_engine(e);
        return cuda_fail(err, "sort set-up");
    }
    if (sh.mo) {
        st = nsga_setup(e->nsga, e->pop, e->dd, e->hd[0], e->tile, e->grid, e->stage);
        if (st != BRKGA_OK) {
            destroy_engine(e);
            return st;
        }
        e->nsga.gscratch = e->gscratch;
        e->nsga.gstride = e->gstride;
    }
    *out = e;
    return BRKGA_OK;
}

int32_t brkga_destroy(brkga_engine* e) {
    if (!e) return BRKGA_OK;
    destroy_engine(e);
    return BRKGA_OK;
}

int32_t brkga_initialize(brkga_engine* e) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (e->external) {
        // the next brkga_external_begin builds a new initial population
        e->initialized = false;
        e->ext_state = 0;
        e->gen = 0;
        return BRKGA_OK;
    }
    const Shape& sh = e->pop.sh;
    // reset generation counters / buffer index on the device
    for (auto& d : e->hd) {
        d.cur = 0;
        d.gen = 0;
    }
    cudaError_t err = cudaMemcpyAsync(e->dd, e->hd.data(), sizeof(PopDesc) * e->hd.size(),
                                      cudaMemcpyHostToDevice, e->stream);
    if (err != cudaSuccess) return cuda_fail(err, "descriptor upload");
    if (sh.mo) {
        err = nsga_enqueue_init(e->nsga, e->stream);
    } else {
        RowLaunch L = base_launch(e, MODE_INIT);
        L.tasks = (sh.k > 1) ? e->d_tasks_all : nullptr;
        L.ntasks = e->nt_all;
        err = launch_rows(L, e->pop.pd->kind, e->tile, e->grid, e->stream);
        if (err == cudaSuccess) err = launch_sort_pops(e->dd, sh.k, sh.Pi, 0, e->stream);
    }
    if (err != cudaSuccess) return cuda_fail(err, "initialize");
    e->gen = 0;
    e->initialized = true;
    return BRKGA_OK;
}

int32_t brkga_evolve(brkga_engine* e, int32_t generations) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    if (generations < 0) return fail(BRKGA_ERR_INVALID, "negative generation count");
    if (e->external)
        return fail(BRKGA_ERR_UNSUPPORTED, "external-fitness engine: use brkga_external_begin / _commit");
    if (!e->initialized) {
        int32_t st = brkga_initialize(e);
        if (st != BRKGA_OK) return st;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    int32_t st = grow_history(e, (int)e->gen + generations + 1);
    if (st != BRKGA_OK) return st;
    cudaError_t err = cudaSuccess;
    int left = generations;
    NvtxRange all("brkga_evolve", e->gen + 1u, e->gen + (unsigned)generations);
    while (left > 0 && err == cudaSuccess) {
        // plain generations until (and excluding) the next special one, in captured runs of
        // 16, then 8, 4, 2, 1
        const uint32_t next = next_special(e);
        int plain = next ? std::min<int>(left, (int)(next - e->gen - 1u)) : left;
        while (plain > 0 && err == cudaSuccess) {
            int k = kMaxRunLog;
            while ((1 << k) > plain) --k;
            NvtxRange run("generations", e->gen + 1u, e->gen + (1u << k));
            if (!e->gx_run[k]) err = capture(e, 1 << k, false, &e->gx_run[k]);
            if (err == cudaSuccess) err = cudaGraphLaunch(e->gx_run[k], e->stream);
            plain -= 1 << k;
            left -= 1 << k;
            e->gen += 1u << k;
        }
        if (left > 0 && err == cudaSuccess) {
            // here e->gen + 1 == next
            NvtxRange run("generation (migration / diversity / local search)", e->gen + 1u, e->gen + 1u);
            if (!e->gx_special) err = capture(e, 1, true, &e->gx_special);
            if (err == cudaSuccess) err = cudaGraphLaunch(e->gx_special, e->stream);
            --left;
            ++e->gen;
        }
    }
    if (err != cudaSuccess) return cuda_fail(err, "evolve");
    return BRKGA_OK;
}

int32_t brkga_synchronize(brkga_engine* e) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    DeviceGuard g(e->device);
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_fail(err, "engine stream");
    return BRKGA_OK;
}

int32_t brkga_run(brkga_engine* e) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    if (e->external)
        return fail(BRKGA_ERR_UNSUPPORTED, "external-fitness engine: use brkga_external_begin / _commit");
    int32_t st = brkga_initialize(e);
    if (st != BRKGA_OK) return st;
    st = brkga_evolve(e, e->pop.prm.max_generations);
    if (st != BRKGA_OK) return st;
    return brkga_synchronize(e);
}

int32_t brkga_generation(const brkga_engine* e) { return e ? (int32_t)e->gen : BRKGA_ERR_INVALID; }

int32_t brkga_engine_info(brkga_engine* e, int32_t* info, int32_t cap) {
    if (!e || !info || cap < 4) return fail(BRKGA_ERR_INVALID, "need an engine and cap >= 4");
    info[0] = e->tile.block;
    info[1] = e->tile.groups;
    info[2] = e->grid;
    info[3] = e->stage ? 1 : 0;
    return BRKGA_OK;
}

int32_t brkga_get_stream(brkga_engine* e, void** stream) {
    if (!e || !stream) return fail(BRKGA_ERR_INVALID, "null argument");
    *stream = (void*)e->stream;
    return BRKGA_OK;
}

int32_t brkga_get_population(brkga_engine* e, float* keys, float* fitness) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    std::lock_guard<std::mutex> lk(e->mu);
    if (e->external && (e->ext_state != 0 || !e->initialized))
        return fail(BRKGA_ERR_INVALID, "no ranked population yet: commit the pending rows first");
    DeviceGuard g(e->device);
    if (e->pop.sh.mo) return nsga_get_population(e->nsga, e->stream, keys, fitness);
    int32_t st = sync_descs_to_host(e);
    if (st != BRKGA_OK) return st;
    const Shape& sh = e->pop.sh;
    const int cur = e->hd[0].cur;
    const int rows = sh.k * sh.Pi;
    std::vector<float> hk((size_t)rows * sh.ld), hf((size_t)rows * sh.m);
    std::vector<int32_t> hs(rows);
    cudaMemcpy(hk.data(), e->pop.keys[cur], hk.size() * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hf.data(), e->pop.fit[cur], hf.size() * 4, cudaMemcpyDeviceToHost);
    cudaError_t err = cudaMemcpy(hs.data(), e->pop.sorted, hs.size() * 4, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "population read-back");
    for (int i = 0; i < sh.k; ++i)
        for (int r = 0; r < sh.Pi; ++r) {
            const int src = i * sh.Pi + hs[(size_t)i * sh.Pi + r];
            const int dst = i * sh.Pi + r;
            if (keys) std::memcpy(keys + (size_t)dst * sh.n, hk.data() + (size_t)src * sh.ld, (size_t)sh.n * 4);
            if (fitness) std::memcpy(fitness + (size_t)dst * sh.m, hf.data() + (size_t)src * sh.m, (size_t)sh.m * 4);
        }
    return BRKGA_OK;
}

int32_t brkga_set_population(brkga_engine* e, const float* keys) {
    if (!e || !keys) return fail(BRKGA_ERR_INVALID, "null argument");
    if (e->external) return fail(BRKGA_ERR_UNSUPPORTED, "the engine cannot evaluate an external-fitness population");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (e->pop.sh.mo) {
        int32_t st = nsga_set_population(e->nsga, e->stream, keys);
        if (st == BRKGA_OK) e->initialized = true;
        return st;
    }
    int32_t st = sync_descs_to_host(e);
    if (st != BRKGA_OK) return st;
    const Shape& sh = e->pop.sh;
    const int cur = e->hd[0].cur;
    const int rows = sh.k * sh.Pi;
    std::vector<float> hk((size_t)rows * sh.ld, 0.0f);
    for (int r = 0; r < rows; ++r) std::memcpy(hk.data() + (size_t)r * sh.ld, keys + (size_t)r * sh.n, (size_t)sh.n * 4);
    cudaError_t err = cudaMemcpy(e->pop.keys[cur], hk.data(), hk.size() * 4, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_fail(err, "population upload");
    RowLaunch L = base_launch(e, MODE_EVAL);
    L.tasks = (sh.k > 1) ? e->d_tasks_all : nullptr;
    L.ntasks = e->nt_all;
    err = launch_rows(L, e->pop.pd->kind, e->tile, e->grid, e->stream);
    if (err == cudaSuccess) err = launch_sort_pops(e->dd, sh.k, sh.Pi, 0, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_fail(err, "population evaluate");
    if (!e->initialized) {
        e->initialized = true;
        e->gen = e->hd[0].gen;
    }
    return BRKGA_OK;
}

int32_t brkga_get_best(brkga_engine* e, float* keys, int32_t* perm, float* fitness) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    if (e->external && perm) return fail(BRKGA_ERR_UNSUPPORTED, "an external-fitness problem is not decoded here");
    std::lock_guard<std::mutex> lk(e->mu);
    if (e->external && (e->ext_state != 0 || !e->initialized))
        return fail(BRKGA_ERR_INVALID, "no ranked population yet: commit the pending rows first");
    DeviceGuard g(e->device);
    if (e->pop.sh.mo) return nsga_get_best(e->nsga, e->stream, keys, perm, fitness);
    int32_t st = sync_descs_to_host(e);
    if (st != BRKGA_OK) return st;
    const Shape& sh = e->pop.sh;
    const ProblemData& pd = *e->pop.pd;
    // best island: compare each island's rank-0 fitness in the problem's order
    int best_i = 0, best_row = 0;
    float best_f = 0.0f;
    for (int i = 0; i < sh.k; ++i) {
        const PopDesc& d = e->hd[i];
        int32_t r0 = 0;
        float f0 = 0.0f;
        cudaMemcpy(&r0, d.sorted, 4, cudaMemcpyDeviceToHost);
        cudaError_t err = cudaMemcpy(&f0, d.fit[d.cur] + (size_t)r0 * sh.m, 4, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return cuda_fail(err, "best read-back");
        const bool better = (i == 0) || (pd.maximize ? (f0 > best_f) : (f0 < best_f));
        if (better) {
            best_i = i;
            best_row = r0;
            best_f = f0;
        }
    }
    const PopDesc& d = e->hd[best_i];
    const float* row = d.keys[d.cur] + (size_t)best_row * sh.ld;
    if (fitness) *fitness = best_f;
    if (keys) {
        cudaError_t err = cudaMemcpy(keys, row, (size_t)sh.n * 4, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return cuda_fail(err, "best keys read-back");
    }
    if (perm) {
        // decode on the device (same argsort as the generation kernel)
        RowLaunch L;
        std::memset(&L, 0, sizeof(L));
        fill_instance(L.single, pd);
        L.single.keys[0] = const_cast<float*>(row);
        L.single.fit[0] = e->d_tmpfit;
        L.single.P = 1;
        L.ntasks = 1;
        L.mode = MODE_EVAL;
        L.perm_out = e->d_perm;
        L.max_n = sh.n;
        L.max_points = points_of(pd);
        L.stage_xy = e->stage ? 1 : 0;
        L.gscratch = e->gscratch;
        L.gstride = e->gstride;
        cudaError_t err = launch_rows(L, pd.kind, e->tile, 1, e->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
        if (err == cudaSuccess) err = cudaMemcpy(perm, e->d_perm, (size_t)sh.n * 4, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) return cuda_fail(err, "best decode");
    }
    return BRKGA_OK;
}

int32_t brkga_get_fitness_history(brkga_engine* e, float* history, int32_t cap, int32_t* len) {
    if (!e || !history || !len) return fail(BRKGA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_fail(err, "engine stream");
    const Shape& sh = e->pop.sh;
    const int have = std::min<int>((int)e->gen + 1, e->pop.hist_cap);
    const int cnt = std::min(have, (int)cap);
    std::vector<float> h((size_t)sh.k * e->pop.hist_cap);
    err = cudaMemcpy(h.data(), e->pop.history, h.size() * 4, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "history read-back");
    const bool mx = e->pop.pd->maximize != 0;
    for (int g2 = 0; g2 < cnt; ++g2) {
        float b = h[g2];
        for (int i = 1; i < sh.k; ++i) {
            const float v = h[(size_t)i * e->pop.hist_cap + g2];
            if (mx ? (v > b) : (v < b)) b = v;
        }
        history[g2] = b;
    }
    *len = cnt;
    return BRKGA_OK;
}

int32_t brkga_get_pareto_front(brkga_engine* e, float* objectives, float* keys, int32_t cap, int32_t* count) {
    if (!e || !count) return fail(BRKGA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (!e->pop.sh.mo) return fail(BRKGA_ERR_INVALID, "not a multi-objective problem");
    return nsga_get_front(e->nsga, e->stream, objectives, keys, cap, count);
}

// ---- external fitness --------------------------------------------------------------------
// The rows are built by the global-memory row kernel, which stores them without evaluating
// an external problem (elite copies keep their fitness); the caller fills the fitness of
// the pending rows; the commit is the elite partition (BRKGA: initially on the current
// buffer, then with the buffer swap and generation advance of an ordinary generation) or
// the NSGA-II selection (survivors moved into the other buffer) and, when due, the
// diversity pass.

// rows [first, first + count) of keys / fit (m values per row) are pending
static void ext_pending(brkga_engine* e, int state, float* keys, float* fit, int first, int count) {
    const Shape& sh = e->pop.sh;
    const int m = e->pop.pd->m;
    e->ext_state = state;
    e->ext_keys = keys + (size_t)first * sh.ld;
    e->ext_fit = fit + (size_t)first * m;
    e->ext_first = first;
    e->ext_count = count;
}

int32_t brkga_external_begin(brkga_engine* e, int32_t dense, float** d_keys, float** d_fitness, int32_t* ld,
                             int32_t* first, int32_t* count) {
    if (!e || !d_keys || !d_fitness || !ld || !first || !count) return fail(BRKGA_ERR_INVALID, "null argument");
    if (!e->external) return fail(BRKGA_ERR_INVALID, "not an external-fitness engine");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (e->ext_state != 0 && e->ext_state != 3)
        return fail(BRKGA_ERR_INVALID, "rows are pending: call brkga_external_commit first");
    const Shape& sh = e->pop.sh;
    cudaError_t err = cudaSuccess;
    if (e->ext_state == 3) {
        // NSGA-II refill rows, built by the commit that reported them
    } else if (!e->initialized) {
        // Population::initialize (core/population.hpp:107-124)
        for (auto& d : e->hd) {
            d.cur = 0;
            d.gen = 0;
        }
        err = cudaMemcpyAsync(e->dd, e->hd.data(), sizeof(PopDesc) * e->hd.size(), cudaMemcpyHostToDevice, e->stream);
        if (err == cudaSuccess) {
            if (sh.mo) {
                err = nsga_enqueue_rows(e->nsga, MODE_INIT, e->stream);
            } else {
                RowLaunch L = base_launch(e, MODE_INIT);
                L.ntasks = e->nt_all;
                err = launch_rows(L, e->pop.pd->kind, e->tile, e->grid, e->stream);
            }
        }
        e->ext_cur = 0;
        e->gen = 0;
        ext_pending(e, 1, e->pop.keys[0], e->pop.fit[0], 0, sh.Pi);
    } else if (sh.mo) {
        // offspring into pool rows [P, 2P) of the current buffer (core/solver.hpp:1019-1091)
        int32_t st = grow_history(e, (int)e->gen + 2);
        if (st == BRKGA_OK) st = sync_descs_to_host(e);
        if (st != BRKGA_OK) return st;
        const int cur = e->hd[0].cur;
        err = nsga_enqueue_rows(e->nsga, MODE_NSGA_OFF, e->stream);
        ext_pending(e, 2, e->pop.keys[cur], e->pop.fit[cur], sh.Pi, sh.Pi);
    } else {
        int32_t st = grow_history(e, (int)e->gen + 2);
        if (st != BRKGA_OK) return st;
        RowLaunch L = base_launch(e, MODE_GEN);
        L.ntasks = e->nt_gen;
        err = launch_rows(L, e->pop.pd->kind, e->tile, e->grid, e->stream);
        const int buf = e->ext_cur ^ 1;
        ext_pending(e, 2, e->pop.keys[buf], e->pop.fit[buf], sh.Ei, sh.Pi - sh.Ei);
    }
    float* keys = e->ext_keys;
    int stride = sh.ld;
    if (err == cudaSuccess && dense && sh.ld != sh.n && e->ext_count > 0) {
        if (!e->ext_dense) {
            void* p = nullptr;
            int32_t st = dalloc(e->pop, &p, (size_t)sh.Pi * sh.n * 4);
            if (st != BRKGA_OK) {
                e->ext_state = 0;
                return st;
            }
            e->ext_dense = (float*)p;
        }
        err = cudaMemcpy2DAsync(e->ext_dense, (size_t)sh.n * 4, e->ext_keys, (size_t)sh.ld * 4, (size_t)sh.n * 4,
                                (size_t)e->ext_count, cudaMemcpyDeviceToDevice, e->stream);
        keys = e->ext_dense;
        stride = sh.n;
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) {
        e->ext_state = 0;
        return cuda_fail(err, "external rows");
    }
    *d_keys = keys;
    *d_fitness = e->ext_fit;
    *ld = stride;
    *first = e->ext_first;
    *count = e->ext_count;
    return BRKGA_OK;
}

int32_t brkga_external_get_rows(brkga_engine* e, float* keys) {
    if (!e || !keys) return fail(BRKGA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (!e->external || e->ext_state == 0) return fail(BRKGA_ERR_INVALID, "no rows pending");
    const Shape& sh = e->pop.sh;
    if (e->ext_count == 0) return BRKGA_OK;
    cudaError_t err = cudaMemcpy2D(keys, (size_t)sh.n * 4, e->ext_keys, (size_t)sh.ld * 4, (size_t)sh.n * 4,
                                   (size_t)e->ext_count, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return cuda_fail(err, "external rows read-back");
    return BRKGA_OK;
}

int32_t brkga_external_set_fitness(brkga_engine* e, const float* fitness) {
    if (!e || !fitness) return fail(BRKGA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (!e->external || e->ext_state == 0) return fail(BRKGA_ERR_INVALID, "no rows pending");
    if (e->ext_count == 0) return BRKGA_OK;
    cudaError_t err = cudaMemcpy(e->ext_fit, fitness, (size_t)e->ext_count * e->pop.pd->m * 4, cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_fail(err, "external fitness upload");
    return BRKGA_OK;
}

int32_t brkga_external_commit(brkga_engine* e) {
    if (!e) return fail(BRKGA_ERR_INVALID, "null engine");
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard g(e->device);
    if (!e->external || e->ext_state == 0) return fail(BRKGA_ERR_INVALID, "no rows pending");
    const Shape& sh = e->pop.sh;
    // fitness the caller's own kernels wrote, on any stream, is in place before the ranking
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return cuda_fail(err, "external fitness");
    const int state = e->ext_state;
    e->ext_state = 0;
    // the ranking is enqueued; every later call that reads the population (or builds the
    // next rows) waits for the engine's stream first
    if (!sh.mo) {
        err = launch_sort_pops(e->dd, sh.k, sh.Pi, state == 1 ? 0 : 1, e->stream);
        if (err != cudaSuccess) return cuda_fail(err, "external commit");
        if (state == 1) {
            e->initialized = true;
            e->gen = 0;
        } else {
            e->ext_cur ^= 1;
            ++e->gen;
        }
        return BRKGA_OK;
    }
    // NSGA-II (core/population.hpp:409-517; ensure_minimum_diversity :130-182)
    if (state == 1) {
        err = nsga_enqueue_select(e->dd, 1, sh.Pi, 1, e->stream);
    } else if (state == 3) {
        err = nsga_enqueue_select(e->dd, 1, sh.Pi, 2, e->stream);  // re-rank the rebuilt population
    } else {
        err = nsga_enqueue_select(e->dd, 1, sh.Pi, 0, e->stream);  // survivors, rows, buffer swap
        if (err == cudaSuccess && nsga_diversity_due(e->nsga, e->gen + 1)) {
            err = nsga_enqueue_diversity(e->dd, 1, sh.Pi, e->stream);
            int32_t nu = sh.Pi;
            if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
            if (err == cudaSuccess) err = cudaMemcpy(&nu, e->hd[0].nu, 4, cudaMemcpyDeviceToHost);
            if (err == cudaSuccess && nu < sh.Pi) {
                // kept rows were gathered into the other buffer, now current: rows [nu, P)
                // take fresh keys and need the caller's objectives
                ++e->gen;
                int32_t st = sync_descs_to_host(e);
                if (st != BRKGA_OK) return st;
                const int cur = e->hd[0].cur;
                err = nsga_enqueue_rows(e->nsga, MODE_NSGA_REFILL, e->stream);
                if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
                if (err != cudaSuccess) return cuda_fail(err, "external refill rows");
                ext_pending(e, 3, e->pop.keys[cur], e->pop.fit[cur], nu, sh.Pi - nu);
                return fail(BRKGA_ERR_NOT_READY, "diversity refill rows pending: evaluate them and commit again");
            }
        }
        if (err == cudaSuccess) ++e->gen;
    }
    if (err != cudaSuccess) return cuda_fail(err, "external commit");
    if (state == 1) {
        e->initialized = true;
        e->gen = 0;
    }
    return BRKGA_OK;
}

}  // extern "C"
