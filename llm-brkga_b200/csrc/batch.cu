// batch.cu -- many independent populations advanced together, and the serving loop.
//
// A Group holds every population (instances x islands, single- and multi-objective) as
// descriptors in one device array: single-objective populations first, NSGA-II ones
// after.  One generation of the whole group is, per tile bucket, one launch of the fused
// row kernel over a task list of (population, row) with the costly rows first; one
// rank launch over every single-objective population; then the grouped NSGA-II launches.
// Instances with small n and P that would leave the GPU idle alone fill it together.
// A population whose generation reached its limit is left untouched by every kernel, so
// requests with different budgets share launches (the serving loop relies on this).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "nsga2.h"

namespace bk {

struct Member {
    std::shared_ptr<ProblemData> pd;
    brkga_params prm{};
    Shape sh;
    Population pop;
    int first = 0;       // first descriptor
    int ndesc = 0;
    uint32_t limit = 0;  // generation limit (0 = none)
    int prm_index = 0;   // position in the caller's list
};

struct Bucket {
    RowTile tile{};
    int grid = 0;
    bool stage = false;
    int max_n = 0, max_pts = 0, kind = 0;
    Task* d_gen = nullptr;   // generation / NSGA offspring tasks
    Task* d_all = nullptr;   // every row (initialisation, refill)
    int nt_gen = 0, nt_all = 0;
};

struct Group {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<Member*> members;
    std::vector<PopDesc> hd;
    PopDesc* dd = nullptr;
    int cap_desc = 0;
    int nb = 0, nn = 0;           // single-objective / NSGA-II descriptor counts
    int maxP_b = 0, maxP_n = 0;
    int k_mig = 0, mig_interval = 0, mig_count = 0, n_mig_inst = 0;
    std::vector<Bucket> bb, nbk;  // row-kernel buckets for each kind of population
    std::vector<void*> plan_allocs;
    bool any_div = false;
    cudaGraphExec_t gx_chunk = nullptr, gx_one = nullptr, gx_mig = nullptr;
    int chunk = 0;
    // consecutive rows a CTA takes per visit of the task list (measured on B200: 8 helps a
    // batch of same-kind instances, +12%; 1 keeps the served mix of kinds and sizes
    // balanced, 8 there cost 8%)
    int task_group = 1;
    int32_t* work = nullptr;  // the row kernel's dynamic dealing counter (launches on `stream`)
};

// the group's stream and its zeroed row-dealing counter
static int32_t group_start(Group& g) {
    cudaError_t e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "stream");
    int32_t st = dev_alloc((void**)&g.work, 8, g.stream);
    if (st != BRKGA_OK) return st;
    if ((e = cudaMemsetAsync(g.work, 0, 8, g.stream)) != cudaSuccess) return cuda_fail(e, "work counter");
    return BRKGA_OK;
}

static void group_stop(Group& g) {
    if (!g.stream) return;
    if (g.work) dev_free(g.work, g.stream);
    g.work = nullptr;
    cudaStreamSynchronize(g.stream);
    cudaStreamDestroy(g.stream);
    g.stream = nullptr;
}

static void free_plan(Group& g) {
    for (void* p : g.plan_allocs) dev_free(p, g.stream);
    g.plan_allocs.clear();
    g.bb.clear();
    g.nbk.clear();
    if (g.gx_chunk) cudaGraphExecDestroy(g.gx_chunk);
    if (g.gx_one) cudaGraphExecDestroy(g.gx_one);
    if (g.gx_mig) cudaGraphExecDestroy(g.gx_mig);
    g.gx_chunk = g.gx_one = g.gx_mig = nullptr;
}

static int32_t upload_tasks(Group& g, const std::vector<Task>& t, Task** out) {
    *out = nullptr;
    if (t.empty()) return BRKGA_OK;
    void* p = nullptr;
    int32_t st = dev_alloc(&p, t.size() * sizeof(Task), g.stream);
    if (st != BRKGA_OK) return st;
    g.plan_allocs.push_back(p);
    cudaError_t e = cudaMemcpyAsync(p, t.data(), t.size() * sizeof(Task), cudaMemcpyHostToDevice, g.stream);
    if (e != cudaSuccess) return cuda_fail(e, "task upload");
    *out = (Task*)p;
    return BRKGA_OK;
}

// build buckets for descriptors [d0, d1) (all of one kind)
static int32_t build_buckets(Group& g, int d0, int d1, bool nsga, std::vector<Bucket>* out) {
    std::map<std::pair<int, int>, std::vector<int>> by_tile;
    for (int i = d0; i < d1; ++i) {
        const RowTile t = pick_tile(g.hd[i].n);
        by_tile[{t.block, t.groups}].push_back(i);
    }
    for (auto& kv : by_tile) {
        Bucket b;
        b.tile = RowTile{kv.first.first, kv.first.second};
        int kind = 0;
        for (int i : kv.second) {
            const PopDesc& d = g.hd[i];
            const int pts = (d.kind == BITSP_COORDS) ? d.n + 1 : d.n;
            b.max_n = std::max(b.max_n, d.n);
            b.max_pts = std::max(b.max_pts, pts);
            if (d.kind == BITSP_COORDS) kind = BITSP_COORDS;
            else if (d.kind == TSP_COORDS && kind != BITSP_COORDS) kind = TSP_COORDS;
            else if (kind == 0) kind = d.kind;
        }
        b.kind = kind;
        b.stage = stage_fits(b.tile, b.max_n, b.max_pts, kind);
        const size_t smem = row_smem_bytes(b.tile, b.max_n, b.max_pts, kind, b.stage);
        int per_sm = 0;
        cudaError_t e = prepare_rows(b.tile, smem, &per_sm);
        if (e != cudaSuccess || per_sm <= 0) return fail(BRKGA_ERR_UNSUPPORTED, "row kernel does not fit");
        b.grid = per_sm * device_sm_count();
        // each population's rows stay together: its children, then its elite copies
        std::vector<Task> tg, ta;
        for (int i : kv.second) {
            const PopDesc& d = g.hd[i];
            const int first = nsga ? 0 : d.E;
            for (int r = first; r < d.P; ++r) tg.push_back({i, r});
            for (int r = 0; r < first; ++r) tg.push_back({i, r});
            for (int r = 0; r < d.P; ++r) ta.push_back({i, r});
        }
        int32_t st = upload_tasks(g, tg, &b.d_gen);
        if (st == BRKGA_OK) st = upload_tasks(g, ta, &b.d_all);
        b.nt_gen = (int)tg.size();
        b.nt_all = (int)ta.size();
        if (st != BRKGA_OK) return st;
        out->push_back(b);
    }
    return BRKGA_OK;
}

static RowLaunch bucket_launch(const Group& g, const Bucket& b, int mode, bool all) {
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.descs = g.dd;
    L.mode = mode;
    L.tasks = all ? b.d_all : b.d_gen;
    L.ntasks = all ? b.nt_all : b.nt_gen;
    // groups of consecutive rows per CTA visit, while every CTA keeps work
    L.task_group = std::max(1, std::min(g.task_group, L.ntasks / std::max(1, b.grid)));
    L.max_n = b.max_n;
    L.max_points = b.max_pts;
    L.stage_xy = b.stage ? 1 : 0;
    // rows dealt from the work counter when a CTA takes several at a time (a batch: +8 %
    // on 256 island instances); one row per grab (the server's mix) costs more than it
    // balances (-4 %), so those launches deal statically
    L.work = (L.task_group > 1) ? g.work : nullptr;
    return L;
}

// (re)build descriptors and the launch plan from the members; uploads the descriptors
static int32_t build_plan(Group& g) {
    free_plan(g);
    // descriptor order: single-objective members' islands, then NSGA-II members
    // (migrating instances first: the migration kernel takes their islands as one run)
    auto migrates = [](const Member* m) {
        return !m->sh.mo && m->sh.k > 1 && m->prm.migration_interval > 0 && m->prm.num_migrants > 0;
    };
    std::vector<Member*> order;
    for (Member* m : g.members)
        if (migrates(m)) order.push_back(m);
    for (Member* m : g.members)
        if (!m->sh.mo && !migrates(m)) order.push_back(m);
    for (Member* m : g.members)
        if (m->sh.mo) order.push_back(m);
    g.members = order;
    g.hd.clear();
    g.nb = g.nn = g.maxP_b = g.maxP_n = 0;
    g.any_div = false;
    g.k_mig = g.mig_interval = g.mig_count = g.n_mig_inst = 0;
    for (Member* m : g.members) {
        m->first = (int)g.hd.size();
        m->ndesc = m->sh.k;
        for (int i = 0; i < m->sh.k; ++i) g.hd.push_back(m->pop.hd_template[i]);
        for (int i = 0; i < m->sh.k; ++i) g.hd[m->first + i].gen_limit = m->limit;
        if (m->sh.mo) {
            ++g.nn;
            g.maxP_n = std::max(g.maxP_n, m->sh.Pi);
            g.any_div = g.any_div || m->prm.diversity_interval > 0;
        } else {
            g.nb += m->sh.k;
            g.maxP_b = std::max(g.maxP_b, m->sh.Pi);
            if (m->sh.k > 1 && m->prm.migration_interval > 0 && m->prm.num_migrants > 0) {
                g.k_mig = m->sh.k;
                g.mig_interval = m->prm.migration_interval;
                g.mig_count = m->prm.num_migrants;
                ++g.n_mig_inst;
            }
        }
    }
    const int nd = (int)g.hd.size();
    if (nd > g.cap_desc) {
        if (g.dd) dev_free(g.dd, g.stream);
        int cap = std::max(16, g.cap_desc);
        while (cap < nd) cap *= 2;
        void* p = nullptr;
        int32_t st = dev_alloc(&p, sizeof(PopDesc) * cap, g.stream);
        if (st != BRKGA_OK) return st;
        g.dd = (PopDesc*)p;
        g.cap_desc = cap;
    }
    int32_t st = build_buckets(g, 0, g.nb, false, &g.bb);
    if (st == BRKGA_OK) st = build_buckets(g, g.nb, nd, true, &g.nbk);
    if (st != BRKGA_OK) return st;
    if (g.maxP_b > 0) {
        cudaError_t e = prepare_sort(g.maxP_b);
        if (e != cudaSuccess) return cuda_fail(e, "sort set-up");
    }
    if (g.maxP_n > 0) {
        cudaError_t e = nsga_prepare(g.maxP_n);
        if (e != cudaSuccess) return cuda_fail(e, "NSGA-II set-up");
    }
    if (nd > 0) {
        cudaError_t e = cudaMemcpyAsync(g.dd, g.hd.data(), sizeof(PopDesc) * nd, cudaMemcpyHostToDevice, g.stream);
        if (e != cudaSuccess) return cuda_fail(e, "descriptor upload");
    }
    return BRKGA_OK;
}

// the device descriptors carry the live state (buffer index, generation): read them back
// into the members' templates before a rebuild
static int32_t pull_state(Group& g) {
    const int nd = (int)g.hd.size();
    if (nd == 0) return BRKGA_OK;
    cudaError_t e = cudaStreamSynchronize(g.stream);
    if (e == cudaSuccess) e = cudaMemcpy(g.hd.data(), g.dd, sizeof(PopDesc) * nd, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "descriptor read-back");
    for (Member* m : g.members)
        for (int i = 0; i < m->ndesc; ++i) m->pop.hd_template[i] = g.hd[m->first + i];
    return BRKGA_OK;
}

static cudaError_t enqueue_generation(Group& g, bool mig) {
    cudaError_t e = cudaSuccess;
    for (const Bucket& b : g.bb)
        if ((e = launch_rows(bucket_launch(g, b, MODE_GEN, false), b.kind, b.tile, b.grid, g.stream)) != cudaSuccess)
            return e;
    if (g.nb > 0) {
        if ((e = launch_sort_pops(g.dd, g.nb, g.maxP_b, 1, g.stream)) != cudaSuccess) return e;
        if (mig && g.n_mig_inst > 0) {
            if ((e = launch_migrate(g.dd, g.n_mig_inst, g.k_mig, g.mig_count, 0, g.stream)) != cudaSuccess) return e;
            if ((e = launch_sort_pops(g.dd, g.nb, g.maxP_b, 0, g.stream)) != cudaSuccess) return e;
        }
    }
    if (g.nn > 0) {
        PopDesc* dn = g.dd + g.nb;
        for (const Bucket& b : g.nbk)
            if ((e = launch_rows(bucket_launch(g, b, MODE_NSGA_OFF, false), b.kind, b.tile, b.grid, g.stream)) !=
                cudaSuccess)
                return e;
        // survivors, their rows into the other buffer and the buffer swap
        if ((e = nsga_enqueue_select(dn, g.nn, g.maxP_n, 0, g.stream)) != cudaSuccess) return e;
        if (g.any_div) {
            if ((e = nsga_enqueue_diversity(dn, g.nn, g.maxP_n, g.stream)) != cudaSuccess) return e;
            for (const Bucket& b : g.nbk)
                if ((e = launch_rows(bucket_launch(g, b, MODE_NSGA_REFILL, true), b.kind, b.tile, b.grid, g.stream)) !=
                    cudaSuccess)
                    return e;
            e = nsga_enqueue_select(dn, g.nn, g.maxP_n, 2, g.stream);
        }
    }
    return e;
}

static cudaError_t capture_group(Group& g, int gens, bool mig, cudaGraphExec_t* out) {
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < gens && e == cudaSuccess; ++i) e = enqueue_generation(g, mig && i == gens - 1);
    cudaError_t end = cudaStreamEndCapture(g.stream, &gr);
    if (e != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        return e;
    }
    if (end != cudaSuccess) return end;
    e = cudaGraphInstantiate(out, gr, 0);
    cudaGraphDestroy(gr);
    return e;
}

// advance every member by `gens` generations; migration generations are host-known
// because the batch advances in lockstep from generation `gen0`
// advance every member by `gens` generations (graph replay when use_graphs)
static cudaError_t run_generations(Group& g, uint32_t gen0, int gens, bool use_graphs) {
    cudaError_t e = cudaSuccess;
    uint32_t gen = gen0;
    int left = gens;
    const int chunk = 16;
    while (left > 0 && e == cudaSuccess) {
        int plain = left;
        if (g.n_mig_inst > 0 && g.mig_interval > 0) {
            const uint32_t iv = (uint32_t)g.mig_interval;
            const uint32_t next = (gen / iv + 1) * iv;
            plain = std::min<int>(left, (int)(next - gen - 1));
        }
        while (plain > 0 && e == cudaSuccess) {
            const int step = (use_graphs && plain >= chunk) ? chunk : 1;
            if (use_graphs) {
                cudaGraphExec_t* gx = (step == chunk) ? &g.gx_chunk : &g.gx_one;
                if (!*gx) e = capture_group(g, step, false, gx);
                if (e == cudaSuccess) e = cudaGraphLaunch(*gx, g.stream);
            } else {
                e = enqueue_generation(g, false);
            }
            plain -= step;
            left -= step;
            gen += step;
        }
        if (left > 0 && e == cudaSuccess) {
            const bool mig = g.n_mig_inst > 0 && g.mig_interval > 0 && (gen + 1) % (uint32_t)g.mig_interval == 0;
            if (use_graphs) {
                cudaGraphExec_t* gx = mig ? &g.gx_mig : &g.gx_one;
                if (!*gx) e = capture_group(g, 1, mig, gx);
                if (e == cudaSuccess) e = cudaGraphLaunch(*gx, g.stream);
            } else {
                e = enqueue_generation(g, mig);
            }
            --left;
            ++gen;
        }
    }
    return e;
}

// allocate a member's buffers and descriptor templates (islands), ordered on `stream`
static int32_t make_member(std::shared_ptr<ProblemData> pd, const brkga_params& prm, cudaStream_t stream,
                           Member** out) {
    Shape sh;
    int32_t st = make_shape(*pd, prm, &sh);
    if (st != BRKGA_OK) return st;
    if (pd->kind == BRKGA_TSPJ && prm.local_search_interval > 0)
        return fail(BRKGA_ERR_UNSUPPORTED, "local search runs in brkga_create engines, not in batches or the server");
    if (pd->kind == BRKGA_MOVRP)
        return fail(BRKGA_ERR_UNSUPPORTED, "MO-VRP runs in brkga_create engines, not in batches or the server");
    if (pd->kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "external-fitness problems run in brkga_create engines");
    if (row_needs_global(pd->n, points_of(*pd), pd->kind))
        return fail(BRKGA_ERR_UNSUPPORTED, "batched and served rows must fit the shared-memory row kernel (n = " +
                                               std::to_string(pd->n) + " does not); solve it with brkga_create");
    auto* m = new Member;
    m->pd = pd;
    m->prm = prm;
    m->sh = sh;
    m->pop.pd = pd;
    m->pop.prm = prm;
    m->pop.sh = sh;
    m->pop.stream = stream;
    if ((st = m->pop.allocate(pd->device)) != BRKGA_OK) {
        m->pop.release(pd->device);
        delete m;
        return st;
    }
    m->pop.hd_template.resize(sh.k);
    for (int i = 0; i < sh.k; ++i) {
        PopDesc& d = m->pop.hd_template[i];
        fill_instance(d, *pd);
        d.P = sh.Pi;
        d.E = sh.Ei;
        d.M = sh.Mi;
        d.rhoT = prob_threshold(prm.elite_prob);
        d.seed = prm.seed;
        d.island = (uint32_t)i;
        for (int b = 0; b < 2; ++b) {
            d.keys[b] = m->pop.keys[b] + (size_t)i * sh.Pi * sh.ld;
            d.fit[b] = m->pop.fit[b] + (size_t)i * sh.Pi * sh.m;
        }
        d.sorted = m->pop.sorted + (size_t)i * sh.Pi;
        d.parents = sh.mo ? nullptr : m->pop.parents + (size_t)i * sh.Pi;
        d.done = m->pop.done + i;
        d.history = m->pop.history + (size_t)i * m->pop.hist_cap;
        d.hist_cap = m->pop.hist_cap;
    }
    if (sh.mo) {
        const double rate = (prm.mutation_rate > 0.0) ? prm.mutation_rate : 5.0 / (double)sh.n;
        st = nsga_alloc(m->pop.hd_template[0], sh.Pi, rate, prm.diversity_interval, sh.Mn, m->pop.allocs,
                        &m->pop.bytes, stream);
        if (st != BRKGA_OK) {
            m->pop.release(pd->device);
            delete m;
            return st;
        }
    }
    *out = m;
    return BRKGA_OK;
}

// initialise members [from, to) of the group's member list (their descriptors must be
// uploaded): keys of generation 0, fitness, rank order / NSGA-II ranks
static cudaError_t init_members(Group& g, const std::vector<Member*>& ms) {
    cudaError_t e = cudaSuccess;
    for (Member* m : ms) {
        const RowTile t = pick_tile(m->sh.n);
        const int pts = points_of(*m->pd);
        const bool stage = stage_fits(t, m->sh.n, pts, m->pd->kind);
        int per_sm = 0;
        if ((e = prepare_rows(t, row_smem_bytes(t, m->sh.n, pts, m->pd->kind, stage), &per_sm)) != cudaSuccess)
            return e;
        for (int i = 0; i < m->ndesc; ++i) {
            RowLaunch L;
            std::memset(&L, 0, sizeof(L));
            L.descs = g.dd + m->first + i;
            L.mode = MODE_INIT;
            L.ntasks = m->sh.Pi;
            L.max_n = m->sh.n;
            L.max_points = pts;
            L.stage_xy = stage ? 1 : 0;
            if ((e = launch_rows(L, m->pd->kind, t, per_sm * device_sm_count(), g.stream)) != cudaSuccess) return e;
        }
        if (m->sh.mo) {
            if ((e = nsga_prepare(m->sh.Pi)) != cudaSuccess) return e;
            e = nsga_enqueue_select(g.dd + m->first, 1, m->sh.Pi, 1, g.stream);
        } else {
            if ((e = prepare_sort(m->sh.Pi)) != cudaSuccess) return e;
            e = launch_sort_pops(g.dd + m->first, m->ndesc, m->sh.Pi, 0, g.stream);
        }
        if (e != cudaSuccess) return e;
    }
    return e;
}

// best objective values of a member from its descriptors (host copies current)
static int32_t member_best(Group& g, Member* m, float* best2) {
    const bool mx = m->pd->maximize != 0;
    best2[0] = best2[1] = NAN;
    if (m->sh.mo) {
        const PopDesc& d = g.hd[m->first];
        const int P = m->sh.Pi;
        std::vector<int32_t> r(P);
        std::vector<float> c(P), o((size_t)P * 2);
        cudaMemcpy(r.data(), d.nrank, (size_t)P * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(c.data(), d.ncd, (size_t)P * 4, cudaMemcpyDeviceToHost);
        cudaError_t e = cudaMemcpy(o.data(), d.fit[d.cur], o.size() * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "best read-back");
        int b = -1;
        for (int i = 0; i < P; ++i)
            if (r[i] == 0 && (b < 0 || c[i] > c[b])) b = i;
        if (b < 0) b = 0;
        best2[0] = o[2 * b];
        best2[1] = o[2 * b + 1];
        return BRKGA_OK;
    }
    for (int i = 0; i < m->ndesc; ++i) {
        const PopDesc& d = g.hd[m->first + i];
        int32_t r0 = 0;
        float f0 = 0.0f;
        cudaMemcpy(&r0, d.sorted, 4, cudaMemcpyDeviceToHost);
        cudaError_t e = cudaMemcpy(&f0, d.fit[d.cur] + (size_t)r0 * d.m, 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "best read-back");
        if (i == 0 || (mx ? f0 > best2[0] : f0 < best2[0])) best2[0] = f0;
    }
    return BRKGA_OK;
}

// best-so-far of every population (its history entry for the current generation)
__global__ void best_gather_kernel(const PopDesc* dd, int nd, float* out, uint32_t* gens) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nd) {
        const PopDesc& d = dd[i];
        const int g = min((int)d.gen, d.hist_cap - 1);
        out[i] = d.history ? d.history[g] : 0.0f;
        gens[i] = d.gen;
    }
}

static void release_member(Member* m, cudaStream_t st) {
    m->pop.stream = st;
    m->pop.release(m->pd->device);
    delete m;
}

}  // namespace bk

using namespace bk;

// ---------------------------------------------------------------------------------------
// batch API
// ---------------------------------------------------------------------------------------
struct brkga_batch {
    std::mutex mu;
    Group g;
    uint32_t gen = 0;
};

extern "C" {

int32_t brkga_batch_create(brkga_problem* const* problems, const brkga_params* params, int32_t count,
                           brkga_batch** out) {
    if (!problems || !params || !out || count <= 0) return fail(BRKGA_ERR_INVALID, "need problems, params, count > 0");
    *out = nullptr;
    const int dev = params[0].device;
    DeviceGuard guard(dev);
    if (!guard.ok()) return fail(BRKGA_ERR_CUDA, "cannot select device");
    int mig_k = -1, mig_iv = -1, mig_n = -1;
    for (int i = 0; i < count; ++i) {
        if (!problems[i]) return fail(BRKGA_ERR_INVALID, "null problem in batch");
        auto pd = problem_data(problems[i]);
        if (pd->device != dev || params[i].device != dev) return fail(BRKGA_ERR_INVALID, "batch spans devices");
        if (pd->m == 1 && params[i].num_islands > 1 && params[i].migration_interval > 0) {
            if (mig_k >= 0 && (mig_k != params[i].num_islands || mig_iv != params[i].migration_interval ||
                               mig_n != params[i].num_migrants))
                return fail(BRKGA_ERR_UNSUPPORTED, "islands / migration settings must agree across a batch");
            mig_k = params[i].num_islands;
            mig_iv = params[i].migration_interval;
            mig_n = params[i].num_migrants;
        }
    }
    auto* b = new brkga_batch;
    b->g.device = dev;
    b->g.task_group = 8;
    int32_t st = group_start(b->g);
    if (st != BRKGA_OK) {
        brkga_batch_destroy(b);
        return st;
    }
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < count && st == BRKGA_OK; ++i) {
        Member* m = nullptr;
        st = make_member(problem_data(problems[i]), params[i], b->g.stream, &m);
        if (st == BRKGA_OK) {
            m->prm_index = i;
            b->g.members.push_back(m);
        }
    }
    if (st == BRKGA_OK) st = build_plan(b->g);
    if (st == BRKGA_OK) {
        std::vector<Member*> ms = b->g.members;
        e = init_members(b->g, ms);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->g.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "batch initialisation");
    }
    if (st != BRKGA_OK) {
        brkga_batch_destroy(b);
        return st;
    }
    *out = b;
    return BRKGA_OK;
}

int32_t brkga_batch_destroy(brkga_batch* b) {
    if (!b) return BRKGA_OK;
    DeviceGuard guard(b->g.device);
    cudaStreamSynchronize(b->g.stream);
    free_plan(b->g);
    for (Member* m : b->g.members) release_member(m, b->g.stream);
    if (b->g.dd) dev_free(b->g.dd, b->g.stream);
    group_stop(b->g);
    delete b;
    return BRKGA_OK;
}

int32_t brkga_batch_evolve(brkga_batch* b, int32_t generations) {
    if (!b || generations < 0) return fail(BRKGA_ERR_INVALID, "bad arguments");
    std::lock_guard<std::mutex> lk(b->mu);
    DeviceGuard guard(b->g.device);
    // history capacity: every member was sized for its max_generations
    for (Member* m : b->g.members)
        if ((int)b->gen + generations + 1 > m->pop.hist_cap)
            return fail(BRKGA_ERR_INVALID, "batch evolved past a member's max_generations");
    NvtxRange range("batch generations", b->gen + 1u, b->gen + (unsigned)generations);
    cudaError_t e = run_generations(b->g, b->gen, generations, true);
    if (e != cudaSuccess) return cuda_fail(e, "batch evolve");
    b->gen += generations;
    return BRKGA_OK;
}

int32_t brkga_batch_synchronize(brkga_batch* b) {
    if (!b) return fail(BRKGA_ERR_INVALID, "null batch");
    DeviceGuard guard(b->g.device);
    cudaError_t e = cudaStreamSynchronize(b->g.stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch stream");
    return BRKGA_OK;
}

int32_t brkga_batch_get_best(brkga_batch* b, float* best) {
    if (!b || !best) return fail(BRKGA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    DeviceGuard guard(b->g.device);
    int32_t st = pull_state(b->g);
    if (st != BRKGA_OK) return st;
    // members are stored single-objective first; report in creation order
    for (size_t i = 0; i < b->g.members.size(); ++i) {
        Member* m = b->g.members[i];
        float v[2];
        if ((st = member_best(b->g, m, v)) != BRKGA_OK) return st;
        best[2 * m->prm_index + 0] = v[0];
        best[2 * m->prm_index + 1] = v[1];
    }
    return BRKGA_OK;
}

int32_t brkga_batch_get_best_keys(brkga_batch* b, int32_t index, float* keys, float* fitness) {
    if (!b || index < 0) return fail(BRKGA_ERR_INVALID, "bad arguments");
    std::lock_guard<std::mutex> lk(b->mu);
    DeviceGuard guard(b->g.device);
    int32_t st = pull_state(b->g);
    if (st != BRKGA_OK) return st;
    Member* m = nullptr;
    for (Member* x : b->g.members)
        if (x->prm_index == index) m = x;
    if (!m) return fail(BRKGA_ERR_INVALID, "index out of range");
    float v[2];
    if ((st = member_best(b->g, m, v)) != BRKGA_OK) return st;
    if (fitness) {
        fitness[0] = v[0];
        if (m->sh.m > 1) fitness[1] = v[1];
    }
    if (keys && !m->sh.mo) {
        const bool mx = m->pd->maximize != 0;
        int bi = 0;
        float bf = 0.0f;
        int32_t br = 0;
        for (int i = 0; i < m->ndesc; ++i) {
            const PopDesc& d = b->g.hd[m->first + i];
            int32_t r0 = 0;
            float f0 = 0.0f;
            cudaMemcpy(&r0, d.sorted, 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(&f0, d.fit[d.cur] + (size_t)r0 * d.m, 4, cudaMemcpyDeviceToHost);
            if (i == 0 || (mx ? f0 > bf : f0 < bf)) {
                bi = i;
                bf = f0;
                br = r0;
            }
        }
        const PopDesc& d = b->g.hd[m->first + bi];
        cudaError_t e = cudaMemcpy(keys, d.keys[d.cur] + (size_t)br * d.ld, (size_t)d.n * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "keys read-back");
    }
    return BRKGA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// serving: continuous batching of solve requests
// ---------------------------------------------------------------------------------------
namespace {

enum ReqState { REQ_QUEUED = 0, REQ_ACTIVE = 1, REQ_DONE = 2, REQ_CANCELLED = 3, REQ_FAILED = 4 };

struct Request {
    int64_t id = 0;
    brkga_problem_desc desc{};
    std::vector<float> coords, coords2, matrix, matrix2;
    std::vector<int32_t> weights, values;
    brkga_params prm{};
    int stall = 0;
    std::chrono::steady_clock::time_point t_submit;
    int state = REQ_QUEUED;
    Member* m = nullptr;
    size_t bytes = 0;
    float best[2] = {NAN, NAN};
    float last = NAN;
    int since = 0;
    int gens = 0;
    double latency = 0.0;
    int err = BRKGA_OK;
};

size_t estimate_bytes(const brkga_problem_desc& d, const brkga_params& p) {
    const size_t n = (size_t)std::max(1, d.n);
    const size_t genes = (d.kind == BRKGA_TSPJ) ? 2 * n : n, ld = (genes + 3) / 4 * 4;
    const bool mo = d.kind == BRKGA_BITSP_COORDS || d.kind == BRKGA_BITSP_MATRIX;
    const size_t P = (size_t)std::max(1, p.population_size);
    const size_t rows = mo ? 2 * P : P;
    const size_t m = mo ? 2 : 1;
    size_t b = 2 * rows * ld * 4 + 2 * rows * m * 4 + rows * 4 + rows * 8 + 64 + (size_t)(p.max_generations + 2) * 4 * 4;
    if (mo) b += rows * 4 * 4 + rows * ((rows + 31) / 32) * 4 + 64;
    switch (d.kind) {
    case BRKGA_TSP_COORDS: b += n * 8; break;
    case BRKGA_TSP_MATRIX: b += n * n * 4; break;
    case BRKGA_BITSP_COORDS: b += 2 * (n + 1) * 8; break;
    case BRKGA_BITSP_MATRIX: b += 2 * (n + 1) * (n + 1) * 4; break;
    case BRKGA_TSPJ: b += 2 * (n + 1) * (n + 1) * 4; break;
    case BRKGA_KNAP_THRESHOLD:
    case BRKGA_KNAP_GREEDY: b += n * 16; break;  // weights, values and the (weight, value) pairs
    default: b += n * 8;
    }
    return b + 4096;
}

}  // namespace

struct brkga_server {
    std::mutex mu;
    brkga_server_config cfg{};
    Group g;
    std::deque<Request*> queue;
    std::unordered_map<int64_t, Request*> all;
    std::vector<Request*> active;
    int64_t next_id = 1;
    size_t budget = 0, in_use = 0;
    float* d_best = nullptr;
    uint32_t* d_gens = nullptr;
    int cap_best = 0;
    int finished = 0;
};

static int32_t server_copy_desc(Request* r, const brkga_problem_desc* d) {
    r->desc = *d;
    const size_t n = (size_t)std::max(1, d->n);
    auto cp_f = [](const float* src, size_t cnt, std::vector<float>& dst) -> const float* {
        if (!src) return nullptr;
        dst.assign(src, src + cnt);
        return dst.data();
    };
    auto cp_i = [](const int32_t* src, size_t cnt, std::vector<int32_t>& dst) -> const int32_t* {
        if (!src) return nullptr;
        dst.assign(src, src + cnt);
        return dst.data();
    };
    switch (d->kind) {
    case BRKGA_TSP_COORDS: r->desc.coords = cp_f(d->coords, n * 2, r->coords); break;
    case BRKGA_TSP_MATRIX: r->desc.matrix = cp_f(d->matrix, n * n, r->matrix); break;
    case BRKGA_BITSP_COORDS:
        r->desc.coords = cp_f(d->coords, (n + 1) * 2, r->coords);
        r->desc.coords2 = cp_f(d->coords2, (n + 1) * 2, r->coords2);
        break;
    case BRKGA_BITSP_MATRIX:
        r->desc.matrix = cp_f(d->matrix, (n + 1) * (n + 1), r->matrix);
        r->desc.matrix2 = cp_f(d->matrix2, (n + 1) * (n + 1), r->matrix2);
        break;
    case BRKGA_KNAP_THRESHOLD:
    case BRKGA_KNAP_GREEDY:
        r->desc.weights = cp_i(d->weights, n, r->weights);
        r->desc.values = cp_i(d->values, n, r->values);
        break;
    case BRKGA_TSPJ:
        r->desc.matrix = cp_f(d->matrix, (n + 1) * (n + 1), r->matrix);
        r->desc.matrix2 = cp_f(d->matrix2, (n + 1) * (n + 1), r->matrix2);
        break;
    case BRKGA_JOBSCHED: r->desc.job_times = cp_f(d->job_times, n, r->coords); break;
    case BRKGA_CONTINUOUS: break;
    default: return fail(BRKGA_ERR_INVALID, "unknown problem kind");
    }
    return BRKGA_OK;
}

static void server_retire(brkga_server* s, Request* r, int state) {
    if (r->m) {
        float v[2];
        if (member_best(s->g, r->m, v) == BRKGA_OK) {
            r->best[0] = v[0];
            r->best[1] = v[1];
        }
        release_member(r->m, s->g.stream);
        r->m = nullptr;
    }
    s->in_use -= r->bytes;
    r->state = state;
    r->latency = std::chrono::duration<double>(std::chrono::steady_clock::now() - r->t_submit).count();
    ++s->finished;
    // the problem data can go now
    r->coords.clear();
    r->coords2.clear();
    r->matrix.clear();
    r->matrix2.clear();
    r->weights.clear();
    r->values.clear();
}

extern "C" {

int32_t brkga_server_create(const brkga_server_config* cfg, brkga_server** out) {
    if (!cfg || !out) return fail(BRKGA_ERR_INVALID, "null argument");
    if (cfg->max_active <= 0 || cfg->generations_per_tick <= 0)
        return fail(BRKGA_ERR_INVALID, "need max_active > 0 and generations_per_tick > 0");
    DeviceGuard guard(cfg->device);
    if (!guard.ok()) return fail(BRKGA_ERR_CUDA, "cannot select device");
    auto* s = new brkga_server;
    s->cfg = *cfg;
    s->g.device = cfg->device;
    int32_t st = group_start(s->g);
    if (st != BRKGA_OK) {
        brkga_server_destroy(s);
        return st;
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->budget = cfg->memory_budget > 0 ? (size_t)cfg->memory_budget : (size_t)(0.8 * (double)fr);
    *out = s;
    return BRKGA_OK;
}

int32_t brkga_server_destroy(brkga_server* s) {
    if (!s) return BRKGA_OK;
    DeviceGuard guard(s->g.device);
    cudaStreamSynchronize(s->g.stream);
    free_plan(s->g);
    for (Request* r : s->active)
        if (r->m) release_member(r->m, s->g.stream);
    for (auto& kv : s->all) delete kv.second;
    if (s->g.dd) dev_free(s->g.dd, s->g.stream);
    if (s->d_best) dev_free(s->d_best, s->g.stream);
    if (s->d_gens) dev_free(s->d_gens, s->g.stream);
    group_stop(s->g);
    delete s;
    return BRKGA_OK;
}

int32_t brkga_server_submit(brkga_server* s, const brkga_problem_desc* desc, const brkga_params* params,
                            int32_t stall_generations, int64_t* request_id) {
    if (!s || !desc || !params || !request_id) return fail(BRKGA_ERR_INVALID, "null argument");
    if (params->max_generations <= 0) return fail(BRKGA_ERR_INVALID, "max_generations must be > 0");
    if (params->num_islands > 1) return fail(BRKGA_ERR_UNSUPPORTED, "served requests run one population each");
    if (desc->kind == BRKGA_MOVRP)
        return fail(BRKGA_ERR_UNSUPPORTED, "MO-VRP runs in brkga_create engines, not in batches or the server");
    if (desc->kind == BRKGA_EXTERNAL)
        return fail(BRKGA_ERR_UNSUPPORTED, "external-fitness problems run in brkga_create engines");
    const long long genes = (desc->kind == BRKGA_TSPJ) ? 2ll * desc->n : (long long)desc->n;
    if (desc->n < 1 || genes > row_max_n()) return fail(BRKGA_ERR_UNSUPPORTED, "chromosome length out of range");
    {
        const int pts = (desc->kind == BRKGA_BITSP_COORDS) ? desc->n + 1 : (int)genes;
        if (row_needs_global((int)genes, pts, desc->kind))
            return fail(BRKGA_ERR_UNSUPPORTED, "served rows must fit the shared-memory row kernel (" +
                                                   std::to_string(genes) + " genes do not)");
    }
    auto* r = new Request;
    int32_t st = server_copy_desc(r, desc);
    if (st != BRKGA_OK) {
        delete r;
        return st;
    }
    r->prm = *params;
    r->prm.device = s->cfg.device;
    r->stall = stall_generations;
    r->bytes = estimate_bytes(*desc, *params);
    r->t_submit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->bytes > s->budget) {
        delete r;
        return fail(BRKGA_ERR_BUSY, "request larger than the server's memory budget");
    }
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->queue.push_back(r);
    *request_id = r->id;
    return BRKGA_OK;
}

int32_t brkga_server_step(brkga_server* s) {
    if (!s) return fail(BRKGA_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    DeviceGuard guard(s->g.device);
    Group& g = s->g;
    const int tick = s->cfg.generations_per_tick;
    cudaError_t e;
    int32_t st;
    // 1. advance every active request by one tick (each stops at its own budget)
    if (!s->active.empty()) {
        NvtxRange range("server tick");
        // membership changes often, so the tick launches directly instead of capturing
        e = run_generations(g, 0, tick, false);
        if (e != cudaSuccess) return cuda_fail(e, "server tick");
        const int nd = (int)g.hd.size();
        if (nd > s->cap_best) {
            if (s->d_best) dev_free(s->d_best, g.stream);
            if (s->d_gens) dev_free(s->d_gens, g.stream);
            s->cap_best = std::max(64, 2 * nd);
            if ((st = dev_alloc((void**)&s->d_best, (size_t)s->cap_best * 4, g.stream)) != BRKGA_OK) return st;
            if ((st = dev_alloc((void**)&s->d_gens, (size_t)s->cap_best * 4, g.stream)) != BRKGA_OK) return st;
        }
        best_gather_kernel<<<(nd + 127) / 128, 128, 0, g.stream>>>(g.dd, nd, s->d_best, s->d_gens);
        std::vector<float> hb(nd);
        std::vector<uint32_t> hg(nd);
        e = cudaMemcpyAsync(hb.data(), s->d_best, (size_t)nd * 4, cudaMemcpyDeviceToHost, g.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hg.data(), s->d_gens, (size_t)nd * 4, cudaMemcpyDeviceToHost, g.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
        if (e != cudaSuccess) return cuda_fail(e, "server progress read-back");
        // 2. retire requests at their budget, or stalled
        std::vector<Request*> keep;
        bool changed = false;
        if ((st = pull_state(g)) != BRKGA_OK) return st;
        for (Request* r : s->active) {
            Member* m = r->m;
            const bool mx = m->pd->maximize != 0;
            float b = hb[m->first];
            for (int i = 1; i < m->ndesc; ++i) b = mx ? std::max(b, hb[m->first + i]) : std::min(b, hb[m->first + i]);
            const int gens = (int)hg[m->first];
            const bool improved = std::isnan(r->last) || (mx ? b > r->last : b < r->last);
            r->since = improved ? 0 : r->since + tick;
            r->last = b;
            r->gens = gens;
            if (gens >= r->prm.max_generations || (r->stall > 0 && r->since >= r->stall)) {
                server_retire(s, r, REQ_DONE);
                changed = true;
            } else {
                keep.push_back(r);
            }
        }
        s->active.swap(keep);
        if (changed) {
            g.members.clear();
            for (Request* r : s->active) g.members.push_back(r->m);
        }
        if (changed && (st = build_plan(g)) != BRKGA_OK) return st;
    }
    // 3. admit queued requests while slots and memory allow.  Besides the server's own
    // budget, each admission round re-reads the device's free memory (other processes and
    // engines come and go) plus what the library's pool holds unused, and keeps a reserve
    // of 1/64 of the device free.
    std::vector<Member*> fresh;
    size_t avail = 0;
    if (!s->queue.empty() && (int)s->active.size() < s->cfg.max_active) {
        size_t fr = 0, tot = 0;
        if ((e = cudaMemGetInfo(&fr, &tot)) != cudaSuccess) return cuda_fail(e, "free memory");
        const size_t spare = pool_spare(s->cfg.device), reserve = tot / 64;
        avail = (fr + spare > reserve) ? fr + spare - reserve : 0;
    }
    while (!s->queue.empty() && (int)s->active.size() < s->cfg.max_active) {
        Request* r = s->queue.front();
        if (s->in_use + r->bytes > s->budget) break;
        if (r->bytes > avail) break;
        avail -= r->bytes;
        s->queue.pop_front();
        std::shared_ptr<ProblemData> pd;
        Member* m = nullptr;
        st = make_problem(&r->desc, s->cfg.device, &pd);
        if (st == BRKGA_OK) st = make_member(pd, r->prm, g.stream, &m);
        if (st != BRKGA_OK) {
            r->err = st;
            r->state = REQ_FAILED;
            r->latency = std::chrono::duration<double>(std::chrono::steady_clock::now() - r->t_submit).count();
            ++s->finished;
            continue;
        }
        m->limit = (uint32_t)r->prm.max_generations;
        r->m = m;
        r->state = REQ_ACTIVE;
        s->in_use += r->bytes;
        s->active.push_back(r);
        fresh.push_back(m);
    }
    if (!fresh.empty()) {
        if ((st = pull_state(g)) != BRKGA_OK) return st;
        g.members.clear();
        for (Request* r : s->active) g.members.push_back(r->m);
        if ((st = build_plan(g)) != BRKGA_OK) return st;
        e = init_members(g, fresh);
        if (e != cudaSuccess) return cuda_fail(e, "request initialisation");
    }
    return BRKGA_OK;
}

int32_t brkga_server_poll(brkga_server* s, int64_t request_id, float* best, int32_t* generations, double* latency_s) {
    if (!s) return fail(BRKGA_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail(BRKGA_ERR_INVALID, "unknown request id");
    Request* r = it->second;
    if (r->state == REQ_QUEUED || r->state == REQ_ACTIVE) return BRKGA_ERR_NOT_READY;
    if (best) {
        best[0] = r->best[0];
        best[1] = r->best[1];
    }
    if (generations) *generations = r->gens;
    if (latency_s) *latency_s = r->latency;
    if (r->state == REQ_CANCELLED) return BRKGA_ERR_CANCELLED;
    if (r->state == REQ_FAILED) return r->err;
    return BRKGA_OK;
}

int32_t brkga_server_cancel(brkga_server* s, int64_t request_id) {
    if (!s) return fail(BRKGA_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    DeviceGuard guard(s->g.device);
    auto it = s->all.find(request_id);
    if (it == s->all.end()) return fail(BRKGA_ERR_INVALID, "unknown request id");
    Request* r = it->second;
    if (r->state == REQ_QUEUED) {
        s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
        r->state = REQ_CANCELLED;
        r->latency = std::chrono::duration<double>(std::chrono::steady_clock::now() - r->t_submit).count();
        ++s->finished;
    } else if (r->state == REQ_ACTIVE) {
        int32_t st = pull_state(s->g);
        if (st != BRKGA_OK) return st;
        server_retire(s, r, REQ_CANCELLED);
        s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
        s->g.members.clear();
        for (Request* q : s->active) s->g.members.push_back(q->m);
        if ((st = build_plan(s->g)) != BRKGA_OK) return st;
    }
    return BRKGA_OK;
}

int32_t brkga_server_stats(brkga_server* s, int32_t* queued, int32_t* active, int32_t* finished) {
    if (!s) return fail(BRKGA_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int32_t)s->queue.size();
    if (active) *active = (int32_t)s->active.size();
    if (finished) *finished = s->finished;
    return BRKGA_OK;
}

}  // extern "C"
