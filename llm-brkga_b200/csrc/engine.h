// engine.h -- host-side pieces shared by the C-ABI translation units.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/brkga_b200.h"
#include "kernels.h"

namespace bk {

constexpr size_t kMaxSmem = 227 * 1024;  // opt-in dynamic shared memory per CTA on sm_100
constexpr int kMaxPop = 16384;           // largest population the in-shared-memory sort handles

int32_t fail(int32_t code, const std::string& msg);
// stream-ordered device memory from the library's pool (memory.cu)
int32_t dev_alloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);
size_t pool_reserved(int dev);
size_t pool_spare(int dev);
int32_t cuda_fail(cudaError_t e, const char* what);

// An NVTX range around a stretch of host work (named like "generations 17-32").  With no
// profiler attached NVTX calls return at once; under Nsight Systems the ranges line up with
// the CUDA graphs each stretch launches.
class NvtxRange {
   public:
    NvtxRange(const char* what, unsigned first, unsigned last) {
        char buf[80];
        snprintf(buf, sizeof buf, "%s %u-%u", what, first, last);
        nvtxRangePushA(buf);
    }
    explicit NvtxRange(const char* what) { nvtxRangePushA(what); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

class DeviceGuard {
public:
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
    bool ok() const { return ok_; }

private:
    int prev_ = 0;
    bool ok_ = false;
};

// device-resident instance data (the reference's per-device matrix map,
// configs/tsp_config.hpp:32, 125-165), shared by every engine built on it
struct ProblemData {
    int device = 0;
    int kind = 0, n = 0, m = 1, maximize = 0;
    float cap = 0.0f;
    long long capi = 0;
    float* xy = nullptr;
    float* xy2 = nullptr;
    float* mat = nullptr;
    float* mat2 = nullptr;
    int32_t* w = nullptr;
    int32_t* v = nullptr;
    int2* wv = nullptr;      // knapsack: (weight, value) interleaved, one load per item
    float* jt = nullptr;     // job scheduling: job times
    int machines = 0;
    int function = 0;        // continuous: brkga_function, bounds
    float lo = 0.0f, hi = 0.0f;
    size_t bytes = 0;
    std::vector<void*> allocs;
    ~ProblemData();
};

int32_t make_problem(const brkga_problem_desc* d, int device, std::shared_ptr<ProblemData>* out);
std::shared_ptr<ProblemData> problem_data(brkga_problem* pb);
void fill_instance(PopDesc& d, const ProblemData& pd);
int points_of(const ProblemData& pd);
bool stage_fits(const RowTile& t, int n, int pts, int kind);
uint32_t prob_threshold(double p);

// Tile autotuner: times every candidate tile (capacity covering n) on `launch`, which
// must enqueue one representative row-kernel launch for the tile and grid it is given on
// `stream`; returns the fastest with its grid.  Results are cached per (kind, n, rows) in
// the process and, when BRKGA_TUNE_CACHE names a file, persisted there.  BRKGA_TILE=
// "block,groups" forces a tile.
struct TunedTile {
    RowTile tile{};
    int grid = 0;
    bool stage = false;
};
template <typename F>
int32_t autotune_tile(int kind, int n, int pts, int rows, cudaStream_t stream, F&& launch, TunedTile* out);
int32_t tune_lookup(int kind, int n, int rows, RowTile* t);
void tune_store(int kind, int n, int rows, const RowTile& t);
int32_t tile_setup(const RowTile& t, int kind, int n, int pts, TunedTile* out);

// validated, per-island GA shape
struct Shape {
    int k = 1;        // islands
    int Pi = 0, Ei = 0, Mi = 0;
    int n = 0, ld = 0, m = 1;
    bool mo = false;  // NSGA-II
    int Mn = 0;       // NSGA-II fresh random offspring
};
int32_t make_shape(const ProblemData& pd, const brkga_params& p, Shape* s);

// one population family (all islands of one instance) on the device
struct Population {
    std::shared_ptr<ProblemData> pd;
    brkga_params prm{};
    Shape sh;
    uint64_t seed = 0;
    int rows = 0;           // rows per key buffer (k * Pi, or 2P pool for NSGA-II)
    float* keys[2] = {nullptr, nullptr};
    float* fit[2] = {nullptr, nullptr};
    int32_t* sorted = nullptr;
    int2* parents = nullptr;   // next generation's parent ranks per child row
    int32_t* done = nullptr;   // rank-kernel completion counters, one per island
    float* history = nullptr;
    int hist_cap = 0;
    // NSGA-II state
    int32_t* rank = nullptr;   // [2P] pool ranks, then survivors' ranks in [0,P)
    float* cd = nullptr;       // [2P]
    int32_t* sel = nullptr;    // [P]
    float* nsga_hist = nullptr;
    std::vector<void*> allocs;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;  // allocations are ordered on the owner's stream
    std::vector<PopDesc> hd_template;  // descriptors (live state copied back before plan rebuilds)
    int32_t allocate(int device);
    void release(int device);
};

template <typename F>
int32_t autotune_tile(int kind, int n, int pts, int rows, cudaStream_t stream, F&& launch, TunedTile* out) {
    RowTile forced{};
    if (tune_lookup(kind, n, rows, &forced) == BRKGA_OK) return tile_setup(forced, kind, n, pts, out);
    RowTile cand[16];
    const int nc = tile_candidates(n, cand, 16);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    // each candidate: one warm-up, then the best of three separately timed launches; the
    // default tile (smallest that covers n) is kept unless another is 5% faster
    const RowTile def = pick_tile(n);
    float best_ms = 1e30f, def_ms = 1e30f;
    TunedTile best, deft;
    for (int c = 0; c < nc; ++c) {
        TunedTile tt;
        if (tile_setup(cand[c], kind, n, pts, &tt) != BRKGA_OK) continue;
        if (launch(tt) != cudaSuccess) continue;  // warm-up
        float ms = 1e30f;
        for (int r = 0; r < 3; ++r) {
            cudaEventRecord(a, stream);
            launch(tt);
            cudaEventRecord(b, stream);
            if (cudaEventSynchronize(b) != cudaSuccess) break;
            float x = 0.0f;
            cudaEventElapsedTime(&x, a, b);
            ms = x < ms ? x : ms;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = tt;
        }
        if (cand[c].block == def.block && cand[c].groups == def.groups) {
            def_ms = ms;
            deft = tt;
        }
    }
    if (deft.grid > 0 && best_ms > 0.95f * def_ms) best = deft;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaGetLastError();
    if (best.grid <= 0) return fail(BRKGA_ERR_UNSUPPORTED, "no row-kernel tile fits this size");
    tune_store(kind, n, rows, best.tile);
    *out = best;
    return BRKGA_OK;
}

}  // namespace bk
