// kernels.h -- host-side launch interface of the engine's CUDA kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace bk {

enum Mode : int32_t {
    MODE_INIT = 0,
    MODE_GEN = 1,
    MODE_EVAL = 2,
    MODE_NSGA_OFF = 3,
    MODE_NSGA_REFILL = 4,
    MODE_LSEARCH = 5,  // TSPJ random 2-opt on the top ranks (task = rank)
};

// one unit of row work: population `pid`, row `row` of that population
struct Task {
    int32_t pid;
    int32_t row;
};

// tile shape chosen per size bucket: threads per row and float4 groups per thread
struct RowTile {
    int block;
    int groups;
};

struct RowLaunch {
    PopDesc* descs;          // device descriptors (nullptr: use `single`)
    PopDesc single;          // descriptor passed by value
    const Task* tasks;       // device task list (nullptr: rows 0..ntasks-1 of `single`)
    int32_t ntasks;
    int32_t mode;
    int32_t* perm_out;       // optional decoded permutations [rows][n] (MODE_EVAL)
    int32_t max_n;           // largest chromosome among the populations launched
    int32_t max_points;      // largest coordinate count (n, or n+1 with a depot)
    int32_t stage_xy;        // stage coordinates in shared memory
    void* gscratch;          // global-scratch kernel (RowTile{0,0}): grid slices of gstride bytes
    size_t gstride;
    int32_t task_group;      // tasks dealt to CTAs in groups of this many consecutive tasks (0, 1: one)
    int32_t* work;           // dynamic dealing (batches and the server): [next group, CTAs done],
                             // zero before the launch and left zero by its last CTA; nullptr:
                             // group g goes to CTA g % grid
    int32_t ls_moves;        // MODE_LSEARCH: segment reversals per individual
    int32_t ls_force;        // MODE_LSEARCH: run whatever the generation (operator); rank q = row q
};

// smallest tile whose capacity (4 * block * groups) covers n
RowTile pick_tile(int n);
// every compiled tile whose capacity covers n without being far larger (autotuning set)
int tile_candidates(int n, RowTile* out, int cap);
// shared memory bytes for one CTA of the row kernel
size_t row_smem_bytes(const RowTile& t, int max_n, int max_points, int kind, bool stage_xy);
// largest n the in-shared-memory row kernel supports
int row_max_n();
// Rows whose sort does not fit in shared memory are decoded by a kernel with its sort
// scratch in global memory: launch_rows with kGlobalTile and RowLaunch::gscratch /
// gstride set (row_global_stride(max_n) bytes for each of the grid's CTAs).
constexpr RowTile kGlobalTile{0, 0};
int row_max_n_global();
bool row_needs_global(int n, int pts, int kind);
size_t row_global_stride(int max_n);
int row_global_grid(int rows, int max_n);
// one-time set-up for a tile / shared-memory size: raises the dynamic shared-memory limit
// and returns the resident CTAs per SM (0 if the tile cannot run with that much memory)
cudaError_t prepare_rows(const RowTile& tile, size_t smem, int* per_sm);
// launch the fused row kernel (generation / init / evaluate / NSGA-II offspring) on
// `grid` CTAs (<= resident capacity); prepare_rows must have run for this tile and size
cudaError_t launch_rows(const RowLaunch& L, int kind, const RowTile& tile, int grid, cudaStream_t s);
// convenience for one-off launches: prepare + launch with an occupancy-sized grid
cudaError_t launch_rows_auto(const RowLaunch& L, int kind, const RowTile& tile, cudaStream_t s);
// raise the shared-memory limit of the sort kernels for populations of up to maxP rows
cudaError_t prepare_sort(int maxP);
// raise (never lower) the dynamic shared-memory limit of a kernel on the current device
cudaError_t raise_smem_limit(const void* fn, size_t smem);

// elite partition of raw fitness segments: sorted[seg*P + r]
cudaError_t launch_sort_raw(const float* fit, int P, int segments, int maximize, int32_t* sorted,
                            cudaStream_t s);
// re-rank after a local search pass: only populations for which it was due
cudaError_t launch_sort_pops_after_ls(PopDesc* descs, int npops, int maxP, cudaStream_t s);
// engine sort: for each population, sort fit[cur^flip]; when flip, swap buffers and gen++;
// history[gen] = best
cudaError_t launch_sort_pops(PopDesc* descs, int npops, int maxP, int flip, cudaStream_t s);
// ring migration between `k` consecutive island descriptors starting at first_pid, for
// `ninst` instances laid out back to back (island descriptors of one instance adjacent)
cudaError_t launch_migrate(PopDesc* descs, int ninst, int k, int migrants, int max_n, cudaStream_t s);

int device_sm_count();

// Launch with programmatic stream serialization: the kernel is scheduled as the one before
// it in the stream drains, and waits for it (dep_wait) before it touches global memory.
// Only kernels that call dep_wait before any global-memory access are launched this way.
template <typename... Args>
inline cudaError_t launch_dep(void (*fn)(Args...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, fn, args...);
    if (e != cudaSuccess) cudaGetLastError();  // the status is returned, not left behind
    return e;
}

}  // namespace bk
