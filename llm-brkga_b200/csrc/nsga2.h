// nsga2.h -- NSGA-II on the device (core/solver.hpp:751-817, core/population.hpp:130-517).
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "kernels.h"

namespace bk {

struct Population;

struct NsgaState {
    PopDesc* dd = nullptr;   // device descriptor of the population (buffers live in it)
    int P = 0, N = 0, n = 0, ld = 0, kind = 0, max_points = 0;
    RowTile tile{};
    int grid = 0;
    bool stage = false;
    float* history = nullptr;
    int hist_cap = 0;
    int div_interval = 0;
    bool ready = false;
    void* gscratch = nullptr;  // global-memory row kernel scratch (tile kGlobalTile)
    size_t gstride = 0;
};

int32_t nsga_setup(NsgaState& s, Population& pop, PopDesc* dd, PopDesc& hdesc, const RowTile& tile, int grid,
                   bool stage);
// allocate one population's NSGA-II buffers and fill its descriptor fields
int32_t nsga_alloc(PopDesc& d, int P, double mut_rate, int div_interval, int Mn, std::vector<void*>& allocs,
                   size_t* bytes, cudaStream_t stream);
int nsga_max_population();
cudaError_t nsga_prepare(int maxP);
// group launches over `npops` consecutive NSGA-II descriptors; mode 0 (a generation's
// pool) also moves the survivors' rows into the other buffer, swaps the buffers and
// advances the generation
cudaError_t nsga_enqueue_select(PopDesc* dd, int npops, int maxP, int mode, cudaStream_t st);
cudaError_t nsga_enqueue_diversity(PopDesc* dd, int npops, int maxP, cudaStream_t st);
void nsga_release(NsgaState& s);
void nsga_set_history(NsgaState& s, float* h, int cap);
cudaError_t nsga_enqueue_init(NsgaState& s, cudaStream_t st);
// one row launch of the population in the given mode (MODE_INIT, MODE_NSGA_OFF, ...)
cudaError_t nsga_enqueue_rows(NsgaState& s, int mode, cudaStream_t st);
// one generation; with_diversity = false leaves out the diversity pass's launches (they
// exit at once unless the pass is due after this generation: nsga_diversity_due)
cudaError_t nsga_enqueue_generation(NsgaState& s, cudaStream_t st, bool with_diversity = true);
// the diversity pass runs after generation g (counted from 1) when (g - 1) % interval == 0
// (core/population.hpp:130-182 via core/solver.hpp:751-817), for a population with no
// generation limit
bool nsga_diversity_due(const NsgaState& s, uint32_t g);
int32_t nsga_get_population(NsgaState& s, cudaStream_t st, float* keys, float* obj);
int32_t nsga_set_population(NsgaState& s, cudaStream_t st, const float* keys);
int32_t nsga_get_best(NsgaState& s, cudaStream_t st, float* keys, int32_t* perm, float* obj);
int32_t nsga_get_front(NsgaState& s, cudaStream_t st, float* obj, float* keys, int32_t cap, int32_t* count);

}  // namespace bk
