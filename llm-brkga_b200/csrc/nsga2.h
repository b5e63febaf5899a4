// nsga2.h -- NSGA-II on the device (core/solver.hpp:751-817, core/population.hpp:130-517).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace bk {

struct Population;

struct NsgaState {
    PopDesc* dd = nullptr;   // device descriptor of the population
    int P = 0, N = 0, n = 0, ld = 0, kind = 0, max_points = 0;
    RowTile tile{};
    int grid = 0;
    bool stage = false;
    float* keys[2] = {nullptr, nullptr};  // [2P][ld] pools
    float* fit[2] = {nullptr, nullptr};   // [2P][2]
    int32_t* rank = nullptr;              // [2P]
    float* cd = nullptr;                  // [2P]
    int32_t* sel = nullptr;               // [P]
    int32_t* d_nu = nullptr;              // diversity: unique count (P when no rebuild)
    float* history = nullptr;
    int hist_cap = 0;
    int Mn = 0;
    uint32_t mutT = 0;
    int div_interval = 0;
    bool ready = false;
};

int32_t nsga_setup(NsgaState& s, Population& pop, PopDesc* dd, const RowTile& tile, int grid, bool stage);
void nsga_release(NsgaState& s);
void nsga_set_history(NsgaState& s, float* h, int cap);
cudaError_t nsga_enqueue_init(NsgaState& s, cudaStream_t st);
cudaError_t nsga_enqueue_generation(NsgaState& s, cudaStream_t st);
int32_t nsga_get_population(NsgaState& s, cudaStream_t st, float* keys, float* obj);
int32_t nsga_set_population(NsgaState& s, cudaStream_t st, const float* keys);
int32_t nsga_get_best(NsgaState& s, cudaStream_t st, float* keys, int32_t* perm, float* obj);
int32_t nsga_get_front(NsgaState& s, cudaStream_t st, float* obj, float* keys, int32_t cap, int32_t* count);

}  // namespace bk
