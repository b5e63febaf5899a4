// common.cuh -- device primitives shared by every kernel of the engine:
// the Philox4x32-10 counter-based stream, the order-preserving key map, the
// population descriptor and small block-level collectives.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bk {

// ---------------------------------------------------------------------------------------
// problem kinds (mirror include/brkga_b200.h)
// ---------------------------------------------------------------------------------------
enum Kind : int32_t {
    TSP_COORDS = 1,
    TSP_MATRIX = 2,
    KNAP_THRESHOLD = 3,
    KNAP_GREEDY = 4,
    BITSP_COORDS = 5,
    BITSP_MATRIX = 6,
    TSPJ = 7,
    JOBSCHED = 8,
    CONTINUOUS = 9,
    MOVRP = 10,  // xy = depot + customers, w = demands, capi = vehicle capacity, machines = vehicles
    EXTERNAL = 11,  // fitness from the caller: rows are built, never evaluated on the device
};

enum Function : int32_t { FN_SPHERE = 0, FN_RASTRIGIN = 1, FN_ROSENBROCK = 2 };

// stream tags: Philox counter word 3 = (island << 8) | tag
enum Tag : uint32_t {
    TAG_INIT = 1,
    TAG_MUTANT = 2,
    TAG_COIN = 3,
    TAG_PARENT = 4,
    TAG_NSGA_TOUR = 5,
    TAG_NSGA_COIN = 6,
    TAG_NSGA_MUTP = 7,
    TAG_NSGA_MUTK = 8,
    TAG_NSGA_REFILL = 9,
    TAG_LS = 10,
};

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): replaces the reference's stateful
// cuRAND XORWOW states (core/cuda_kernels.cuh:10-15) -- nothing is stored per individual,
// every draw is a pure function of (seed, generation, row, gene).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint4 draw4(uint64_t seed, uint32_t word, uint32_t row, uint32_t gen,
                                       uint32_t stream) {
    return philox(make_uint4(word, row, gen, stream), (uint32_t)seed, (uint32_t)(seed >> 32));
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization
// is scheduled as the kernel before it in the stream drains, instead of after that kernel's
// completion has been processed.  Every such kernel calls dep_wait() before its first
// global-memory access: the wait returns once the preceding grid has completed and its
// writes are visible, so nothing is read or written early.  No kernel here releases its
// dependents before it exits (griddepcontrol.launch_dependents): row CTAs placed while the
// previous kernel still held SMs took SMs out of order, and the CTAs with the most rows
// then shared SMs (TSPJ -20 %).  Without the launch attribute the wait is a no-op.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// top 24 bits -> float in [0,1): exact (24-bit integer times 2^-24)
__device__ __forceinline__ float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
// floor(x * k / 2^32)
__device__ __forceinline__ uint32_t pick(uint32_t x, uint32_t k) { return __umulhi(x, k); }

// order-preserving float -> uint32 (-0 folded onto +0, every NaN above +inf)
__device__ __forceinline__ uint32_t okey(float f) {
    uint32_t b = __float_as_uint(f);
    if ((b & 0x7F800000u) == 0x7F800000u && (b & 0x007FFFFFu)) return 0xFFFFFFFFu;
    if (b == 0x80000000u) b = 0u;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// fitness order key: ascending for minimisation, descending for maximisation; NaN last
__device__ __forceinline__ uint32_t fitkey(float f, int maximize) {
    const uint32_t k = okey(f);
    if (!maximize || k == 0xFFFFFFFFu) return k;
    return ~k;
}

// ---------------------------------------------------------------------------------------
// population descriptor.  Device-resident copies are updated in place by the sort kernel
// (ping-pong buffer index and generation counter), so a captured CUDA graph of
// [generation kernel, sort kernel] can be replayed any number of times.
// ---------------------------------------------------------------------------------------
struct PopDesc {
    // instance
    int32_t kind, n, ld, m;   // m = number of objectives (1 or 2)
    const float* xy;          // TSP [n][2]; bi-TSP [n+1][2]
    const float* xy2;
    const float* mat;         // TSP [n][n]; bi-TSP [n+1][n+1]; TSPJ travel times [c+1][c+1] (n = 2c)
    const float* mat2;        // bi-TSP second matrix; TSPJ job durations [c+1][c+1]
    const int32_t* w;
    const int2* wv;           // knapsack: (weight, value) pairs (one load per item in key order)
    const float* jt;          // job scheduling: job times [n]
    int32_t machines;
    int32_t function;         // continuous: Function and bounds
    float lo, hi;
    float cap;                // knapsack capacity (threshold fitness, float like the reference)
    int32_t maximize;
    long long capi;           // floor(cap) for the greedy decoder
    // GA parameters
    int32_t P, E, M;
    uint32_t rhoT;            // coin threshold: elite gene iff (x >> 8) < rhoT
    uint64_t seed;
    uint32_t island;          // stream high bits (island << 8)
    int32_t row0;             // first row of this population inside the key buffers
    // state
    float* keys[2];
    float* fit[2];            // [rows][m]
    int32_t* sorted;          // rank -> row (relative to row0) of keys[cur]
    int2* parents;            // per child row of the next generation: (elite rank, non-elite rank)
    int32_t* done;            // completion counter of the rank kernel (last CTA flips the state)
    float* history;           // best fitness per generation
    int32_t hist_cap;
    int32_t cur;
    uint32_t gen;
    // NSGA-II state (null for single-objective populations)
    int32_t Mn;               // fresh random offspring per generation
    uint32_t mutT;            // per-gene reset threshold
    int32_t div_interval;     // ensure_minimum_diversity period (0 = off)
    int32_t domW;             // row stride (words) of the dominance matrix
    int32_t* nrank;           // [2P] pool ranks; [0,P) the survivors'
    float* ncd;               // [2P] crowding distances
    int32_t* nsel;            // [P] survivor pool indices / unique list of the diversity pass
    uint32_t* domS;           // [2P][domW] dominance rows
    int32_t* domcnt;          // [2P] domination counts
    int32_t* nu;              // diversity pass: unique count, P when nothing was rebuilt
    int32_t* nord;            // [2][2P] pool points in (rank, objective o, index) order, then
                              // [2P] the pool's dominator counts (zero between generations)
    int32_t* nft;             // front table of the last peel: [0] ranks, [1] cut rank (-1: none),
                              // [2 + r] first position of rank r in rank order, [2 + ranks] = N
    float* ncdp;              // [2P] crowding distance of every pool point
    int32_t* nlist;           // [2P] the last peel's fronts (members in no set order), fronts in rank
                              // order (front r at [nft[2 + r], nft[3 + r]); not the last front
                              // of a peel stopped at the cut)
    uint32_t* nfmin;          // survivors' smallest first objective (order key; all ones: none)
    // shared launches: a population whose generation has reached gen_limit (> 0) is left
    // unchanged by every kernel; `advanced` records whether the last generation ran
    uint32_t gen_limit;
    int32_t advanced;
    // TSPJ random 2-opt local search period (0 = off)
    int32_t ls_interval;
};

__host__ __device__ __forceinline__ bool at_limit(const PopDesc& d) { return d.gen_limit != 0u && d.gen >= d.gen_limit; }

// local search after generation gen (the reference's counter is gen - 1, core/solver.hpp:459-460)
__host__ __device__ __forceinline__ bool ls_due(const PopDesc& d) {
    return d.ls_interval > 0 && d.gen >= 2u && ((d.gen - 1u) % (uint32_t)d.ls_interval) == 0u;
}

// ---------------------------------------------------------------------------------------
// block collectives
// ---------------------------------------------------------------------------------------
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = (lane < NW) ? warp_tot[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NW) warp_tot[lane] = s;
    }
    __syncthreads();
    const uint32_t base = (w > 0) ? warp_tot[w - 1] : 0u;
    if (total) *total = warp_tot[NW - 1];
    return base + x - v;
}

template <int BLOCK>
__device__ __forceinline__ long long block_sum_ll(long long v, long long* red) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w] = v;
    __syncthreads();
    long long s = 0;
#pragma unroll
    for (int i = 0; i < NW; ++i) s += red[i];
    __syncthreads();
    return s;
}

__host__ __device__ __forceinline__ int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace bk
