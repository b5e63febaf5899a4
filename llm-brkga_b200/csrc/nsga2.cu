// nsga2.cu -- NSGA-II selection on the device.
//
// Reference: Solver::evolve_generation_nsga2 (core/solver.hpp:751-817) and
// Population::fast_non_dominated_sort / calculate_crowding_distance /
// select_next_generation_nsga2 / ensure_minimum_diversity (core/population.hpp:130-517).
//
// The reference pushes every first-front point into fronts[0] twice (once in
// fast_non_dominated_sort, core/population.hpp:431-434, again in
// build_fronts_from_domination, :335-340).  Its ranks therefore come from a peeling in
// which the first front decrements twice, its crowding pass sees every first-front point
// as two adjacent entries, and its survivor list takes first-front points twice.  All
// three are reproduced here (ties fixed by index), bit for bit against the oracle.
//
// Ranks: bit-packed dominance matrix + bit-sliced front peeling (below).
// Crowding: per objective a bitonic sort of (rank, objective, index) makes every front a
// contiguous ordered run; each entry adds (next - prev) / range in list order.
// Survivors: bitonic sort of the entry list (first-front points twice) by (rank, last
// objective or -crowding for the front that is cut, index, copy); the first P entries.
#include <algorithm>
#include <cfloat>
#include <map>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "engine.h"
#include "nsga2.h"

namespace bk {

constexpr int kNsgaBlock = 1024;
constexpr int kMaxPool = 4096;  // largest pool (2P) of the in-shared-memory select kernel

__host__ __device__ inline int npow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Ascending bitonic sort of s[0, N2) (N2 a power of two) by the whole block.  Strides of 64
// and more go through shared memory with a barrier each; strides 32 .. 1 run in registers:
// warp w owns the 64-element blocks w, w + warps, ..., lane l holding elements l and l + 32
// of a block (stride 32 inside the lane, strides 16 .. 1 by shuffles), so each k costs one
// barrier for all of its small strides instead of six.
__device__ __forceinline__ unsigned long long cx_keep(unsigned long long x, unsigned long long y, int g, int j,
                                                      int k) {
    // element g of the pair (g, g ^ j): the lower index keeps the minimum in an ascending
    // run ((g & k) == 0), the maximum in a descending one
    const bool keep_min = ((g & j) == 0) == ((g & k) == 0);
    return keep_min ? (x < y ? x : y) : (x < y ? y : x);
}

template <int BLOCK>
__device__ void bitonic_u64(unsigned long long* s, int N2) {
    const int t = threadIdx.x;
    if (N2 < 64) {
        for (int k = 2; k <= N2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int p = t; p < (N2 >> 1); p += BLOCK) {
                    const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
                    const int ixj = i + j;
                    const bool up = (i & k) == 0;
                    const unsigned long long a = s[i], b = s[ixj];
                    if ((a > b) == up) {
                        s[i] = b;
                        s[ixj] = a;
                    }
                }
                __syncthreads();
            }
        return;
    }
    constexpr int NW = BLOCK / 32;
    const int lane = t & 31, warp = t >> 5;
    // strides min(32, k / 2) .. 1 of step k on every 64-element block, in registers
    auto small_strides = [&](int k, int jmax) {
        for (int base = warp * 64; base < N2; base += NW * 64) {
            const int g0 = base + lane, g1 = g0 + 32;
            unsigned long long x0 = s[g0], x1 = s[g1];
            if (jmax >= 32) {
                const unsigned long long lo = x0 < x1 ? x0 : x1, hi = x0 < x1 ? x1 : x0;
                const bool up = (g0 & k) == 0;
                x0 = up ? lo : hi;
                x1 = up ? hi : lo;
            }
            for (int j = (jmax >= 32 ? 16 : jmax); j > 0; j >>= 1) {
                const unsigned long long y0 = __shfl_xor_sync(0xffffffffu, x0, j);
                const unsigned long long y1 = __shfl_xor_sync(0xffffffffu, x1, j);
                x0 = cx_keep(x0, y0, g0, j, k);
                x1 = cx_keep(x1, y1, g1, j, k);
            }
            s[g0] = x0;
            s[g1] = x1;
        }
        __syncthreads();
    };
    for (int k = 2; k <= 64; k <<= 1) small_strides(k, k >> 1);
    for (int k = 128; k <= N2; k <<= 1) {
        for (int j = k >> 1; j >= 64; j >>= 1) {
            for (int p = t; p < (N2 >> 1); p += BLOCK) {
                const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
                const int ixj = i + j;
                const bool up = (i & k) == 0;
                const unsigned long long a = s[i], b = s[ixj];
                if ((a > b) == up) {
                    s[i] = b;
                    s[ixj] = a;
                }
            }
            __syncthreads();
        }
        small_strides(k, 32);
    }
}

constexpr int kCB = 16;  // count planes (two's complement)
constexpr int kDB = 15;  // decrement planes

__device__ __forceinline__ bool dominates_m(const float* a, const float* b, int m) {
    bool better = false;
    for (int o = 0; o < m; ++o) {
        if (a[o] > b[o]) return false;
        if (a[o] < b[o]) better = true;
    }
    return better;
}

struct DomArgs {
    PopDesc* dd;          // engine mode: the P population blockIdx.y (objectives fit[cur], buffers);
                          // a generation's 2P pool goes through dom2_pool_kernel
    int only_rebuilt;     // engine mode: skip populations whose diversity pass kept them (*nu >= P)
    const float* obj;     // raw mode
    int rawN, m;
    uint32_t* S;          // raw mode: [N][Wmax]
    int32_t* cnt;         // raw mode: [N]
    int Wmax;
};

__global__ void dom_build_kernel(DomArgs a) {
    const float* obj;
    int N, m, Wmax;
    uint32_t* S;
    int32_t* cnt;
    if (a.dd) {
        const PopDesc& d = a.dd[blockIdx.y];
        if (a.only_rebuilt && (!d.advanced || __ldg(d.nu) >= d.P)) return;
        N = d.P;
        m = d.m;
        obj = d.fit[d.cur];
        S = d.domS;
        cnt = d.domcnt;
        Wmax = d.domW;
    } else {
        N = a.rawN;
        m = a.m;
        obj = a.obj;
        S = a.S;
        cnt = a.cnt;
        Wmax = a.Wmax;
    }
    const int W = (N + 31) / 32;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < N; i += nwarps) {
        float oi[4];
        for (int o = 0; o < m && o < 4; ++o) oi[o] = __ldg(obj + (size_t)i * m + o);
        int c = 0;
        for (int w = 0; w < W; ++w) {
            const int j = 32 * w + lane;
            bool dij = false, dji = false;
            if (j < N && j != i) {
                float oj[4];
                for (int o = 0; o < m && o < 4; ++o) oj[o] = __ldg(obj + (size_t)j * m + o);
                dij = dominates_m(oi, oj, m);
                dji = dominates_m(oj, oi, m);
            }
            const uint32_t si = __ballot_sync(0xffffffffu, dij);
            const uint32_t di = __ballot_sync(0xffffffffu, dji);
            if (lane == 0) S[(size_t)i * Wmax + w] = si;
            c += __popc(di);
        }
        if (lane == 0) cnt[i] = c;
    }
}

// Two objectives (every NSGA-II problem of the engine): the objectives are staged in
// shared memory and each warp tests four rows against 32 columns per step.  The four
// comparisons of a pair give both directions: i dominates j iff !(a0 > b0) && !(a1 > b1)
// && (a0 < b0 || a1 < b1), the reference's Individual::dominates (core/individual.hpp:99-114)
// with its NaN behaviour; padding columns are NaN, which dominates nothing either way.
// Element i of [0, count) for i = threadIdx.x + k * T: a thread issues the loads of K of
// its elements before the first store, so staging takes one memory round trip per K
// elements instead of one per element.
template <int T, int K, typename Ld, typename St>
__device__ __forceinline__ void staged(int count, Ld ld, St st) {
    for (int i0 = (int)threadIdx.x; i0 < count; i0 += T * K) {
        decltype(ld(0)) v[K];
#pragma unroll
        for (int u = 0; u < K; ++u)
            if (i0 + u * T < count) v[u] = ld(i0 + u * T);
#pragma unroll
        for (int u = 0; u < K; ++u)
            if (i0 + u * T < count) st(i0 + u * T, v[u]);
    }
}

// A generation's pool (two objectives): the dominator counts are accumulated into a slot
// after the two orders (nord + 2N, N = 2P), which is zero between generations: the peel
// reads each count and clears it.
__host__ __device__ inline int32_t* pool_counts(const PopDesc& d) { return d.nord + 4 * (size_t)d.P; }

// 32 x 32 bit transpose across a warp: lane l holds row l on entry (bit c = element (l, c))
// and column l on exit (bit r = element (r, l)); five exchange steps of halving blocks.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t w, int lane) {
    const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int s = 16 >> k;
        const uint32_t m = masks[k];
        const uint32_t y = __shfl_xor_sync(0xffffffffu, w, s);
        w = (lane & s) ? ((w & ~m) | ((y & ~m) >> s)) : ((w & m) | ((y & m) << s));
    }
    return w;
}

// The pool's dominance rows, each unordered pair of 32-point blocks (I <= J) visited once
// by one warp: for row r of block I against lane j of block J the four compares give
// both directions.  Row words: block I's rows at word J directly; block J's rows at word
// I from the other direction's ballots by a bit transpose.  Dominator counts by atomic
// adds into pool_counts (a diagonal block adds only once).  The same compares as
// dom2_build_kernel, so the same matrix and counts bit for bit; half the pair tests.
constexpr int kSymWarps = 16;

__global__ void __launch_bounds__(kSymWarps * 32) dom2_pool_kernel(PopDesc* dd) {
    dep_wait();
    __shared__ float2 srow[kSymWarps][32];
    PopDesc& d = dd[blockIdx.y];
    if (at_limit(d)) return;
    const int N = 2 * d.P, W = (N + 31) / 32, Wmax = d.domW;
    const int T = W * (W + 1) / 2;
    const float2* __restrict__ o2 = reinterpret_cast<const float2*>(d.fit[d.cur]);
    uint32_t* const S = d.domS;
    int32_t* const acc = pool_counts(d);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2* const rows = srow[warp];
    // consecutive tiles go to different CTAs, so that every CTA (and SM) gets the same
    // share; each warp loads the next tile's objectives before it works on the current one
    const int nw = gridDim.x * kSymWarps;
    auto block_pair = [](int tile, int& I, int& J) {  // tile = J (J + 1) / 2 + I with I <= J
        J = (int)((sqrtf(8.0f * (float)tile + 1.0f) - 1.0f) * 0.5f);
        while (J * (J + 1) / 2 > tile) --J;
        while ((J + 1) * (J + 2) / 2 <= tile) ++J;
        I = tile - J * (J + 1) / 2;
    };
    auto objectives = [&](int I, int J, float2& oi, float2& oj) {
        const int i = 32 * I + lane, j = 32 * J + lane;
        oi = (i < N) ? __ldg(o2 + i) : make_float2(NAN, NAN);
        oj = (j < N) ? __ldg(o2 + j) : make_float2(NAN, NAN);
    };
    int tile = warp * gridDim.x + blockIdx.x, I = 0, J = 0;
    float2 oi = make_float2(NAN, NAN), oj = make_float2(NAN, NAN);
    if (tile < T) {
        block_pair(tile, I, J);
        objectives(I, J, oi, oj);
    }
    for (; tile < T; tile += nw) {
        int nI = 0, nJ = 0;
        float2 noi = make_float2(NAN, NAN), noj = make_float2(NAN, NAN);
        if (tile + nw < T) {
            block_pair(tile + nw, nI, nJ);
            objectives(nI, nJ, noi, noj);
        }
        const int i = 32 * I + lane, j = 32 * J + lane;
        __syncwarp();
        rows[lane] = oi;
        __syncwarp();
        uint32_t rw = 0u, cw = 0u;
        int cj = 0;
#pragma unroll 8
        for (int r = 0; r < 32; ++r) {
            const float2 a = rows[r];
            const bool gt0 = a.x > oj.x, gt1 = a.y > oj.y;
            const bool lt0 = a.x < oj.x, lt1 = a.y < oj.y;
            const bool rdj = !gt0 && !gt1 && (lt0 || lt1);  // row 32 I + r dominates 32 J + lane
            const uint32_t s1 = __ballot_sync(0xffffffffu, rdj);
            const uint32_t s2 = __ballot_sync(0xffffffffu, !lt0 && !lt1 && (gt0 || gt1));
            cj += rdj ? 1 : 0;
            if (lane == r) {
                rw = s1;
                cw = s2;
            }
        }
        if (i < N) {
            S[(size_t)i * Wmax + J] = rw;
            const int c = __popc(cw);  // points of block J dominating i
            if (c) atomicAdd(acc + i, c);
        }
        if (I != J) {
            const uint32_t tw = warp_transpose32(cw, lane);  // row j, word I
            if (j < N) {
                S[(size_t)j * Wmax + I] = tw;
                if (cj) atomicAdd(acc + j, cj);
            }
        }
        I = nI;
        J = nJ;
        oi = noi;
        oj = noj;
    }
}

constexpr int kDom2Rows = 4;       // rows per warp
constexpr int kDom2RowWarps = 4;   // row groups per CTA
constexpr int kDom2ColGroups = 4;  // column groups: warp g of a row group takes the 32-word blocks b % 4 == g
constexpr int kDom2Warps = kDom2RowWarps * kDom2ColGroups;

__global__ void __launch_bounds__(kDom2Warps * 32) dom2_build_kernel(DomArgs a) {
    dep_wait();
    extern __shared__ float2 so[];  // [32 * ceil(N / 32)] objectives
    __shared__ int cpart[kDom2ColGroups][kDom2RowWarps * kDom2Rows];
    const float* obj;
    int N, Wmax;
    uint32_t* S;
    int32_t* cnt;
    if (a.dd) {
        const PopDesc& d = a.dd[blockIdx.y];
        if (a.only_rebuilt && (!d.advanced || __ldg(d.nu) >= d.P)) return;
        N = d.P;
        obj = d.fit[d.cur];
        S = d.domS;
        cnt = d.domcnt;
        Wmax = d.domW;
    } else {
        N = a.rawN;
        obj = a.obj;
        S = a.S;
        cnt = a.cnt;
        Wmax = a.Wmax;
    }
    constexpr int RPC = kDom2Rows * kDom2RowWarps;  // rows per CTA
    const int row0 = blockIdx.x * RPC;
    if (row0 >= N) return;
    const int W = (N + 31) / 32;
    const float2* o2 = reinterpret_cast<const float2*>(obj);
    staged<kDom2Warps * 32, 8>(
        32 * W, [&](int j) { return (j < N) ? __ldg(o2 + j) : make_float2(NAN, NAN); },
        [&](int j, float2 v) { so[j] = v; });
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rg = warp % kDom2RowWarps, cg = warp / kDom2RowWarps;
    const int i0 = row0 + rg * kDom2Rows;
    float2 oi[kDom2Rows];
    int c[kDom2Rows];
#pragma unroll
    for (int r = 0; r < kDom2Rows; ++r) {
        oi[r] = so[min(i0 + r, N - 1)];
        c[r] = 0;
    }
    const int nblk = (W + 31) / 32;
    for (int b = cg; b < nblk; b += kDom2ColGroups) {
        uint32_t buf[kDom2Rows];
#pragma unroll
        for (int r = 0; r < kDom2Rows; ++r) buf[r] = 0u;
        const int wend = min(W, 32 * b + 32);
        for (int w = 32 * b; w < wend; ++w) {
            const float2 oj = so[32 * w + lane];
#pragma unroll
            for (int r = 0; r < kDom2Rows; ++r) {
                const bool gt0 = oi[r].x > oj.x, gt1 = oi[r].y > oj.y;
                const bool lt0 = oi[r].x < oj.x, lt1 = oi[r].y < oj.y;
                const uint32_t si = __ballot_sync(0xffffffffu, !gt0 && !gt1 && (lt0 || lt1));
                const uint32_t di = __ballot_sync(0xffffffffu, !lt0 && !lt1 && (gt0 || gt1));
                c[r] += __popc(di);
                if (lane == (w & 31)) buf[r] = si;
            }
        }
        // lane l holds word 32 b + l of each row: one coalesced store per row
        const int wl = 32 * b + lane;
#pragma unroll
        for (int r = 0; r < kDom2Rows; ++r)
            if (i0 + r < N && wl < wend) S[(size_t)(i0 + r) * Wmax + wl] = buf[r];
    }
    // dominator counts: the column groups' partial counts, added in a fixed order
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < kDom2Rows; ++r) cpart[cg][rg * kDom2Rows + r] = c[r];
    }
    __syncthreads();
    if (threadIdx.x < RPC && row0 + (int)threadIdx.x < N) {
        int sum = 0;
#pragma unroll
        for (int g = 0; g < kDom2ColGroups; ++g) sum += cpart[g][threadIdx.x];
        cnt[row0 + threadIdx.x] = sum;
    }
}

struct PeelSmem {
    uint32_t* C;      // [kCB][W] count planes
    uint32_t* A;      // [W] ranked
    uint32_t* F;      // [W] current front
    uint32_t* V;      // [W] valid points
    uint16_t* list;   // [N] front members
};

__host__ __device__ inline size_t peel_smem_bytes(int N) {
    const int W = (N + 31) / 32;
    return (size_t)(kCB + 4) * W * 4 + (((size_t)N * 2 + 15) / 16) * 16;
}

__device__ inline PeelSmem peel_carve(unsigned char* base, int N) {
    const int W = (N + 31) / 32;
    PeelSmem p;
    p.C = (uint32_t*)base;
    p.A = p.C + (size_t)kCB * W;
    p.F = p.A + W;
    p.V = p.F + W;
    p.list = (uint16_t*)(p.V + 2 * W);  // V[W..2W) stages the next front
    return p;
}

// ranks of N points into rank[] (shared memory); S rows of stride Wmax, counts cnt[]
template <int T>
__device__ int peel_ranks(int N, const uint32_t* __restrict__ S, int Wmax, const int32_t* __restrict__ cnt,
                          uint16_t* rank, const PeelSmem& ps, uint32_t* wt32) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int W = (N + 31) / 32;
    // counts -> planes, valid mask
    for (int w = warp; w < W; w += T / 32) {
        const int i = 32 * w + lane;
        const int c = (i < N) ? __ldg(cnt + i) : 0;
#pragma unroll
        for (int b = 0; b < kCB; ++b) {
            const uint32_t pl = __ballot_sync(0xffffffffu, (c >> b) & 1);
            if (lane == 0) ps.C[(size_t)b * W + w] = pl;
        }
        const uint32_t v = __ballot_sync(0xffffffffu, i < N);
        if (lane == 0) ps.V[w] = v;
    }
    __syncthreads();
    // first front: zero counts
    for (int w = t; w < W; w += T) {
        uint32_t z = ps.V[w];
#pragma unroll
        for (int b = 0; b < kCB; ++b) z &= ~ps.C[(size_t)b * W + w];
        ps.F[w] = z;
        ps.A[w] = z;
        for (uint32_t x = z; x; x &= x - 1) rank[32 * w + __ffs(x) - 1] = 0;
    }
    __syncthreads();
    // lanes per word for the column sums: a power of two, at most 32, SP * W <= T
    int SP = 32;
    while (SP > 1 && SP * W > T) SP >>= 1;
    int k = 0;
    for (; k < N; ++k) {
        // front member list
        const uint32_t pc = (t < W) ? __popc(ps.F[t]) : 0u;
        uint32_t nf = 0;
        uint32_t base = block_exclusive_scan<T>(pc, wt32, &nf);
        if (t < W)
            for (uint32_t x = ps.F[t]; x; x &= x - 1) ps.list[base++] = (uint16_t)(32 * t + __ffs(x) - 1);
        __syncthreads();
        if (nf == 0) break;
        const int w = t / SP, sl = t % SP;
        uint32_t acc[kDB];
#pragma unroll
        for (int b = 0; b < kDB; ++b) acc[b] = 0u;
        if (w < W) {
            // bit-sliced column sums: the member rows' words are loaded eight at a time
            // (eight L2 requests in flight per lane), counted in a 4-plane counter and
            // added into the kDB-plane accumulator once per batch
            constexpr int kBatch = 8;
            for (int j0 = sl; j0 < (int)nf; j0 += kBatch * SP) {
                uint32_t xs[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int j = j0 + u * SP;
                    xs[u] = (j < (int)nf) ? __ldg(S + (size_t)ps.list[j] * Wmax + w) : 0u;
                }
                uint32_t s0 = 0u, s1 = 0u, s2 = 0u, s3 = 0u;
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const uint32_t c0 = s0 & xs[u];
                    s0 ^= xs[u];
                    const uint32_t c1 = s1 & c0;
                    s1 ^= c0;
                    const uint32_t c2 = s2 & c1;
                    s2 ^= c1;
                    s3 ^= c2;
                }
                uint32_t cy = 0u;
                const uint32_t sv[4] = {s0, s1, s2, s3};
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const uint32_t x = acc[b], y = sv[b];
                    acc[b] = x ^ y ^ cy;
                    cy = (x & y) | (cy & (x ^ y));
                }
#pragma unroll
                for (int b = 4; b < kDB; ++b) {
                    const uint32_t x = acc[b];
                    acc[b] = x ^ cy;
                    cy = x & cy;
                }
            }
        }
        // combine the SP partial sums of a word (consecutive lanes) with full adders
        for (int off = 1; off < SP; off <<= 1) {
            uint32_t c = 0u;
#pragma unroll
            for (int b = 0; b < kDB; ++b) {
                const uint32_t o = __shfl_xor_sync(0xffffffffu, acc[b], off);
                const uint32_t s2 = acc[b] ^ o ^ c;
                c = (acc[b] & o) | (c & (acc[b] ^ o));
                acc[b] = s2;
            }
        }
        if (w < W && sl == 0) {
            // decrement: doubled for the first front
            uint32_t dec[kCB];
#pragma unroll
            for (int b = 0; b < kCB; ++b) dec[b] = 0u;
            if (k == 0) {
#pragma unroll
                for (int b = 1; b < kCB; ++b) dec[b] = (b - 1 < kDB) ? acc[b - 1] : 0u;
            } else {
#pragma unroll
                for (int b = 0; b < kDB; ++b) dec[b] = acc[b];
            }
            uint32_t bor = 0u, any = 0u;
#pragma unroll
            for (int b = 0; b < kCB; ++b) {
                const uint32_t x = ps.C[(size_t)b * W + w];
                const uint32_t d = x ^ dec[b] ^ bor;
                bor = (~x & dec[b]) | (~(x ^ dec[b]) & bor);
                ps.C[(size_t)b * W + w] = d;
                any |= d;
            }
            const uint32_t sign = ps.C[(size_t)(kCB - 1) * W + w];
            const uint32_t nz = (sign | ~any) & ~ps.A[w] & ps.V[w];
            ps.A[w] |= nz;
            for (uint32_t x = nz; x; x &= x - 1) rank[32 * w + __ffs(x) - 1] = (uint16_t)(k + 1);
            ps.V[W + w] = nz;  // next front, staged after the valid mask
        }
        __syncthreads();
        if (t < W) ps.F[t] = ps.V[W + t];
        __syncthreads();
    }
    return k;
}


// ---------------------------------------------------------------------------------------
// crowding and survivors (two objectives), one CTA per population
// ---------------------------------------------------------------------------------------
struct SelSmem {
    float* obj;                 // [N][2]
    uint16_t* rank;             // [N]
    float* cd;                  // [N]
    unsigned long long* key;    // [K2]: next_pow2(2N) sort entries
    uint16_t* fs;               // [N] first sorted position of each rank
    uint16_t* fe;               // [N] last sorted position of each rank
    uint32_t* rb;               // [N + 1] survivor entries before each rank
    unsigned char* peel;        // peel_smem_bytes(N)
};

__host__ __device__ inline size_t sel_smem_bytes(int N) {
    const int K2 = npow2(2 * N);
    size_t b = (size_t)N * 8;
    b += ((size_t)N * 2 + 15) / 16 * 16;
    b += ((size_t)N * 4 + 15) / 16 * 16;
    b += (size_t)K2 * 8;
    b += ((size_t)N * 2 + 15) / 16 * 16 * 2;
    b += ((size_t)(N + 1) * 4 + 15) / 16 * 16;
    b += peel_smem_bytes(N);
    return (b + 15) / 16 * 16;
}

__device__ inline SelSmem sel_carve(unsigned char* base, int N) {
    const int K2 = npow2(2 * N);
    SelSmem s;
    size_t off = 0;
    s.obj = (float*)(base + off);
    off += (size_t)N * 8;
    s.rank = (uint16_t*)(base + off);
    off += ((size_t)N * 2 + 15) / 16 * 16;
    s.cd = (float*)(base + off);
    off += ((size_t)N * 4 + 15) / 16 * 16;
    s.key = (unsigned long long*)(base + off);
    off += (size_t)K2 * 8;
    s.fs = (uint16_t*)(base + off);
    off += ((size_t)N * 2 + 15) / 16 * 16;
    s.fe = (uint16_t*)(base + off);
    off += ((size_t)N * 2 + 15) / 16 * 16;
    s.rb = (uint32_t*)(base + off);
    off += ((size_t)(N + 1) * 4 + 15) / 16 * 16;
    s.peel = base + off;
    return s;
}

__device__ __forceinline__ uint32_t cd_key(float c) {
    const uint32_t k = okey(c);
    return (k == 0xFFFFFFFFu) ? 0xFFFFFFFFu : ~k;
}

// front bounds of the (rank, objective, index) order held in s.key[0, N)
template <int T>
__device__ void front_bounds(int N, const SelSmem& s) {
    for (int p = threadIdx.x; p < N; p += T) {
        const int r = (int)(s.key[p] >> 48);
        if (p == 0 || (int)(s.key[p - 1] >> 48) != r) s.fs[r] = (uint16_t)p;
        if (p == N - 1 || (int)(s.key[p + 1] >> 48) != r) s.fe[r] = (uint16_t)p;
    }
}

// one objective's contribution to the crowding distance (core/population.hpp:453-489) over
// the reference's front lists, s.key[0, N) in (rank, objective o, index) order: rank-0
// points are two adjacent entries (index, copy 0/1), other points one
template <int T>
__device__ void crowding_pass(int N, int o, const SelSmem& s) {
#define VAL(pos) s.obj[2 * (int)(s.key[pos] & 0xFFFFu) + o]
    for (int p = threadIdx.x; p < N; p += T) {
        const int i = (int)(s.key[p] & 0xFFFFu);
        const int r = (int)(s.key[p] >> 48);
        const int f = s.fs[r], l = s.fe[r];
        const int size = l - f + 1;
        if (r == 0) {
            // entries 2(p-f) and 2(p-f)+1 of the doubled list of 2*size entries
            if (size == 1 || p == f || p == l) {
                s.cd[i] = INFINITY;
            } else {
                const float range = __fsub_rn(VAL(l), VAL(f));
                if (range > 0.0f) {
                    const float v = VAL(p);
                    const float da = __fdiv_rn(__fsub_rn(v, VAL(p - 1)), range);
                    const float db = __fdiv_rn(__fsub_rn(VAL(p + 1), v), range);
                    s.cd[i] = __fadd_rn(__fadd_rn(s.cd[i], da), db);
                }
            }
        } else {
            if (size <= 2 || p == f || p == l) {
                s.cd[i] = INFINITY;
            } else {
                const float range = __fsub_rn(VAL(l), VAL(f));
                if (range > 0.0f)
                    s.cd[i] = __fadd_rn(s.cd[i], __fdiv_rn(__fsub_rn(VAL(p + 1), VAL(p - 1)), range));
            }
        }
    }
#undef VAL
}

__device__ __forceinline__ unsigned long long order_key(int rank, float v, int i) {
    return ((unsigned long long)rank << 48) | ((unsigned long long)okey(v) << 16) | (unsigned long long)i;
}

// crowding from the orders nsga_order_kernel computed (ord[o * ostride + position]); leaves
// s.key holding the objective-1 order and s.fs / s.fe its front bounds
template <int T>
__device__ void crowding_given(int N, const SelSmem& s, const int32_t* __restrict__ ord, int ostride) {
    const int t = threadIdx.x;
    for (int i = t; i < N; i += T) s.cd[i] = 0.0f;
    for (int o = 0; o < 2; ++o) {
        __syncthreads();
        staged<T, 4>(
            N, [&](int p) { return __ldg(ord + (size_t)o * ostride + p); },
            [&](int p, int i) { s.key[p] = order_key(s.rank[i], s.obj[2 * i + o], i); });
        __syncthreads();
        front_bounds<T>(N, s);
        __syncthreads();
        crowding_pass<T>(N, o, s);
    }
    __syncthreads();
}

// survivors (core/population.hpp:491-517): whole fronts while they fit, ordered by
// (last objective, index, copy) -- the objective-1 order in s.key with every rank-0 point
// taken twice -- then the cut front by (-crowding, index, copy), sorted alone
template <int T>
__device__ void select_given(int N, int P, const SelSmem& s, int32_t* g_sel, int32_t* g_rank, float* g_cd,
                             float* fmin_out, uint32_t* wt32) {
    const int t = threadIdx.x;
    __shared__ int s_cut;
    const int R = (int)(s.key[N - 1] >> 48) + 1;  // ranks 0 .. R-1 all occur
    // survivor entries of each rank (rank 0 counts twice), prefix over ranks
    const int ch = (R + T - 1) / T;
    const int r0 = min(R, t * ch), r1 = min(R, r0 + ch);
    uint32_t loc = 0;
    for (int r = r0; r < r1; ++r) loc += (uint32_t)(s.fe[r] - s.fs[r] + 1) * (r == 0 ? 2u : 1u);
    if (t == 0) s_cut = R;
    uint32_t run = block_exclusive_scan<T>(loc, wt32, nullptr);
    for (int r = r0; r < r1; ++r) {
        s.rb[r] = run;
        run += (uint32_t)(s.fe[r] - s.fs[r] + 1) * (r == 0 ? 2u : 1u);
        if (run > (uint32_t)P && s.rb[r] <= (uint32_t)P) s_cut = r;  // exactly one rank crosses P
    }
    __syncthreads();
    const int cut = s_cut;
    float fmin = INFINITY;
    // whole fronts before the cut
    for (int p = t; p < N; p += T) {
        const int r = (int)(s.key[p] >> 48);
        if (r >= cut) continue;
        const int i = (int)(s.key[p] & 0xFFFFu);
        const int k = p - s.fs[r];
        const int q = (int)s.rb[r] + (r == 0 ? 2 * k : k);
        for (int c = 0; c < (r == 0 ? 2 : 1); ++c) {
            g_sel[q + c] = i;
            g_rank[q + c] = r;
            g_cd[q + c] = s.cd[i];
        }
        fmin = fminf(fmin, s.obj[2 * i]);
    }
    const int f = (cut < R) ? s.fs[cut] : 0;
    const int nc = (cut < R) ? s.fe[cut] - f + 1 : 0;
    __syncthreads();
    if (cut < R) {
        // the cut front's points, in order, into s.fs; then its entries sorted by
        // (cd descending, index, copy) in s.key (sized for 2N entries)
        for (int k = t; k < nc; k += T) s.fs[k] = (uint16_t)(s.key[f + k] & 0xFFFFu);
        __syncthreads();
        const int mult = (cut == 0) ? 2 : 1;
        const int E = nc * mult, K2 = npow2(E);
        const int take = P - (int)s.rb[cut];
        for (int e = t; e < K2; e += T) {
            unsigned long long kk = ~0ull;
            if (e < E) {
                const int i = s.fs[e / mult];
                kk = ((unsigned long long)cd_key(s.cd[i]) << 32) | ((unsigned long long)i << 1) |
                     (unsigned long long)(e % mult);
            }
            s.key[e] = kk;
        }
        __syncthreads();
        bitonic_u64<T>(s.key, K2);
        for (int k = t; k < take; k += T) {
            const int i = (int)((s.key[k] >> 1) & 0x7FFFu);
            const int q = (int)s.rb[cut] + k;
            g_sel[q] = i;
            g_rank[q] = cut;
            g_cd[q] = s.cd[i];
            fmin = fminf(fmin, s.obj[2 * i]);
        }
    }
    *fmin_out = fmin;
}

__device__ float block_min_f(float v, float* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) red[w] = v;
    __syncthreads();
    float r = red[0];
    for (int i = 1; i < (int)(blockDim.x / 32); ++i) r = fminf(r, red[i]);
    __syncthreads();
    return r;
}

// Selection launches (core/population.hpp:409-517): mode 0 works on the 2P pool of fit[cur]
// and picks the survivors; mode 1 ranks the P population (initialisation); mode 2 does
// the same only for populations the diversity pass rebuilt (*nu < P).
__device__ __forceinline__ bool select_active(const PopDesc& d, int mode) {
    if (mode == 0) return !at_limit(d);
    if (mode == 2) return d.advanced && __ldg(d.nu) < d.P;
    return true;
}

// Ranks by bit-sliced peeling on a cluster of kPeelCluster CTAs per population.  CTA c
// owns columns [512c, 512c + 512) (16 words): their count planes, and for every front the
// sum of the member rows' words over those columns.  The front masks are exchanged through
// distributed shared memory with one cluster barrier per front, so the dominance rows are
// read by eight SMs instead of one.  Ranks -> domcnt[0, N).
//
// The pool of a generation (mode 0) is peeled only up to the front where the survivors
// (rank-0 points counted twice) first exceed P: that front is cut by crowding, and no
// later front is selected.  The points left then get that front's rank + 1 as one last
// front.  Selection, crowding of every selected point and the ranks kept for the next
// generation are the same as with every front peeled.
constexpr int kPeelCluster = 8, kPeelWords = 16, kPeelThreads = 256;
constexpr int kPeelSlices = kPeelThreads / kPeelWords, kPeelWarps = kPeelThreads / 32;

__global__ void __cluster_dims__(kPeelCluster, 1, 1) __launch_bounds__(kPeelThreads)
    nsga_peel_cluster_kernel(PopDesc* dd, int mode) {
    dep_wait();
    namespace cg = cooperative_groups;
    __shared__ uint32_t C[kCB][kPeelWords];  // count planes of the own words (two's complement)
    __shared__ uint32_t A[kPeelWords], V[kPeelWords];
    __shared__ uint32_t Floc[2][kPeelWords];  // own words of the next front, by front parity
    __shared__ uint16_t list[kMaxPool];
    __shared__ uint32_t s_nf[2];              // member count of front k, by front parity
    __shared__ uint32_t part[kPeelWarps][kDB][kPeelWords];
    __shared__ uint16_t r16[kPeelWords * 32];
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    PopDesc& d = dd[blockIdx.x / kPeelCluster];
    if (!select_active(d, mode)) return;  // the same decision in every CTA of the cluster
    const int N = (mode == 0) ? 2 * d.P : d.P;
    const int W = (N + 31) / 32;
    const uint32_t* __restrict__ S = d.domS;
    const int Wmax = d.domW;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int w0 = crank * kPeelWords;
    // domination counts of the own columns -> count planes; a generation's pool takes them
    // from the pool build's accumulator and leaves it zero for the next generation
    int32_t* const pacc = (mode == 0) ? pool_counts(d) : nullptr;
    for (int wl = warp; wl < kPeelWords; wl += kPeelWarps) {
        const int w = w0 + wl, i = 32 * w + lane;
        int c = 0;
        if (w < W && i < N) {
            if (pacc) {
                c = pacc[i];
                pacc[i] = 0;
            } else {
                c = __ldg(d.domcnt + i);
            }
        }
#pragma unroll
        for (int b = 0; b < kCB; ++b) {
            const uint32_t pl = __ballot_sync(0xffffffffu, (c >> b) & 1);
            if (lane == 0) C[b][wl] = pl;
        }
        const uint32_t v = __ballot_sync(0xffffffffu, w < W && i < N);
        if (lane == 0) V[wl] = v;
    }
    __syncthreads();
    // first front: zero counts
    if (t < kPeelWords) {
        uint32_t z = V[t];
#pragma unroll
        for (int b = 0; b < kCB; ++b) z &= ~C[b][t];
        A[t] = z;
        Floc[0][t] = z;
        for (uint32_t x = z; x; x &= x - 1) r16[32 * t + __ffs(x) - 1] = 0;
    }
    if (t == 0) {
        s_nf[0] = 0;
        s_nf[1] = 0;
    }
    cluster.sync();
    constexpr int NW = kPeelCluster * kPeelWords;
    int survivors = 0, rest = 0;
    // thread 0 of the cluster's first CTA records the front table (start of each front in
    // rank order, the cut front) for the grid-wide crowding and placement of mode 0
    int32_t* const ft = (crank == 0 && t == 0) ? d.nft : nullptr;
    int start = 0;
    for (int k = 0; k < N; ++k) {
        // the whole front k, gathered from every CTA of the cluster; its member list is
        // filled through one shared-memory atomic per warp (the order of the list does
        // not matter: the column sums, the crowding scan and the cut-front sort do not
        // depend on it)
        uint32_t fw = 0u;
        if (t < NW) fw = cluster.map_shared_rank(&Floc[k & 1][0], t / kPeelWords)[t % kPeelWords];
        {
            const uint32_t pc = __popc(fw);
            uint32_t inc = pc;  // inclusive prefix of the warp's counts
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            uint32_t wbase = 0u;
            if (lane == 31 && inc) wbase = atomicAdd(&s_nf[k & 1], inc);
            uint32_t base = __shfl_sync(0xffffffffu, wbase, 31) + inc - pc;
            for (uint32_t x = fw; x; x &= x - 1) list[base++] = (uint16_t)(32 * t + __ffs(x) - 1);
            if (t == 0) s_nf[(k + 1) & 1] = 0u;  // read by every thread before the last barrier
        }
        __syncthreads();
        const uint32_t nf = s_nf[k & 1];
        if (nf == 0) {  // every CTA sees the same front
            if (ft) {
                ft[0] = k;
                ft[1] = -1;
                ft[2 + k] = start;
            }
            break;
        }
        if (ft) ft[2 + k] = start;
        if (crank == 0 && d.nlist)
            for (int j = t; j < (int)nf; j += kPeelThreads) d.nlist[start + j] = list[j];
        start += (int)nf;
        if (mode == 0) {
            survivors += (k == 0) ? 2 * (int)nf : (int)nf;
            if (survivors > d.P) {
                rest = k + 1;
                if (ft) {  // the cut front k, then the points left as one last front
                    ft[1] = k;
                    ft[3 + k] = start;
                    ft[4 + k] = N;
                    ft[0] = (start < N) ? k + 2 : k + 1;
                }
                break;
            }
        }
        // column sums over the front's rows: thread (word t % 16, slice t / 16); the member
        // rows' words are loaded sixteen at a time (one L2 round trip for fronts of up to
        // 256 members) into 5-plane counters
        const int wl = t % kPeelWords, sl = t / kPeelWords, w = w0 + wl;
        uint32_t acc[kDB];
#pragma unroll
        for (int b = 0; b < kDB; ++b) acc[b] = 0u;
        if (w < W) {
            constexpr int kBatch = 16, kSP = 5;  // a batch counts up to 16: 5 planes
            for (int j0 = sl; j0 < (int)nf; j0 += kBatch * kPeelSlices) {
                uint32_t xs[kBatch];
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    const int j = j0 + u * kPeelSlices;
                    xs[u] = (j < (int)nf) ? __ldg(S + (size_t)list[j] * Wmax + w) : 0u;
                }
                uint32_t sv[kSP];
#pragma unroll
                for (int b = 0; b < kSP; ++b) sv[b] = 0u;
#pragma unroll
                for (int u = 0; u < kBatch; ++u) {
                    uint32_t c = xs[u];
#pragma unroll
                    for (int b = 0; b < kSP; ++b) {
                        const uint32_t nc = sv[b] & c;
                        sv[b] ^= c;
                        c = nc;
                    }
                }
                uint32_t cy = 0u;
#pragma unroll
                for (int b = 0; b < kSP; ++b) {
                    const uint32_t x = acc[b], y = sv[b];
                    acc[b] = x ^ y ^ cy;
                    cy = (x & y) | (cy & (x ^ y));
                }
#pragma unroll
                for (int b = kSP; b < kDB; ++b) {
                    const uint32_t x = acc[b];
                    acc[b] = x ^ cy;
                    cy = x & cy;
                }
            }
        }
        {  // the two slices of a warp (lanes l and l ^ 16 share a word)
            uint32_t cy = 0u;
#pragma unroll
            for (int b = 0; b < kDB; ++b) {
                const uint32_t o = __shfl_xor_sync(0xffffffffu, acc[b], 16);
                const uint32_t s2 = acc[b] ^ o ^ cy;
                cy = (acc[b] & o) | (cy & (acc[b] ^ o));
                acc[b] = s2;
            }
        }
        if (lane < kPeelWords)
#pragma unroll
            for (int b = 0; b < kDB; ++b) part[warp][b][wl] = acc[b];
        __syncthreads();
        if (t < kPeelWords) {
            uint32_t nz = 0u;
            if (w0 + t < W) {
                uint32_t sum[kDB];
#pragma unroll
                for (int b = 0; b < kDB; ++b) sum[b] = part[0][b][t];
                for (int wp = 1; wp < kPeelWarps; ++wp) {
                    uint32_t cy = 0u;
#pragma unroll
                    for (int b = 0; b < kDB; ++b) {
                        const uint32_t x = sum[b], y = part[wp][b][t];
                        sum[b] = x ^ y ^ cy;
                        cy = (x & y) | (cy & (x ^ y));
                    }
                }
                // decrement: doubled for the first front (its points are listed twice)
                uint32_t dec[kCB];
#pragma unroll
                for (int b = 0; b < kCB; ++b) dec[b] = 0u;
                if (k == 0) {
#pragma unroll
                    for (int b = 1; b < kCB; ++b) dec[b] = (b - 1 < kDB) ? sum[b - 1] : 0u;
                } else {
#pragma unroll
                    for (int b = 0; b < kDB; ++b) dec[b] = sum[b];
                }
                uint32_t bor = 0u, any = 0u;
#pragma unroll
                for (int b = 0; b < kCB; ++b) {
                    const uint32_t x = C[b][t];
                    const uint32_t dd2 = x ^ dec[b] ^ bor;
                    bor = (~x & dec[b]) | (~(x ^ dec[b]) & bor);
                    C[b][t] = dd2;
                    any |= dd2;
                }
                const uint32_t sign = C[kCB - 1][t];
                nz = (sign | ~any) & ~A[t] & V[t];
                A[t] |= nz;
                for (uint32_t x = nz; x; x &= x - 1) r16[32 * t + __ffs(x) - 1] = (uint16_t)(k + 1);
            }
            Floc[(k + 1) & 1][t] = nz;
        }
        cluster.sync();
    }
    cluster.sync();  // no CTA leaves while another may still read its front words
    for (int x = t; x < kPeelWords * 32; x += kPeelThreads) {
        const int i = 32 * w0 + x;
        if (i < N) d.domcnt[i] = ((A[x >> 5] >> (x & 31)) & 1u) ? r16[x] : (uint16_t)rest;
    }
}

// The pool ordered by (rank, objective o, index) for o = blockIdx.y, by exact counting:
// position(i) = #{j : key_j < key_i} over unique composite keys.  N^2 compares per
// objective spread over the grid; one warp per point.
constexpr int kOrdThreads = 1024, kOrdPerCta = kOrdThreads / 32;

__global__ void __launch_bounds__(kOrdThreads) nsga_order_kernel(PopDesc* dd, int mode) {
    dep_wait();
    extern __shared__ unsigned long long okeys[];  // [N]
    const PopDesc& d = dd[blockIdx.z];
    if (!select_active(d, mode)) return;
    const int N = (mode == 0) ? 2 * d.P : d.P;
    const int base = blockIdx.x * kOrdPerCta;
    if (base >= N) return;
    const int o = blockIdx.y, t = threadIdx.x;
    const float* f = d.fit[d.cur];
    staged<kOrdThreads, 4>(
        N, [&](int i) { return make_int2(__ldg(d.domcnt + i), __float_as_int(__ldg(f + 2 * i + o))); },
        [&](int i, int2 v) { okeys[i] = order_key(v.x, __int_as_float(v.y), i); });
    __syncthreads();
    const int lane = t & 31, i = base + (t >> 5);
    const unsigned long long me = (i < N) ? okeys[i] : 0ull;
    int cnt = 0;
#pragma unroll 8
    for (int j = lane; j < N; j += 32) cnt += (okeys[j] < me) ? 1 : 0;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    if (lane == 0 && i < N) d.nord[(size_t)o * 2 * d.P + cnt] = i;
}

// Mode 0 (the pool of a generation), one warp per pool point, over the members of its own
// front only (the peel's lists): its position in the front in each objective order, its
// neighbours and the front's extremes in both orders, so its crowding distance (the float
// operations of crowding_pass in the same order) and, for whole fronts before the cut, its
// survivor entries: front r starts at survivor entry first(r) + size(0) (rank-0 points
// count twice), members in objective-1 order, a rank-0 point as two adjacent entries; and
// the smallest first objective among them (atomic minimum of order keys).  Keys are
// (okey(value) << 32 | index); a value is recovered from its key.  CTAs take the points in
// rank order, kFrontWarps at a time, so a CTA's warps share a front, whose members' keys
// the CTA stages in shared memory once (a warp whose point lies in a later front reads
// that front from global memory).  Points of the last front of a peel stopped at the cut
// are never selected and are skipped.  Work: the sum of the squared front sizes instead
// of N^2 per objective.
constexpr int kFrontWarps = 8;

__device__ __forceinline__ float key_value(unsigned long long k) {
    const uint32_t o = (uint32_t)(k >> 32);
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// one member's two keys -> the running position, neighbours and extremes of the point
struct FrontScan {
    unsigned long long me0, me1;
    int below0 = 0, below1 = 0;
    unsigned long long lo0 = 0ull, hi0 = ~0ull, lo1 = 0ull, hi1 = ~0ull;  // neighbours (0 / ~0: none)
    unsigned long long mn0 = ~0ull, mx0 = 0ull, mn1 = ~0ull, mx1 = 0ull;  // front extremes
    __device__ __forceinline__ void add(unsigned long long k0, unsigned long long k1) {
        below0 += (k0 < me0) ? 1 : 0;
        below1 += (k1 < me1) ? 1 : 0;
        if (k0 < me0 && k0 > lo0) lo0 = k0;
        if (k0 > me0 && k0 < hi0) hi0 = k0;
        if (k1 < me1 && k1 > lo1) lo1 = k1;
        if (k1 > me1 && k1 < hi1) hi1 = k1;
        mn0 = k0 < mn0 ? k0 : mn0;
        mx0 = k0 > mx0 ? k0 : mx0;
        mn1 = k1 < mn1 ? k1 : mn1;
        mx1 = k1 > mx1 ? k1 : mx1;
    }
    __device__ __forceinline__ void reduce() {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            below0 += __shfl_xor_sync(0xffffffffu, below0, off);
            below1 += __shfl_xor_sync(0xffffffffu, below1, off);
            unsigned long long x;
            x = __shfl_xor_sync(0xffffffffu, lo0, off);
            lo0 = x > lo0 ? x : lo0;
            x = __shfl_xor_sync(0xffffffffu, hi0, off);
            hi0 = x < hi0 ? x : hi0;
            x = __shfl_xor_sync(0xffffffffu, lo1, off);
            lo1 = x > lo1 ? x : lo1;
            x = __shfl_xor_sync(0xffffffffu, hi1, off);
            hi1 = x < hi1 ? x : hi1;
            x = __shfl_xor_sync(0xffffffffu, mn0, off);
            mn0 = x < mn0 ? x : mn0;
            x = __shfl_xor_sync(0xffffffffu, mx0, off);
            mx0 = x > mx0 ? x : mx0;
            x = __shfl_xor_sync(0xffffffffu, mn1, off);
            mn1 = x < mn1 ? x : mn1;
            x = __shfl_xor_sync(0xffffffffu, mx1, off);
            mx1 = x > mx1 ? x : mx1;
        }
    }
};

__device__ __forceinline__ unsigned long long obj_key(float v, int j) {
    return ((unsigned long long)okey(v) << 32) | (uint32_t)j;
}

// one pool point of nsga_front_crowd_kernel (one warp): the scan of its front, then lane
// 0's crowding distance and survivor entries
// A survivor's keys and objectives into the other buffer, at entry q (and q2 >= 0: the
// second entry of a first-front point), by one warp: four 128-bit loads in flight per lane.
__device__ __forceinline__ void copy_survivor(const PopDesc& d, int src_row, int q, int q2, int lane) {
    const int ld4 = d.ld / 4, m = d.m, cur = d.cur;
    const float4* src = reinterpret_cast<const float4*>(d.keys[cur]) + (size_t)src_row * ld4;
    float4* dst = reinterpret_cast<float4*>(d.keys[cur ^ 1]) + (size_t)q * ld4;
    float4* dst2 = (q2 >= 0) ? reinterpret_cast<float4*>(d.keys[cur ^ 1]) + (size_t)q2 * ld4 : nullptr;
    int c = lane;
    for (; c + 96 < ld4; c += 128) {
        const float4 a0 = src[c], a1 = src[c + 32], a2 = src[c + 64], a3 = src[c + 96];
        dst[c] = a0;
        dst[c + 32] = a1;
        dst[c + 64] = a2;
        dst[c + 96] = a3;
        if (dst2) {
            dst2[c] = a0;
            dst2[c + 32] = a1;
            dst2[c + 64] = a2;
            dst2[c + 96] = a3;
        }
    }
    for (; c < ld4; c += 32) {
        const float4 a = src[c];
        dst[c] = a;
        if (dst2) dst2[c] = a;
    }
    if (lane < m) {
        const float v = d.fit[cur][(size_t)src_row * m + lane];
        d.fit[cur ^ 1][(size_t)q * m + lane] = v;
        if (q2 >= 0) d.fit[cur ^ 1][(size_t)q2 * m + lane] = v;
    }
}

__device__ __forceinline__ void front_crowd_point(const PopDesc& d, const int32_t* __restrict__ ft,
                                                  const float2* __restrict__ f2, const int32_t* __restrict__ list,
                                                  const uint2* fkeys, int r0, int lane, int i, int cut,
                                                  uint32_t* s_min) {
    const int r = __ldg(d.domcnt + i);
    const int fs = __ldg(ft + 2 + r), size = __ldg(ft + 3 + r) - fs;
    const float2 vi = __ldg(f2 + i);
    FrontScan sc;
    sc.me0 = obj_key(vi.x, i);
    sc.me1 = obj_key(vi.y, i);
    if (r == r0) {
        for (int j = lane; j < size; j += 32) {
            const uint2 k = fkeys[j];
            const int m = __ldg(list + fs + j);
            sc.add(((unsigned long long)k.x << 32) | (uint32_t)m, ((unsigned long long)k.y << 32) | (uint32_t)m);
        }
    } else {
        for (int j = lane; j < size; j += 32) {
            const int m = __ldg(list + fs + j);
            const float2 v = __ldg(f2 + m);
            sc.add(obj_key(v.x, m), obj_key(v.y, m));
        }
    }
    sc.reduce();  // every lane holds the front's figures
    float cd = 0.0f;
#pragma unroll
    for (int o = 0; o < 2; ++o) {
        const int p = o ? sc.below1 : sc.below0;  // position inside the front
        const bool edge = (r == 0) ? (size == 1 || p == 0 || p == size - 1) : (size <= 2 || p == 0 || p == size - 1);
        if (edge) {
            cd = INFINITY;
            continue;
        }
        const float range = __fsub_rn(key_value(o ? sc.mx1 : sc.mx0), key_value(o ? sc.mn1 : sc.mn0));
        if (range > 0.0f) {
            const float vp = key_value(o ? sc.lo1 : sc.lo0), vn = key_value(o ? sc.hi1 : sc.hi0);
            if (r == 0) {
                const float v = key_value(o ? sc.me1 : sc.me0);
                cd = __fadd_rn(__fadd_rn(cd, __fdiv_rn(__fsub_rn(v, vp), range)), __fdiv_rn(__fsub_rn(vn, v), range));
            } else {
                cd = __fadd_rn(cd, __fdiv_rn(__fsub_rn(vn, vp), range));
            }
        }
    }
    if (lane == 0) d.ncdp[i] = cd;
    if (r < cut) {
        const int q = (r == 0) ? 2 * sc.below1 : fs + __ldg(ft + 3) + sc.below1;
        if (lane == 0) {
            d.nsel[q] = i;
            d.nrank[q] = r;
            d.ncd[q] = cd;
            if (r == 0) {
                d.nsel[q + 1] = i;
                d.nrank[q + 1] = r;
                d.ncd[q + 1] = cd;
            }
            atomicMin(s_min, (uint32_t)(sc.me0 >> 32));
        }
        copy_survivor(d, i, q, (r == 0) ? q + 1 : -1, lane);
    }
}

__global__ void __launch_bounds__(kFrontWarps * 32) nsga_front_crowd_kernel(PopDesc* dd) {
    dep_wait();
    extern __shared__ uint2 fkeys[];  // [front size]: the staged front's (okey0, okey1)
    __shared__ int s_front[3];        // staged front: rank, first position, size
    __shared__ uint32_t s_min;        // the CTA's smallest first-objective key among survivors
    const PopDesc& d = dd[blockIdx.y];
    if (!select_active(d, 0)) return;
    const int N = 2 * d.P;
    const int32_t* __restrict__ ft = d.nft;
    const int cut = __ldg(ft + 1);
    const int end = (cut >= 0) ? __ldg(ft + 3 + cut) : N;  // positions of the fronts up to the cut
    const int pos0 = blockIdx.x * kFrontWarps;
    if (pos0 >= end) return;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const float2* __restrict__ f2 = reinterpret_cast<const float2*>(d.fit[d.cur]);
    const int32_t* __restrict__ list = d.nlist;
    if (t == 0) {
        const int r0 = __ldg(d.domcnt + __ldg(list + pos0));
        s_front[0] = r0;
        s_front[1] = __ldg(ft + 2 + r0);
        s_front[2] = __ldg(ft + 3 + r0) - s_front[1];
        s_min = 0xFFFFFFFFu;
    }
    __syncthreads();
    const int r0 = s_front[0], fs0 = s_front[1], size0 = s_front[2];
    staged<kFrontWarps * 32, 4>(
        size0, [&](int j) { return __ldg(f2 + __ldg(list + fs0 + j)); },
        [&](int j, float2 v) { fkeys[j] = make_uint2(okey(v.x), okey(v.y)); });
    __syncthreads();
    const int pos = pos0 + w;
    if (pos < end) front_crowd_point(d, ft, f2, list, fkeys, r0, lane, __ldg(list + pos), cut, &s_min);
    __syncthreads();
    if (t == 0 && s_min != 0xFFFFFFFFu) atomicMin(d.nfmin, s_min);
}

// Mode 0, over the grid, one warp per member of the cut front: the member's place among
// the front's entries in (crowding descending, index, copy) order, by counting the members
// with a smaller (crowding key, index) (every CTA stages the front's keys), a first-front
// point as two adjacent entries; entries before P - (entries of the whole fronts) become
// survivors, and the warp copies their rows into the other buffer (the front kernel has
// copied the whole fronts' rows).  The population's last CTA (completion counter) then
// finishes the generation: the history entry from the survivors' smallest first objective
// (the atomic minimum of order keys that both kernels feed), the buffer swap and the
// generation count.
__global__ void __launch_bounds__(kFrontWarps * 32) nsga_cut_kernel(PopDesc* dd) {
    dep_wait();
    extern __shared__ unsigned long long ckeys[];  // [cut front size]
    __shared__ uint32_t s_min;
    PopDesc& d = dd[blockIdx.y];
    if (at_limit(d)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) d.advanced = 0;
        return;
    }
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int32_t* __restrict__ ft = d.nft;
    const int cut = __ldg(ft + 1);
    const int fs = __ldg(ft + 2 + cut), nc = __ldg(ft + 3 + cut) - fs;
    const int j0 = blockIdx.x * kFrontWarps;
    if (t == 0) s_min = 0xFFFFFFFFu;
    if (j0 < nc) {  // every CTA reaches the completion count below
        const int mult = (cut == 0) ? 2 : 1;
        const int rb = (cut == 0) ? 0 : fs + __ldg(ft + 3);
        const int take = d.P - rb;
        const int32_t* __restrict__ mem = d.nlist + fs;
        staged<kFrontWarps * 32, 4>(
            nc, [&](int j) { return __ldg(mem + j); },
            [&](int j, int m) { ckeys[j] = ((unsigned long long)cd_key(__ldg(d.ncdp + m)) << 32) | (uint32_t)m; });
        __syncthreads();
        const int j = j0 + w;
        if (j < nc) {
            const unsigned long long me = ckeys[j];
            int c = 0;
            for (int k = lane; k < nc; k += 32) c += (ckeys[k] < me) ? 1 : 0;
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
            const int m = (int)(uint32_t)me, q0 = rb + mult * c;
            if (lane < mult && mult * c + lane < take) {
                const int q = q0 + lane;
                d.nsel[q] = m;
                d.nrank[q] = cut;
                d.ncd[q] = __ldg(d.ncdp + m);
                atomicMin(&s_min, okey(__ldg(d.fit[d.cur] + 2 * m)));
            }
            if (mult * c < take) copy_survivor(d, m, q0, (mult == 2 && 2 * c + 1 < take) ? q0 + 1 : -1, lane);
        }
    }
    __syncthreads();
    if (t == 0) {
        if (s_min != 0xFFFFFFFFu) atomicMin(d.nfmin, s_min);
        __threadfence();
        if (atomicAdd(d.done, 1) == (int)gridDim.x - 1) {
            // +inf when no survivor's first objective is a number; then the minimum's reset
            const uint32_t k = atomicExch(d.nfmin, 0xFFFFFFFFu);
            const uint32_t g = d.gen + 1;
            if (d.history && (int)g < d.hist_cap)
                d.history[g] = (k == 0xFFFFFFFFu) ? INFINITY
                                                  : __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
            d.cur ^= 1;
            d.gen = g;
            d.advanced = 1;
            *d.done = 0;
            __threadfence();
        }
    }
}

// crowding and (mode 0) survivors from the ranks and orders above; one CTA per population
__global__ void __launch_bounds__(kNsgaBlock, 1) nsga_select_kernel(PopDesc* dd, int mode) {
    dep_wait();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t wt32[32];
    __shared__ float redf[32];
    PopDesc& d = dd[blockIdx.x];
    if (!select_active(d, mode)) return;
    const int t = threadIdx.x;
    const int P = d.P;
    const int N = (mode == 0) ? 2 * P : P;
    const float* f = d.fit[d.cur];
    const SelSmem s = sel_carve(smem, N);
    staged<kNsgaBlock, 8>(2 * N, [&](int i) { return __ldg(f + i); }, [&](int i, float v) { s.obj[i] = v; });
    staged<kNsgaBlock, 4>(N, [&](int i) { return __ldg(d.domcnt + i); },
                          [&](int i, int v) { s.rank[i] = (uint16_t)v; });
    crowding_given<kNsgaBlock>(N, s, d.nord, 2 * P);
    float fmin = INFINITY;
    if (mode == 0) {
        select_given<kNsgaBlock>(N, P, s, d.nsel, d.nrank, d.ncd, &fmin, wt32);
    } else {
        for (int i = t; i < P; i += kNsgaBlock) {
            d.nrank[i] = s.rank[i];
            d.ncd[i] = s.cd[i];
            fmin = fminf(fmin, s.obj[2 * i]);
        }
    }
    fmin = block_min_f(fmin, redf);
    if (t == 0 && d.history) {
        const uint32_t g = (mode == 0) ? d.gen + 1 : d.gen;
        if ((int)g < d.hist_cap) d.history[g] = fmin;
    }
}

// ranks only (op API, any number of objectives): one CTA
__global__ void __launch_bounds__(kNsgaBlock) peel_op_kernel(int N, const uint32_t* S, const int32_t* cnt, int Wmax,
                                                             int32_t* rank) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t wt32[32];
    uint16_t* r16 = reinterpret_cast<uint16_t*>(smem);
    const PeelSmem ps = peel_carve(smem + (((size_t)N * 2 + 15) / 16) * 16, N);
    peel_ranks<kNsgaBlock>(N, S, Wmax, cnt, r16, ps, wt32);
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += kNsgaBlock) rank[i] = r16[i];
}

// ensure_minimum_diversity (core/population.hpp:130-182) runs after generation g when
// (g - 1) % interval == 0 (the reference's counter is g - 1).
__device__ __forceinline__ bool div_due(const PopDesc& d) {
    return d.advanced && d.div_interval > 0 && d.gen >= 1u && ((d.gen - 1u) % (uint32_t)d.div_interval) == 0u;
}

// The reference keeps a point when no earlier KEPT point is within distance 0.001 in
// objective space (float differences, squared and summed in double).  near_build_kernel
// records, per point c, which earlier points u < c are that close (bit u of row c of the
// dominance scratch); nsga_diversity_kernel then settles keep / drop in rounds: c is
// dropped as soon as a kept point is near it, kept once every near earlier point is
// settled as dropped.  The result is the reference's greedy in-order pass.
constexpr int kNearWarps = 4, kNearRows = 4;

__global__ void __launch_bounds__(kNearWarps * 32) near_build_kernel(PopDesc* dd) {
    dep_wait();
    extern __shared__ float2 so[];  // [32 * ceil(P / 32)]
    const PopDesc& d = dd[blockIdx.y];
    if (!div_due(d)) return;
    const int P = d.P, W = (P + 31) / 32;
    const int row0 = blockIdx.x * kNearWarps * kNearRows;
    if (row0 >= P) return;
    const float2* o2 = reinterpret_cast<const float2*>(d.fit[d.cur]);
    for (int j = threadIdx.x; j < 32 * W; j += blockDim.x) so[j] = (j < P) ? o2[j] : make_float2(0.0f, 0.0f);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = 0; r < kNearRows; ++r) {
        const int c = row0 + warp * kNearRows + r;
        if (c >= P) break;
        const float2 pc = so[c];
        uint32_t* row = d.domS + (size_t)c * d.domW;
        for (int w = 0; w <= c / 32; ++w) {
            const int u = 32 * w + lane;
            bool near = false;
            if (u < c) {
                const float2 pu = so[u];
                const double d0 = (double)__fsub_rn(pc.x, pu.x);
                const double d1 = (double)__fsub_rn(pc.y, pu.y);
                near = __dsqrt_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1))) < 0.001;
            }
            const uint32_t bits = __ballot_sync(0xffffffffu, near);
            if (lane == 0) row[w] = bits;
        }
    }
}

// Settles the pass (one CTA per population).  When fewer than 70% are kept, the kept rows
// are gathered in order into the other key buffer, which becomes the current one, and
// *nu < P tells the refill and re-rank launches to run; otherwise *nu = P.
__global__ void __launch_bounds__(kNsgaBlock) nsga_diversity_kernel(PopDesc* dd) {
    dep_wait();
    constexpr int WP = kMaxPool / 2 / 32;
    __shared__ uint32_t U[WP], D[WP], Un[WP], Dn[WP];
    __shared__ uint32_t wt32[32];
    PopDesc& d = dd[blockIdx.x];
    const int t = threadIdx.x, P = d.P, W = (P + 31) / 32;
    if (!div_due(d)) {
        if (t == 0) *d.nu = P;
        return;
    }
    for (int w = t; w < W; w += kNsgaBlock) U[w] = D[w] = Un[w] = Dn[w] = 0u;
    __syncthreads();
    // every round settles at least the lowest unsettled point, so P rounds suffice
    for (int round = 0; round <= P; ++round) {
        int open = 0;
        for (int c = t; c < P; c += kNsgaBlock) {
            if ((D[c >> 5] >> (c & 31)) & 1u) continue;
            const uint32_t* row = d.domS + (size_t)c * d.domW;
            const int last = c >> 5;
            bool kept_near = false, unsettled = false;
            for (int w = 0; w <= last; ++w) {
                uint32_t nb = __ldg(row + w);
                if (w == last) nb &= (1u << (c & 31)) - 1u;
                kept_near |= (nb & U[w]) != 0u;
                unsettled |= (nb & ~D[w]) != 0u;
            }
            if (kept_near) {
                atomicOr(&Dn[c >> 5], 1u << (c & 31));
            } else if (!unsettled) {
                atomicOr(&Un[c >> 5], 1u << (c & 31));
                atomicOr(&Dn[c >> 5], 1u << (c & 31));
            } else {
                open = 1;
            }
        }
        __syncthreads();
        for (int w = t; w < W; w += kNsgaBlock) {
            U[w] |= Un[w];
            D[w] |= Dn[w];
        }
        if (!__syncthreads_or(open)) break;
    }
    // kept points in index order -> nsel[0, nu)
    const int pc = (t < W) ? __popc(U[t]) : 0;
    uint32_t nu = 0;
    uint32_t pos = block_exclusive_scan<kNsgaBlock>((uint32_t)pc, wt32, &nu);
    if (t < W)
        for (uint32_t x = U[t]; x; x &= x - 1) d.nsel[pos++] = 32 * t + __ffs(x) - 1;
    __syncthreads();
    const double ratio = (double)nu / (double)P;
    if (!(ratio < 0.70)) {
        if (t == 0) *d.nu = P;
        return;
    }
    // gather the kept rows, in order, into the other buffer and make it current
    const int cur = d.cur, ld4 = d.ld / 4;
    const float4* src = reinterpret_cast<const float4*>(d.keys[cur]);
    float4* dst = reinterpret_cast<float4*>(d.keys[cur ^ 1]);
    const float* fs = d.fit[cur];
    float* fd = d.fit[cur ^ 1];
    const size_t total = (size_t)nu * ld4;
    for (size_t x = t; x < total; x += kNsgaBlock) {
        const int q = (int)(x / ld4), col = (int)(x % ld4);
        dst[x] = src[(size_t)d.nsel[q] * ld4 + col];
    }
    for (int q = t; q < (int)nu; q += kNsgaBlock) {
        fd[2 * q] = fs[2 * d.nsel[q]];
        fd[2 * q + 1] = fs[2 * d.nsel[q] + 1];
    }
    __syncthreads();
    if (t == 0) {
        d.cur = cur ^ 1;
        *d.nu = (int)nu;
    }
}

// ---------------------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------------------
int nsga_max_population() { return kMaxPool / 2; }

size_t nsga_select_smem(int maxP) { return sel_smem_bytes(2 * maxP); }

cudaError_t nsga_prepare(int maxP) {
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(nsga_select_kernel), sel_smem_bytes(2 * maxP));
    if (e == cudaSuccess)
        e = raise_smem_limit(reinterpret_cast<const void*>(nsga_order_kernel), (size_t)2 * maxP * 8);
    if (e == cudaSuccess)
        e = raise_smem_limit(reinterpret_cast<const void*>(near_build_kernel), (size_t)((maxP + 31) / 32) * 32 * 8);
    if (e == cudaSuccess)
        e = raise_smem_limit(reinterpret_cast<const void*>(nsga_cut_kernel), (size_t)2 * maxP * 8);
    if (e == cudaSuccess)
        e = raise_smem_limit(reinterpret_cast<const void*>(nsga_front_crowd_kernel), (size_t)2 * maxP * sizeof(uint2));
    return e;
}

// two-objective dominance rows of up to maxN points per population (grid.y)
static cudaError_t launch_dom2(const DomArgs& a, int maxN, int npops, cudaStream_t st) {
    constexpr int RPC = kDom2Rows * kDom2RowWarps;
    const size_t smem = (size_t)((maxN + 31) / 32) * 32 * sizeof(float2);
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(dom2_build_kernel), smem);
    if (e != cudaSuccess) return e;
    return launch_dep(dom2_build_kernel, dim3((maxN + RPC - 1) / RPC, npops), dim3(kDom2Warps * 32), smem, st, a);
}

static cudaError_t launch_dom(PopDesc* dd, int npops, int maxN, int only_rebuilt, cudaStream_t st) {
    DomArgs a;
    std::memset(&a, 0, sizeof(a));
    a.dd = dd;
    a.only_rebuilt = only_rebuilt;
    return launch_dom2(a, maxN, npops, st);
}

// ranks, crowding and (mode 0) survivors of every population of the group
cudaError_t nsga_enqueue_select(PopDesc* dd, int npops, int maxP, int mode, cudaStream_t st) {
    const int maxN = (mode == 0) ? 2 * maxP : maxP;
    cudaError_t e;
    if (mode == 0)
        e = launch_dep(dom2_pool_kernel, dim3(2 * device_sm_count(), npops), dim3(kSymWarps * 32), 0, st, dd);
    else
        e = launch_dom(dd, npops, maxN, mode == 2 ? 1 : 0, st);
    if (e != cudaSuccess) return e;
    e = launch_dep(nsga_peel_cluster_kernel, dim3(npops * kPeelCluster), dim3(kPeelThreads), 0, st, dd, mode);
    if (e != cudaSuccess) return e;
    if (mode == 0) {
        // a generation's pool: crowding and whole fronts from each point's own front, then
        // the cut front
        e = launch_dep(nsga_front_crowd_kernel, dim3((maxN + kFrontWarps - 1) / kFrontWarps, npops),
                       dim3(kFrontWarps * 32), (size_t)maxN * sizeof(uint2), st, dd);
        if (e != cudaSuccess) return e;
        return launch_dep(nsga_cut_kernel, dim3((maxN + kFrontWarps - 1) / kFrontWarps, npops), dim3(kFrontWarps * 32),
                          (size_t)maxN * 8, st, dd);
    }
    e = launch_dep(nsga_order_kernel, dim3((maxN + kOrdPerCta - 1) / kOrdPerCta, 2, npops), dim3(kOrdThreads),
                   (size_t)maxN * 8, st, dd, mode);
    if (e != cudaSuccess) return e;
    return launch_dep(nsga_select_kernel, dim3(npops), dim3(kNsgaBlock), sel_smem_bytes(maxN), st, dd, mode);
}

cudaError_t nsga_enqueue_diversity(PopDesc* dd, int npops, int maxP, cudaStream_t st) {
    constexpr int RPC = kNearWarps * kNearRows;
    const size_t smem = (size_t)((maxP + 31) / 32) * 32 * sizeof(float2);
    const cudaError_t e =
        launch_dep(near_build_kernel, dim3((maxP + RPC - 1) / RPC, npops), dim3(kNearWarps * 32), smem, st, dd);
    if (e != cudaSuccess) return e;
    return launch_dep(nsga_diversity_kernel, dim3(npops), dim3(kNsgaBlock), 0, st, dd);
}

int32_t nsga_alloc(PopDesc& d, int P, double mut_rate, int div_interval, int Mn, std::vector<void*>& allocs,
                   size_t* bytes, cudaStream_t stream) {
    const int N = 2 * P;
    const int W = (N + 31) / 32;
    auto get = [&](size_t b, void** p) -> int32_t {
        int32_t rc = dev_alloc(p, b ? b : 16, stream);
        if (rc != BRKGA_OK) return rc;
        allocs.push_back(*p);
        *bytes += b;
        return BRKGA_OK;
    };
    void* p = nullptr;
    int32_t st;
    if ((st = get((size_t)N * 4, &p)) != BRKGA_OK) return st;
    d.nrank = (int32_t*)p;
    if ((st = get((size_t)N * 4, &p)) != BRKGA_OK) return st;
    d.ncd = (float*)p;
    if ((st = get((size_t)P * 4, &p)) != BRKGA_OK) return st;
    d.nsel = (int32_t*)p;
    if ((st = get((size_t)N * W * 4, &p)) != BRKGA_OK) return st;
    d.domS = (uint32_t*)p;
    if ((st = get((size_t)N * 4, &p)) != BRKGA_OK) return st;
    d.domcnt = (int32_t*)p;
    if ((st = get(16, &p)) != BRKGA_OK) return st;
    d.nu = (int32_t*)p;
    if ((st = get((size_t)3 * N * 4, &p)) != BRKGA_OK) return st;  // two orders, then the pool counts
    d.nord = (int32_t*)p;
    if (cudaMemsetAsync(d.nord + 2 * (size_t)N, 0, (size_t)N * 4, stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(BRKGA_ERR_CUDA, "NSGA-II state initialisation");
    }
    if ((st = get((size_t)(N + 4) * 4, &p)) != BRKGA_OK) return st;
    d.nft = (int32_t*)p;
    if ((st = get((size_t)N * 4, &p)) != BRKGA_OK) return st;
    d.ncdp = (float*)p;
    if ((st = get((size_t)N * 4, &p)) != BRKGA_OK) return st;
    d.nlist = (int32_t*)p;
    if ((st = get(16, &p)) != BRKGA_OK) return st;
    d.nfmin = (uint32_t*)p;
    if (cudaMemsetAsync(d.nfmin, 0xFF, 4, stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(BRKGA_ERR_CUDA, "NSGA-II state initialisation");
    }
    d.domW = W;
    d.Mn = Mn;
    d.mutT = prob_threshold(mut_rate);
    d.div_interval = div_interval;
    return BRKGA_OK;
}

int32_t nsga_setup(NsgaState& s, Population& pop, PopDesc* dd, PopDesc& hdesc, const RowTile& tile, int grid,
                   bool stage) {
    s.dd = dd;
    s.P = pop.sh.Pi;
    s.N = 2 * pop.sh.Pi;
    if (s.P > nsga_max_population())
        return fail(BRKGA_ERR_UNSUPPORTED, "NSGA-II population above " + std::to_string(nsga_max_population()));
    s.n = pop.sh.n;
    s.ld = pop.sh.ld;
    s.kind = pop.pd->kind;
    s.max_points = points_of(*pop.pd);
    s.tile = tile;
    s.grid = grid;
    s.stage = stage;
    const double rate = (pop.prm.mutation_rate > 0.0) ? pop.prm.mutation_rate : 5.0 / (double)pop.sh.n;
    int32_t st = nsga_alloc(hdesc, s.P, rate, pop.prm.diversity_interval, pop.sh.Mn, pop.allocs, &pop.bytes,
                            pop.stream);
    if (st != BRKGA_OK) return st;
    s.div_interval = pop.prm.diversity_interval;
    cudaError_t e = cudaStreamSynchronize(pop.stream);
    if (e == cudaSuccess) e = cudaMemcpy(dd, &hdesc, sizeof(PopDesc), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "descriptor upload");
    e = nsga_prepare(s.P);
    if (e != cudaSuccess) return cuda_fail(e, "NSGA-II set-up");
    s.ready = true;
    return BRKGA_OK;
}

void nsga_release(NsgaState& s) { s.ready = false; }

void nsga_set_history(NsgaState& s, float* h, int cap) {
    s.history = h;
    s.hist_cap = cap;
}

static RowLaunch nsga_rows(const NsgaState& s, int mode) {
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.descs = s.dd;
    L.mode = mode;
    L.ntasks = s.P;
    L.max_n = s.n;
    L.max_points = s.max_points;
    L.stage_xy = s.stage ? 1 : 0;
    L.gscratch = s.gscratch;
    L.gstride = s.gstride;
    return L;
}

cudaError_t nsga_enqueue_rows(NsgaState& s, int mode, cudaStream_t st) {
    return launch_rows(nsga_rows(s, mode), s.kind, s.tile, s.grid, st);
}

cudaError_t nsga_enqueue_init(NsgaState& s, cudaStream_t st) {
    cudaError_t e = launch_rows(nsga_rows(s, MODE_INIT), s.kind, s.tile, s.grid, st);
    if (e != cudaSuccess) return e;
    return nsga_enqueue_select(s.dd, 1, s.P, 1, st);
}

bool nsga_diversity_due(const NsgaState& s, uint32_t g) {
    return s.div_interval > 0 && g >= 1u && ((g - 1u) % (uint32_t)s.div_interval) == 0u;
}

cudaError_t nsga_enqueue_generation(NsgaState& s, cudaStream_t st, bool with_diversity) {
    // offspring into pool rows [P, 2P) (core/solver.hpp:1019-1032) + their objectives
    cudaError_t e = launch_rows(nsga_rows(s, MODE_NSGA_OFF), s.kind, s.tile, s.grid, st);
    if (e != cudaSuccess) return e;
    // ranks, crowding and survivors of the pool (core/population.hpp:409-517), the
    // survivors' rows into the other buffer and the buffer swap
    if ((e = nsga_enqueue_select(s.dd, 1, s.P, 0, st)) != cudaSuccess) return e;
    if (with_diversity && s.div_interval > 0) {
        // decided on the device: due this generation, and fewer than 70% unique
        if ((e = nsga_enqueue_diversity(s.dd, 1, s.P, st)) != cudaSuccess) return e;
        if ((e = launch_rows(nsga_rows(s, MODE_NSGA_REFILL), s.kind, s.tile, s.grid, st)) != cudaSuccess) return e;
        e = nsga_enqueue_select(s.dd, 1, s.P, 2, st);
    }
    return e;
}

static int32_t read_desc(NsgaState& s, cudaStream_t st, PopDesc* d) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaMemcpy(d, s.dd, sizeof(PopDesc), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "descriptor read-back");
    return BRKGA_OK;
}

int32_t nsga_get_population(NsgaState& s, cudaStream_t st, float* keys, float* obj) {
    PopDesc d;
    int32_t rc = read_desc(s, st, &d);
    if (rc != BRKGA_OK) return rc;
    std::vector<float> hk((size_t)s.P * s.ld);
    cudaError_t e = cudaMemcpy(hk.data(), d.keys[d.cur], hk.size() * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && obj) e = cudaMemcpy(obj, d.fit[d.cur], (size_t)s.P * 2 * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "population read-back");
    if (keys)
        for (int r = 0; r < s.P; ++r) std::memcpy(keys + (size_t)r * s.n, hk.data() + (size_t)r * s.ld, (size_t)s.n * 4);
    return BRKGA_OK;
}

int32_t nsga_set_population(NsgaState& s, cudaStream_t st, const float* keys) {
    PopDesc d;
    int32_t rc = read_desc(s, st, &d);
    if (rc != BRKGA_OK) return rc;
    std::vector<float> hk((size_t)s.P * s.ld, 0.0f);
    for (int r = 0; r < s.P; ++r) std::memcpy(hk.data() + (size_t)r * s.ld, keys + (size_t)r * s.n, (size_t)s.n * 4);
    cudaError_t e = cudaMemcpy(d.keys[d.cur], hk.data(), hk.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "population upload");
    e = launch_rows(nsga_rows(s, MODE_EVAL), s.kind, s.tile, s.grid, st);
    if (e == cudaSuccess) e = nsga_enqueue_select(s.dd, 1, s.P, 1, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "population evaluate");
    return BRKGA_OK;
}

// best = the first-front member with the largest crowding distance (update_best_from_front,
// core/population.hpp:684-698), the first such index on ties
int32_t nsga_get_best(NsgaState& s, cudaStream_t st, float* keys, int32_t* perm, float* obj) {
    PopDesc d;
    int32_t rc = read_desc(s, st, &d);
    if (rc != BRKGA_OK) return rc;
    std::vector<int32_t> hr(s.P);
    std::vector<float> hc(s.P), ho((size_t)s.P * 2);
    cudaMemcpy(hr.data(), d.nrank, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), d.ncd, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
    cudaError_t e = cudaMemcpy(ho.data(), d.fit[d.cur], ho.size() * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "best read-back");
    int best = -1;
    for (int i = 0; i < s.P; ++i)
        if (hr[i] == 0 && (best < 0 || hc[i] > hc[best])) best = i;
    if (best < 0) best = 0;
    if (obj) {
        obj[0] = ho[2 * best];
        obj[1] = ho[2 * best + 1];
    }
    const float* row = d.keys[d.cur] + (size_t)best * s.ld;
    if (keys) {
        e = cudaMemcpy(keys, row, (size_t)s.n * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "best keys");
    }
    if (perm) {
        // decode on the device with the row kernel (same argsort as the generation step)
        float* tmpf = nullptr;
        int32_t* tmpp = nullptr;
        if (dev_alloc((void**)&tmpf, 16, st) != BRKGA_OK || dev_alloc((void**)&tmpp, (size_t)s.n * 4, st) != BRKGA_OK) {
            dev_free(tmpf, st);
            return fail(BRKGA_ERR_OOM, "decode scratch");
        }
        RowLaunch L;
        std::memset(&L, 0, sizeof(L));
        L.single = d;
        L.single.keys[0] = const_cast<float*>(row);
        L.single.fit[0] = tmpf;
        L.single.cur = 0;
        L.ntasks = 1;
        L.mode = MODE_EVAL;
        L.perm_out = tmpp;
        L.max_n = s.n;
        L.max_points = s.max_points;
        L.stage_xy = s.stage ? 1 : 0;
        L.gscratch = s.gscratch;
        L.gstride = s.gstride;
        e = launch_rows(L, s.kind, s.tile, 1, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaMemcpy(perm, tmpp, (size_t)s.n * 4, cudaMemcpyDeviceToHost);
        dev_free(tmpf, st);
        dev_free(tmpp, st);
        if (e != cudaSuccess) return cuda_fail(e, "best decode");
    }
    return BRKGA_OK;
}

int32_t nsga_get_front(NsgaState& s, cudaStream_t st, float* obj, float* keys, int32_t cap, int32_t* count) {
    PopDesc d;
    int32_t rc = read_desc(s, st, &d);
    if (rc != BRKGA_OK) return rc;
    std::vector<int32_t> hr(s.P);
    std::vector<float> ho((size_t)s.P * 2), hk((size_t)s.P * s.ld);
    cudaMemcpy(hr.data(), d.nrank, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(ho.data(), d.fit[d.cur], ho.size() * 4, cudaMemcpyDeviceToHost);
    cudaError_t e = cudaMemcpy(hk.data(), d.keys[d.cur], hk.size() * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "front read-back");
    int c = 0;
    for (int i = 0; i < s.P; ++i) {
        if (hr[i] != 0) continue;
        if (c < cap) {
            if (obj) {
                obj[2 * c] = ho[2 * i];
                obj[2 * c + 1] = ho[2 * i + 1];
            }
            if (keys) std::memcpy(keys + (size_t)c * s.n, hk.data() + (size_t)i * s.ld, (size_t)s.n * 4);
        }
        ++c;
    }
    *count = c;
    return BRKGA_OK;
}

// ---------------------------------------------------------------------------------------
// Pareto ranks for callers that cannot allocate device memory.  The dominance rows and
// counts live in a file-scope device array of fixed size (every GPU that loads the
// library holds it until the process exits); host code finds its device address with
// cudaGetSymbolAddress once per device, with that device current.
// ---------------------------------------------------------------------------------------
constexpr int kStaticMaxN = 2048;                       // largest point count it accepts
constexpr int kStaticW = (kStaticMaxN + 31) / 32;       // dominance row words
constexpr size_t kStaticWords = (size_t)kStaticMaxN * kStaticW + kStaticMaxN;  // rows + counts (532 KiB)
static __device__ __align__(256) uint32_t g_static_scratch[kStaticWords];

static std::mutex g_static_mu;
static std::map<int, uint32_t*> g_static_addr;  // device -> address of g_static_scratch

// per-device set-up on first use: the array's device address and the peel kernel's
// shared-memory limit (neither allocates device memory)
static int32_t static_scratch(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_static_mu);
    auto it = g_static_addr.find(dev);
    if (it != g_static_addr.end()) {
        *out = it->second;
        return BRKGA_OK;
    }
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress (static scratch)");
    const size_t smem = (((size_t)kStaticMaxN * 2 + 15) / 16) * 16 + peel_smem_bytes(kStaticMaxN);
    e = raise_smem_limit(reinterpret_cast<const void*>(peel_op_kernel), smem);
    if (e != cudaSuccess) return cuda_fail(e, "peel set-up");
    g_static_addr[dev] = (uint32_t*)ptr;
    *out = (uint32_t*)ptr;
    return BRKGA_OK;
}

// scratch of the operator entry points (grow-only, per device)
static std::mutex g_op_mu;
static std::map<int, std::pair<void*, size_t>> g_op_buf;

static int32_t op_scratch(size_t need, void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    auto& b = g_op_buf[dev];
    if (b.second < need) {
        if (b.first) {
            cudaDeviceSynchronize();
            cudaFree(b.first);
        }
        b = {nullptr, 0};
        if ((e = cudaMalloc(&b.first, need)) != cudaSuccess) {
            b.first = nullptr;
            cudaGetLastError();  // a failed allocation must not surface as a later launch's error
            return fail(BRKGA_ERR_OOM, std::string("operator scratch: ") + cudaGetErrorString(e));
        }
        b.second = need;
    }
    *out = b.first;
    return BRKGA_OK;
}

}  // namespace bk

using namespace bk;

extern "C" {

int32_t brkga_pareto_rank_bitmatrix(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream) {
    if (!d_obj || !d_rank) return fail(BRKGA_ERR_INVALID, "null argument");
    if (N < 0 || m < 1 || m > 4) return fail(BRKGA_ERR_INVALID, "need N >= 0 and 1 <= m <= 4");
    if (N == 0) return BRKGA_OK;
    if (N > 8192) return fail(BRKGA_ERR_UNSUPPORTED, "more than 8192 points");
    cudaStream_t st = (cudaStream_t)stream;
    const int W = (N + 31) / 32;
    const size_t sbytes = (size_t)N * W * 4, cbytes = (size_t)N * 4;
    const size_t doff = ((sbytes + cbytes + 255) / 256) * 256;  // a descriptor for the cluster peel
    std::lock_guard<std::mutex> lk(g_op_mu);
    void* buf = nullptr;
    int32_t rc = op_scratch(doff + sizeof(PopDesc), &buf);
    if (rc != BRKGA_OK) return rc;
    DomArgs a;
    std::memset(&a, 0, sizeof(a));
    a.obj = d_obj;
    a.rawN = N;
    a.m = m;
    a.S = (uint32_t*)buf;
    a.cnt = (int32_t*)((char*)buf + sbytes);
    a.Wmax = W;
    cudaError_t e;
    if (m == 2) {
        e = launch_dom2(a, N, 1, st);
    } else {
        dom_build_kernel<<<(N + 7) / 8, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "dominance launch");
    if (N <= kMaxPool) {
        // the engine's peel on a cluster of CTAs (ranks left in the counts), as for a
        // population of N rows in mode 1
        PopDesc hd;
        std::memset(&hd, 0, sizeof(hd));
        hd.P = N;
        hd.m = m;
        hd.domS = a.S;
        hd.domW = W;
        hd.domcnt = a.cnt;
        PopDesc* dd = reinterpret_cast<PopDesc*>((char*)buf + doff);
        if ((e = cudaMemcpyAsync(dd, &hd, sizeof(hd), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cuda_fail(e, "peel descriptor");
        nsga_peel_cluster_kernel<<<kPeelCluster, kPeelThreads, 0, st>>>(dd, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "peel launch");
        if ((e = cudaMemcpyAsync(d_rank, a.cnt, cbytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return cuda_fail(e, "rank copy");
    } else {
        const size_t smem = (((size_t)N * 2 + 15) / 16) * 16 + peel_smem_bytes(N);
        if ((e = raise_smem_limit(reinterpret_cast<const void*>(peel_op_kernel), smem)) != cudaSuccess)
            return cuda_fail(e, "peel set-up");
        peel_op_kernel<<<1, kNsgaBlock, smem, st>>>(N, a.S, a.cnt, W, d_rank);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "peel launch");
    }
    // the scratch is shared by later calls: finish before returning
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "peel");
    return BRKGA_OK;
}

int32_t brkga_pareto_rank_noalloc(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream) {
    if (!d_obj || !d_rank) return fail(BRKGA_ERR_INVALID, "null argument");
    if (N < 0 || m < 1 || m > 4) return fail(BRKGA_ERR_INVALID, "need N >= 0 and 1 <= m <= 4");
    if (N > kStaticMaxN)
        return fail(BRKGA_ERR_UNSUPPORTED, "brkga_pareto_rank_noalloc takes at most " + std::to_string(kStaticMaxN) +
                                               " points (got " + std::to_string(N) + "); use brkga_pareto_rank");
    if (N == 0) return BRKGA_OK;
    uint32_t* base = nullptr;
    int32_t rc = static_scratch(&base);
    if (rc != BRKGA_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int W = (N + 31) / 32;
    DomArgs a;
    std::memset(&a, 0, sizeof(a));
    a.obj = d_obj;
    a.rawN = N;
    a.m = m;
    a.S = base;                                        // rows [N][W]: every word is written
    a.cnt = (int32_t*)(base + (size_t)kStaticMaxN * kStaticW);  // counts [N]: every entry is written
    a.Wmax = W;
    dom_build_kernel<<<(N + 7) / 8, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "dominance launch");
    const size_t smem = (((size_t)N * 2 + 15) / 16) * 16 + peel_smem_bytes(N);
    peel_op_kernel<<<1, kNsgaBlock, smem, st>>>(N, a.S, a.cnt, W, d_rank);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "peel launch");
    return BRKGA_OK;
}

int32_t brkga_pareto_rank(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream) {
    return brkga_pareto_rank_bitmatrix(d_obj, N, m, d_rank, stream);
}

int32_t brkga_crowding(const float* d_obj, const int32_t* d_rank, int32_t N, int32_t m, float* d_cd, void* stream) {
    if (!d_obj || !d_rank || !d_cd) return fail(BRKGA_ERR_INVALID, "null argument");
    if (m != 2) return fail(BRKGA_ERR_UNSUPPORTED, "crowding kernel handles two objectives");
    if (N < 0 || N > kMaxPool) return fail(BRKGA_ERR_UNSUPPORTED, "N outside [0, 4096]");
    if (N == 0) return BRKGA_OK;
    cudaStream_t st = (cudaStream_t)stream;
    // the engine's crowding: orders by (rank, objective, index) on the grid, then the crowding
    // over them, as for a population of N points in mode 1; scratch from the stream-ordered
    // pool (orders [2][2N], ranks [N], the descriptor), returned behind the launches
    const size_t doff = (((size_t)5 * N * 4 + 255) / 256) * 256;
    void* p = nullptr;
    int32_t rc = dev_alloc(&p, doff + sizeof(PopDesc), st);
    if (rc != BRKGA_OK) return rc;
    PopDesc hd;
    std::memset(&hd, 0, sizeof(hd));
    hd.P = N;
    hd.m = 2;
    hd.fit[0] = const_cast<float*>(d_obj);
    hd.domcnt = const_cast<int32_t*>(d_rank);
    hd.nord = static_cast<int32_t*>(p);
    hd.nrank = static_cast<int32_t*>(p) + 4 * (size_t)N;
    hd.ncd = d_cd;
    PopDesc* dd = reinterpret_cast<PopDesc*>(static_cast<char*>(p) + doff);
    cudaError_t e = nsga_prepare((N + 1) / 2);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dd, &hd, sizeof(hd), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        nsga_order_kernel<<<dim3((N + kOrdPerCta - 1) / kOrdPerCta, 2, 1), kOrdThreads, (size_t)N * 8, st>>>(dd, 1);
        nsga_select_kernel<<<1, kNsgaBlock, sel_smem_bytes(N), st>>>(dd, 1);
        e = cudaGetLastError();
    }
    dev_free(p, st);
    if (e != cudaSuccess) return cuda_fail(e, "crowding launch");
    return BRKGA_OK;
}

}  // extern "C"
