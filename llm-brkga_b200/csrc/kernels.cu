// kernels.cu -- the per-generation hot path on sm_100a.
//
// One CTA owns one chromosome row at a time (persistent grid, rows strided over CTAs):
//   1. build the row in registers: elite copy, biased crossover of two parent rows
//      (128-bit loads, Philox coins), mutant fill, or a load of given keys;
//   2. write it to the next population buffer (128-bit stores);
//   3. decode it: stable argsort of the keys in shared memory -- a bucket scatter
//      (bucket = floor(key * B), monotone in key) followed by an exact rank inside each
//      bucket by (key, index), so ties go to the lower index exactly like the
//      reference's std::sort over (key, index) pairs (configs/tsp_config.hpp:206-225);
//   4. fitness from the permutation: closed tour length from coordinates staged in
//      shared memory (or a distance matrix), the depot tour of the bi-objective TSP,
//      or the knapsack decoders; FP32 tour sums use one fixed order (256 virtual lanes,
//      xor butterflies, fixed 8-way tree) that the oracle restates bit for bit.
// The elite partition ranks (fitness key, row) composites by exact counting across the
// grid (rank_kernel below).
#include <climits>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.h"

namespace bk {

// ---------------------------------------------------------------------------------------
// shared-memory carve-up for the row kernel
// ---------------------------------------------------------------------------------------
struct RowSmem {
    uint32_t* cnt;            // bucket counters / offsets, NB + 1
    unsigned long long* sc;   // scattered (okey << 32 | index) composites, n
    int32_t* perm;            // decoded permutation, n
    float* xy;                // staged coordinates (1 or 2 sets)
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// bucket counters: 4 * groups * block buckets (>= n) plus a sentinel, padded to 16 bytes
__host__ __device__ inline size_t cnt_words(int block, int groups) { return (size_t)4 * groups * block + 4; }

constexpr size_t kRowSmemCap = 227 * 1024;  // opt-in dynamic shared memory per CTA

size_t row_smem_bytes(const RowTile& t, int max_n, int max_points, int kind, bool stage_xy) {
    size_t b = align_up(cnt_words(t.block, t.groups) * 4, 16);
    b += align_up((size_t)max_n * 8, 16);
    b += align_up((size_t)max_n * 4, 16);
    if (stage_xy && (kind == TSP_COORDS || kind == BITSP_COORDS))
        b += (size_t)max_points * 8 * (kind == BITSP_COORDS ? 2 : 1);
    return b;
}

__device__ __forceinline__ RowSmem carve(unsigned char* base, int block, int groups, int max_n, int max_points) {
    RowSmem s;
    size_t off = 0;
    s.cnt = reinterpret_cast<uint32_t*>(base + off);
    off += align_up(cnt_words(block, groups) * 4, 16);
    s.sc = reinterpret_cast<unsigned long long*>(base + off);
    off += align_up((size_t)max_n * 8, 16);
    s.perm = reinterpret_cast<int32_t*>(base + off);
    off += align_up((size_t)max_n * 4, 16);
    s.xy = reinterpret_cast<float*>(base + off);
    (void)max_points;
    return s;
}

// ---------------------------------------------------------------------------------------
// decode: stable argsort of one row held in registers (k[g][l] is key index
// 4 * (threadIdx.x + g * BLOCK) + l)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int bucket_of(float key, float nbf, int nb) {
    // monotone in okey order: negatives -> 0; [0,1) -> floor(key * nb); >= 1, +inf, NaN -> nb-1
    if (!(key >= 0.0f)) return (key != key) ? nb - 1 : 0;
    const float t = __fmul_rn(key, nbf);
    const int b = (t < nbf) ? (int)t : nb - 1;
    return b < nb - 1 ? b : nb - 1;
}

// The exact rank inside a bucket scans the bucket, so its cost is the sum of the squared
// bucket sizes.  Keys in [0,1) spread over about one per bucket; equal keys, keys outside
// [0,1) (one bucket each side) or NaNs (the last bucket) pile into few buckets.  A row with
// a bucket above kHeavyBucket keys is sorted instead by an ascending bitonic network over
// its composites: O(n log^2 n) on any input, and the same (key, index) order.
constexpr uint32_t kHeavyBucket = 32;

// Ascending sort of a[0, n) (shared or global memory) by the whole block, any n: the
// bitonic network in its one-direction form (each merge of size k first compares i with
// its mirror inside the k-block, then half-cleaners of stride k/4 .. 1), with a[i] for
// i >= n taken as +infinity.  Such an element is always the higher index of its pair and
// would stay put, so pairs that reach past n are skipped and nothing is padded.
template <int BLOCK>
__device__ void block_sort_u64(unsigned long long* a, int n) {
    const int t = threadIdx.x;
    int n2 = 1;
    while (n2 < n) n2 <<= 1;
    const int half = n2 >> 1;
    for (int k = 2; k <= n2; k <<= 1) {
        const int hk = k >> 1;
        for (int p = t; p < half; p += BLOCK) {
            const int base = (p / hk) * k, x = p % hk;
            const int i = base + x, j = base + k - 1 - x;
            if (j < n) {
                const unsigned long long u = a[i], v = a[j];
                if (v < u) {
                    a[i] = v;
                    a[j] = u;
                }
            }
        }
        __syncthreads();
        for (int st = k >> 2; st > 0; st >>= 1) {
            for (int p = t; p < half; p += BLOCK) {
                const int i = ((p & ~(st - 1)) << 1) | (p & (st - 1));
                const int j = i + st;
                if (j < n) {
                    const unsigned long long u = a[i], v = a[j];
                    if (v < u) {
                        a[i] = v;
                        a[j] = u;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// the permutation of a heavy row: each segment's composites sorted, then their indices;
// called rather than inlined, so the row kernels keep their registers for the common path
template <int BLOCK>
__device__ __noinline__ void heavy_row_perm(unsigned long long* sc, int32_t* perm, int n, int split) {
    block_sort_u64<BLOCK>(sc, split);
    if (split < n) block_sort_u64<BLOCK>(sc + split, n - split);
    for (int p = threadIdx.x; p < n; p += BLOCK) perm[p] = (int32_t)(uint32_t)sc[p];
    __syncthreads();
}

// Counters must be zero on entry; they are left holding bucket offsets (the caller
// re-zeroes them while it no longer needs them).  Bucket count NB = 4 * G * BLOCK >= n,
// thread t owns the contiguous buckets [4Gt, 4Gt + 4G) for the scan.
// Keys [split, n) form a second segment sorted on its own (TSPJ's job keys after its city
// keys): it takes the upper half of the buckets, so no bucket mixes the segments and
// positions [split, n) of the permutation hold the second segment's order.  A heavy row
// sorts each segment's composites on its own: the scatter has put the first segment's in
// [0, split).
template <int BLOCK, int G>
__device__ void row_argsort(const float (&k)[G][4], int n, int split, const RowSmem& s, uint32_t* warp_tot) {
    constexpr int KB = 4 * G, NB = KB * BLOCK;
    const int t = threadIdx.x;
    const int nbs = (split < n) ? NB / 2 : NB;
    const float nbf = (float)nbs;
    uint32_t bs[G][4];  // (bucket << 16) | slot
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n) {
                const int b = bucket_of(k[g][l], nbf, nbs) + ((i >= split) ? nbs : 0);
                const uint32_t slot = atomicAdd(&s.cnt[b], 1u);
                bs[g][l] = ((uint32_t)b << 16) | slot;
            }
        }
    __syncthreads();
    uint4 c[G];
    uint32_t sum = 0, big = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        c[g] = reinterpret_cast<const uint4*>(s.cnt)[t * G + g];
        sum += c[g].x + c[g].y + c[g].z + c[g].w;
        big = max(big, max(max(c[g].x, c[g].y), max(c[g].z, c[g].w)));
    }
    uint32_t run = block_exclusive_scan<BLOCK>(sum, warp_tot, nullptr);
#pragma unroll
    for (int g = 0; g < G; ++g) {
        uint4 o;
        o.x = run;
        o.y = o.x + c[g].x;
        o.z = o.y + c[g].y;
        o.w = o.z + c[g].z;
        run = o.w + c[g].w;
        reinterpret_cast<uint4*>(s.cnt)[t * G + g] = o;
    }
    if (t == 0) s.cnt[NB] = (uint32_t)n;
    const bool heavy = __syncthreads_or(big > kHeavyBucket) != 0;
    // scatter composites
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n) {
                const uint32_t b = bs[g][l] >> 16, slot = bs[g][l] & 0xFFFFu;
                s.sc[s.cnt[b] + slot] = ((unsigned long long)okey(k[g][l]) << 32) | (uint32_t)i;
            }
        }
    __syncthreads();
    if (heavy) {
        heavy_row_perm<BLOCK>(s.sc, s.perm, n, split);
        return;
    }
    // exact rank inside the bucket
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n) {
                const uint32_t b = bs[g][l] >> 16;
                const uint32_t b0 = s.cnt[b], b1 = s.cnt[b + 1];
                const unsigned long long me = ((unsigned long long)okey(k[g][l]) << 32) | (uint32_t)i;
                uint32_t r = b0;
                if constexpr (G > 1) {
                    // long rows: buckets of up to four keys (nearly all of them for keys in
                    // [0,1)) take predicated steps without a loop, larger ones continue in
                    // the loop (TSP n = 5000 and knapsack n = 10 000 rows 3 % faster; the
                    // one-group tiles measured 1 % slower with it and keep the plain loop)
#pragma unroll
                    for (uint32_t u = 0; u < 4; ++u)
                        if (b0 + u < b1) r += (s.sc[b0 + u] < me) ? 1u : 0u;
                    for (uint32_t q = b0 + 4; q < b1; ++q) r += (s.sc[q] < me) ? 1u : 0u;
                } else {
                    for (uint32_t q = b0; q < b1; ++q) r += (s.sc[q] < me) ? 1u : 0u;
                }
                s.perm[r] = i;
            }
        }
    __syncthreads();
}

// zero the bucket counters (4 * G * BLOCK + 1 words) with 128-bit stores
template <int BLOCK, int G>
__device__ __forceinline__ void zero_counters(const RowSmem& s) {
    uint4* c = reinterpret_cast<uint4*>(s.cnt);
    for (int i = threadIdx.x; i < G * BLOCK + 1; i += BLOCK) c[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ---------------------------------------------------------------------------------------
// fitness
// ---------------------------------------------------------------------------------------
// Euclidean edge exactly as the reference builds its matrix (configs/tsp_config.hpp:366-368):
// float dx, dy; sqrt(dx*dx + dy*dy), no contraction, correctly rounded sqrt
__device__ __forceinline__ float edge_xy(const float* xy, int a, int b) {
    const float2 pa = reinterpret_cast<const float2*>(xy)[a];
    const float2 pb = reinterpret_cast<const float2*>(xy)[b];
    const float dx = __fsub_rn(pa.x, pb.x);
    const float dy = __fsub_rn(pa.y, pb.y);
    return __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

// canonical FP32 sum of nedges edge terms: 256 virtual lanes, xor butterflies inside each
// group of 32 lanes, fixed tree over the 8 group totals
template <int BLOCK, int NOBJ, typename EdgeF>
__device__ __forceinline__ void canon_sum(int nedges, EdgeF edge, float* red, float* out) {
    constexpr int LPT = BLOCK >= 256 ? 1 : 256 / BLOCK;
    const int t = threadIdx.x, lane = t & 31;
    float acc[LPT][NOBJ];
#pragma unroll
    for (int j = 0; j < LPT; ++j) {
#pragma unroll
        for (int o = 0; o < NOBJ; ++o) acc[j][o] = 0.0f;
        const int vl = t + j * BLOCK;
        if (vl < 256) {
            for (int e = vl; e < nedges; e += 256) {
                float d[NOBJ];
                edge(e, d);
#pragma unroll
                for (int o = 0; o < NOBJ; ++o) acc[j][o] = __fadd_rn(acc[j][o], d[o]);
            }
        }
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1)
#pragma unroll
        for (int j = 0; j < LPT; ++j)
#pragma unroll
            for (int o = 0; o < NOBJ; ++o) acc[j][o] = __fadd_rn(acc[j][o], __shfl_xor_sync(0xffffffffu, acc[j][o], m));
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < LPT; ++j) {
            const int vl = t + j * BLOCK;
            if (vl < 256) {
#pragma unroll
                for (int o = 0; o < NOBJ; ++o) red[o * 8 + (vl >> 5)] = acc[j][o];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int o = 0; o < NOBJ; ++o) {
        const float* g = red + o * 8;
        out[o] = __fadd_rn(__fadd_rn(__fadd_rn(g[0], g[1]), __fadd_rn(g[2], g[3])),
                           __fadd_rn(__fadd_rn(g[4], g[5]), __fadd_rn(g[6], g[7])));
    }
}

// exclusive block scan of two 64-bit values at once (red: 64 entries)
template <int BLOCK>
__device__ __forceinline__ void block_excl_scan_ll2(long long a, long long b, long long* red, long long* ea,
                                                    long long* eb, long long* ta, long long* tb) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = a, y = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long xu = __shfl_up_sync(0xffffffffu, x, o);
        const long long yu = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) {
            x += xu;
            y += yu;
        }
    }
    if (lane == 31) {
        red[w] = x;
        red[32 + w] = y;
    }
    __syncthreads();
    if (w == 0) {
        long long sx = (lane < NW) ? red[lane] : 0ll, sy = (lane < NW) ? red[32 + lane] : 0ll;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long xu = __shfl_up_sync(0xffffffffu, sx, o);
            const long long yu = __shfl_up_sync(0xffffffffu, sy, o);
            if (lane >= o) {
                sx += xu;
                sy += yu;
            }
        }
        if (lane < NW) {
            red[lane] = sx;
            red[32 + lane] = sy;
        }
    }
    __syncthreads();
    *ea = ((w > 0) ? red[w - 1] : 0ll) + x - a;
    *eb = ((w > 0) ? red[32 + w - 1] : 0ll) + y - b;
    *ta = red[NW - 1];
    *tb = red[32 + NW - 1];
    __syncthreads();
}

// knapsack greedy in key order: prefix of the sorted items that fits, then a
// first-fit scan of the rest by warp 0 (weights must be >= 0).  The items' (weight, value)
// pairs are first gathered in key order into wv ([n], free scratch after the argsort) by
// the whole block, so the scans read on-chip data instead of one dependent round of loads
// per 32 items.
template <int BLOCK>
__device__ float knap_greedy(const int32_t* perm, int n, const int2* __restrict__ items, long long C,
                             long long* red, long long* shared_misc, int2* wv) {
    const int t = threadIdx.x;
    // one 8-byte load per item from the interleaved (weight, value) table: an item's pair
    // sits in one cache line, so the random gather touches half the lines of two tables
    for (int p = t; p < n; p += BLOCK) wv[p] = __ldg(items + perm[p]);
    __syncthreads();
    const int ch = (n + BLOCK - 1) / BLOCK;
    const int p0 = t * ch, p1 = min(n, p0 + ch);
    long long ws = 0, vs = 0;
    for (int p = p0; p < p1; ++p) {
        const int2 x = wv[p];
        ws += x.x;
        vs += x.y;
    }
    long long S, V, totw, totv;
    block_excl_scan_ll2<BLOCK>(ws, vs, red, &S, &V, &totw, &totv);
    // the prefix: positions whose inclusive prefix weight stays <= C.  Weights are >= 0, so
    // the prefix weight only grows and exactly one position breaks it (none when every item
    // fits); the thread holding it records the prefix's weight, length and value
    if (t == 0 && totw <= C) {
        shared_misc[0] = totw;
        shared_misc[1] = n;
        shared_misc[2] = totv;
    }
    for (int p = p0; p < p1; ++p) {
        const int2 x = wv[p];
        if (S <= C && S + x.x > C) {
            shared_misc[0] = S;
            shared_misc[1] = p;
            shared_misc[2] = V;
        }
        S += x.x;
        V += x.y;
    }
    __syncthreads();
    const long long f = shared_misc[1], v0 = shared_misc[2];
    long long vt = 0;
    if (t < 32 && f < n) {
        // the spare capacity left by the prefix is below the weight of the item that broke
        // it, so it fits in 32 bits from here on; four chunks of 32 items are loaded before
        // they are walked, so the walk waits for one load round per 128 items
        int r = (int)(C - shared_misc[0]);
        for (int b0 = (int)f + 1; b0 < n; b0 += 128) {
            int2 x[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int pos = b0 + 32 * c + t;
                x[c] = (pos < n) ? wv[pos] : make_int2(INT_MAX, 0);
            }
            // one vote for the 128 items: once the spare capacity is small most groups hold
            // no item that fits, and the walk passes them without stepping chunk by chunk
            if (!__any_sync(0xffffffffu, x[0].x <= r || x[1].x <= r || x[2].x <= r || x[3].x <= r)) continue;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                int cur = 0;
                for (;;) {
                    const unsigned mask = __ballot_sync(0xffffffffu, t >= cur && x[c].x <= r);
                    if (!mask) break;
                    const int j = __ffs(mask) - 1;
                    r -= __shfl_sync(0xffffffffu, x[c].x, j);
                    vt += __shfl_sync(0xffffffffu, x[c].y, j);
                    cur = j + 1;
                }
            }
        }
    }
    __syncthreads();
    return (float)(v0 + vt);
}

// the same, called rather than inlined: in the one-group row kernels (48 registers) an
// inlined copy spills registers on every kind's path
template <int BLOCK>
__device__ __noinline__ float knap_greedy_call(const int32_t* perm, int n, const int2* __restrict__ items,
                                               long long C, long long* red, long long* shared_misc, int2* wv) {
    return knap_greedy<BLOCK>(perm, n, items, C, red, shared_misc, wv);
}

// TSPJ makespan (configs/tspj_config.hpp:555-585): the city tour from the depot (node 0)
// and back; at each position the arrival time plus the duration of the job type assigned
// to that position; the larger of the tour length and the latest job completion.  perm[0,
// c) is the city order (cities perm+1), perm[c, 2c) the job order (types perm-c+1).  One
// warp adds in the reference's own sequential order, so the value equals the reference's
// fitness function bit for bit.
template <int BLOCK>
__device__ float tspj_makespan(const int32_t* perm, int nc, const float* __restrict__ travel,
                               const float* __restrict__ jobs, float* red) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        const size_t D = (size_t)nc + 1;
        float run = 0.0f, mjc = 0.0f;
        for (int c0 = 0; c0 < nc; c0 += 32) {
            const int i = c0 + lane;
            float e = 0.0f, jd = 0.0f;
            if (i < nc) {
                const int city = perm[i] + 1;
                const int prev = (i == 0) ? 0 : perm[i - 1] + 1;
                const int job = perm[nc + i] - nc + 1;
                e = __ldg(travel + (size_t)prev * D + city);
                jd = __ldg(jobs + (size_t)city * D + job);
            }
            const int cnt = min(32, nc - c0);
            for (int q = 0; q < cnt; ++q) {
                run = __fadd_rn(run, __shfl_sync(0xffffffffu, e, q));
                const float jc = __fadd_rn(run, __shfl_sync(0xffffffffu, jd, q));
                mjc = (mjc < jc) ? jc : mjc;
            }
        }
        const float tt = __fadd_rn(run, __ldg(travel + (size_t)(perm[nc - 1] + 1) * D));
        if (lane == 0) red[0] = (tt < mjc) ? mjc : tt;
    }
    __syncthreads();
    const float v = red[0];
    __syncthreads();
    return v;
}

// The same for tours of up to 128 cities, called rather than inlined (one-group row
// kernels): every lane issues the loads of all its positions before the first sequential
// step, so the walk waits for one round of loads instead of one per 32 cities.
template <int BLOCK>
__device__ __noinline__ float tspj_makespan_call(const int32_t* perm, int nc, const float* __restrict__ travel,
                                                 const float* __restrict__ jobs, float* red) {
    constexpr int kChunks = 4;
    if (nc > 32 * kChunks) return tspj_makespan<BLOCK>(perm, nc, travel, jobs, red);
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        const size_t D = (size_t)nc + 1;
        float e[kChunks], jd[kChunks];
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            const int i = 32 * c + lane;
            e[c] = 0.0f;
            jd[c] = 0.0f;
            if (i < nc) {
                const int city = perm[i] + 1;
                const int prev = (i == 0) ? 0 : perm[i - 1] + 1;
                const int job = perm[nc + i] - nc + 1;
                e[c] = __ldg(travel + (size_t)prev * D + city);
                jd[c] = __ldg(jobs + (size_t)city * D + job);
            }
        }
        float run = 0.0f, mjc = 0.0f;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            const int cnt = min(32, nc - 32 * c);
            for (int q = 0; q < cnt; ++q) {
                run = __fadd_rn(run, __shfl_sync(0xffffffffu, e[c], q));
                const float jc = __fadd_rn(run, __shfl_sync(0xffffffffu, jd[c], q));
                mjc = (mjc < jc) ? jc : mjc;
            }
        }
        const float tt = __fadd_rn(run, __ldg(travel + (size_t)(perm[nc - 1] + 1) * D));
        if (lane == 0) red[0] = (tt < mjc) ? mjc : tt;
    }
    __syncthreads();
    const float v = red[0];
    __syncthreads();
    return v;
}

// ContinuousOptGPUConfig (configs/continuous_opt_gpu_config.hpp:114-173): x = key * (upper -
// lower) + lower; sphere sum x^2; Rastrigin 10 n + sum (x^2 - 10 cos(2 pi x)); Rosenbrock
// sum 100 (x_{i+1} - x_i^2)^2 + (1 - x_i)^2.  keys in index order (shared or global memory).
// One warp adds the terms in the reference's sequential order, so sphere and Rosenbrock
// equal the reference's values bit for bit; Rastrigin goes through the device cosf.
template <int BLOCK>
__device__ float continuous_fitness(const float* keys, int n, int fn, float lo, float hi, float* red) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        const float range = __fsub_rn(hi, lo);
        const float two_pi = __fmul_rn(2.0f, 3.14159265358979323846f);
        float sum = (fn == FN_RASTRIGIN) ? __fmul_rn(10.0f, (float)n) : 0.0f;
        const int terms = (fn == FN_ROSENBROCK) ? n - 1 : n;
        for (int c0 = 0; c0 < terms; c0 += 32) {
            const int i = c0 + lane;
            float term = 0.0f;
            if (i < terms) {
                const float x = __fadd_rn(__fmul_rn(keys[i], range), lo);
                if (fn == FN_SPHERE) {
                    term = __fmul_rn(x, x);
                } else if (fn == FN_RASTRIGIN) {
                    term = __fsub_rn(__fmul_rn(x, x), __fmul_rn(10.0f, cosf(__fmul_rn(two_pi, x))));
                } else {
                    const float xn = __fadd_rn(__fmul_rn(keys[i + 1], range), lo);
                    const float t1 = __fsub_rn(xn, __fmul_rn(x, x));
                    const float t2 = __fsub_rn(1.0f, x);
                    term = __fadd_rn(__fmul_rn(__fmul_rn(100.0f, t1), t1), __fmul_rn(t2, t2));
                }
            }
            const int cnt = min(32, terms - c0);
            for (int q = 0; q < cnt; ++q) sum = __fadd_rn(sum, __shfl_sync(0xffffffffu, term, q));
        }
        if (lane == 0) red[0] = sum;
    }
    __syncthreads();
    const float v = red[0];
    __syncthreads();
    return v;
}

// JobSchedulingGPUConfig (configs/job_scheduling_gpu_config.hpp:132-148): job i goes to
// machine (int)(key_i * machines), capped at machines - 1; each machine's load adds its
// jobs in index order; the makespan is the largest load.  Lane l of warp w keeps machine
// 32 w + l (and every BLOCK-th after it) and adds the jobs of each 32-job chunk in order,
// so every load equals the reference's sequential float sum bit for bit.
template <int BLOCK>
__device__ float jobsched_makespan(const float* keys, int n, const float* __restrict__ jt, int M, float* red) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float mf = (float)M;
    float best = -INFINITY;
    for (int m0 = warp * 32; m0 < M; m0 += BLOCK) {
        float load = 0.0f;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int i = c0 + lane;
            int mid = -1;
            float v = 0.0f;
            if (i < n) {
                int mm = (int)__fmul_rn(keys[i], mf);
                mid = mm >= M ? M - 1 : (mm < 0 ? 0 : mm);
                v = __ldg(jt + i);
            }
            const int cnt = min(32, n - c0);
            for (int q = 0; q < cnt; ++q) {
                const int mq = __shfl_sync(0xffffffffu, mid, q);
                const float vq = __shfl_sync(0xffffffffu, v, q);
                if (mq == m0 + lane) load = __fadd_rn(load, vq);
            }
        }
        if (m0 + lane < M) best = (best < load) ? load : best;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const float other = __shfl_xor_sync(0xffffffffu, best, o);
        best = (best < other) ? other : best;
    }
    if (lane == 0) red[warp] = best;
    __syncthreads();
    float r = red[0];
    for (int w = 1; w < NW; ++w) r = (r < red[w]) ? red[w] : r;
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------------------
// the fused row kernel
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int tourn(int i1, int i2, const int32_t* rank, const float* cd) {
    const int r1 = __ldg(rank + i1), r2 = __ldg(rank + i2);
    if (r1 < r2) return i1;
    if (r2 < r1) return i2;
    if (__ldg(cd + i1) > __ldg(cd + i2)) return i1;
    return i2;
}

// residency target: 1280 threads per SM for one float4 group per thread, 1024 otherwise
// (measured at n = 1000: 5 CTAs of 256 with 51 registers beat 6 with 40 and 8 with 32)
template <int BLOCK, int G>
struct RowResidency {
    static constexpr int want = (G == 1 ? 1280 : 1024) / BLOCK;
    static constexpr int value = want < 1 ? 1 : (want > 32 ? 32 : want);
};

template <int BLOCK, int G, bool DYN>
__global__ void __launch_bounds__(BLOCK, RowResidency<BLOCK, G>::value) row_kernel(RowLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ PopDesc sd;
    __shared__ uint32_t warp_tot[32];
    __shared__ long long red_ll[64];
    __shared__ float red_f[32];
    __shared__ long long misc[4];

    __shared__ int grab[2];

    const int t = threadIdx.x;
    const RowSmem s = carve(smem_raw, BLOCK, G, L.max_n, L.max_points);
    int cur_pid = -1;
    zero_counters<BLOCK, G>(s);
    dep_wait();  // shared memory only above this line

    // tasks are dealt to CTAs in groups of K consecutive tasks: neighbouring rows of one
    // population stay in one CTA (its descriptor and coordinates are staged once per
    // group).  Statically, group g goes to CTA g % grid.  With dynamic dealing (DYN, the
    // shared launches of batches and the server, whose rows differ in length and kind), a
    // CTA takes the next group from the work counter whenever it finishes one, so no SM
    // idles while another still holds several long rows.
    const int K = L.task_group > 1 ? L.task_group : 1;
    if (DYN) {
        if (t == 0) grab[0] = atomicAdd(L.work, K);
        __syncthreads();
    }
    int round = 0;
    for (int g0 = DYN ? grab[0] : blockIdx.x * K; g0 < L.ntasks;) {
        int next = 0;
        if (DYN && t == 0) next = atomicAdd(L.work, K);  // the following group, used after this one
    for (int task = g0; task < min(L.ntasks, g0 + K); ++task) {
        int pid = 0, r = task;
        if (L.tasks) {
            const Task tk = L.tasks[task];
            pid = tk.pid;
            r = tk.row;
        }
        if (pid != cur_pid) {
            __syncthreads();
            if (t == 0) sd = L.descs ? L.descs[pid] : L.single;
            __syncthreads();
            if (L.stage_xy && (sd.kind == TSP_COORDS || sd.kind == BITSP_COORDS)) {
                const int npts = (sd.kind == BITSP_COORDS) ? sd.n + 1 : sd.n;
                const float2* g0 = reinterpret_cast<const float2*>(sd.xy);
                float2* d0 = reinterpret_cast<float2*>(s.xy);
                for (int i = t; i < npts; i += BLOCK) d0[i] = g0[i];
                if (sd.kind == BITSP_COORDS) {
                    const float2* g1 = reinterpret_cast<const float2*>(sd.xy2);
                    for (int i = t; i < npts; i += BLOCK) d0[npts + i] = g1[i];
                }
            }
            __syncthreads();
            cur_pid = pid;
        }
        const int n = sd.n, ld = sd.ld, P = sd.P, E = sd.E, M = sd.M, m = sd.m;
        const int cur = sd.cur;
        if ((L.mode == MODE_GEN || L.mode == MODE_NSGA_OFF) && at_limit(sd)) continue;
        if (L.mode == MODE_NSGA_REFILL && !sd.advanced) continue;
        if (!L.tasks && L.mode == MODE_GEN) r = (task < P - E) ? E + task : task - (P - E);
        // local search: task = rank q; the row is the q-th best (the operator form works on
        // rows in rank order already)
        const int lsq = r;
        if (L.mode == MODE_LSEARCH) {
            if (!L.ls_force && (!ls_due(sd) || at_limit(sd))) continue;
            if (!L.ls_force) r = __ldg(sd.sorted + lsq);
        }

        float k[G][4];
        float* dst = nullptr;
        float* dfit = nullptr;
        bool eval = true, store = true;
        const uint32_t isl = sd.island << 8;
        // how the row is built: BUILD_LOAD (given keys), BUILD_COPY (elite), BUILD_RANDOM
        // (fresh keys from one stream), BUILD_CROSS (biased crossover), BUILD_NSGA
        // (uniform crossover + per-gene reset)
        enum { BUILD_LOAD, BUILD_COPY, BUILD_RANDOM, BUILD_CROSS, BUILD_NSGA };
        int build = BUILD_LOAD;
        uint32_t gdraw = 0, tag0 = 0;
        const float* src = sd.keys[cur];
        int pa = 0, pb = 0;
        if (L.mode == MODE_GEN) {
            dst = sd.keys[cur ^ 1];
            dfit = sd.fit[cur ^ 1];
            gdraw = sd.gen + 1;
            if (r < E) {
                build = BUILD_COPY;
            } else if (r < P - M) {
                // biased crossover (core/solver.hpp:1109-1135; core/cuda_kernels.cuh:120-134)
                build = BUILD_CROSS;
                tag0 = isl | TAG_COIN;
                int2 prk;
                if (sd.parents) {
                    prk = sd.parents[r];
                } else {
                    const uint4 pr = draw4(sd.seed, 0u, (uint32_t)r, gdraw, isl | TAG_PARENT);
                    prk = make_int2((int)pick(pr.x, (uint32_t)E), E + (int)pick(pr.y, (uint32_t)(P - E)));
                }
                pa = __ldg(sd.sorted + prk.x);
                pb = __ldg(sd.sorted + prk.y);
            } else {
                build = BUILD_RANDOM;  // mutant (core/solver.hpp:1244-1258)
                tag0 = isl | TAG_MUTANT;
            }
        } else if (L.mode == MODE_INIT) {
            // Population::initialize keys (core/population.hpp:107-110)
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            build = BUILD_RANDOM;
            tag0 = isl | TAG_INIT;
        } else if (L.mode == MODE_NSGA_OFF) {
            // NSGA-II offspring (core/solver.hpp:1019-1091): pool rows [P, 2P) of keys[cur]
            dst = sd.keys[cur] + (size_t)P * ld;
            dfit = sd.fit[cur] + (size_t)P * m;
            gdraw = sd.gen + 1;
            if (r >= P - sd.Mn) {
                build = BUILD_RANDOM;
                tag0 = TAG_MUTANT;
            } else {
                build = BUILD_NSGA;
                tag0 = TAG_NSGA_COIN;
                const uint4 pk = draw4(sd.seed, 0u, (uint32_t)r, gdraw, TAG_NSGA_TOUR);
                pa = tourn(pick(pk.x, P), pick(pk.y, P), sd.nrank, sd.ncd);
                pb = tourn(pick(pk.z, P), pick(pk.w, P), sd.nrank, sd.ncd);
            }
        } else if (L.mode == MODE_NSGA_REFILL) {
            // ensure_minimum_diversity refill (core/population.hpp:166-171): rows from the
            // unique count on are replaced by fresh random keys of generation sd.gen
            if (r < __ldg(sd.nu)) continue;
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            gdraw = sd.gen;
            build = BUILD_RANDOM;
            tag0 = TAG_NSGA_REFILL;
        } else if (L.mode == MODE_LSEARCH) {
            // random 2-opt (core/cuda_kernels.cuh:166-246): the row is rewritten in place, and
            // only when the search improved it
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            store = false;
        } else {  // MODE_EVAL: given keys
            dfit = sd.fit[cur];
            store = false;
        }

        if (build == BUILD_COPY) {
            // elite copy (core/population.hpp:700-714), fitness kept
            const int sr = __ldg(sd.sorted + r);
            const float4* a = reinterpret_cast<const float4*>(src + (size_t)sr * ld);
            float4* o = reinterpret_cast<float4*>(dst + (size_t)r * ld);
            for (int q = t; q < ld / 4; q += BLOCK) o[q] = __ldg(a + q);
            if (t < m) dfit[(size_t)r * m + t] = __ldg(sd.fit[cur] + (size_t)sr * m + t);
            eval = false;
            store = false;
        } else if (build == BUILD_LOAD) {
            const float* row = src + (size_t)r * ld;
            const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
#pragma unroll
            for (int gg = 0; gg < G; ++gg) {
                const int q = t + gg * BLOCK;
                if (vec && 4 * q + 3 < ld) {
                    const float4 a = __ldg(reinterpret_cast<const float4*>(row) + q);
                    k[gg][0] = a.x;
                    k[gg][1] = a.y;
                    k[gg][2] = a.z;
                    k[gg][3] = a.w;
                } else {
#pragma unroll
                    for (int l = 0; l < 4; ++l) k[gg][l] = (4 * q + l < n) ? __ldg(row + 4 * q + l) : 0.0f;
                }
            }
        } else {
            const float4* A = reinterpret_cast<const float4*>(src + (size_t)pa * ld);
            const float4* Bv = reinterpret_cast<const float4*>(src + (size_t)pb * ld);
#pragma unroll
            for (int gg = 0; gg < G; ++gg) {
                const int q = t + gg * BLOCK;
                if (4 * q < n) {
                    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
                    if (build != BUILD_RANDOM) {
                        a = __ldg(A + q);
                        b = __ldg(Bv + q);
                    }
                    // one Philox call site per group for every way a row is built
                    const uint4 x = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, tag0);
                    if (build == BUILD_RANDOM) {
                        k[gg][0] = u24(x.x);
                        k[gg][1] = u24(x.y);
                        k[gg][2] = u24(x.z);
                        k[gg][3] = u24(x.w);
                    } else {
                        const uint32_t T = sd.rhoT;
                        k[gg][0] = ((x.x >> 8) < T) ? a.x : b.x;
                        k[gg][1] = ((x.y >> 8) < T) ? a.y : b.y;
                        k[gg][2] = ((x.z >> 8) < T) ? a.z : b.z;
                        k[gg][3] = ((x.w >> 8) < T) ? a.w : b.w;
                    }
                    if (build == BUILD_NSGA) {
                        const uint4 mp = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTP);
                        const uint4 mk = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTK);
                        const uint32_t T = sd.mutT;
                        if ((mp.x >> 8) < T) k[gg][0] = u24(mk.x);
                        if ((mp.y >> 8) < T) k[gg][1] = u24(mk.y);
                        if ((mp.z >> 8) < T) k[gg][2] = u24(mk.z);
                        if ((mp.w >> 8) < T) k[gg][3] = u24(mk.w);
                    }
                }
            }
        }

        if (L.mode == MODE_LSEARCH) {
            // reverse random segments [i, j] of the city keys (the first n/2 genes), as the
            // reference's random_2opt_kernel: i, j uniform over the cities, ordered, skipped
            // when j - i < 2; the composites buffer is free until the decode
            const int c = n / 2;
            float* sk = reinterpret_cast<float*>(s.sc);
#pragma unroll
            for (int gg = 0; gg < G; ++gg)
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const int i = 4 * (t + gg * BLOCK) + l;
                    if (i < c) sk[i] = k[gg][l];
                }
            __syncthreads();
            for (int mv = 0; mv < L.ls_moves; ++mv) {
                const uint4 x = draw4(sd.seed, (uint32_t)mv, (uint32_t)lsq, sd.gen, isl | TAG_LS);
                int i = (int)pick(x.x, (uint32_t)c), j = (int)pick(x.y, (uint32_t)c);
                if (i > j) {
                    const int tmp = i;
                    i = j;
                    j = tmp;
                }
                if (j - i >= 2)
                    for (int p = t; p < (j - i + 1) / 2; p += BLOCK) {
                        const float u = sk[i + p];
                        sk[i + p] = sk[j - p];
                        sk[j - p] = u;
                    }
                __syncthreads();
            }
#pragma unroll
            for (int gg = 0; gg < G; ++gg)
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const int i = 4 * (t + gg * BLOCK) + l;
                    if (i < c) k[gg][l] = sk[i];
                }
            __syncthreads();
        }

        if (store) {
            // write the new row with 128-bit stores; padding lanes (>= n) are zero
            float4* o = reinterpret_cast<float4*>(dst + (size_t)r * ld);
#pragma unroll
            for (int gg = 0; gg < G; ++gg) {
                const int q = t + gg * BLOCK;
                if (4 * q < ld) {
                    float4 v;
                    v.x = (4 * q + 0 < n) ? k[gg][0] : 0.0f;
                    v.y = (4 * q + 1 < n) ? k[gg][1] : 0.0f;
                    v.z = (4 * q + 2 < n) ? k[gg][2] : 0.0f;
                    v.w = (4 * q + 3 < n) ? k[gg][3] : 0.0f;
                    o[q] = v;
                }
            }
        }

        if (eval) {
            float res[2] = {0.0f, 0.0f};
            const int kind = sd.kind;
            if (kind == KNAP_THRESHOLD) {
                // configs/knapsack_config.hpp:43-62 (integer sums are exact as floats below 2^24)
                long long tw = 0, tv = 0;
#pragma unroll
                for (int gg = 0; gg < G; ++gg)
#pragma unroll
                    for (int l = 0; l < 4; ++l) {
                        const int i = 4 * (t + gg * BLOCK) + l;
                        if (i < n && k[gg][l] > 0.5f) {
                            tw += __ldg(sd.w + i);
                            tv += __ldg(&sd.wv[i].y);
                        }
                    }
                tw = block_sum_ll<BLOCK>(tw, red_ll);
                tv = block_sum_ll<BLOCK>(tv, red_ll);
                const float twf = (float)tw, tvf = (float)tv;
                res[0] = (twf > sd.cap) ? __fsub_rn(tvf, __fmul_rn(__fsub_rn(twf, sd.cap), 1000.0f)) : tvf;
            } else if (kind == CONTINUOUS || kind == JOBSCHED) {
                // no decode: the keys in index order, staged where the sort composites go
                float* sk = reinterpret_cast<float*>(s.sc);
#pragma unroll
                for (int gg = 0; gg < G; ++gg)
#pragma unroll
                    for (int l = 0; l < 4; ++l) {
                        const int i = 4 * (t + gg * BLOCK) + l;
                        if (i < n) sk[i] = k[gg][l];
                    }
                __syncthreads();
                res[0] = (kind == CONTINUOUS) ? continuous_fitness<BLOCK>(sk, n, sd.function, sd.lo, sd.hi, red_f)
                                              : jobsched_makespan<BLOCK>(sk, n, sd.jt, sd.machines, red_f);
            } else {
                row_argsort<BLOCK, G>(k, n, (kind == TSPJ) ? n / 2 : n, s, warp_tot);
                zero_counters<BLOCK, G>(s);  // ready for the next row (separated by the row-end barrier)
                const int32_t* perm = s.perm;
                if (kind == TSP_COORDS) {
                    const float* xy = L.stage_xy ? s.xy : sd.xy;
                    canon_sum<BLOCK, 1>(n, [&](int e, float* d) {
                        const int a = perm[e], b = perm[(e + 1 < n) ? e + 1 : 0];
                        d[0] = edge_xy(xy, a, b);
                    }, red_f, res);
                } else if (kind == TSP_MATRIX) {
                    const float* mat = sd.mat;
                    canon_sum<BLOCK, 1>(n, [&](int e, float* d) {
                        const int a = perm[e], b = perm[(e + 1 < n) ? e + 1 : 0];
                        d[0] = __ldg(mat + (size_t)a * n + b);
                    }, red_f, res);
                } else if (kind == BITSP_COORDS) {
                    const int npts = n + 1;
                    const float* xy0 = L.stage_xy ? s.xy : sd.xy;
                    const float* xy1 = L.stage_xy ? s.xy + 2 * npts : sd.xy2;
                    canon_sum<BLOCK, 2>(n + 1, [&](int e, float* d) {
                        const int a = (e == 0) ? 0 : perm[e - 1] + 1;
                        const int b = (e == n) ? 0 : perm[e] + 1;
                        d[0] = edge_xy(xy0, a, b);
                        d[1] = edge_xy(xy1, a, b);
                    }, red_f, res);
                } else if (kind == BITSP_MATRIX) {
                    const float* m0 = sd.mat;
                    const float* m1 = sd.mat2;
                    const size_t np1 = (size_t)n + 1;
                    canon_sum<BLOCK, 2>(n + 1, [&](int e, float* d) {
                        const int a = (e == 0) ? 0 : perm[e - 1] + 1;
                        const int b = (e == n) ? 0 : perm[e] + 1;
                        d[0] = __ldg(m0 + (size_t)a * np1 + b);
                        d[1] = __ldg(m1 + (size_t)a * np1 + b);
                    }, red_f, res);
                } else if (kind == KNAP_GREEDY) {
                    if constexpr (G == 1)
                        res[0] = knap_greedy_call<BLOCK>(s.perm, n, sd.wv, sd.capi, red_ll, misc,
                                                         reinterpret_cast<int2*>(s.sc));
                    else
                        res[0] = knap_greedy<BLOCK>(s.perm, n, sd.wv, sd.capi, red_ll, misc,
                                                    reinterpret_cast<int2*>(s.sc));
                } else if (kind == TSPJ) {
                    if constexpr (G == 1)
                        res[0] = tspj_makespan_call<BLOCK>(perm, n / 2, sd.mat, sd.mat2, red_f);
                    else
                        res[0] = tspj_makespan<BLOCK>(perm, n / 2, sd.mat, sd.mat2, red_f);
                }
                if (L.perm_out) {
                    int32_t* po = L.perm_out + (size_t)r * n;
                    for (int i = t; i < n; i += BLOCK) po[i] = perm[i];
                }
            }
            if (L.mode == MODE_LSEARCH) {
                // keep the searched row only if it is better (restore_if_worse_kernel)
                const float old = dfit[(size_t)r * m];
                if (sd.maximize ? (res[0] > old) : (res[0] < old)) {
                    __syncthreads();  // every thread has read the old value
                    float4* o = reinterpret_cast<float4*>(dst + (size_t)r * ld);
#pragma unroll
                    for (int gg = 0; gg < G; ++gg) {
                        const int q = t + gg * BLOCK;
                        if (4 * q < ld) {
                            float4 v;
                            v.x = (4 * q + 0 < n) ? k[gg][0] : 0.0f;
                            v.y = (4 * q + 1 < n) ? k[gg][1] : 0.0f;
                            v.z = (4 * q + 2 < n) ? k[gg][2] : 0.0f;
                            v.w = (4 * q + 3 < n) ? k[gg][3] : 0.0f;
                            o[q] = v;
                        }
                    }
                    if (t == 0) dfit[(size_t)r * m] = res[0];
                }
            } else {
                if (t == 0) dfit[(size_t)r * m] = res[0];
                if (t == 1 && m > 1) dfit[(size_t)r * m + 1] = res[1];
            }
        }
        __syncthreads();
    }
        if (DYN) {
            ++round;
            if (t == 0) grab[round & 1] = next;
            __syncthreads();
            g0 = grab[round & 1];
        } else {
            g0 += gridDim.x * K;
        }
    }
    if (DYN && t == 0 && atomicAdd(L.work + 1, 1) == (int)gridDim.x - 1) {
        // every CTA has taken its last group: leave the counter zero for the next launch
        L.work[0] = 0;
        L.work[1] = 0;
    }
}

// ---------------------------------------------------------------------------------------
// rows beyond shared memory: the same build, bucket argsort and canonical sums, with the
// sort's counters, composites and permutation in a per-CTA slice of global scratch
// (L2-resident at these sizes) and the keys re-read from the row between passes.  One CTA
// of 1024 threads per row; results equal the in-shared-memory kernel's bit for bit (the
// sort order and the summation order do not depend on the tile).
// ---------------------------------------------------------------------------------------
constexpr int kBigBlock = 1024;

__host__ __device__ inline size_t big_cnt_bytes(int max_n) {
    return align_up((size_t)(round_up(max_n, kBigBlock) + 1) * 4, 256);
}
__host__ __device__ inline size_t big_perm_bytes(int max_n) { return align_up((size_t)max_n * 4, 256); }

size_t row_global_stride(int max_n) { return big_cnt_bytes(max_n) + big_perm_bytes(max_n) + align_up((size_t)max_n * 8, 256); }

__global__ void __launch_bounds__(kBigBlock) row_kernel_big(RowLaunch L) {
    constexpr int BLOCK = kBigBlock;
    __shared__ PopDesc sd;
    __shared__ uint32_t warp_tot[32];
    __shared__ long long red_ll[64];
    __shared__ float red_f[32];
    __shared__ long long misc[4];
    const int t = threadIdx.x;
    unsigned char* base = static_cast<unsigned char*>(L.gscratch) + (size_t)blockIdx.x * L.gstride;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base);                               // [NB + 1]
    int32_t* perm = reinterpret_cast<int32_t*>(base + big_cnt_bytes(L.max_n));       // slots, then the permutation
    unsigned long long* sc =
        reinterpret_cast<unsigned long long*>(base + big_cnt_bytes(L.max_n) + big_perm_bytes(L.max_n));
    const int NBmax = round_up(L.max_n, BLOCK);
    for (int j = t; j <= NBmax; j += BLOCK) cnt[j] = 0u;
    __syncthreads();
    int cur_pid = -1;

    for (int task = blockIdx.x; task < L.ntasks; task += gridDim.x) {
        int pid = 0, r = task;
        if (L.tasks) {
            const Task tk = L.tasks[task];
            pid = tk.pid;
            r = tk.row;
        }
        if (pid != cur_pid) {
            __syncthreads();
            if (t == 0) sd = L.descs ? L.descs[pid] : L.single;
            __syncthreads();
            cur_pid = pid;
        }
        const int n = sd.n, ld = sd.ld, P = sd.P, E = sd.E, M = sd.M, m = sd.m;
        const int cur = sd.cur;
        if ((L.mode == MODE_GEN || L.mode == MODE_NSGA_OFF) && at_limit(sd)) continue;
        if (L.mode == MODE_NSGA_REFILL && !sd.advanced) continue;
        if (!L.tasks && L.mode == MODE_GEN) r = (task < P - E) ? E + task : task - (P - E);
        // local search: task = rank q; the row is the q-th best (the operator form works on
        // rows in rank order already)
        const int lsq = r;
        if (L.mode == MODE_LSEARCH) {
            if (!L.ls_force && (!ls_due(sd) || at_limit(sd))) continue;
            if (!L.ls_force) r = __ldg(sd.sorted + lsq);
        }

        enum { BUILD_LOAD, BUILD_COPY, BUILD_RANDOM, BUILD_CROSS, BUILD_NSGA };
        int build = BUILD_LOAD;
        float* dst = nullptr;
        float* dfit = nullptr;
        bool store = true;
        const uint32_t isl = sd.island << 8;
        uint32_t gdraw = 0, tag0 = 0;
        const float* src = sd.keys[cur];
        int pa = 0, pb = 0;
        if (L.mode == MODE_GEN) {
            dst = sd.keys[cur ^ 1];
            dfit = sd.fit[cur ^ 1];
            gdraw = sd.gen + 1;
            if (r < E) {
                build = BUILD_COPY;
            } else if (r < P - M) {
                build = BUILD_CROSS;  // core/solver.hpp:1109-1135
                tag0 = isl | TAG_COIN;
                int2 prk;
                if (sd.parents) {
                    prk = sd.parents[r];
                } else {
                    const uint4 pr = draw4(sd.seed, 0u, (uint32_t)r, gdraw, isl | TAG_PARENT);
                    prk = make_int2((int)pick(pr.x, (uint32_t)E), E + (int)pick(pr.y, (uint32_t)(P - E)));
                }
                pa = __ldg(sd.sorted + prk.x);
                pb = __ldg(sd.sorted + prk.y);
            } else {
                build = BUILD_RANDOM;  // core/solver.hpp:1244-1258
                tag0 = isl | TAG_MUTANT;
            }
        } else if (L.mode == MODE_INIT) {
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            build = BUILD_RANDOM;
            tag0 = isl | TAG_INIT;
        } else if (L.mode == MODE_NSGA_OFF) {
            dst = sd.keys[cur] + (size_t)P * ld;
            dfit = sd.fit[cur] + (size_t)P * m;
            gdraw = sd.gen + 1;
            if (r >= P - sd.Mn) {
                build = BUILD_RANDOM;
                tag0 = TAG_MUTANT;
            } else {
                build = BUILD_NSGA;
                tag0 = TAG_NSGA_COIN;
                const uint4 pk = draw4(sd.seed, 0u, (uint32_t)r, gdraw, TAG_NSGA_TOUR);
                pa = tourn(pick(pk.x, P), pick(pk.y, P), sd.nrank, sd.ncd);
                pb = tourn(pick(pk.z, P), pick(pk.w, P), sd.nrank, sd.ncd);
            }
        } else if (L.mode == MODE_NSGA_REFILL) {
            if (r < __ldg(sd.nu)) continue;
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            gdraw = sd.gen;
            build = BUILD_RANDOM;
            tag0 = TAG_NSGA_REFILL;
        } else {
            dfit = sd.fit[cur];
            store = false;
        }

        if (build == BUILD_COPY) {
            const int sr = __ldg(sd.sorted + r);
            const float4* a = reinterpret_cast<const float4*>(src + (size_t)sr * ld);
            float4* o = reinterpret_cast<float4*>(dst + (size_t)r * ld);
            for (int q = t; q < ld / 4; q += BLOCK) o[q] = __ldg(a + q);
            if (t < m) dfit[(size_t)r * m + t] = __ldg(sd.fit[cur] + (size_t)sr * m + t);
            __syncthreads();
            continue;
        }
        const float* row = src + (size_t)r * ld;
        if (store) {
            const float4* A = reinterpret_cast<const float4*>(src + (size_t)pa * ld);
            const float4* Bv = reinterpret_cast<const float4*>(src + (size_t)pb * ld);
            float4* o = reinterpret_cast<float4*>(dst + (size_t)r * ld);
            for (int q = t; q < ld / 4; q += BLOCK) {
                float k[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (4 * q < n) {
                    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
                    if (build != BUILD_RANDOM) {
                        a = __ldg(A + q);
                        b = __ldg(Bv + q);
                    }
                    const uint4 x = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, tag0);
                    if (build == BUILD_RANDOM) {
                        k[0] = u24(x.x);
                        k[1] = u24(x.y);
                        k[2] = u24(x.z);
                        k[3] = u24(x.w);
                    } else {
                        const uint32_t T = sd.rhoT;
                        k[0] = ((x.x >> 8) < T) ? a.x : b.x;
                        k[1] = ((x.y >> 8) < T) ? a.y : b.y;
                        k[2] = ((x.z >> 8) < T) ? a.z : b.z;
                        k[3] = ((x.w >> 8) < T) ? a.w : b.w;
                    }
                    if (build == BUILD_NSGA) {
                        const uint4 mp = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTP);
                        const uint4 mk = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTK);
                        const uint32_t T = sd.mutT;
                        if ((mp.x >> 8) < T) k[0] = u24(mk.x);
                        if ((mp.y >> 8) < T) k[1] = u24(mk.y);
                        if ((mp.z >> 8) < T) k[2] = u24(mk.z);
                        if ((mp.w >> 8) < T) k[3] = u24(mk.w);
                    }
#pragma unroll
                    for (int l = 0; l < 4; ++l)
                        if (4 * q + l >= n) k[l] = 0.0f;
                }
                o[q] = make_float4(k[0], k[1], k[2], k[3]);
            }
            row = dst + (size_t)r * ld;
        }
        __syncthreads();  // the row's keys are visible to the whole block
        if (sd.kind == EXTERNAL) continue;  // the caller computes the fitness

        float res[2] = {0.0f, 0.0f};
        const int kind = sd.kind;
        if (kind == KNAP_THRESHOLD) {
            long long tw = 0, tv = 0;
            for (int i = t; i < n; i += BLOCK)
                if (row[i] > 0.5f) {
                    tw += __ldg(sd.w + i);
                    tv += __ldg(&sd.wv[i].y);
                }
            tw = block_sum_ll<BLOCK>(tw, red_ll);
            tv = block_sum_ll<BLOCK>(tv, red_ll);
            const float twf = (float)tw, tvf = (float)tv;
            res[0] = (twf > sd.cap) ? __fsub_rn(tvf, __fmul_rn(__fsub_rn(twf, sd.cap), 1000.0f)) : tvf;
        } else if (kind == CONTINUOUS) {
            res[0] = continuous_fitness<BLOCK>(row, n, sd.function, sd.lo, sd.hi, red_f);
        } else if (kind == JOBSCHED) {
            res[0] = jobsched_makespan<BLOCK>(row, n, sd.jt, sd.machines, red_f);
        } else {
            // stable argsort by (okey, index): bucket histogram, scan, scatter, rank in bucket
            const int NB = round_up(n, BLOCK);
            const int split = (kind == TSPJ) ? n / 2 : n;  // two segments: buckets split in halves
            const int nbs = (split < n) ? NB / 2 : NB;
            const float nbf = (float)nbs;
            auto bucket = [&](float k, int i) { return bucket_of(k, nbf, nbs) + ((i >= split) ? nbs : 0); };
            for (int i = t; i < n; i += BLOCK) perm[i] = (int32_t)atomicAdd(&cnt[bucket(row[i], i)], 1u);
            __syncthreads();
            bool heavy;
            {
                const int ch = NB / BLOCK;
                uint32_t sum = 0, big = 0;
                for (int j = t * ch; j < t * ch + ch; ++j) {
                    const uint32_t c = cnt[j];
                    sum += c;
                    big = max(big, c);
                }
                uint32_t run = block_exclusive_scan<BLOCK>(sum, warp_tot, nullptr);
                for (int j = t * ch; j < t * ch + ch; ++j) {
                    const uint32_t c = cnt[j];
                    cnt[j] = run;
                    run += c;
                }
                if (t == 0) cnt[NB] = (uint32_t)n;
                heavy = __syncthreads_or(big > kHeavyBucket) != 0;
            }
            for (int i = t; i < n; i += BLOCK) {
                const float k = row[i];
                sc[cnt[bucket(k, i)] + (uint32_t)perm[i]] = ((unsigned long long)okey(k) << 32) | (uint32_t)i;
            }
            __syncthreads();
            if (heavy) {
                // equal or extreme keys in few buckets: sort each segment's composites
                heavy_row_perm<BLOCK>(sc, perm, n, split);
            } else {
                for (int i = t; i < n; i += BLOCK) {
                    const float k = row[i];
                    const int b = bucket(k, i);
                    const uint32_t b0 = cnt[b], b1 = cnt[b + 1];
                    const unsigned long long me = ((unsigned long long)okey(k) << 32) | (uint32_t)i;
                    uint32_t rk = b0;
                    for (uint32_t q = b0; q < b1; ++q) rk += (sc[q] < me) ? 1u : 0u;
                    perm[rk] = i;
                }
            }
            __syncthreads();
            for (int j = t; j <= NB; j += BLOCK) cnt[j] = 0u;  // for the next row
            if (kind == TSP_COORDS) {
                const float* xy = sd.xy;
                canon_sum<BLOCK, 1>(n, [&](int e, float* d) {
                    const int a = perm[e], b = perm[(e + 1 < n) ? e + 1 : 0];
                    d[0] = edge_xy(xy, a, b);
                }, red_f, res);
            } else if (kind == TSP_MATRIX) {
                const float* mat = sd.mat;
                canon_sum<BLOCK, 1>(n, [&](int e, float* d) {
                    const int a = perm[e], b = perm[(e + 1 < n) ? e + 1 : 0];
                    d[0] = __ldg(mat + (size_t)a * n + b);
                }, red_f, res);
            } else if (kind == BITSP_COORDS) {
                const float* xy0 = sd.xy;
                const float* xy1 = sd.xy2;
                canon_sum<BLOCK, 2>(n + 1, [&](int e, float* d) {
                    const int a = (e == 0) ? 0 : perm[e - 1] + 1;
                    const int b = (e == n) ? 0 : perm[e] + 1;
                    d[0] = edge_xy(xy0, a, b);
                    d[1] = edge_xy(xy1, a, b);
                }, red_f, res);
            } else if (kind == BITSP_MATRIX) {
                const float* m0 = sd.mat;
                const float* m1 = sd.mat2;
                const size_t np1 = (size_t)n + 1;
                canon_sum<BLOCK, 2>(n + 1, [&](int e, float* d) {
                    const int a = (e == 0) ? 0 : perm[e - 1] + 1;
                    const int b = (e == n) ? 0 : perm[e] + 1;
                    d[0] = __ldg(m0 + (size_t)a * np1 + b);
                    d[1] = __ldg(m1 + (size_t)a * np1 + b);
                }, red_f, res);
            } else if (kind == KNAP_GREEDY) {
                res[0] = knap_greedy<BLOCK>(perm, n, sd.wv, sd.capi, red_ll, misc, reinterpret_cast<int2*>(sc));
            } else if (kind == TSPJ) {
                res[0] = tspj_makespan<BLOCK>(perm, n / 2, sd.mat, sd.mat2, red_f);
            }
            if (L.perm_out) {
                int32_t* po = L.perm_out + (size_t)r * n;
                for (int i = t; i < n; i += BLOCK) po[i] = perm[i];
            }
        }
        if (t == 0) dfit[(size_t)r * m] = res[0];
        if (t == 1 && m > 1) dfit[(size_t)r * m + 1] = res[1];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// elite partition by exact rank counting: the composite key (fitness key << 32 | row) is
// unique, so rank(i) = #{j : key_j < key_i} is a permutation and sorted[rank(i)] = i is
// the stable order.  P^2 compares spread over ceil(P / RK_CH) CTAs per population, TPE
// threads per element (each counts a slice of j), no sort network and no atomics on the
// ranks.  In engine mode the last CTA of a population (completion counter) swaps the
// buffer index and advances the generation; every CTA also draws the parent ranks of its
// slice of the next generation's child rows (they depend only on seed, row, generation).
// ---------------------------------------------------------------------------------------
constexpr int RK_THREADS = 256, RK_TPE = 32, RK_CH = RK_THREADS / RK_TPE;

struct RankArgs {
    PopDesc* descs;       // engine mode (nullptr: raw mode)
    const float* fit;     // raw mode: segments of P fitness values
    int32_t* sorted;
    int P, maximize, flip;
    int only_ls;          // engine mode: only populations whose local search was due
};

__host__ __device__ inline int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

__global__ void __launch_bounds__(RK_THREADS) rank_kernel(RankArgs a) {
    extern __shared__ unsigned long long rk_keys[];
    const int t = threadIdx.x, pop = blockIdx.y;
    dep_wait();
    PopDesc* d = a.descs ? a.descs + pop : nullptr;
    int P, mx, m, buf = 0;
    const float* f;
    int32_t* sorted;
    uint32_t gen_new = 0;
    if (d) {
        // every descriptor field is read before the first branch, so the reads go out
        // together: one round trip before the fitness loads instead of two
        const uint32_t gen = d->gen, gen_limit = d->gen_limit;
        const int ls_interval = d->ls_interval, cur = d->cur;
        const float* f0 = d->fit[0];
        const float* f1 = d->fit[1];
        P = d->P;
        mx = d->maximize;
        m = d->m;
        sorted = d->sorted;
        const bool lim = gen_limit != 0u && gen >= gen_limit;
        if (a.flip && lim) return;
        if (a.only_ls) {
            const bool due = ls_interval > 0 && gen >= 2u && ((gen - 1u) % (uint32_t)ls_interval) == 0u;
            if (!due || lim) return;
        }
        buf = a.flip ? (cur ^ 1) : cur;
        f = buf ? f1 : f0;
        gen_new = a.flip ? gen + 1 : gen;
    } else {
        P = a.P;
        mx = a.maximize;
        m = 1;
        f = a.fit + (size_t)pop * P;
        sorted = a.sorted + (size_t)pop * P;
    }
    const int base = blockIdx.x * RK_CH;
    if (base >= P) return;
    const int e = t / RK_TPE, part = t % RK_TPE;
    const int i = base + e;
    // a batch of this thread's global loads is issued before the first use (one round trip)
    constexpr int RK_BATCH = 8;
    float v[RK_BATCH];
    auto load = [&](int i0) {
#pragma unroll
        for (int u = 0; u < RK_BATCH; ++u) {
            const int j = i0 + u * RK_THREADS;
            v[u] = (j < P) ? __ldg(f + (size_t)j * m) : 0.0f;
        }
    };
    auto store = [&](int i0) {
#pragma unroll
        for (int u = 0; u < RK_BATCH; ++u) {
            const int j = i0 + u * RK_THREADS;
            if (j < P) rk_keys[j] = ((unsigned long long)fitkey(v[u], mx) << 32) | (uint32_t)j;
        }
    };
    load(t);
    if (d && part == 1 && d->parents && i >= d->E && i < P - d->M) {
        // parent ranks of child row i of generation gen_new + 1 (core/solver.hpp:1117-1118);
        // they do not depend on the fitness, so they are drawn while its loads are in flight
        const uint4 pr = draw4(d->seed, 0u, (uint32_t)i, gen_new + 1, (d->island << 8) | TAG_PARENT);
        d->parents[i] = make_int2((int)pick(pr.x, (uint32_t)d->E), d->E + (int)pick(pr.y, (uint32_t)(P - d->E)));
    }
    store(t);
    for (int i0 = t + RK_THREADS * RK_BATCH; i0 < P; i0 += RK_THREADS * RK_BATCH) {
        load(i0);
        store(i0);
    }
    __syncthreads();
    const unsigned long long me = (i < P) ? rk_keys[i] : 0ull;
    // part p counts j = p, p + TPE, ...: the TPE parts of a warp read consecutive keys
    int cnt = 0;
#pragma unroll 8
    for (int j = part; j < P; j += RK_TPE) cnt += (rk_keys[j] < me) ? 1 : 0;
#pragma unroll
    for (int o = RK_TPE / 2; o >= 1; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o, RK_TPE);
    if (part == 0 && i < P) {
        sorted[cnt] = i;
        if (cnt == 0 && d && d->history && (int)gen_new < d->hist_cap) d->history[gen_new] = f[(size_t)i * m];
    }
    if (d) {
        if (a.flip) {
            __syncthreads();
            if (t == 0) {
                __threadfence();
                const int nblocks = (P + RK_CH - 1) / RK_CH;
                if (atomicAdd(d->done, 1) == nblocks - 1) {
                    d->cur = buf;
                    d->gen = gen_new;
                    *d->done = 0;
                    __threadfence();
                }
            }
        }
    }
}

// ring migration (core/solver.hpp:517-558), migrating the true best rows: island i's
// top `mig` rows by rank overwrite island (i+1)%k's worst `mig` rows; one CTA per instance
__global__ void migrate_kernel(PopDesc* descs, int k, int mig) {
    const int inst = blockIdx.x;
    for (int i = 0; i < k; ++i) {
        const PopDesc& a = descs[inst * k + i];
        const PopDesc& b = descs[inst * k + (i + 1) % k];
        const int ld = a.ld, m = a.m;
        for (int q = 0; q < mig; ++q) {
            const int sr = a.sorted[q];
            const int dr = b.sorted[b.P - mig + q];
            const float4* src = reinterpret_cast<const float4*>(a.keys[a.cur] + (size_t)sr * ld);
            float4* dst = reinterpret_cast<float4*>(b.keys[b.cur] + (size_t)dr * ld);
            for (int j = threadIdx.x; j < ld / 4; j += blockDim.x) dst[j] = src[j];
            if (threadIdx.x < m) b.fit[b.cur][(size_t)dr * m + threadIdx.x] = a.fit[a.cur][(size_t)sr * m + threadIdx.x];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// MO-VRP rows (MultiObjectiveVRPConfig, configs/multi_objective_vrp_config.hpp).  A kernel of
// their own, so the other kinds' row kernel keeps its registers: it builds rows exactly as
// the row kernel does in the modes an NSGA-II population uses (initial keys, offspring,
// diversity refill, given keys), then decodes and scores them:
//   1. h = the FP32 sum of key_i * (i + 1) in index order (one warp, keys staged in shared
//      memory); the sort value of gene i is key_i + (i * 1e-5 + h * 1e-5)  (:219-230);
//   2. a stable argsort of the values, ties to the lower index (std::sort over (value,
//      customer) pairs);
//   3. one warp walks the order, closing a route when the next demand would take a
//      non-empty route over capacity, and forms both objectives with the overload and
//      fleet penalties in the reference's order of float additions (:233-313).
// ---------------------------------------------------------------------------------------

// the bucket argsort of row_argsort with buckets over (value - lo) * inv, lo = h * 1e-5 and
// inv = 1 / (1 + n * 1e-5): the values span about [lo, lo + 1 + n * 1e-5], and any
// non-decreasing bucket map gives the same (value, index) order
template <int BLOCK, int G>
__device__ void movrp_argsort(const float (&v)[G][4], int n, float lo, float inv, const RowSmem& s,
                              uint32_t* warp_tot) {
    constexpr int NB = 4 * G * BLOCK;
    const int t = threadIdx.x;
    uint32_t bs[G][4];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n) {
                const int b = bucket_of(__fmul_rn(__fsub_rn(v[g][l], lo), inv), (float)NB, NB);
                bs[g][l] = ((uint32_t)b << 16) | atomicAdd(&s.cnt[b], 1u);
            }
        }
    __syncthreads();
    uint4 c[G];
    uint32_t sum = 0, big = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        c[g] = reinterpret_cast<const uint4*>(s.cnt)[t * G + g];
        sum += c[g].x + c[g].y + c[g].z + c[g].w;
        big = max(big, max(max(c[g].x, c[g].y), max(c[g].z, c[g].w)));
    }
    uint32_t run = block_exclusive_scan<BLOCK>(sum, warp_tot, nullptr);
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const uint4 o = make_uint4(run, run + c[g].x, run + c[g].x + c[g].y, run + c[g].x + c[g].y + c[g].z);
        run = o.w + c[g].w;
        reinterpret_cast<uint4*>(s.cnt)[t * G + g] = o;
    }
    if (t == 0) s.cnt[NB] = (uint32_t)n;
    const bool heavy = __syncthreads_or(big > kHeavyBucket) != 0;
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n)
                s.sc[s.cnt[bs[g][l] >> 16] + (bs[g][l] & 0xFFFFu)] =
                    ((unsigned long long)okey(v[g][l]) << 32) | (uint32_t)i;
        }
    __syncthreads();
    if (heavy) {  // equal or extreme values in few buckets: sort the composites instead
        heavy_row_perm<BLOCK>(s.sc, s.perm, n, n);
        return;
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int i = 4 * (t + g * BLOCK) + l;
            if (i < n) {
                const uint32_t b = bs[g][l] >> 16, b0 = s.cnt[b], b1 = s.cnt[b + 1];
                const unsigned long long me = ((unsigned long long)okey(v[g][l]) << 32) | (uint32_t)i;
                uint32_t r = b0;
                for (uint32_t q = b0; q < b1; ++q) r += (s.sc[q] < me) ? 1u : 0u;
                s.perm[r] = i;
            }
        }
    __syncthreads();
}

// routes and objectives of the sorted customers perm[j] + 1.  Lanes fetch the legs (from the
// previous customer, and to the depot) and demands of 128 positions at a time, loads first;
// every lane then replays them in order, so all lanes hold the same state.  d(a, b) = d(b, a)
// bit for bit (dx and -dx have the same square), so the depot leg into a route's first
// customer is its leg to the depot.
__device__ void movrp_objectives(const int32_t* perm, int n, const float* __restrict__ xy,
                                 const int32_t* __restrict__ dem, int cap, int vehicles, float* red, float* out) {
    constexpr int kChunks = 4;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        float dist = 0.0f, total = 0.0f, longest = 0.0f, pen = 0.0f, lastdep = 0.0f;
        int load = 0, size = 0, routes = 0;
        for (int g0 = 0; g0 < n; g0 += 32 * kChunks) {
            float e[kChunks], dep[kChunks];
            int dm[kChunks];
#pragma unroll
            for (int c = 0; c < kChunks; ++c) {
                const int j = g0 + 32 * c + lane;
                e[c] = 0.0f;
                dep[c] = 0.0f;
                dm[c] = 0;
                if (j < n) {
                    const int cust = perm[j] + 1;
                    e[c] = edge_xy(xy, (j == 0) ? 0 : perm[j - 1] + 1, cust);
                    dep[c] = edge_xy(xy, cust, 0);
                    dm[c] = __ldg(dem + cust);
                }
            }
#pragma unroll
            for (int c = 0; c < kChunks; ++c) {
                const int cnt = min(32, n - (g0 + 32 * c));
                for (int q = 0; q < cnt; ++q) {
                    const float eq = __shfl_sync(0xffffffffu, e[c], q);
                    const float dq = __shfl_sync(0xffffffffu, dep[c], q);
                    const int mq = __shfl_sync(0xffffffffu, dm[c], q);
                    if (load + mq > cap && size > 0) {  // close the route: back to the depot
                        dist = __fadd_rn(dist, lastdep);
                        total = __fadd_rn(total, dist);
                        longest = (dist > longest) ? dist : longest;
                        if (load > cap) pen = __fadd_rn(pen, __fmul_rn((float)(load - cap), 100.0f));
                        ++routes;
                        dist = 0.0f;
                        load = 0;
                        size = 0;
                    }
                    dist = __fadd_rn(dist, (size == 0) ? dq : eq);
                    load += mq;
                    ++size;
                    lastdep = dq;
                }
            }
        }
        if (size > 0) {
            dist = __fadd_rn(dist, lastdep);
            total = __fadd_rn(total, dist);
            longest = (dist > longest) ? dist : longest;
            if (load > cap) pen = __fadd_rn(pen, __fmul_rn((float)(load - cap), 100.0f));
            ++routes;
        }
        float o0 = __fadd_rn(total, pen), o1 = longest;
        if (routes > vehicles) {
            const float vp = __fmul_rn((float)(routes - vehicles), 500.0f);
            o0 = __fadd_rn(o0, vp);
            o1 = __fadd_rn(o1, vp);
        }
        if (lane == 0) {
            red[0] = o0;
            red[1] = o1;
        }
    }
    __syncthreads();
    out[0] = red[0];
    out[1] = red[1];
    __syncthreads();
}

template <int BLOCK, int G>
__global__ void __launch_bounds__(BLOCK, RowResidency<BLOCK, G>::value) movrp_row_kernel(RowLaunch L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ PopDesc sd;
    __shared__ uint32_t warp_tot[32];
    __shared__ float red_f[32];
    const int t = threadIdx.x;
    const RowSmem s = carve(smem_raw, BLOCK, G, L.max_n, L.max_points);
    int cur_pid = -1;
    zero_counters<BLOCK, G>(s);
    dep_wait();  // shared memory only above this line

    for (int task = blockIdx.x; task < L.ntasks; task += gridDim.x) {
        int pid = 0, r = task;
        if (L.tasks) {
            const Task tk = L.tasks[task];
            pid = tk.pid;
            r = tk.row;
        }
        if (pid != cur_pid) {
            __syncthreads();
            if (t == 0) sd = L.descs ? L.descs[pid] : L.single;
            __syncthreads();
            cur_pid = pid;
        }
        const int n = sd.n, ld = sd.ld, P = sd.P, m = sd.m, cur = sd.cur;
        if (L.mode == MODE_NSGA_OFF && at_limit(sd)) continue;
        if (L.mode == MODE_NSGA_REFILL && (!sd.advanced || r < __ldg(sd.nu))) continue;
        const float* src = sd.keys[cur];
        float* dst = nullptr;
        float* dfit = nullptr;
        enum { LOAD, RANDOM, NSGA } build = RANDOM;
        uint32_t gdraw = 0, tag = 0;
        int pa = 0, pb = 0;
        if (L.mode == MODE_INIT) {  // core/population.hpp:107-110
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            tag = (sd.island << 8) | TAG_INIT;
        } else if (L.mode == MODE_NSGA_OFF) {  // core/solver.hpp:1019-1091, pool rows [P, 2P)
            dst = sd.keys[cur] + (size_t)P * ld;
            dfit = sd.fit[cur] + (size_t)P * m;
            gdraw = sd.gen + 1;
            if (r >= P - sd.Mn) {
                tag = TAG_MUTANT;
            } else {
                build = NSGA;
                tag = TAG_NSGA_COIN;
                const uint4 pk = draw4(sd.seed, 0u, (uint32_t)r, gdraw, TAG_NSGA_TOUR);
                pa = tourn(pick(pk.x, P), pick(pk.y, P), sd.nrank, sd.ncd);
                pb = tourn(pick(pk.z, P), pick(pk.w, P), sd.nrank, sd.ncd);
            }
        } else if (L.mode == MODE_NSGA_REFILL) {  // core/population.hpp:166-171
            dst = sd.keys[cur];
            dfit = sd.fit[cur];
            gdraw = sd.gen;
            tag = TAG_NSGA_REFILL;
        } else if (L.mode == MODE_EVAL) {
            dfit = sd.fit[cur];
            build = LOAD;
        } else {
            continue;  // single-objective modes do not apply
        }

        float k[G][4];
        const float* row = src + (size_t)r * ld;
        const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
#pragma unroll
        for (int gg = 0; gg < G; ++gg) {
            const int q = t + gg * BLOCK;
#pragma unroll
            for (int l = 0; l < 4; ++l) k[gg][l] = 0.0f;
            if (build == LOAD) {
                if (vec && 4 * q + 3 < ld) {
                    const float4 a = __ldg(reinterpret_cast<const float4*>(row) + q);
                    k[gg][0] = a.x, k[gg][1] = a.y, k[gg][2] = a.z, k[gg][3] = a.w;
                } else {
#pragma unroll
                    for (int l = 0; l < 4; ++l) k[gg][l] = (4 * q + l < n) ? __ldg(row + 4 * q + l) : 0.0f;
                }
            } else if (4 * q < n) {
                const uint4 x = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, tag);
                if (build == RANDOM) {
                    k[gg][0] = u24(x.x), k[gg][1] = u24(x.y), k[gg][2] = u24(x.z), k[gg][3] = u24(x.w);
                } else {
                    const float4 a = __ldg(reinterpret_cast<const float4*>(src + (size_t)pa * ld) + q);
                    const float4 b = __ldg(reinterpret_cast<const float4*>(src + (size_t)pb * ld) + q);
                    const uint32_t T = sd.rhoT, MT = sd.mutT;
                    k[gg][0] = ((x.x >> 8) < T) ? a.x : b.x;
                    k[gg][1] = ((x.y >> 8) < T) ? a.y : b.y;
                    k[gg][2] = ((x.z >> 8) < T) ? a.z : b.z;
                    k[gg][3] = ((x.w >> 8) < T) ? a.w : b.w;
                    const uint4 mp = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTP);
                    const uint4 mk = draw4(sd.seed, (uint32_t)q, (uint32_t)r, gdraw, TAG_NSGA_MUTK);
                    if ((mp.x >> 8) < MT) k[gg][0] = u24(mk.x);
                    if ((mp.y >> 8) < MT) k[gg][1] = u24(mk.y);
                    if ((mp.z >> 8) < MT) k[gg][2] = u24(mk.z);
                    if ((mp.w >> 8) < MT) k[gg][3] = u24(mk.w);
                }
            }
            if (build != LOAD && 4 * q < ld) {
                float4 o;
                o.x = (4 * q + 0 < n) ? k[gg][0] : 0.0f;
                o.y = (4 * q + 1 < n) ? k[gg][1] : 0.0f;
                o.z = (4 * q + 2 < n) ? k[gg][2] : 0.0f;
                o.w = (4 * q + 3 < n) ? k[gg][3] : 0.0f;
                reinterpret_cast<float4*>(dst + (size_t)r * ld)[q] = o;
            }
        }

        // 1. the row hash and the sort values
        float* sk = reinterpret_cast<float*>(s.sc);
#pragma unroll
        for (int gg = 0; gg < G; ++gg)
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const int i = 4 * (t + gg * BLOCK) + l;
                if (i < n) sk[i] = k[gg][l];
            }
        __syncthreads();
        if (t < 32) {
            float h = 0.0f;
            for (int c0 = 0; c0 < n; c0 += 32) {
                const int i = c0 + t;
                const float term = (i < n) ? __fmul_rn(sk[i], (float)(i + 1)) : 0.0f;
                const int cnt = min(32, n - c0);
                for (int q = 0; q < cnt; ++q) h = __fadd_rn(h, __shfl_sync(0xffffffffu, term, q));
            }
            if (t == 0) red_f[0] = h;
        }
        __syncthreads();
        const float hb = __fmul_rn(red_f[0], 1.0e-5f);
#pragma unroll
        for (int gg = 0; gg < G; ++gg)
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const int i = 4 * (t + gg * BLOCK) + l;
                k[gg][l] = (i < n) ? __fadd_rn(k[gg][l], __fadd_rn(__fmul_rn((float)i, 1.0e-5f), hb)) : 0.0f;
            }
        __syncthreads();  // red_f[0] and the staged keys are read
        // 2. the visiting order
        movrp_argsort<BLOCK, G>(k, n, hb, __frcp_rn(__fadd_rn(1.0f, __fmul_rn((float)n, 1.0e-5f))), s, warp_tot);
        zero_counters<BLOCK, G>(s);  // ready for the next row (separated by the row-end barrier)
        // 3. routes and objectives
        float res[2];
        movrp_objectives(s.perm, n, sd.xy, sd.w, (int)sd.capi, sd.machines, red_f, res);
        if (L.perm_out) {
            int32_t* po = L.perm_out + (size_t)r * n;
            for (int i = t; i < n; i += BLOCK) po[i] = s.perm[i];
        }
        if (t < 2) dfit[(size_t)r * m + t] = res[t];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
int device_sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// default tile per size (smallest capacity 4 * block * groups that covers n); the
// autotuner may pick any other tile whose capacity covers n
static constexpr RowTile kTiles[] = {
    {32, 1}, {64, 1}, {128, 1}, {256, 1}, {256, 2}, {512, 2}, {512, 4}, {1024, 3}, {1024, 4},
};
static constexpr RowTile kAllTiles[] = {
    {32, 1}, {64, 1}, {64, 2}, {128, 1}, {128, 2}, {128, 4}, {256, 1}, {256, 2}, {256, 4},
    {512, 1}, {512, 2}, {512, 4}, {1024, 1}, {1024, 2}, {1024, 3}, {1024, 4},
};

int tile_candidates(int n, RowTile* out, int cap) {
    int c = 0;
    for (const RowTile& t : kAllTiles)
        if (4 * t.block * t.groups >= n && 4 * t.block * t.groups <= 8 * n + 128 && c < cap) out[c++] = t;
    return c;
}

RowTile pick_tile(int n) {
    for (const RowTile& t : kTiles)
        if (4 * t.block * t.groups >= n) return t;
    return RowTile{0, 0};
}

int row_max_n() { return 4 * 1024 * 4; }

int row_max_n_global() { return 1 << 22; }

bool row_needs_global(int n, int pts, int kind) {
    // rows of an external-fitness problem are only built: the global kernel builds them
    // without a sort buffer in shared memory
    if (kind == EXTERNAL) return true;
    if (n > row_max_n()) return true;
    const RowTile t = pick_tile(n);
    return row_smem_bytes(t, n, pts, kind, false) > kRowSmemCap;
}

int row_global_grid(int rows, int max_n) {
    const size_t budget = (size_t)2 << 30;  // scratch for at most 2 GiB of CTAs
    int g = 2 * device_sm_count();
    const size_t by_mem = budget / row_global_stride(max_n);
    if ((size_t)g > by_mem) g = (int)by_mem;
    if (g > rows) g = rows;
    return g < 1 ? 1 : g;
}

using RowFn = void (*)(RowLaunch);

static RowFn row_fn(const RowTile& t, bool dyn = false) {
#define BK_TILE(B, G) \
    if (t.block == B && t.groups == G) return dyn ? row_kernel<B, G, true> : row_kernel<B, G, false>;
    BK_TILE(32, 1)
    BK_TILE(64, 1)
    BK_TILE(64, 2)
    BK_TILE(128, 1)
    BK_TILE(128, 2)
    BK_TILE(128, 4)
    BK_TILE(256, 1)
    BK_TILE(256, 2)
    BK_TILE(256, 4)
    BK_TILE(512, 1)
    BK_TILE(512, 2)
    BK_TILE(512, 4)
    BK_TILE(1024, 1)
    BK_TILE(1024, 2)
    BK_TILE(1024, 3)
    BK_TILE(1024, 4)
#undef BK_TILE
    return nullptr;
}

static RowFn movrp_fn(const RowTile& t) {
#define BK_TILE(B, G) \
    if (t.block == B && t.groups == G) return movrp_row_kernel<B, G>;
    BK_TILE(32, 1)
    BK_TILE(64, 1)
    BK_TILE(64, 2)
    BK_TILE(128, 1)
    BK_TILE(128, 2)
    BK_TILE(128, 4)
    BK_TILE(256, 1)
    BK_TILE(256, 2)
    BK_TILE(256, 4)
    BK_TILE(512, 1)
    BK_TILE(512, 2)
    BK_TILE(512, 4)
    BK_TILE(1024, 1)
    BK_TILE(1024, 2)
    BK_TILE(1024, 3)
    BK_TILE(1024, 4)
#undef BK_TILE
    return nullptr;
}

// the dynamic shared-memory limit of a kernel is only ever raised, so a later launch
// that needs less never takes it away from a live engine that needs more
static std::mutex g_attr_mu;
static std::map<std::pair<int, const void*>, size_t> g_attr;

cudaError_t raise_smem_limit(const void* fn, size_t smem) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_attr_mu);
    size_t& cur = g_attr[{dev, fn}];
    if (smem <= cur) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cur = smem;
    return e;
}

cudaError_t prepare_rows(const RowTile& tile, size_t smem, int* per_sm) {
    RowFn fn = row_fn(tile);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(fn), smem);
    if (e == cudaSuccess) e = raise_smem_limit(reinterpret_cast<const void*>(row_fn(tile, true)), smem);
    // the MO-VRP kernel has the same launch bounds and shared memory
    if (e == cudaSuccess) e = raise_smem_limit(reinterpret_cast<const void*>(movrp_fn(tile)), smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, tile.block, smem);
}

cudaError_t launch_rows(const RowLaunch& L, int kind, const RowTile& tile, int grid, cudaStream_t s) {
    if (tile.block == 0) {  // rows beyond shared memory: global-scratch kernel
        if (!L.gscratch || L.gstride < row_global_stride(L.max_n)) return cudaErrorInvalidValue;
        if (kind == MOVRP) return cudaErrorInvalidValue;  // MO-VRP rows fit in shared memory only
        if (L.ntasks <= 0 || grid <= 0) return cudaSuccess;
        if (grid > L.ntasks) grid = L.ntasks;
        row_kernel_big<<<grid, kBigBlock, 0, s>>>(L);
        return cudaGetLastError();
    }
    RowFn fn = (kind == MOVRP) ? movrp_fn(tile) : row_fn(tile, L.work != nullptr);
    if (!fn) return cudaErrorInvalidValue;
    if (L.ntasks <= 0 || grid <= 0) return cudaSuccess;
    if (grid > L.ntasks) grid = L.ntasks;
    const size_t smem = row_smem_bytes(tile, L.max_n, L.max_points, kind, L.stage_xy != 0);
    return launch_dep(fn, dim3(grid), dim3(tile.block), smem, s, L);
}

cudaError_t launch_rows_auto(const RowLaunch& L, int kind, const RowTile& tile, cudaStream_t s) {
    const size_t smem = row_smem_bytes(tile, L.max_n, L.max_points, kind, L.stage_xy != 0);
    int per_sm = 0;
    cudaError_t e = prepare_rows(tile, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    return launch_rows(L, kind, tile, per_sm * device_sm_count(), s);
}

cudaError_t prepare_sort(int maxP) {
    return raise_smem_limit(reinterpret_cast<const void*>(rank_kernel), (size_t)(maxP > 0 ? maxP : 1) * 8);
}

cudaError_t launch_sort_raw(const float* fit, int P, int segments, int maximize, int32_t* sorted,
                            cudaStream_t s) {
    if (P <= 0 || segments <= 0) return cudaSuccess;
    RankArgs a{nullptr, fit, sorted, P, maximize, 0, 0};
    dim3 grid((P + RK_CH - 1) / RK_CH, segments);
    return launch_dep(rank_kernel, grid, dim3(RK_THREADS), (size_t)P * 8, s, a);
}

cudaError_t launch_sort_pops(PopDesc* descs, int npops, int maxP, int flip, cudaStream_t s) {
    if (npops <= 0) return cudaSuccess;
    RankArgs a{descs, nullptr, nullptr, 0, 0, flip, 0};
    dim3 grid((maxP + RK_CH - 1) / RK_CH, npops);
    return launch_dep(rank_kernel, grid, dim3(RK_THREADS), (size_t)maxP * 8, s, a);
}

cudaError_t launch_sort_pops_after_ls(PopDesc* descs, int npops, int maxP, cudaStream_t s) {
    if (npops <= 0) return cudaSuccess;
    RankArgs a{descs, nullptr, nullptr, 0, 0, 0, 1};
    dim3 grid((maxP + RK_CH - 1) / RK_CH, npops);
    return launch_dep(rank_kernel, grid, dim3(RK_THREADS), (size_t)maxP * 8, s, a);
}

cudaError_t launch_migrate(PopDesc* descs, int ninst, int k, int migrants, int max_n, cudaStream_t s) {
    (void)max_n;
    if (ninst <= 0 || k < 2 || migrants <= 0) return cudaSuccess;
    migrate_kernel<<<ninst, 256, 0, s>>>(descs, k, migrants);
    return cudaGetLastError();
}

}  // namespace bk
