// nsga2.cu -- NSGA-II selection on the device.
//
// Reference: Solver::evolve_generation_nsga2 (core/solver.hpp:751-817) and
// Population::fast_non_dominated_sort / calculate_crowding_distance /
// select_next_generation_nsga2 / ensure_minimum_diversity (core/population.hpp:130-517).
//
// Pareto ranks, two objectives (the bi-objective TSP): the pool is sorted by
// (f0, f1); a point is then dominated exactly when the lexicographic minimum of (f1, f0)
// over the points before it is below its own (f1, f0), so each front is one block-wide
// exclusive min-scan over the points still unranked, and peeling repeats the scan on
// the compacted remainder.  Any number of objectives: a bit-packed dominance matrix
// (row i, bit j = "j dominates i") built 32 columns at a time with __ballot_sync,
// domination counts and front peeling with __popc over the row & front-mask words.
// Crowding: per objective a bitonic sort of (rank, objective, index) so each front is
// contiguous and ordered; interior points add (next - prev) / range in the reference's
// accumulation order.  Survivors: bitonic sort of (rank, -crowding, index), first P.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "nsga2.h"

namespace bk {

constexpr int kNsgaBlock = 1024;
constexpr int kMaxPool = 8192;  // largest pool of the in-shared-memory select kernel

__host__ __device__ inline int npow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// ---------------------------------------------------------------------------------------
// block helpers
// ---------------------------------------------------------------------------------------
template <int BLOCK>
__device__ unsigned long long block_excl_min_u64(unsigned long long v, unsigned long long* wt) {
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = (y < x) ? y : x;
    }
    unsigned long long prev = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) prev = ~0ull;
    if (lane == 31) wt[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned long long s = (lane < NW) ? wt[lane] : ~0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s = (y < s) ? y : s;
        }
        if (lane < NW) wt[lane] = s;
    }
    __syncthreads();
    const unsigned long long base = (w > 0) ? wt[w - 1] : ~0ull;
    __syncthreads();
    return (base < prev) ? base : prev;
}

template <int BLOCK>
__device__ void bitonic_u64(unsigned long long* s, int N2) {
    const int t = threadIdx.x;
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
}

template <int BLOCK>
__device__ void bitonic_kv(unsigned long long* s, uint16_t* v, int N2) {
    const int t = threadIdx.x;
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
                    const uint16_t x = v[i];
                    v[i] = v[ixj];
                    v[ixj] = x;
                }
            }
            __syncthreads();
        }
}

// ---------------------------------------------------------------------------------------
// shared-memory working set of the select kernel (N <= kMaxPool points, 2 objectives)
// ---------------------------------------------------------------------------------------
struct SelSmem {
    float* obj;                // [N][2]
    uint16_t* rank;            // [N]
    float* cd;                 // [N]
    unsigned long long* key;   // [N2]
    uint16_t* sidx;            // [N2]
    uint16_t* ra;              // [N]
    uint16_t* rb;              // [N]
};

__host__ __device__ inline size_t sel_smem_bytes(int N) {
    const int N2 = npow2(N);
    size_t b = (size_t)N * 8;           // obj
    b += ((size_t)N * 2 + 15) / 16 * 16;  // rank
    b += (size_t)N * 4;                 // cd
    b = (b + 15) / 16 * 16;
    b += (size_t)N2 * 8;                // key
    b += (size_t)N2 * 2;                // sidx
    b += (size_t)N * 2 * 2;             // ra, rb
    return (b + 15) / 16 * 16;
}

__device__ inline SelSmem sel_carve(unsigned char* base, int N) {
    const int N2 = npow2(N);
    SelSmem s;
    size_t off = 0;
    s.obj = (float*)(base + off);
    off += (size_t)N * 8;
    s.rank = (uint16_t*)(base + off);
    off += ((size_t)N * 2 + 15) / 16 * 16;
    s.cd = (float*)(base + off);
    off += (size_t)N * 4;
    off = (off + 15) / 16 * 16;
    s.key = (unsigned long long*)(base + off);
    off += (size_t)N2 * 8;
    s.sidx = (uint16_t*)(base + off);
    off += (size_t)N2 * 2;
    s.ra = (uint16_t*)(base + off);
    off += (size_t)N * 2;
    s.rb = (uint16_t*)(base + off);
    return s;
}

__device__ __forceinline__ unsigned long long lex10(const float* obj, int i) {
    return ((unsigned long long)okey(obj[2 * i + 1]) << 32) | okey(obj[2 * i]);
}

// two-objective Pareto ranks by staircase peeling; returns the number of fronts
template <int BLOCK>
__device__ int rank2_staircase(int N, const SelSmem& s, unsigned long long* wt64, uint32_t* wt32) {
    const int t = threadIdx.x;
    const int N2 = npow2(N);
    for (int i = t; i < N2; i += BLOCK) {
        s.key[i] = (i < N) ? (((unsigned long long)okey(s.obj[2 * i]) << 32) | okey(s.obj[2 * i + 1])) : ~0ull;
        s.sidx[i] = (uint16_t)i;
    }
    __syncthreads();
    bitonic_kv<BLOCK>(s.key, s.sidx, N2);
    // the padding (~0 keys) sorts last, so the first N entries are the points
    for (int p = t; p < N; p += BLOCK) s.ra[p] = s.sidx[p];
    __syncthreads();
    uint16_t* ra = s.ra;
    uint16_t* rb = s.rb;
    int nr = N, k = 0;
    while (nr > 0) {
        const int ch = (nr + BLOCK - 1) / BLOCK;
        const int p0 = t * ch, p1 = min(nr, p0 + ch);
        unsigned long long lmin = ~0ull;
        for (int p = p0; p < p1; ++p) {
            const unsigned long long v = lex10(s.obj, ra[p]);
            lmin = (v < lmin) ? v : lmin;
        }
        const unsigned long long pm0 = block_excl_min_u64<BLOCK>(lmin, wt64);
        unsigned long long pm = pm0;
        uint32_t kept = 0;
        for (int p = p0; p < p1; ++p) {
            const int i = ra[p];
            const unsigned long long me = lex10(s.obj, i);
            if (pm < me) ++kept;
            else s.rank[i] = (uint16_t)k;
            pm = (me < pm) ? me : pm;
        }
        uint32_t total;
        uint32_t base = block_exclusive_scan<BLOCK>(kept, wt32, &total);
        pm = pm0;
        for (int p = p0; p < p1; ++p) {
            const int i = ra[p];
            const unsigned long long me = lex10(s.obj, i);
            if (pm < me) rb[base++] = (uint16_t)i;
            pm = (me < pm) ? me : pm;
        }
        __syncthreads();
        uint16_t* tmp = ra;
        ra = rb;
        rb = tmp;
        nr = (int)total;
        ++k;
    }
    return k;
}

// crowding distance per front, objectives processed in order (core/population.hpp:453-489)
template <int BLOCK>
__device__ void crowding2(int N, const SelSmem& s) {
    const int t = threadIdx.x;
    const int N2 = npow2(N);
    uint16_t* fs = s.ra;  // front first position, indexed by rank
    uint16_t* fe = s.rb;  // front last position
    for (int i = t; i < N; i += BLOCK) s.cd[i] = 0.0f;
    for (int o = 0; o < 2; ++o) {
        __syncthreads();
        for (int i = t; i < N2; i += BLOCK)
            s.key[i] = (i < N) ? (((unsigned long long)s.rank[i] << 48) |
                                  ((unsigned long long)okey(s.obj[2 * i + o]) << 16) | (unsigned long long)i)
                               : ~0ull;
        __syncthreads();
        bitonic_u64<BLOCK>(s.key, N2);
        for (int p = t; p < N; p += BLOCK) {
            const int r = (int)(s.key[p] >> 48);
            if (p == 0 || (int)(s.key[p - 1] >> 48) != r) fs[r] = (uint16_t)p;
            if (p == N - 1 || (int)(s.key[p + 1] >> 48) != r) fe[r] = (uint16_t)p;
        }
        __syncthreads();
        for (int p = t; p < N; p += BLOCK) {
            const int i = (int)(s.key[p] & 0xFFFFu);
            const int r = (int)(s.key[p] >> 48);
            const int f = fs[r], l = fe[r];
            if (l - f + 1 <= 2 || p == f || p == l) {
                s.cd[i] = INFINITY;
            } else {
                const float lo = s.obj[2 * (int)(s.key[f] & 0xFFFFu) + o];
                const float hi = s.obj[2 * (int)(s.key[l] & 0xFFFFu) + o];
                const float range = __fsub_rn(hi, lo);
                if (range > 0.0f) {
                    const float a = s.obj[2 * (int)(s.key[p + 1] & 0xFFFFu) + o];
                    const float b = s.obj[2 * (int)(s.key[p - 1] & 0xFFFFu) + o];
                    s.cd[i] = __fadd_rn(s.cd[i], __fdiv_rn(__fsub_rn(a, b), range));
                }
            }
        }
    }
    __syncthreads();
}

__device__ __forceinline__ uint32_t cd_key(float c) {
    const uint32_t k = okey(c);
    return (k == 0xFFFFFFFFu) ? 0xFFFFFFFFu : ~k;
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

// mode 0: select P survivors from the 2P pool of fit[cur];
// mode 1: ranks + crowding of the P population (initialisation);
// mode 2: as mode 1, only when the diversity pass rebuilt the population (*nu < P)
__global__ void __launch_bounds__(kNsgaBlock) nsga_select_kernel(PopDesc* dd, int32_t* g_rank, float* g_cd,
                                                                 int32_t* g_sel, const int32_t* d_nu, int mode) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long wt64[32];
    __shared__ uint32_t wt32[32];
    __shared__ float redf[32];
    PopDesc& d = dd[blockIdx.x];
    const int t = threadIdx.x;
    const int P = d.P;
    if (mode == 2 && __ldg(d_nu) >= P) return;
    const int N = (mode == 0) ? 2 * P : P;
    const float* f = d.fit[d.cur];
    const SelSmem s = sel_carve(smem, N);
    for (int i = t; i < 2 * N; i += kNsgaBlock) s.obj[i] = f[i];
    __syncthreads();
    rank2_staircase<kNsgaBlock>(N, s, wt64, wt32);
    __syncthreads();
    crowding2<kNsgaBlock>(N, s);
    float fmin = INFINITY;
    if (mode == 0) {
        const int N2 = npow2(N);
        for (int i = t; i < N2; i += kNsgaBlock)
            s.key[i] = (i < N) ? (((unsigned long long)s.rank[i] << 48) | ((unsigned long long)cd_key(s.cd[i]) << 16) |
                                  (unsigned long long)i)
                               : ~0ull;
        __syncthreads();
        bitonic_u64<kNsgaBlock>(s.key, N2);
        for (int q = t; q < P; q += kNsgaBlock) {
            const int i = (int)(s.key[q] & 0xFFFFu);
            g_sel[q] = i;
            g_rank[q] = s.rank[i];
            g_cd[q] = s.cd[i];
            fmin = fminf(fmin, s.obj[2 * i]);
        }
    } else {
        for (int i = t; i < P; i += kNsgaBlock) {
            g_rank[i] = s.rank[i];
            g_cd[i] = s.cd[i];
            fmin = fminf(fmin, s.obj[2 * i]);
        }
    }
    fmin = block_min_f(fmin, redf);
    if (t == 0 && d.history) {
        const uint32_t g = (mode == 0) ? d.gen + 1 : d.gen;
        if ((int)g < d.hist_cap) d.history[g] = fmin;
    }
}

// survivors -> the other pool buffer, rows [0, P)
__global__ void nsga_gather_kernel(PopDesc* dd, const int32_t* sel) {
    const PopDesc& d = dd[0];
    const int P = d.P, ld4 = d.ld / 4, m = d.m;
    const float4* src = reinterpret_cast<const float4*>(d.keys[d.cur]);
    float4* dst = reinterpret_cast<float4*>(d.keys[d.cur ^ 1]);
    const float* fs = d.fit[d.cur];
    float* fd = d.fit[d.cur ^ 1];
    const size_t total = (size_t)P * ld4;
    for (size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(x / ld4), c = (int)(x % ld4);
        const size_t sq = (size_t)__ldg(sel + q);
        dst[x] = src[sq * ld4 + c];
        if (c == 0)
            for (int o = 0; o < m; ++o) fd[(size_t)q * m + o] = fs[sq * m + o];
    }
}

__global__ void nsga_finish_kernel(PopDesc* dd) {
    if (threadIdx.x == 0) {
        dd[0].cur ^= 1;
        dd[0].gen += 1;
    }
}

// ensure_minimum_diversity (core/population.hpp:130-182): greedy in-order dedupe in
// objective space (distance < 0.001, float differences squared and summed in double);
// when fewer than 70% are unique, the unique rows move to the front in order and
// *nu < P tells the refill and re-rank launches to run.  Runs after generation g
// when (g - 1) % interval == 0.
__global__ void __launch_bounds__(kNsgaBlock) nsga_diversity_kernel(PopDesc* dd, int interval, int32_t* d_nu,
                                                                    int32_t* g_uniq) {
    PopDesc& d = dd[0];
    const int t = threadIdx.x, P = d.P;
    const uint32_t g = d.gen;
    if (interval <= 0 || g < 1 || ((g - 1) % (uint32_t)interval) != 0) {
        if (t == 0) *d_nu = P;
        return;
    }
    extern __shared__ float2 uobj[];  // [P]
    float* f = d.fit[d.cur];
    int nu = 0;
    for (int c = 0; c < P; ++c) {
        const float c0 = f[2 * c], c1 = f[2 * c + 1];
        int near = 0;
        for (int u = t; u < nu; u += kNsgaBlock) {
            const double d0 = (double)__fsub_rn(c0, uobj[u].x);
            const double d1 = (double)__fsub_rn(c1, uobj[u].y);
            const double dist = __dsqrt_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)));
            near |= (dist < 0.001) ? 1 : 0;
        }
        near = __syncthreads_or(near);
        if (!near) {
            if (t == 0) {
                uobj[nu] = make_float2(c0, c1);
                g_uniq[nu] = c;
            }
            ++nu;
        }
        __syncthreads();
    }
    const double ratio = (double)nu / (double)P;
    if (!(ratio < 0.70)) {
        if (t == 0) *d_nu = P;
        return;
    }
    // compact the unique rows to the front, in order (sources never precede targets)
    float4* keys = reinterpret_cast<float4*>(d.keys[d.cur]);
    const int ld4 = d.ld / 4;
    for (int i = 0; i < nu; ++i) {
        const int src = g_uniq[i];
        if (src != i) {
            for (int c = t; c < ld4; c += kNsgaBlock) keys[(size_t)i * ld4 + c] = keys[(size_t)src * ld4 + c];
            if (t < 2) f[2 * i + t] = f[2 * src + t];
        }
        __syncthreads();
    }
    if (t == 0) *d_nu = nu;
}

// ---------------------------------------------------------------------------------------
// general-m Pareto ranks: bit-packed dominance matrix
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ bool dominates_m(const float* a, const float* b, int m) {
    bool better = false;
    for (int o = 0; o < m; ++o) {
        if (a[o] > b[o]) return false;
        if (a[o] < b[o]) better = true;
    }
    return better;
}

// D[i][w] bit b: point j = 32w + b dominates point i
__global__ void dom_matrix_kernel(const float* __restrict__ obj, int N, int m, int W, uint32_t* __restrict__ D) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long x = warp; x < (long long)N * W; x += nwarps) {
        const int i = (int)(x / W), w = (int)(x % W);
        const int j = 32 * w + lane;
        const bool dom = (j < N && j != i) ? dominates_m(obj + (size_t)j * m, obj + (size_t)i * m, m) : false;
        const uint32_t word = __ballot_sync(0xffffffffu, dom);
        if (lane == 0) D[(size_t)i * W + w] = word;
    }
}

// domination counts and front peeling: count_i -= popc(D[i] & front) per front
__global__ void __launch_bounds__(kNsgaBlock) dom_peel_kernel(const uint32_t* __restrict__ D, int N, int W,
                                                             int32_t* rank) {
    extern __shared__ uint32_t sm[];
    int32_t* cnt = reinterpret_cast<int32_t*>(sm);  // [N], -1 once ranked
    uint32_t* F = sm + N;                           // [W]
    const int t = threadIdx.x;
    for (int i = t; i < N; i += kNsgaBlock) {
        int c = 0;
        for (int w = 0; w < W; ++w) c += __popc(__ldg(D + (size_t)i * W + w));
        cnt[i] = c;
    }
    __syncthreads();
    for (int k = 0; k < N; ++k) {
        for (int w = t; w < W; w += kNsgaBlock) F[w] = 0u;
        __syncthreads();
        int any = 0;
        for (int i = t; i < N; i += kNsgaBlock)
            if (cnt[i] == 0) {
                rank[i] = k;
                atomicOr(&F[i >> 5], 1u << (i & 31));
                any = 1;
            }
        any = __syncthreads_or(any);
        if (!any) break;
        for (int i = t; i < N; i += kNsgaBlock) {
            if (cnt[i] == 0) {
                cnt[i] = -1;
            } else if (cnt[i] > 0) {
                int c = 0;
                for (int w = 0; w < W; ++w)
                    if (F[w]) c += __popc(__ldg(D + (size_t)i * W + w) & F[w]);
                cnt[i] -= c;
            }
        }
        __syncthreads();
    }
}

// ranks (+ crowding) of an arbitrary two-objective point set, one CTA: op API
__global__ void __launch_bounds__(kNsgaBlock) rank2_op_kernel(const float* obj, int N, int32_t* rank, float* cd) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long wt64[32];
    __shared__ uint32_t wt32[32];
    const SelSmem s = sel_carve(smem, N);
    for (int i = threadIdx.x; i < 2 * N; i += kNsgaBlock) s.obj[i] = obj[i];
    __syncthreads();
    rank2_staircase<kNsgaBlock>(N, s, wt64, wt32);
    __syncthreads();
    if (cd) crowding2<kNsgaBlock>(N, s);
    for (int i = threadIdx.x; i < N; i += kNsgaBlock) {
        if (rank) rank[i] = s.rank[i];
        if (cd) cd[i] = s.cd[i];
    }
}

// crowding from given ranks, one CTA: op API
__global__ void __launch_bounds__(kNsgaBlock) crowd2_op_kernel(const float* obj, const int32_t* rank, int N, float* cd) {
    extern __shared__ __align__(16) unsigned char smem[];
    const SelSmem s = sel_carve(smem, N);
    for (int i = threadIdx.x; i < 2 * N; i += kNsgaBlock) s.obj[i] = obj[i];
    for (int i = threadIdx.x; i < N; i += kNsgaBlock) s.rank[i] = (uint16_t)rank[i];
    __syncthreads();
    crowding2<kNsgaBlock>(N, s);
    for (int i = threadIdx.x; i < N; i += kNsgaBlock) cd[i] = s.cd[i];
}

// ---------------------------------------------------------------------------------------
// host: engine integration
// ---------------------------------------------------------------------------------------
static cudaError_t prep_select(int N) {
    const size_t smem = sel_smem_bytes(N);
    const void* fns[] = {reinterpret_cast<const void*>(nsga_select_kernel),
                         reinterpret_cast<const void*>(rank2_op_kernel),
                         reinterpret_cast<const void*>(crowd2_op_kernel)};
    for (const void* f : fns) {
        cudaError_t e = raise_smem_limit(f, smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int32_t nsga_setup(NsgaState& s, Population& pop, PopDesc* dd, const RowTile& tile, int grid, bool stage) {
    s.dd = dd;
    s.P = pop.sh.Pi;
    s.N = 2 * pop.sh.Pi;
    if (s.N > kMaxPool) return fail(BRKGA_ERR_UNSUPPORTED, "NSGA-II pool above " + std::to_string(kMaxPool));
    s.n = pop.sh.n;
    s.ld = pop.sh.ld;
    s.kind = pop.pd->kind;
    s.max_points = points_of(*pop.pd);
    s.tile = tile;
    s.grid = grid;
    s.stage = stage;
    for (int b = 0; b < 2; ++b) {
        s.keys[b] = pop.keys[b];
        s.fit[b] = pop.fit[b];
    }
    s.rank = pop.rank;
    s.cd = pop.cd;
    s.sel = pop.sel;
    s.history = pop.history;
    s.hist_cap = pop.hist_cap;
    s.Mn = pop.sh.Mn;
    const double rate = (pop.prm.mutation_rate > 0.0) ? pop.prm.mutation_rate : 5.0 / (double)pop.sh.n;
    s.mutT = prob_threshold(rate);
    s.div_interval = pop.prm.diversity_interval;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, 16);
    if (e != cudaSuccess) return fail(BRKGA_ERR_OOM, "cudaMalloc nu");
    pop.allocs.push_back(p);
    s.d_nu = (int32_t*)p;
    e = prep_select(s.N);
    if (e != cudaSuccess) return cuda_fail(e, "select set-up");
    e = raise_smem_limit(reinterpret_cast<const void*>(nsga_diversity_kernel), (size_t)s.P * 8);
    if (e != cudaSuccess) return cuda_fail(e, "diversity set-up");
    s.ready = true;
    return BRKGA_OK;
}

void nsga_release(NsgaState& s) { s.ready = false; }

void nsga_set_history(NsgaState& s, float* h, int cap) {
    s.history = h;
    s.hist_cap = cap;
}

static RowLaunch nsga_launch(const NsgaState& s, int mode) {
    RowLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.descs = s.dd;
    L.mode = mode;
    L.ntasks = s.P;
    L.max_n = s.n;
    L.max_points = s.max_points;
    L.stage_xy = s.stage ? 1 : 0;
    L.nsga_rank = s.rank;
    L.nsga_cd = s.cd;
    L.nsga_Mn = s.Mn;
    L.nsga_mutT = s.mutT;
    L.refill_from = s.d_nu;
    return L;
}

cudaError_t nsga_enqueue_init(NsgaState& s, cudaStream_t st) {
    RowLaunch L = nsga_launch(s, MODE_INIT);
    cudaError_t e = launch_rows(L, s.kind, s.tile, s.grid, st);
    if (e != cudaSuccess) return e;
    nsga_select_kernel<<<1, kNsgaBlock, sel_smem_bytes(s.P), st>>>(s.dd, s.rank, s.cd, s.sel, s.d_nu, 1);
    return cudaGetLastError();
}

cudaError_t nsga_enqueue_generation(NsgaState& s, cudaStream_t st) {
    // offspring into pool rows [P, 2P) (core/solver.hpp:1019-1032) + objectives
    RowLaunch L = nsga_launch(s, MODE_NSGA_OFF);
    cudaError_t e = launch_rows(L, s.kind, s.tile, s.grid, st);
    if (e != cudaSuccess) return e;
    // ranks, crowding, survivors of the 2P pool (core/population.hpp:409-517)
    nsga_select_kernel<<<1, kNsgaBlock, sel_smem_bytes(s.N), st>>>(s.dd, s.rank, s.cd, s.sel, s.d_nu, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int sms = device_sm_count();
    nsga_gather_kernel<<<sms * 4, 256, 0, st>>>(s.dd, s.sel);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    nsga_finish_kernel<<<1, 32, 0, st>>>(s.dd);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (s.div_interval > 0) {
        // the diversity pass decides on the device whether it is due and needed
        nsga_diversity_kernel<<<1, kNsgaBlock, (size_t)s.P * 8, st>>>(s.dd, s.div_interval, s.d_nu, s.sel);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        RowLaunch R = nsga_launch(s, MODE_NSGA_REFILL);
        e = launch_rows(R, s.kind, s.tile, s.grid, st);
        if (e != cudaSuccess) return e;
        nsga_select_kernel<<<1, kNsgaBlock, sel_smem_bytes(s.P), st>>>(s.dd, s.rank, s.cd, s.sel, s.d_nu, 2);
        e = cudaGetLastError();
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
    RowLaunch L = nsga_launch(s, MODE_EVAL);
    e = launch_rows(L, s.kind, s.tile, s.grid, st);
    if (e == cudaSuccess) {
        nsga_select_kernel<<<1, kNsgaBlock, sel_smem_bytes(s.P), st>>>(s.dd, s.rank, s.cd, s.sel, s.d_nu, 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "population evaluate");
    return BRKGA_OK;
}

// best = the front-0 member with the largest crowding distance (update_best_from_front,
// core/population.hpp:684-698), first such index on ties
int32_t nsga_get_best(NsgaState& s, cudaStream_t st, float* keys, int32_t* perm, float* obj) {
    PopDesc d;
    int32_t rc = read_desc(s, st, &d);
    if (rc != BRKGA_OK) return rc;
    std::vector<int32_t> hr(s.P);
    std::vector<float> hc(s.P), ho((size_t)s.P * 2);
    cudaMemcpy(hr.data(), s.rank, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), s.cd, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
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
        std::vector<float> k(s.n);
        cudaMemcpy(k.data(), row, (size_t)s.n * 4, cudaMemcpyDeviceToHost);
        // decode on the device through the evaluate entry point's kernel
        RowLaunch L;
        std::memset(&L, 0, sizeof(L));
        L.single = d;
        L.single.keys[0] = const_cast<float*>(row);
        L.single.cur = 0;
        float* tmpf = nullptr;
        int32_t* tmpp = nullptr;
        e = cudaMalloc(&tmpf, 16);
        if (e == cudaSuccess) e = cudaMalloc(&tmpp, (size_t)s.n * 4);
        if (e != cudaSuccess) {
            cudaFree(tmpf);
            return fail(BRKGA_ERR_OOM, "decode scratch");
        }
        L.single.fit[0] = tmpf;
        L.ntasks = 1;
        L.mode = MODE_EVAL;
        L.perm_out = tmpp;
        L.max_n = s.n;
        L.max_points = s.max_points;
        L.stage_xy = s.stage ? 1 : 0;
        e = launch_rows(L, s.kind, s.tile, 1, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaMemcpy(perm, tmpp, (size_t)s.n * 4, cudaMemcpyDeviceToHost);
        cudaFree(tmpf);
        cudaFree(tmpp);
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
    cudaMemcpy(hr.data(), s.rank, (size_t)s.P * 4, cudaMemcpyDeviceToHost);
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

// scratch for the dominance matrix of the op API (grow-only, per process)
static std::mutex g_dom_mu;
static void* g_dom_buf = nullptr;
static size_t g_dom_cap = 0;
static int g_dom_dev = -1;

}  // namespace bk

using namespace bk;

extern "C" {

int32_t brkga_pareto_rank(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream) {
    if (!d_obj || !d_rank) return fail(BRKGA_ERR_INVALID, "null argument");
    if (N < 0 || m < 1) return fail(BRKGA_ERR_INVALID, "need N >= 0 and m >= 1");
    if (N == 0) return BRKGA_OK;
    if (N > 65535) return fail(BRKGA_ERR_UNSUPPORTED, "more than 65535 points");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (m == 2 && N <= kMaxPool) {
        if ((e = prep_select(N)) != cudaSuccess) return cuda_fail(e, "rank set-up");
        rank2_op_kernel<<<1, kNsgaBlock, sel_smem_bytes(N), st>>>(d_obj, N, d_rank, nullptr);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "rank launch");
        return BRKGA_OK;
    }
    return brkga_pareto_rank_bitmatrix(d_obj, N, m, d_rank, stream);
}

int32_t brkga_pareto_rank_bitmatrix(const float* d_obj, int32_t N, int32_t m, int32_t* d_rank, void* stream) {
    if (!d_obj || !d_rank) return fail(BRKGA_ERR_INVALID, "null argument");
    if (N < 0 || m < 1) return fail(BRKGA_ERR_INVALID, "need N >= 0 and m >= 1");
    if (N == 0) return BRKGA_OK;
    const int W = (N + 31) / 32;
    const size_t smem = (size_t)N * 4 + (size_t)W * 4;
    if (smem > kMaxSmem) return fail(BRKGA_ERR_UNSUPPORTED, "too many points for the peeling kernel");
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_dom_mu);
    const size_t need = (size_t)N * W * 4;
    cudaError_t e;
    if (g_dom_dev != dev || g_dom_cap < need) {
        if (g_dom_buf) {
            cudaStreamSynchronize(st);
            cudaFree(g_dom_buf);
        }
        g_dom_buf = nullptr;
        g_dom_cap = 0;
        if ((e = cudaMalloc(&g_dom_buf, need)) != cudaSuccess) return fail(BRKGA_ERR_OOM, "dominance matrix");
        g_dom_cap = need;
        g_dom_dev = dev;
    }
    uint32_t* D = (uint32_t*)g_dom_buf;
    const long long warps = (long long)N * W;
    const int blocks = (int)std::min<long long>((warps * 32 + 255) / 256, (long long)device_sm_count() * 16);
    dom_matrix_kernel<<<blocks, 256, 0, st>>>(d_obj, N, m, W, D);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "dominance launch");
    if ((e = raise_smem_limit(reinterpret_cast<const void*>(dom_peel_kernel), smem)) != cudaSuccess)
        return cuda_fail(e, "peel set-up");
    dom_peel_kernel<<<1, kNsgaBlock, smem, st>>>(D, N, W, d_rank);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "peel launch");
    // the scratch is reused by the next call on this stream order; callers on other
    // streams are serialised by waiting here
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "peel");
    return BRKGA_OK;
}

int32_t brkga_crowding(const float* d_obj, const int32_t* d_rank, int32_t N, int32_t m, float* d_cd, void* stream) {
    if (!d_obj || !d_rank || !d_cd) return fail(BRKGA_ERR_INVALID, "null argument");
    if (m != 2) return fail(BRKGA_ERR_UNSUPPORTED, "crowding kernel handles two objectives");
    if (N < 0 || N > kMaxPool) return fail(BRKGA_ERR_UNSUPPORTED, "N outside [0, 8192]");
    if (N == 0) return BRKGA_OK;
    cudaError_t e;
    if ((e = prep_select(N)) != cudaSuccess) return cuda_fail(e, "crowding set-up");
    crowd2_op_kernel<<<1, kNsgaBlock, sel_smem_bytes(N), (cudaStream_t)stream>>>(d_obj, d_rank, N, d_cd);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "crowding launch");
    return BRKGA_OK;
}

}  // extern "C"
