/*
 * brkga_oracle.c -- CPU restatement of the reference BRKGA hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg; never linked into the product library.
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off, so float expressions round
 * exactly as written, like the reference's host code on x86-64).
 */
#include "brkga_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ================================================================================ */
/* Philox4x32-10 (Salmon et al., SC'11): 10 rounds of two 32x32->64 multiplies with   */
/* the published multipliers and Weyl key increments.                                 */
/* ================================================================================ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += PHILOX_W0; k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint32_t orc_draw(uint64_t seed, uint32_t word, uint32_t row, uint32_t gen, uint32_t stream, int lane) {
    uint32_t ctr[4] = {word, row, gen, stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    return out[lane & 3];
}

float orc_u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

uint32_t orc_prob_threshold(double p) {
    if (!(p > 0.0)) return 0u;
    if (p >= 1.0) return 1u << 24;
    double t = ceil(p * 16777216.0);
    if (t > 16777216.0) t = 16777216.0;
    return (uint32_t)t;
}

uint32_t orc_pick(uint32_t x, uint32_t k) { return (uint32_t)(((uint64_t)x * (uint64_t)k) >> 32); }

/* ================================================================================ */
/* keys and decode                                                                  */
/* ================================================================================ */
uint32_t orc_okey(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    if ((b & 0x7F800000u) == 0x7F800000u && (b & 0x007FFFFFu)) return 0xFFFFFFFFu; /* NaN */
    if (b == 0x80000000u) b = 0u;                                                   /* -0 */
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

/* configs/tsp_config.hpp:206-225: std::sort of (key, index) pairs -> tour */
void orc_decode(const float* keys, int n, int32_t* perm) {
    uint64_t* c = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) c[i] = ((uint64_t)orc_okey(keys[i]) << 32) | (uint32_t)i;
    qsort(c, (size_t)n, sizeof(uint64_t), cmp_u64);
    for (int i = 0; i < n; ++i) perm[i] = (int32_t)(uint32_t)c[i];
    free(c);
}

void orc_decode_rows(const float* keys, int rows, int n, int ld, int32_t* perm) {
    for (int r = 0; r < rows; ++r) orc_decode(keys + (size_t)r * ld, n, perm + (size_t)r * n);
}

/* ================================================================================ */
/* problems                                                                         */
/* ================================================================================ */
int orc_num_objectives(const orc_problem* pb) {
    return (pb->kind == ORC_BITSP_COORDS || pb->kind == ORC_BITSP_MATRIX || pb->kind == ORC_MOVRP) ? 2 : 1;
}
int orc_maximize(const orc_problem* pb) {
    return pb->kind == ORC_KNAP_THRESHOLD || pb->kind == ORC_KNAP_GREEDY;
}

float orc_edge(const float* xy, int a, int b) {
    float dx = xy[2 * a] - xy[2 * b];
    float dy = xy[2 * a + 1] - xy[2 * b + 1];
    float s = dx * dx;
    float t = dy * dy;
    return sqrtf(s + t);
}

static double edge64(const float* xy, int a, int b) {
    double dx = (double)xy[2 * a] - (double)xy[2 * b];
    double dy = (double)xy[2 * a + 1] - (double)xy[2 * b + 1];
    return sqrt(dx * dx + dy * dy);
}

float orc_canon_sum(const float* d, int nedges) {
    float s[256], t[256];
    for (int l = 0; l < 256; ++l) s[l] = 0.0f;
    for (int e = 0; e < nedges; ++e) s[e & 255] = s[e & 255] + d[e];
    for (int m = 16; m >= 1; m >>= 1) {
        for (int l = 0; l < 256; ++l) t[l] = s[l] + s[l ^ m];
        memcpy(s, t, sizeof(s));
    }
    float g[8];
    for (int w = 0; w < 8; ++w) g[w] = s[32 * w];
    return ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]));
}

/* node sequence of edge e for the depot tour (bi-objective TSP):
 * nodes 0 (depot) and perm[i]+1, edges depot->p0, p0->p1, ..., p_{n-1}->depot */
static void depot_edge(const int32_t* perm, int n, int e, int* a, int* b) {
    *a = (e == 0) ? 0 : perm[e - 1] + 1;
    *b = (e == n) ? 0 : perm[e] + 1;
}

static float knap_threshold(const orc_problem* pb, const float* keys) {
    /* configs/knapsack_config.hpp:43-62: float sums of integer weights/values
     * (exact below 2^24), then value - (weight - cap) * 1000 when over capacity. */
    int64_t tw = 0, tv = 0;
    for (int i = 0; i < pb->n; ++i)
        if (keys[i] > 0.5f) { tw += pb->w[i]; tv += pb->v[i]; }
    float twf = (float)tw, tvf = (float)tv;
    if (twf > pb->cap) {
        float over = twf - pb->cap;
        float pen = over * 1000.0f;
        return tvf - pen;
    }
    return tvf;
}

/* TSPJConfig::calculate_tspj_fitness (configs/tspj_config.hpp:555-585): perm[0, c) is the
 * city order (city perm+1), perm[c, 2c) the job order (job type perm-c+1).  The travel
 * time and the arrival times are the same sequential float sum; std::max is
 * (a < b) ? b : a. */
static float tspj_makespan(const orc_problem* pb, const int32_t* perm) {
    int c = pb->n / 2;
    size_t D = (size_t)c + 1;
    float travel = 0.0f, mjc = 0.0f;
    int cur = 0;
    for (int i = 0; i < c; ++i) {
        int city = perm[i] + 1, job = perm[c + i] - c + 1;
        travel = travel + pb->mat[(size_t)cur * D + city];
        float jc = travel + pb->mat2[(size_t)city * D + job];
        mjc = (mjc < jc) ? jc : mjc;
        cur = city;
    }
    float tt = travel + pb->mat[(size_t)cur * D];
    return (tt < mjc) ? mjc : tt;
}

static double tspj_makespan64(const orc_problem* pb, const int32_t* perm) {
    int c = pb->n / 2;
    size_t D = (size_t)c + 1;
    double travel = 0.0, mjc = 0.0;
    int cur = 0;
    for (int i = 0; i < c; ++i) {
        int city = perm[i] + 1, job = perm[c + i] - c + 1;
        travel += pb->mat[(size_t)cur * D + city];
        double jc = travel + pb->mat2[(size_t)city * D + job];
        if (mjc < jc) mjc = jc;
        cur = city;
    }
    double tt = travel + pb->mat[(size_t)cur * D];
    return (tt < mjc) ? mjc : tt;
}

/* the decode of one chromosome: one argsort, or for TSPJ one per component (city keys,
 * then job keys: TSPJConfig::decode_solution_internal, configs/tspj_config.hpp:606-626),
 * the second component's positions offset by c */
void orc_movrp_values(const float* keys, int n, float* val) {
    float h = 0.0f;
    for (int i = 0; i < n; ++i) h += keys[i] * (float)(i + 1);
    const float hb = h * 0.00001f;
    for (int i = 0; i < n; ++i) val[i] = keys[i] + ((float)i * 0.00001f + hb);
}

void orc_decode_problem(const orc_problem* pb, const float* keys, int32_t* perm) {
    if (pb->kind == ORC_MOVRP) {
        float* val = (float*)malloc(sizeof(float) * (size_t)(pb->n > 0 ? pb->n : 1));
        orc_movrp_values(keys, pb->n, val);
        orc_decode(val, pb->n, perm);
        free(val);
        return;
    }
    if (pb->kind == ORC_TSPJ) {
        int c = pb->n / 2;
        orc_decode(keys, c, perm);
        orc_decode(keys + c, c, perm + c);
        for (int i = 0; i < c; ++i) perm[c + i] += c;
    } else {
        orc_decode(keys, pb->n, perm);
    }
}

/* JobSchedulingGPUConfig::calculate_scheduling_fitness (configs/job_scheduling_gpu_config.hpp:132-148) */
static float jobsched_makespan(const orc_problem* pb, const float* keys) {
    int M = pb->machines;
    float* load = (float*)calloc((size_t)M, sizeof(float));
    for (int i = 0; i < pb->n; ++i) {
        int m = (int)(keys[i] * (float)M);
        if (m >= M) m = M - 1;
        if (m < 0) m = 0;
        load[m] += pb->jt[i];
    }
    float best = load[0];
    for (int m = 1; m < M; ++m)
        if (best < load[m]) best = load[m];
    free(load);
    return best;
}

/* ContinuousOptGPUConfig::calculate_sphere / _rastrigin / _rosenbrock
 * (configs/continuous_opt_gpu_config.hpp:131-173), float arithmetic in the same order */
static float continuous_value(const orc_problem* pb, const float* keys) {
    const float range = pb->hi - pb->lo;
    const int n = pb->n;
    if (pb->function == 1) {
        const float A = 10.0f, PI = 3.14159265358979323846f;
        float sum = A * (float)n;
        for (int i = 0; i < n; ++i) {
            float x = keys[i] * range + pb->lo;
            sum += x * x - A * cosf(2 * PI * x);
        }
        return sum;
    }
    float sum = 0.0f;
    if (pb->function == 2) {
        for (int i = 0; i + 1 < n; ++i) {
            float x = keys[i] * range + pb->lo;
            float xn = keys[i + 1] * range + pb->lo;
            float t1 = xn - x * x;
            float t2 = 1 - x;
            sum += 100 * t1 * t1 + t2 * t2;
        }
        return sum;
    }
    for (int i = 0; i < n; ++i) {
        float x = keys[i] * range + pb->lo;
        sum += x * x;
    }
    return sum;
}

static double continuous_value64(const orc_problem* pb, const float* keys) {
    const double range = (double)pb->hi - (double)pb->lo;
    const int n = pb->n;
    double sum = (pb->function == 1) ? 10.0 * n : 0.0;
    for (int i = 0; i < n; ++i) {
        double x = keys[i] * range + pb->lo;
        if (pb->function == 0) sum += x * x;
        else if (pb->function == 1) sum += x * x - 10.0 * cos(2.0 * 3.14159265358979323846 * x);
        else if (i + 1 < n) {
            double xn = keys[i + 1] * range + pb->lo;
            sum += 100.0 * (xn - x * x) * (xn - x * x) + (1.0 - x) * (1.0 - x);
        }
    }
    return sum;
}

double orc_continuous_f64(const orc_problem* pb, const float* keys) { return continuous_value64(pb, keys); }

static float knap_greedy(const orc_problem* pb, const int32_t* perm) {
    /* first-fit in key order: take item iff the running weight stays <= capacity */
    int64_t cap = (int64_t)floor((double)pb->cap);
    int64_t cw = 0, cv = 0;
    for (int i = 0; i < pb->n; ++i) {
        int it = perm[i];
        if (cw + pb->w[it] <= cap) { cw += pb->w[it]; cv += pb->v[it]; }
    }
    return (float)cv;
}

/* MultiObjectiveVRPConfig::decode_routes + decode_solution (configs/multi_objective_vrp_config.hpp:
 * 214-313): customers in sorted order; a customer whose demand would push a non-empty route
 * over capacity closes it (back to the depot) and opens the next; route lengths are float
 * sums in visiting order; objectives are the float sum of route lengths in route order plus
 * 100 per unit of overload of a route, and the longest route; each vehicle beyond the fleet
 * adds 500 to both.  route_of (optional) receives the route index of each position. */
static int movrp_walk(const orc_problem* pb, const int32_t* perm, float* out, int32_t* route_of) {
    const int n = pb->n, cap = pb->vcap;
    float dist = 0.0f, total = 0.0f, longest = 0.0f, pen = 0.0f;
    int load = 0, last = 0, size = 0, routes = 0;
    for (int j = 0; j < n; ++j) {
        const int cust = perm[j] + 1, dem = pb->w[cust];
        if (load + dem > cap && size > 0) {
            dist += orc_edge(pb->xy, last, 0);
            total += dist;
            if (dist > longest) longest = dist;
            if (load > cap) pen += (float)(load - cap) * 100.0f;
            ++routes;
            dist = 0.0f;
            load = 0;
            size = 0;
            last = 0;
        }
        dist += orc_edge(pb->xy, last, cust);
        load += dem;
        ++size;
        last = cust;
        if (route_of) route_of[j] = routes;
    }
    if (size > 0) {
        dist += orc_edge(pb->xy, last, 0);
        total += dist;
        if (dist > longest) longest = dist;
        if (load > cap) pen += (float)(load - cap) * 100.0f;
        ++routes;
    }
    if (out) {
        out[0] = total + pen;
        out[1] = longest;
        if (routes > pb->machines) {
            const float vp = (float)(routes - pb->machines) * 500.0f;
            out[0] += vp;
            out[1] += vp;
        }
    }
    return routes;
}

int orc_movrp_routes(const orc_problem* pb, const int32_t* perm, int32_t* route_of) {
    return movrp_walk(pb, perm, NULL, route_of);
}

void orc_eval_perm(const orc_problem* pb, const int32_t* perm, const float* keys, float* out) {
    int n = pb->n;
    switch (pb->kind) {
    case ORC_TSP_COORDS:
    case ORC_TSP_MATRIX: {
        float* d = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
        for (int e = 0; e < n; ++e) {
            int a = perm[e], b = perm[(e + 1) % n];
            d[e] = (pb->kind == ORC_TSP_COORDS) ? orc_edge(pb->xy, a, b) : pb->mat[(size_t)a * n + b];
        }
        out[0] = orc_canon_sum(d, n);
        free(d);
        break;
    }
    case ORC_BITSP_COORDS:
    case ORC_BITSP_MATRIX: {
        float* d0 = (float*)malloc(sizeof(float) * (size_t)(n + 1));
        float* d1 = (float*)malloc(sizeof(float) * (size_t)(n + 1));
        for (int e = 0; e <= n; ++e) {
            int a, b;
            depot_edge(perm, n, e, &a, &b);
            if (pb->kind == ORC_BITSP_COORDS) {
                d0[e] = orc_edge(pb->xy, a, b);
                d1[e] = orc_edge(pb->xy2, a, b);
            } else {
                d0[e] = pb->mat[(size_t)a * (n + 1) + b];
                d1[e] = pb->mat2[(size_t)a * (n + 1) + b];
            }
        }
        out[0] = orc_canon_sum(d0, n + 1);
        out[1] = orc_canon_sum(d1, n + 1);
        free(d0);
        free(d1);
        break;
    }
    case ORC_KNAP_THRESHOLD: out[0] = knap_threshold(pb, keys); break;
    case ORC_KNAP_GREEDY: out[0] = knap_greedy(pb, perm); break;
    case ORC_TSPJ: out[0] = tspj_makespan(pb, perm); break;
    case ORC_JOBSCHED: out[0] = jobsched_makespan(pb, keys); break;
    case ORC_CONTINUOUS: out[0] = continuous_value(pb, keys); break;
    case ORC_MOVRP: movrp_walk(pb, perm, out, NULL); break;
    default: out[0] = NAN;
    }
}

void orc_eval_perm_f64(const orc_problem* pb, const int32_t* perm, double* out) {
    int n = pb->n;
    if (pb->kind == ORC_TSP_COORDS || pb->kind == ORC_TSP_MATRIX) {
        double s = 0.0;
        for (int e = 0; e < n; ++e) {
            int a = perm[e], b = perm[(e + 1) % n];
            s += (pb->kind == ORC_TSP_COORDS) ? edge64(pb->xy, a, b) : (double)pb->mat[(size_t)a * n + b];
        }
        out[0] = s;
    } else if (pb->kind == ORC_BITSP_COORDS || pb->kind == ORC_BITSP_MATRIX) {
        double s0 = 0.0, s1 = 0.0;
        for (int e = 0; e <= n; ++e) {
            int a, b;
            depot_edge(perm, n, e, &a, &b);
            if (pb->kind == ORC_BITSP_COORDS) {
                s0 += edge64(pb->xy, a, b);
                s1 += edge64(pb->xy2, a, b);
            } else {
                s0 += pb->mat[(size_t)a * (n + 1) + b];
                s1 += pb->mat2[(size_t)a * (n + 1) + b];
            }
        }
        out[0] = s0;
        out[1] = s1;
    } else if (pb->kind == ORC_TSPJ) {
        out[0] = tspj_makespan64(pb, perm);
    } else {
        out[0] = NAN;
    }
}

float orc_tsp_len_seq(const orc_problem* pb, const int32_t* perm) {
    int n = pb->n;
    float s = 0.0f;
    for (int e = 0; e < n; ++e) {
        int a = perm[e], b = perm[(e + 1) % n];
        s += (pb->kind == ORC_TSP_COORDS) ? orc_edge(pb->xy, a, b) : pb->mat[(size_t)a * n + b];
    }
    return s;
}

void orc_evaluate(const orc_problem* pb, const float* keys, int rows, int ld, float* fit) {
    int m = orc_num_objectives(pb);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(pb->n > 0 ? pb->n : 1));
    for (int r = 0; r < rows; ++r) {
        const float* k = keys + (size_t)r * ld;
        if (pb->kind != ORC_KNAP_THRESHOLD && pb->kind != ORC_JOBSCHED && pb->kind != ORC_CONTINUOUS)
            orc_decode_problem(pb, k, perm);
        orc_eval_perm(pb, perm, k, fit + (size_t)r * m);
    }
    free(perm);
}

void orc_local_search(const orc_problem* pb, float* pop, float* fit, const int32_t* rows, int count, int ld,
                      int moves, uint64_t seed, uint32_t gen, int island) {
    int c = pb->n / 2;
    float* row = (float*)malloc(sizeof(float) * (size_t)(ld > 0 ? ld : 1));
    for (int q = 0; q < count; ++q) {
        int r = rows[q];
        memcpy(row, pop + (size_t)r * ld, sizeof(float) * (size_t)ld);
        for (int mv = 0; mv < moves; ++mv) {
            uint32_t st = ((uint32_t)island << 8) | ORC_TAG_LS;
            int i = (int)orc_pick(orc_draw(seed, (uint32_t)mv, (uint32_t)q, gen, st, 0), (uint32_t)c);
            int j = (int)orc_pick(orc_draw(seed, (uint32_t)mv, (uint32_t)q, gen, st, 1), (uint32_t)c);
            if (i > j) { int tmp = i; i = j; j = tmp; }
            if (j - i < 2) continue;
            while (i < j) { float u = row[i]; row[i] = row[j]; row[j] = u; ++i; --j; }
        }
        float f;
        orc_evaluate(pb, row, 1, ld, &f);
        if (orc_maximize(pb) ? (f > fit[r]) : (f < fit[r])) {
            memcpy(pop + (size_t)r * ld, row, sizeof(float) * (size_t)ld);
            fit[r] = f;
        }
    }
    free(row);
}

/* ================================================================================ */
/* BRKGA                                                                            */
/* ================================================================================ */
static uint32_t fit_key(float f, int maximize) {
    uint32_t k = orc_okey(f);
    if (!maximize) return k;
    return (k == 0xFFFFFFFFu) ? 0xFFFFFFFFu : ~k;
}

void orc_sort_fitness(const float* fit, int P, int maximize, int32_t* sorted) {
    uint64_t* c = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(P > 0 ? P : 1));
    for (int i = 0; i < P; ++i) c[i] = ((uint64_t)fit_key(fit[i], maximize) << 32) | (uint32_t)i;
    qsort(c, (size_t)P, sizeof(uint64_t), cmp_u64);
    for (int i = 0; i < P; ++i) sorted[i] = (int32_t)(uint32_t)c[i];
    free(c);
}

void orc_generation_core(int P, int E, int M, int n, int ld,
                         const float* pop, const float* fit, const int32_t* sorted,
                         const int32_t* ep, const int32_t* np, const uint8_t* coin,
                         const float* mut, float* newpop, float* newfit) {
    int off = P - E - M;
    for (int r = 0; r < E; ++r) {
        memcpy(newpop + (size_t)r * ld, pop + (size_t)sorted[r] * ld, sizeof(float) * (size_t)n);
        newfit[r] = fit[sorted[r]];
    }
    for (int i = 0; i < off; ++i) {
        const float* a = pop + (size_t)sorted[ep[i]] * ld;
        const float* b = pop + (size_t)sorted[E + np[i]] * ld;
        float* c = newpop + (size_t)(E + i) * ld;
        for (int j = 0; j < n; ++j) c[j] = coin[(size_t)i * n + j] ? a[j] : b[j];
    }
    for (int i = 0; i < M; ++i)
        memcpy(newpop + (size_t)(P - M + i) * ld, mut + (size_t)i * n, sizeof(float) * (size_t)n);
    for (int r = 0; r < P; ++r)
        for (int j = n; j < ld; ++j) newpop[(size_t)r * ld + j] = 0.0f;
}

static uint32_t stream_id(int island, int tag) { return ((uint32_t)island << 8) | (uint32_t)tag; }

void orc_brkga_generation(const orc_problem* pb, const orc_params* pr, uint32_t g,
                          const float* pop, const float* fit, const int32_t* sorted, int ld,
                          float* newpop, float* newfit) {
    int P = pr->P, E = pr->E, M = pr->M, n = pb->n, off = P - E - M;
    int32_t* ep = (int32_t*)malloc(sizeof(int32_t) * (size_t)(off > 0 ? off : 1));
    int32_t* np = (int32_t*)malloc(sizeof(int32_t) * (size_t)(off > 0 ? off : 1));
    uint8_t* coin = (uint8_t*)malloc((size_t)(off > 0 ? off : 1) * (size_t)n);
    float* mut = (float*)malloc(sizeof(float) * (size_t)(M > 0 ? M : 1) * (size_t)n);
    uint32_t T = orc_prob_threshold(pr->rho);
    uint32_t sp = stream_id(pr->island, ORC_TAG_PARENT);
    uint32_t sc = stream_id(pr->island, ORC_TAG_COIN);
    uint32_t sm = stream_id(pr->island, ORC_TAG_MUTANT);
    uint32_t key[2] = {(uint32_t)pr->seed, (uint32_t)(pr->seed >> 32)};
    for (int i = 0; i < off; ++i) {
        uint32_t r = (uint32_t)(E + i), out[4];
        uint32_t ctr[4] = {0u, r, g, sp};
        orc_philox4x32_10(ctr, key, out);
        ep[i] = (int32_t)orc_pick(out[0], (uint32_t)E);
        np[i] = (int32_t)orc_pick(out[1], (uint32_t)(P - E));
        for (int q = 0; q < n; q += 4) {
            uint32_t c4[4] = {(uint32_t)(q >> 2), r, g, sc};
            orc_philox4x32_10(c4, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) coin[(size_t)i * n + q + l] = (out[l] >> 8) < T;
        }
    }
    for (int i = 0; i < M; ++i) {
        uint32_t r = (uint32_t)(P - M + i), out[4];
        for (int q = 0; q < n; q += 4) {
            uint32_t c4[4] = {(uint32_t)(q >> 2), r, g, sm};
            orc_philox4x32_10(c4, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) mut[(size_t)i * n + q + l] = orc_u24(out[l]);
        }
    }
    orc_generation_core(P, E, M, n, ld, pop, fit, sorted, ep, np, coin, mut, newpop, newfit);
    orc_evaluate(pb, newpop + (size_t)E * ld, P - E, ld, newfit + E);
    free(ep); free(np); free(coin); free(mut);
}

void orc_brkga_init(const orc_problem* pb, const orc_params* pr, int ld, float* pop, float* fit) {
    int P = pr->P, n = pb->n;
    uint32_t key[2] = {(uint32_t)pr->seed, (uint32_t)(pr->seed >> 32)};
    uint32_t s = stream_id(pr->island, ORC_TAG_INIT);
    for (int r = 0; r < P; ++r) {
        float* row = pop + (size_t)r * ld;
        for (int q = 0; q < n; q += 4) {
            uint32_t ctr[4] = {(uint32_t)(q >> 2), (uint32_t)r, 0u, s}, out[4];
            orc_philox4x32_10(ctr, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) row[q + l] = orc_u24(out[l]);
        }
        for (int j = n; j < ld; ++j) row[j] = 0.0f;
    }
    orc_evaluate(pb, pop, P, ld, fit);
}

void orc_migrate(int k, int Pi, int m, int n, int ld, int maximize,
                 float* pop, float* fit, int32_t* sorted) {
    if (k < 2 || m <= 0) return;
    float* mk = (float*)malloc(sizeof(float) * (size_t)k * m * n);
    float* mf = (float*)malloc(sizeof(float) * (size_t)k * m);
    for (int i = 0; i < k; ++i)
        for (int q = 0; q < m; ++q) {
            int row = i * Pi + sorted[i * Pi + q];
            memcpy(mk + ((size_t)i * m + q) * n, pop + (size_t)row * ld, sizeof(float) * (size_t)n);
            mf[i * m + q] = fit[row];
        }
    for (int i = 0; i < k; ++i) {
        int src = (i + k - 1) % k;
        for (int q = 0; q < m; ++q) {
            int row = i * Pi + sorted[i * Pi + Pi - m + q];
            memcpy(pop + (size_t)row * ld, mk + ((size_t)src * m + q) * n, sizeof(float) * (size_t)n);
            fit[row] = mf[src * m + q];
        }
    }
    for (int i = 0; i < k; ++i) orc_sort_fitness(fit + (size_t)i * Pi, Pi, maximize, sorted + (size_t)i * Pi);
    free(mk);
    free(mf);
}

void orc_brkga_run(const orc_problem* pb, const orc_params* pr, int G, int ld,
                   float* pop, float* fit, int32_t* sorted, float* history) {
    int P = pr->P, mx = orc_maximize(pb);
    float* np = (float*)malloc(sizeof(float) * (size_t)P * ld);
    float* nf = (float*)malloc(sizeof(float) * (size_t)P);
    orc_brkga_init(pb, pr, ld, pop, fit);
    orc_sort_fitness(fit, P, mx, sorted);
    history[0] = fit[sorted[0]];
    for (int g = 1; g <= G; ++g) {
        orc_brkga_generation(pb, pr, (uint32_t)g, pop, fit, sorted, ld, np, nf);
        memcpy(pop, np, sizeof(float) * (size_t)P * ld);
        memcpy(fit, nf, sizeof(float) * (size_t)P);
        orc_sort_fitness(fit, P, mx, sorted);
        history[g] = fit[sorted[0]];
    }
    free(np);
    free(nf);
}

/* ================================================================================ */
/* NSGA-II                                                                          */
/* ================================================================================ */
/* core/individual.hpp:99-114: <= on every objective and < on at least one */
static int dominates(const float* a, const float* b, int m) {
    int better = 0;
    for (int i = 0; i < m; ++i) {
        if (a[i] > b[i]) return 0;
        if (a[i] < b[i]) better = 1;
    }
    return better;
}

/* Front peeling by domination counts.  `front0_weight` is how many times each member of
 * the first front decrements the points it dominates: the reference pushes every rank-0
 * point into fronts[0] twice -- once in fast_non_dominated_sort (core/population.hpp:
 * 431-434) and again at the top of build_fronts_from_domination (:335-340) -- so its
 * first front decrements twice (weight 2); textbook NSGA-II ranks use weight 1.  A point
 * takes rank k+1 when its count first drops to zero or below while front k is processed. */
static void ranks_impl(const float* obj, int N, int m, int front0_weight, int32_t* rank) {
    int* cnt = (int*)calloc((size_t)(N > 0 ? N : 1), sizeof(int));
    unsigned char* done = (unsigned char*)calloc((size_t)(N > 0 ? N : 1), 1);
    int* front = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    int* next = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    int fs = 0;
    for (int p = 0; p < N; ++p) {
        for (int q = 0; q < N; ++q)
            if (p != q && dominates(obj + (size_t)q * m, obj + (size_t)p * m, m)) cnt[p]++;
        if (cnt[p] == 0) { front[fs++] = p; rank[p] = 0; done[p] = 1; }
    }
    int k = 0;
    while (fs > 0) {
        int ns = 0;
        int wgt = (k == 0) ? front0_weight : 1;
        for (int i = 0; i < fs; ++i)
            for (int q = 0; q < N; ++q) {
                if (done[q] || !dominates(obj + (size_t)front[i] * m, obj + (size_t)q * m, m)) continue;
                cnt[q] -= wgt;
                if (cnt[q] <= 0) { done[q] = 1; rank[q] = k + 1; next[ns++] = q; }
            }
        int* t = front; front = next; next = t;
        fs = ns;
        ++k;
    }
    free(cnt); free(done); free(front); free(next);
}

/* the reference's ranks (front-0 weight 2) */
void orc_pareto_ranks(const float* obj, int N, int m, int32_t* rank) { ranks_impl(obj, N, m, 2, rank); }
/* textbook Pareto ranks */
void orc_pareto_ranks_strict(const float* obj, int N, int m, int32_t* rank) { ranks_impl(obj, N, m, 1, rank); }

/* crowding over the reference's front lists: every rank-0 point appears twice in
 * fronts[0] (see ranks_impl), later fronts once.  Per front and objective the list is
 * sorted by (objective, index, copy); the first and last entries get +inf, interior
 * entries add (next - prev) / range to their point when range > 0; lists of size <= 2
 * are all +inf (core/population.hpp:453-489).  A point listed twice receives both of its
 * entries' contributions in list order. */
typedef struct { uint32_t k; int idx; int copy; } ent_t;
static int cmp_ent(const void* a, const void* b) {
    const ent_t* x = (const ent_t*)a;
    const ent_t* y = (const ent_t*)b;
    if (x->k != y->k) return (x->k > y->k) - (x->k < y->k);
    if (x->idx != y->idx) return (x->idx > y->idx) - (x->idx < y->idx);
    return (x->copy > y->copy) - (x->copy < y->copy);
}

static void crowding_impl(const float* obj, const int32_t* rank, int N, int m, int double0,
                          float* cd32, double* cd64) {
    int maxr = -1;
    for (int i = 0; i < N; ++i) if (rank[i] > maxr) maxr = rank[i];
    ent_t* buf = (ent_t*)malloc(sizeof(ent_t) * 2 * (size_t)(N > 0 ? N : 1));
    for (int r = 0; r <= maxr; ++r) {
        int fs = 0;
        int copies = (r == 0 && double0) ? 2 : 1;
        for (int i = 0; i < N; ++i)
            if (rank[i] == r)
                for (int c = 0; c < copies; ++c) { buf[fs].idx = i; buf[fs].copy = c; ++fs; }
        if (fs == 0) continue;
        if (fs <= 2) {
            for (int i = 0; i < fs; ++i) {
                if (cd32) cd32[buf[i].idx] = INFINITY;
                if (cd64) cd64[buf[i].idx] = INFINITY;
            }
            continue;
        }
        for (int i = 0; i < fs; ++i) {
            if (cd32) cd32[buf[i].idx] = 0.0f;
            if (cd64) cd64[buf[i].idx] = 0.0;
        }
        for (int o = 0; o < m; ++o) {
            for (int i = 0; i < fs; ++i) buf[i].k = orc_okey(obj[(size_t)buf[i].idx * m + o]);
            qsort(buf, (size_t)fs, sizeof(ent_t), cmp_ent);
#define V(i) obj[(size_t)buf[i].idx * m + o]
            int lo = buf[0].idx, hi = buf[fs - 1].idx;
            if (cd32) { cd32[lo] = INFINITY; cd32[hi] = INFINITY; }
            if (cd64) { cd64[lo] = INFINITY; cd64[hi] = INFINITY; }
            float range = V(fs - 1) - V(0);
            double range64 = (double)V(fs - 1) - (double)V(0);
            if (range > 0.0f) {
                for (int i = 1; i < fs - 1; ++i) {
                    if (cd32) {
                        float d = (V(i + 1) - V(i - 1)) / range;
                        cd32[buf[i].idx] = cd32[buf[i].idx] + d;
                    }
                    if (cd64) cd64[buf[i].idx] += ((double)V(i + 1) - (double)V(i - 1)) / range64;
                }
            }
#undef V
        }
    }
    free(buf);
}

void orc_crowding_f32(const float* obj, const int32_t* rank, int N, int m, float* cd) {
    crowding_impl(obj, rank, N, m, 1, cd, NULL);
}
void orc_crowding_f64(const float* obj, const int32_t* rank, int N, int m, double* cd) {
    crowding_impl(obj, rank, N, m, 1, NULL, cd);
}
void orc_crowding_strict_f32(const float* obj, const int32_t* rank, int N, int m, float* cd) {
    crowding_impl(obj, rank, N, m, 0, cd, NULL);
}

/* select_next_generation_nsga2 (core/population.hpp:491-517) over the same front lists:
 * fronts are appended whole while they fit (rank-0 points twice), each in the order the
 * crowding pass left it -- sorted by the last objective, then index; the first front that
 * does not fit is sorted by crowding descending (ties by index) and truncated. */
int orc_nsga2_select(const int32_t* rank, const float* cd, const float* obj, int N, int m, int P,
                     int32_t* sel) {
    int maxr = -1;
    for (int i = 0; i < N; ++i) if (rank[i] > maxr) maxr = rank[i];
    ent_t* buf = (ent_t*)malloc(sizeof(ent_t) * 2 * (size_t)(N > 0 ? N : 1));
    int taken = 0;
    for (int r = 0; r <= maxr && taken < P; ++r) {
        int fs = 0;
        int copies = (r == 0) ? 2 : 1;
        for (int i = 0; i < N; ++i)
            if (rank[i] == r)
                for (int c = 0; c < copies; ++c) { buf[fs].idx = i; buf[fs].copy = c; ++fs; }
        if (taken + fs <= P) {
            for (int i = 0; i < fs; ++i) buf[i].k = orc_okey(obj[(size_t)buf[i].idx * m + (m - 1)]);
        } else {
            for (int i = 0; i < fs; ++i) {
                uint32_t ck = orc_okey(cd[buf[i].idx]);
                buf[i].k = (ck == 0xFFFFFFFFu) ? 0xFFFFFFFFu : ~ck;
            }
        }
        qsort(buf, (size_t)fs, sizeof(ent_t), cmp_ent);
        for (int i = 0; i < fs && taken < P; ++i) sel[taken++] = buf[i].idx;
    }
    free(buf);
    return taken;
}

/* core/solver.hpp:1042-1056: two uniform picks; lower rank wins, then larger crowding,
 * else the second pick */
static int tournament(int i1, int i2, const int32_t* rank, const float* cd) {
    if (rank[i1] < rank[i2]) return i1;
    if (rank[i2] < rank[i1]) return i2;
    if (cd[i1] > cd[i2]) return i1;
    return i2;
}

void orc_nsga2_offspring_core(int P, int n, int ld, const float* pop, const int32_t* rank,
                              const float* cd, const int32_t* picks, const uint8_t* coin,
                              const uint8_t* mflag, const float* mkey, float* off) {
    for (int i = 0; i < P; ++i) {
        float* c = off + (size_t)i * ld;
        int p1 = tournament(picks[4 * i], picks[4 * i + 1], rank, cd);
        int p2 = tournament(picks[4 * i + 2], picks[4 * i + 3], rank, cd);
        const float* a = pop + (size_t)p1 * ld;
        const float* b = pop + (size_t)p2 * ld;
        for (int j = 0; j < n; ++j) {
            size_t q = (size_t)i * n + j;
            float v = coin[q] ? a[j] : b[j];
            if (mflag[q]) v = mkey[q];
            c[j] = v;
        }
        for (int j = n; j < ld; ++j) c[j] = 0.0f;
    }
}

void orc_nsga2_offspring(const orc_nsga2_params* pr, uint32_t g, int n, int ld,
                         const float* pop, const int32_t* rank, const float* cd,
                         float* off) {
    int P = pr->P, Mn = pr->Mn;
    if (Mn < 0) Mn = 0;
    if (Mn > P) Mn = P;
    int Pc = P - Mn;
    uint32_t key[2] = {(uint32_t)pr->seed, (uint32_t)(pr->seed >> 32)};
    uint32_t Tc = orc_prob_threshold(pr->rho);
    uint32_t Tm = orc_prob_threshold(pr->mut_rate);
    size_t cells = (size_t)(Pc > 0 ? Pc : 1) * (size_t)(n > 0 ? n : 1);
    int32_t* picks = (int32_t*)malloc(sizeof(int32_t) * 4 * (size_t)(Pc > 0 ? Pc : 1));
    uint8_t* coin = (uint8_t*)malloc(cells);
    uint8_t* mflag = (uint8_t*)malloc(cells);
    float* mkey = (float*)malloc(sizeof(float) * cells);
    for (int i = 0; i < Pc; ++i) {
        uint32_t out[4], o2[4], o3[4];
        uint32_t ctr[4] = {0u, (uint32_t)i, g, ORC_TAG_NSGA_TOUR};
        orc_philox4x32_10(ctr, key, out);
        for (int l = 0; l < 4; ++l) picks[4 * i + l] = (int32_t)orc_pick(out[l], (uint32_t)P);
        for (int q = 0; q < n; q += 4) {
            uint32_t cc[4] = {(uint32_t)(q >> 2), (uint32_t)i, g, ORC_TAG_NSGA_COIN};
            uint32_t cm[4] = {(uint32_t)(q >> 2), (uint32_t)i, g, ORC_TAG_NSGA_MUTP};
            uint32_t ck[4] = {(uint32_t)(q >> 2), (uint32_t)i, g, ORC_TAG_NSGA_MUTK};
            orc_philox4x32_10(cc, key, out);
            orc_philox4x32_10(cm, key, o2);
            orc_philox4x32_10(ck, key, o3);
            for (int l = 0; l < 4 && q + l < n; ++l) {
                size_t x = (size_t)i * n + q + l;
                coin[x] = (out[l] >> 8) < Tc;
                mflag[x] = (o2[l] >> 8) < Tm;
                mkey[x] = orc_u24(o3[l]);
            }
        }
    }
    orc_nsga2_offspring_core(Pc, n, ld, pop, rank, cd, picks, coin, mflag, mkey, off);
    for (int i = Pc; i < P; ++i) {
        float* c = off + (size_t)i * ld;
        uint32_t out[4];
        for (int q = 0; q < n; q += 4) {
            uint32_t ctr[4] = {(uint32_t)(q >> 2), (uint32_t)i, g, ORC_TAG_MUTANT};
            orc_philox4x32_10(ctr, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) c[q + l] = orc_u24(out[l]);
        }
        for (int j = n; j < ld; ++j) c[j] = 0.0f;
    }
    free(picks); free(coin); free(mflag); free(mkey);
}

static void nsga2_rank_crowd(int N, int m, const float* obj, int32_t* rank, float* cd) {
    orc_pareto_ranks(obj, N, m, rank);
    orc_crowding_f32(obj, rank, N, m, cd);
}

void orc_nsga2_init(const orc_problem* pb, const orc_nsga2_params* pr, int ld,
                    float* pop, float* obj, int32_t* rank, float* cd) {
    orc_params bp;
    memset(&bp, 0, sizeof(bp));
    bp.P = pr->P;
    bp.seed = pr->seed;
    int n = pb->n, P = pr->P;
    uint32_t key[2] = {(uint32_t)pr->seed, (uint32_t)(pr->seed >> 32)};
    for (int r = 0; r < P; ++r) {
        float* row = pop + (size_t)r * ld;
        for (int q = 0; q < n; q += 4) {
            uint32_t ctr[4] = {(uint32_t)(q >> 2), (uint32_t)r, 0u, ORC_TAG_INIT}, out[4];
            orc_philox4x32_10(ctr, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) row[q + l] = orc_u24(out[l]);
        }
        for (int j = n; j < ld; ++j) row[j] = 0.0f;
    }
    orc_evaluate(pb, pop, P, ld, obj);
    nsga2_rank_crowd(P, orc_num_objectives(pb), obj, rank, cd);
}

int orc_nsga2_diversity(const orc_problem* pb, const orc_nsga2_params* pr, uint32_t g, int ld,
                        float* pop, float* obj, int32_t* rank, float* cd) {
    /* core/population.hpp:130-182: greedy in-order dedupe in objective space
     * (Euclidean distance < 0.001 with float differences squared in double);
     * rebuild when fewer than 70% are unique. */
    int P = pr->P, m = orc_num_objectives(pb), n = pb->n;
    int* uniq = (int*)malloc(sizeof(int) * (size_t)P);
    int nu = 0;
    for (int c = 0; c < P; ++c) {
        int ok = 1;
        for (int u = 0; u < nu && ok; ++u) {
            double dist = 0.0;
            for (int o = 0; o < m; ++o) {
                double diff = (double)(obj[(size_t)c * m + o] - obj[(size_t)uniq[u] * m + o]);
                dist += diff * diff;
            }
            if (sqrt(dist) < 0.001) ok = 0;
        }
        if (ok) uniq[nu++] = c;
    }
    double ratio = (double)nu / (double)P;
    if (!(ratio < 0.70)) { free(uniq); return 0; }
    float* np = (float*)malloc(sizeof(float) * (size_t)P * ld);
    float* no = (float*)malloc(sizeof(float) * (size_t)P * m);
    for (int i = 0; i < nu; ++i) {
        memcpy(np + (size_t)i * ld, pop + (size_t)uniq[i] * ld, sizeof(float) * (size_t)ld);
        memcpy(no + (size_t)i * m, obj + (size_t)uniq[i] * m, sizeof(float) * (size_t)m);
    }
    uint32_t key[2] = {(uint32_t)pr->seed, (uint32_t)(pr->seed >> 32)};
    for (int r = nu; r < P; ++r) {
        float* row = np + (size_t)r * ld;
        for (int q = 0; q < n; q += 4) {
            uint32_t ctr[4] = {(uint32_t)(q >> 2), (uint32_t)r, g, ORC_TAG_NSGA_REFILL}, out[4];
            orc_philox4x32_10(ctr, key, out);
            for (int l = 0; l < 4 && q + l < n; ++l) row[q + l] = orc_u24(out[l]);
        }
        for (int j = n; j < ld; ++j) row[j] = 0.0f;
    }
    if (P > nu) orc_evaluate(pb, np + (size_t)nu * ld, P - nu, ld, no + (size_t)nu * m);
    memcpy(pop, np, sizeof(float) * (size_t)P * ld);
    memcpy(obj, no, sizeof(float) * (size_t)P * m);
    nsga2_rank_crowd(P, m, obj, rank, cd);
    free(np);
    free(no);
    free(uniq);
    return 1;
}

void orc_nsga2_generation(const orc_problem* pb, const orc_nsga2_params* pr, uint32_t g, int ld,
                          float* pop, float* obj, int32_t* rank, float* cd) {
    int P = pr->P, N = 2 * P, m = orc_num_objectives(pb), n = pb->n;
    float* pk = (float*)malloc(sizeof(float) * (size_t)N * ld);
    float* po = (float*)malloc(sizeof(float) * (size_t)N * m);
    int32_t* pr_ = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    float* pc = (float*)malloc(sizeof(float) * (size_t)N);
    int32_t* sel = (int32_t*)malloc(sizeof(int32_t) * (size_t)P);
    memcpy(pk, pop, sizeof(float) * (size_t)P * ld);
    memcpy(po, obj, sizeof(float) * (size_t)P * m);
    orc_nsga2_offspring(pr, g, n, ld, pop, rank, cd, pk + (size_t)P * ld);
    orc_evaluate(pb, pk + (size_t)P * ld, P, ld, po + (size_t)P * m);
    nsga2_rank_crowd(N, m, po, pr_, pc);
    orc_nsga2_select(pr_, pc, po, N, m, P, sel);
    for (int i = 0; i < P; ++i) {
        memcpy(pop + (size_t)i * ld, pk + (size_t)sel[i] * ld, sizeof(float) * (size_t)ld);
        memcpy(obj + (size_t)i * m, po + (size_t)sel[i] * m, sizeof(float) * (size_t)m);
        rank[i] = pr_[sel[i]];
        cd[i] = pc[sel[i]];
    }
    /* core/solver.hpp:810-812: diversity check after selection, every 25 generations
     * counted from 0 (the generation being produced is g, the reference's counter g-1) */
    if (pr->diversity_interval > 0 && ((g - 1) % (uint32_t)pr->diversity_interval) == 0)
        orc_nsga2_diversity(pb, pr, g, ld, pop, obj, rank, cd);
    free(pk); free(po); free(pr_); free(pc); free(sel);
}
