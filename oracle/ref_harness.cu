// ref_harness.cu -- drives the UNMODIFIED reference headers (hsaseendran/llm-brkga,
// brkga/core and brkga/configs) on injected inputs, so the oracle can be pinned to the
// reference's own behaviour and the reference's CPU path can be timed.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile from the reference tree into
// oracle/_ref/libref.so (git-ignored); loaded by tests/ (parity pins), by
// tests/golden/make_golden.py and by bench.py's reference arm.
//
// The reference keeps its RNG and generation operators private; this file widens
// access (after every standard header is included) so that a generation can be run
// with a seeded mt19937 and the draws it consumed can be replayed.  Every device
// must be hidden (CUDA_VISIBLE_DEVICES="") so the reference takes its CPU path
// (core/solver.hpp:1353-1386, configs/tsp_config.hpp:114-123).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <future>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <omp.h>
#include <unistd.h>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/gather.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#define private public
#define protected public
#include "core/solver.hpp"
#include "configs/tsp_config.hpp"
#include "configs/knapsack_config.hpp"
#include "configs/multi_tsp_config.hpp"
#include "configs/tspj_config.hpp"
#include "configs/job_scheduling_gpu_config.hpp"
#include "configs/continuous_opt_gpu_config.hpp"
#include "configs/multi_objective_vrp_config.hpp"
#undef private
#undef protected

using Mat = std::vector<std::vector<float>>;

// distance matrix exactly as configs/tsp_config.hpp:359-371 builds it from coordinates
static Mat coords_to_matrix(const float* xy, int n) {
    Mat d(n, std::vector<float>(n, 0.0f));
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            if (i == j) { d[i][j] = 0; continue; }
            float dx = xy[2 * i] - xy[2 * j];
            float dy = xy[2 * i + 1] - xy[2 * j + 1];
            d[i][j] = std::sqrt(dx * dx + dy * dy);
        }
    return d;
}

static Mat flat_to_matrix(const float* m, int n) {
    Mat d(n, std::vector<float>(n));
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) d[i][j] = m[(size_t)i * n + j];
    return d;
}

static void set_keys(Individual<float>& ind, const float* row, int n) {
    auto& c = ind.get_chromosome();
    c.assign(row, row + n);
}

extern "C" {

int ref_version() { return 1; }

// TSPConfig decode + fitness (configs/tsp_config.hpp:180-225)
int ref_tsp_eval(const float* xy, const float* mat, int n, const float* keys, int rows,
                 float* fit, int32_t* perm) {
    try {
        Mat d = xy ? coords_to_matrix(xy, n) : flat_to_matrix(mat, n);
        TSPConfig<float> cfg(d, "ref");
        Individual<float> ind(n);
        for (int r = 0; r < rows; r++) {
            set_keys(ind, keys + (size_t)r * n, n);
            fit[r] = cfg.fitness_function(ind);
            if (perm) {
                auto sol = cfg.decoder(ind);
                for (int i = 0; i < n; i++) perm[(size_t)r * n + i] = (int32_t)sol[0][i];
            }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// KnapsackConfig threshold fitness (configs/knapsack_config.hpp:43-62)
int ref_knap_eval(const float* w, const float* v, float cap, int n, const float* keys, int rows,
                  float* fit) {
    try {
        std::vector<float> W(w, w + n), V(v, v + n);
        KnapsackConfig<float> cfg(W, V, cap, "ref");
        Individual<float> ind(n);
        for (int r = 0; r < rows; r++) {
            set_keys(ind, keys + (size_t)r * n, n);
            fit[r] = cfg.fitness_function(ind);
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// MultiTSPConfig objectives (configs/multi_tsp_config.hpp:54-103); matrices are dim x dim
int ref_bitsp_eval(const float* m0, const float* m1, int dim, const float* keys, int rows,
                   float* obj) {
    try {
        MultiTSPConfig<float> cfg(flat_to_matrix(m0, dim), flat_to_matrix(m1, dim), "ref");
        int n = dim - 1;
        Individual<float> ind(std::vector<int>{n}, 2);
        for (int r = 0; r < rows; r++) {
            set_keys(ind, keys + (size_t)r * n, n);
            obj[2 * r] = cfg.objective_functions[0](ind);
            obj[2 * r + 1] = cfg.objective_functions[1](ind);
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// TSPJConfig decode + makespan (configs/tspj_config.hpp:555-626); matrices are dim x dim
// (depot + c cities), each key row holds the c city keys then the c job keys; perm gets
// the city tour (cities 1..c) then the job order (types 1..c)
int ref_tspj_eval(const float* travel, const float* jobs, int dim, const float* keys, int rows, float* fit,
                  int32_t* perm) {
    try {
        TSPJConfig<float> cfg(flat_to_matrix(travel, dim), flat_to_matrix(jobs, dim), "ref");
        const int c = dim - 1;
        Individual<float> ind(std::vector<int>{c, c});
        for (int r = 0; r < rows; r++) {
            const float* row = keys + (size_t)r * 2 * c;
            ind.chromosomes[0].assign(row, row + c);
            ind.chromosomes[1].assign(row + c, row + 2 * c);
            fit[r] = cfg.fitness_function(ind);
            if (perm) {
                auto sol = cfg.decoder(ind);
                for (int i = 0; i < c; i++) {
                    perm[(size_t)r * 2 * c + i] = (int32_t)sol[0][i];
                    perm[(size_t)r * 2 * c + c + i] = (int32_t)sol[1][i];
                }
            }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// MultiObjectiveVRPConfig (configs/multi_objective_vrp_config.hpp) built through its own file
// reader (load_from_file, :78-165): the instance is written to a temporary file in that format,
// coordinates with 9 significant digits so that they read back as the same floats.  xy [n+1][2]
// with the depot first, demands [n+1]; the fleet goes in the name ("-k<V>").
static std::unique_ptr<MultiObjectiveVRPConfig<float>> load_vrp(const float* xy, const int32_t* demands, int n,
                                                                int capacity, int vehicles) {
    char path[] = "/tmp/ref_movrp_XXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) return nullptr;
    close(fd);
    {
        std::ofstream f(path);
        f << "NAME : ref-n" << (n + 1) << "-k" << vehicles << "\n";
        f << "DIMENSION : " << (n + 1) << "\n";
        f << "CAPACITY : " << capacity << "\n";
        f << "NODE_COORD_SECTION\n";
        char buf[96];
        for (int i = 0; i <= n; i++) {
            std::snprintf(buf, sizeof(buf), "%d %.9g %.9g\n", i + 1, (double)xy[2 * i], (double)xy[2 * i + 1]);
            f << buf;
        }
        f << "DEMAND_SECTION\n";
        for (int i = 0; i <= n; i++) f << (i + 1) << " " << demands[i] << "\n";
    }
    auto cfg = MultiObjectiveVRPConfig<float>::load_from_file(path);
    std::remove(path);
    return cfg;
}

// decode_solution (:280-313) gives both objectives, decode_routes (:214-271) the visiting
// order; perm receives the customers (1-based) in visiting order
int ref_movrp_eval(const float* xy, const int32_t* demands, int n, int capacity, int vehicles, const float* keys,
                   int rows, float* obj, int32_t* perm) {
    try {
        auto cfg = load_vrp(xy, demands, n, capacity, vehicles);
        if (!cfg) return -1;
        if (cfg->get_num_customers() != n || cfg->get_num_vehicles() != vehicles) return -2;
        for (int r = 0; r < rows; r++) {
            const float* row = keys + (size_t)r * n;
            cfg->decode_solution(row, obj + (size_t)r * 2);
            if (perm) {
                auto routes = cfg->decode_routes(row);
                size_t j = 0;
                for (const auto& rt : routes)
                    for (int c : rt.customers) perm[(size_t)r * n + j++] = c;
                if (j != (size_t)n) return -3;
            }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// JobSchedulingGPUConfig::fitness_function (configs/job_scheduling_gpu_config.hpp:132-148)
int ref_job_eval(const float* jt, int n, int machines, const float* keys, int rows, float* fit) {
    try {
        JobSchedulingGPUConfig<float> cfg(std::vector<float>(jt, jt + n), machines, "ref");
        Individual<float> ind(n);
        for (int r = 0; r < rows; r++) {
            set_keys(ind, keys + (size_t)r * n, n);
            fit[r] = cfg.fitness_function(ind);
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// ContinuousOptGPUConfig::fitness_function (configs/continuous_opt_gpu_config.hpp:114-173);
// function 0 sphere, 1 Rastrigin, 2 Rosenbrock
int ref_cont_eval(int function, float lower, float upper, int n, const float* keys, int rows, float* fit) {
    try {
        const OptimizationFunction f = function == 1   ? OptimizationFunction::RASTRIGIN
                                       : function == 2 ? OptimizationFunction::ROSENBROCK
                                                       : OptimizationFunction::SPHERE;
        ContinuousOptGPUConfig<float> cfg(n, lower, upper, f, "ref");
        Individual<float> ind(n);
        for (int r = 0; r < rows; r++) {
            set_keys(ind, keys + (size_t)r * n, n);
            fit[r] = cfg.fitness_function(ind);
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

static MultiTSPConfig<float>* tiny_mo_config() {
    Mat d(2, std::vector<float>(2, 1.0f));
    d[0][0] = d[1][1] = 0.0f;
    return new MultiTSPConfig<float>(d, d, "ref");
}

// Population::fast_non_dominated_sort + calculate_crowding_distance
// (core/population.hpp:409-489) on N points of 2 objectives
int ref_pareto(const float* obj, int N, int32_t* rank, float* cd) {
    try {
        std::unique_ptr<MultiTSPConfig<float>> cfg(tiny_mo_config());
        cfg->population_size = 4;
        Population<float> pop(cfg.get());
        auto& inds = pop.get_individuals();
        inds.assign(N, Individual<float>(cfg->component_lengths, 2));
        for (int i = 0; i < N; i++) inds[i].set_objectives({obj[2 * i], obj[2 * i + 1]});
        pop.fast_non_dominated_sort();
        pop.calculate_crowding_distance();
        for (int i = 0; i < N; i++) {
            rank[i] = inds[i].rank;
            if (cd) cd[i] = inds[i].crowding_distance;
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// Population::sort (core/population.hpp:660-676), the reference's elite partition, on P
// single-objective individuals of n keys with the given fitness values: mean seconds of one
// sort over `reps` sorts of the same unsorted population
double ref_population_sort_seconds(const float* fit, int P, int n, int reps) {
    try {
        std::vector<float> xy(2 * (size_t)n, 0.0f);
        auto cfg = std::make_unique<TSPConfig<float>>(coords_to_matrix(xy.data(), n), "ref");
        cfg->population_size = P;
        Population<float> pop(cfg.get());
        std::vector<Individual<float>> base(P, Individual<float>(n));
        for (int i = 0; i < P; i++) {
            base[i].fitness = fit[i];
            base[i].evaluated = true;
        }
        auto& inds = pop.get_individuals();
        double total = 0.0;
        for (int r = 0; r < reps; r++) {
            inds = base;
            const auto t0 = std::chrono::steady_clock::now();
            pop.sort();
            total += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        return total / (reps > 0 ? reps : 1);
    } catch (...) {
        return -1.0;
    }
}

// select_next_generation_nsga2 (core/population.hpp:491-517): pool indices of survivors
int ref_nsga2_select(const float* obj, int N, int P, int32_t* sel) {
    try {
        std::unique_ptr<MultiTSPConfig<float>> cfg(tiny_mo_config());
        cfg->population_size = P;
        Population<float> pop(cfg.get());
        auto& inds = pop.get_individuals();
        inds.assign(N, Individual<float>(cfg->component_lengths, 2));
        for (int i = 0; i < N; i++) {
            inds[i].set_objectives({obj[2 * i], obj[2 * i + 1]});
            inds[i].get_chromosome()[0] = (float)i;  // tag
        }
        pop.fast_non_dominated_sort();
        pop.calculate_crowding_distance();
        pop.select_next_generation_nsga2();
        auto& out = pop.get_individuals();
        for (int i = 0; i < P && i < (int)out.size(); i++) sel[i] = (int32_t)out[i].get_chromosome()[0];
        return (int)out.size();
    } catch (...) {
        return -1;
    }
}

// One single-objective generation through Solver::evolve_generation on the CPU path
// (core/solver.hpp:213-273) from a population given in sorted order, with the solver's
// mt19937 seeded; also returns the draws it consumed, replayed with identical
// distribution objects in the same call order (core/solver.hpp:1109-1135, 1244-1258).
int ref_brkga_generation(const float* xy, int n, int P, int E, int M, double rho, uint32_t seed,
                         const float* keys_sorted, const float* fit_sorted,
                         float* out_keys, float* out_fit,
                         int32_t* ep, int32_t* np, uint8_t* coin, float* mut) {
    try {
        auto cfg = std::make_unique<TSPConfig<float>>(coords_to_matrix(xy, n), "ref");
        cfg->population_size = P;
        cfg->elite_size = E;
        cfg->mutant_size = M;
        cfg->elite_prob = rho;
        cfg->max_generations = 1;
        Solver<float> solver(std::move(cfg), false, 1000000);
        if (solver.execution_mode != "cpu") return -2;
        auto& inds = solver.population->get_individuals();
        for (int r = 0; r < P; r++) {
            set_keys(inds[r], keys_sorted + (size_t)r * n, n);
            inds[r].fitness = fit_sorted[r];
            inds[r].evaluated = true;
        }
        solver.rng.seed(seed);
        solver.evolve_generation();
        auto& out = solver.population->get_individuals();
        for (int r = 0; r < P; r++) {
            const auto& c = out[r].get_chromosome();
            std::copy(c.begin(), c.end(), out_keys + (size_t)r * n);
            out_fit[r] = out[r].fitness;
        }
        // replay
        std::mt19937 rng(seed);
        int off = P - E - M;
        std::uniform_real_distribution<double> prob_dist(0.0, 1.0);
        std::uniform_int_distribution<int> elite_dist(0, E - 1);
        std::uniform_int_distribution<int> non_elite_dist(0, P - E - 1);
        for (int i = 0; i < off; i++) {
            ep[i] = elite_dist(rng);
            np[i] = non_elite_dist(rng);
            for (int j = 0; j < n; j++) coin[(size_t)i * n + j] = prob_dist(rng) < rho;
        }
        std::uniform_real_distribution<float> dist(0.0, 1.0);
        for (int i = 0; i < M; i++)
            for (int j = 0; j < n; j++) mut[(size_t)i * n + j] = dist(rng);
        return 0;
    } catch (...) {
        return -1;
    }
}

// seconds of one Solver::evolve_generation on the CPU path (core/solver.hpp:213-273: the
// non-elites' evaluation, sort, crossover and mutants) from a population in sorted order
double ref_generation_seconds(const float* xy, int n, int P, int E, int M, double rho, uint32_t seed,
                              const float* keys_sorted, const float* fit_sorted) {
    try {
        auto cfg = std::make_unique<TSPConfig<float>>(coords_to_matrix(xy, n), "ref");
        cfg->population_size = P;
        cfg->elite_size = E;
        cfg->mutant_size = M;
        cfg->elite_prob = rho;
        cfg->max_generations = 1;
        Solver<float> solver(std::move(cfg), false, 1000000);
        if (solver.execution_mode != "cpu") return -2.0;
        auto& inds = solver.population->get_individuals();
        for (int r = 0; r < P; r++) {
            set_keys(inds[r], keys_sorted + (size_t)r * n, n);
            inds[r].fitness = fit_sorted[r];
            inds[r].evaluated = true;
        }
        solver.rng.seed(seed);
        const auto t0 = std::chrono::steady_clock::now();
        solver.evolve_generation();
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } catch (...) {
        return -1.0;
    }
}

// Solver::generate_offspring_cpu (core/solver.hpp:1019-1091) with a seeded mt19937,
// plus the replayed draws (tournament picks, crossover coins, mutation flags/keys).
int ref_nsga2_offspring(const float* m0, const float* m1, int dim, int P, double rho, uint32_t seed,
                        const float* keys, const int32_t* rank, const float* cd,
                        float* out_keys, int32_t* picks, uint8_t* coin, uint8_t* mflag, float* mkey) {
    try {
        auto cfg = std::make_unique<MultiTSPConfig<float>>(flat_to_matrix(m0, dim), flat_to_matrix(m1, dim), "ref");
        cfg->population_size = P;
        cfg->elite_prob = rho;
        int n = dim - 1;
        Solver<float> solver(std::move(cfg), false, 1000000);
        std::vector<Individual<float>> parents(P, Individual<float>(std::vector<int>{n}, 2));
        for (int i = 0; i < P; i++) {
            set_keys(parents[i], keys + (size_t)i * n, n);
            parents[i].rank = rank[i];
            parents[i].crowding_distance = cd[i];
        }
        solver.rng.seed(seed);
        auto kids = solver.generate_offspring_cpu(parents);
        for (int i = 0; i < P; i++) {
            const auto& c = kids[i].get_chromosome();
            std::copy(c.begin(), c.end(), out_keys + (size_t)i * n);
        }
        std::mt19937 rng(seed);
        double rate = 5.0 / n;
        for (int i = 0; i < P; i++) {
            for (int t = 0; t < 2; t++) {
                std::uniform_int_distribution<int> d(0, P - 1);
                picks[4 * i + 2 * t] = d(rng);
                picks[4 * i + 2 * t + 1] = d(rng);
            }
            std::uniform_real_distribution<double> prob_dist(0.0, 1.0);
            for (int j = 0; j < n; j++) coin[(size_t)i * n + j] = prob_dist(rng) < rho;
            std::uniform_real_distribution<float> kd(0.0, 1.0);
            std::uniform_real_distribution<double> mp(0.0, 1.0);
            for (int j = 0; j < n; j++) {
                size_t q = (size_t)i * n + j;
                mflag[q] = mp(rng) < rate;
                mkey[q] = mflag[q] ? kd(rng) : 0.0f;
            }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// ---- the reference's whole CPU generation, for timing --------------------------------
struct RefSolver {
    std::unique_ptr<Solver<float>> s;
};

static void* make_solver(std::unique_ptr<BRKGAConfig<float>> cfg, int P, int E, int M, double rho) {
    cfg->population_size = P;
    cfg->elite_size = E;
    cfg->mutant_size = M;
    cfg->elite_prob = rho;
    cfg->max_generations = 1 << 30;
    auto* h = new RefSolver;
    h->s = std::make_unique<Solver<float>>(std::move(cfg), false, 1 << 30);
    h->s->initialize();
    return h;
}

// kind 1: TSP from coordinates; 3: threshold knapsack; 5: bi-objective TSP (coords of dim points);
// 7: TSPJ (travel and job matrices)
void* ref_solver_create(int kind, int n, const float* xy, const float* xy2, const float* w,
                        const float* v, float cap, int P, int E, int M, double rho) {
    try {
        if (kind == 1) {
            return make_solver(std::make_unique<TSPConfig<float>>(coords_to_matrix(xy, n), "ref"), P, E, M, rho);
        } else if (kind == 3) {
            std::vector<float> W(w, w + n), V(v, v + n);
            return make_solver(std::make_unique<KnapsackConfig<float>>(W, V, cap, "ref"), P, E, M, rho);
        } else if (kind == 7) {  // TSPJ: xy / xy2 carry the (n+1) x (n+1) travel and job matrices
            return make_solver(std::make_unique<TSPJConfig<float>>(flat_to_matrix(xy, n + 1), flat_to_matrix(xy2, n + 1),
                                                                  "ref"),
                               P, E, M, rho);
        } else if (kind == 5) {
            return make_solver(std::make_unique<MultiTSPConfig<float>>(coords_to_matrix(xy, n + 1),
                                                                      coords_to_matrix(xy2, n + 1), "ref"),
                               P, E, M, rho);
        }
    } catch (...) {
    }
    return nullptr;
}

// MO-VRP (NSGA-II) through the same file reader, with the elite / mutant sizes
// configure_for_size uses (P / 5, P / 6; the NSGA-II generation ignores both)
void* ref_solver_create_movrp(const float* xy, const int32_t* demands, int n, int capacity, int vehicles, int P,
                              double rho) {
    try {
        auto cfg = load_vrp(xy, demands, n, capacity, vehicles);
        if (!cfg) return nullptr;
        return make_solver(std::move(cfg), P, P / 5, P / 6, rho);
    } catch (...) {
    }
    return nullptr;
}

// a config that brings only a host fitness_function, the kind the reference's LLM solver
// writes: single-machine weighted completion time (jobs in key order, ties to the lower
// job; sum of w_j * C_j, minimised), with the float arithmetic of the engine's external-
// fitness example (llm-brkga_b200/cpp/examples/solve_external.cu) and its host
// fitness_function, with the instance drawn as that example draws it (std::mt19937(seed):
// processing times U[1, 100), then weights U[1, 10))
// a subclass, as the LLM solver's configs are (a bare BRKGAConfig<float> given to the
// reference's Solver crashed in this -O3 build; at -O1 it ran)
struct RefWctConfig : public BRKGAConfig<float> {
    explicit RefWctConfig(int n) : BRKGAConfig<float>(n) {}
};

void* ref_solver_create_wct(int n, unsigned seed, int P, int E, int M, double rho) {
    try {
        auto cfg = std::make_unique<RefWctConfig>(n);
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> up(1.0f, 100.0f), uw(1.0f, 10.0f);
        std::vector<float> pv(n), wv(n);
        for (int i = 0; i < n; ++i) {
            pv[i] = up(rng);
            wv[i] = uw(rng);
        }
        cfg->fitness_function = [pv, wv](const Individual<float>& ind) {
            const std::vector<float>& keys = ind.chromosomes[0];
            std::vector<int> order(keys.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
            float c = 0.0f, total = 0.0f;
            for (int job : order) {
                c = c + pv[job];
                const float prod = wv[job] * c;
                total = total + prod;
            }
            return total;
        };
        cfg->comparator = [](float a, float b) { return a < b; };
        return make_solver(std::move(cfg), P, E, M, rho);
    } catch (...) {
    }
    return nullptr;
}

const char* ref_solver_mode(void* h) { return static_cast<RefSolver*>(h)->s->execution_mode.c_str(); }

double ref_solver_evolve(void* h, int gens) {
    auto* r = static_cast<RefSolver*>(h);
    auto t0 = std::chrono::steady_clock::now();
    for (int g = 0; g < gens; g++) r->s->evolve_generation();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

double ref_solver_best(void* h) { return static_cast<RefSolver*>(h)->s->get_best_individual().fitness; }

void ref_solver_destroy(void* h) { delete static_cast<RefSolver*>(h); }

}  // extern "C"
