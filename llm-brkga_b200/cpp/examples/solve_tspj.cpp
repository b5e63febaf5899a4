// solve_tspj.cpp -- a reference-style TSPJ program on the drop-in header: writes
// <dir>/synthetic_TT.csv (Euclidean travel times of c+1 points uniform in [0,100)^2) and
// <dir>/synthetic_JT.csv (job durations uniform in [1,100), depot row 0), both from a
// seeded std::mt19937, loads them with TSPJConfig::load_from_file, runs Solver with the
// random 2-opt local search on, and prints one JSON line (makespan, city tour, job order,
// history length).  Usage: solve_tspj <dir> [c] [seed] [pop] [elite] [mutants] [gens]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../brkga_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir> [cities] [seed] [pop] [elite] [mutants] [gens]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int c = argc > 2 ? std::atoi(argv[2]) : 20;
    const unsigned seed = argc > 3 ? (unsigned)std::atoi(argv[3]) : 1u;
    const int pop = argc > 4 ? std::atoi(argv[4]) : 256;
    const int elite = argc > 5 ? std::atoi(argv[5]) : 51;
    const int mutants = argc > 6 ? std::atoi(argv[6]) : 25;
    const int gens = argc > 7 ? std::atoi(argv[7]) : 200;
    {
        std::mt19937 rng(seed);
        std::uniform_real_distribution<double> u(0.0, 100.0), dur(1.0, 100.0);
        std::vector<double> x(c + 1), y(c + 1);
        for (int i = 0; i <= c; ++i) x[i] = u(rng), y[i] = u(rng);
        std::ofstream tt(dir + "/synthetic_TT.csv"), jt(dir + "/synthetic_JT.csv");
        tt << std::setprecision(9);
        jt << std::setprecision(9);
        for (int i = 0; i <= c; ++i) {
            for (int j = 0; j <= c; ++j) {
                tt << (j ? "," : "") << (float)std::hypot(x[i] - x[j], y[i] - y[j]);
                jt << (j ? "," : "") << (i == 0 ? 0.0f : (float)dur(rng));
            }
            tt << "\n";
            jt << "\n";
        }
    }
    try {
        auto config = TSPJConfig<float>::load_from_file(dir + "/synthetic_TT.csv");
        config->population_size = pop;
        config->elite_size = elite;
        config->mutant_size = mutants;
        config->max_generations = gens;
        config->seed = 7;
        config->local_search_interval = 2;
        Solver<float> solver(std::move(config), false);
        solver.run();
        const auto& best = solver.get_best_individual();
        const auto perm = solver.get_best_permutation();
        const auto& hist = solver.get_fitness_history();
        std::printf("{\"best\": %.9g, \"history\": %zu, \"perm\": [", (double)best.fitness, hist.size());
        for (size_t i = 0; i < perm.size(); ++i) std::printf("%s%d", i ? ", " : "", perm[i]);
        std::printf("]}\n");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
