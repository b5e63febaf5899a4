// solve_tsp.cpp -- a reference-style program on the drop-in header: writes a TSPLIB file
// of n cities uniform in [0, scale)^2 (std::mt19937 seeded), loads it with
// TSPConfig::load_from_file, runs Solver and prints one JSON line (best fitness, tour,
// history length).  Usage: solve_tsp <file> [n] [seed] [pop] [elite] [mutants] [gens]
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../brkga_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <tsplib-file> [n] [seed] [pop] [elite] [mutants] [gens]\n", argv[0]);
        return 2;
    }
    const std::string path = argv[1];
    const int n = argc > 2 ? std::atoi(argv[2]) : 52;
    const unsigned seed = argc > 3 ? (unsigned)std::atoi(argv[3]) : 1u;
    const int pop = argc > 4 ? std::atoi(argv[4]) : 256;
    const int elite = argc > 5 ? std::atoi(argv[5]) : 51;
    const int mutants = argc > 6 ? std::atoi(argv[6]) : 25;
    const int gens = argc > 7 ? std::atoi(argv[7]) : 500;
    {
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> u(0.0f, 1000.0f);
        std::ofstream f(path);
        f << "NAME : synthetic" << n << "\nTYPE : TSP\nDIMENSION : " << n << "\nEDGE_WEIGHT_TYPE : EUC_2D\n"
          << "NODE_COORD_SECTION\n" << std::setprecision(9);
        for (int i = 0; i < n; ++i) {
            const float x = u(rng), y = u(rng);
            f << (i + 1) << " " << x << " " << y << "\n";
        }
        f << "EOF\n";
    }
    try {
        auto config = TSPConfig<float>::load_from_file(path);
        config->population_size = pop;
        config->elite_size = elite;
        config->mutant_size = mutants;
        config->elite_prob = 0.7;
        config->max_generations = gens;
        config->seed = 7;
        Solver<float> solver(std::move(config), false);
        solver.run();
        const auto& best = solver.get_best_individual();
        const auto tour = solver.get_best_permutation();
        const auto& hist = solver.get_fitness_history();
        std::printf("{\"best\": %.9g, \"history\": %zu, \"tour\": [", (double)best.fitness, hist.size());
        for (size_t i = 0; i < tour.size(); ++i) std::printf("%s%d", i ? ", " : "", tour[i]);
        std::printf("]}\n");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
