// solve_knapsack.cpp -- knapsack instance files through the drop-in header: writes
// <dir>/items.txt ("num_items capacity" then "weight value" lines) and <dir>/items.csv
// ("weight,value[,capacity]" rows) with the same seeded items, loads each with
// KnapsackConfig::load_from_file (threshold decode) and solves it; prints one JSON line
// with both best values.  Usage: solve_knapsack <dir> [items] [seed] [gens]
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../brkga_b200.hpp"

static double solve(std::unique_ptr<KnapsackConfig<float>> cfg, int gens) {
    KnapsackConfig<float>::configure_for_size(cfg.get(), (int)cfg->get_weights().size());
    cfg->max_generations = gens;
    cfg->seed = 5;
    Solver<float> s(std::move(cfg), false);
    s.run();
    return s.get_best_individual().fitness;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir> [items] [seed] [gens]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int n = argc > 2 ? std::atoi(argv[2]) : 60;
    const unsigned seed = argc > 3 ? (unsigned)std::atoi(argv[3]) : 1u;
    const int gens = argc > 4 ? std::atoi(argv[4]) : 50;
    std::mt19937 rng(seed);
    std::uniform_int_distribution<int> d(1, 100);
    std::vector<int> w(n), v(n);
    long total = 0;
    for (int i = 0; i < n; ++i) w[i] = d(rng), v[i] = d(rng), total += w[i];
    const long cap = total / 2;
    {
        std::ofstream t(dir + "/items.txt"), c(dir + "/items.csv");
        t << "# synthetic knapsack\n" << n << " " << cap << "\n";
        c << "# weight,value,capacity\n";
        for (int i = 0; i < n; ++i) {
            t << w[i] << " " << v[i] << "\n";
            c << w[i] << "," << v[i];
            if (i == 0) c << "," << cap;
            c << "\n";
        }
    }
    try {
        const double a = solve(KnapsackConfig<float>::load_from_file(dir + "/items.txt"), gens);
        const double b = solve(KnapsackConfig<float>::load_from_file(dir + "/items.csv"), gens);
        std::printf("{\"txt\": %.9g, \"csv\": %.9g, \"capacity\": %ld}\n", a, b, cap);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
