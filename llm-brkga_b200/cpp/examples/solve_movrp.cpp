// solve_movrp.cpp -- a reference-style MO-VRP program on the drop-in header: writes
// <dir>/synthetic-n<N>-k<V>.vrp (depot and customers uniform in [0,100)^2, demands uniform in
// {1..30}, capacity 1.1 x total demand / V, from a seeded std::mt19937) in the file format
// MultiObjectiveVRPConfig::load_from_file reads, loads it, runs the Solver (NSGA-II) and
// prints one JSON line: the first front's objectives and the route count of the best point.
// Usage: solve_movrp <dir> [customers] [vehicles] [seed] [pop] [gens]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../brkga_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir> [customers] [vehicles] [seed] [pop] [gens]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int n = argc > 2 ? std::atoi(argv[2]) : 31;
    const int V = argc > 3 ? std::atoi(argv[3]) : 5;
    const unsigned seed = argc > 4 ? (unsigned)std::atoi(argv[4]) : 1u;
    const int pop = argc > 5 ? std::atoi(argv[5]) : 128;
    const int gens = argc > 6 ? std::atoi(argv[6]) : 100;
    const std::string path = dir + "/synthetic-n" + std::to_string(n + 1) + "-k" + std::to_string(V) + ".vrp";
    {
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> u(0.0f, 100.0f);
        std::uniform_int_distribution<int> dem(1, 30);
        std::vector<float> x(n + 1), y(n + 1);
        std::vector<int> d(n + 1, 0);
        long total = 0;
        for (int i = 0; i <= n; ++i) x[i] = u(rng), y[i] = u(rng);
        for (int i = 1; i <= n; ++i) total += (d[i] = dem(rng));
        const int cap = (int)std::ceil(1.1 * (double)total / V);
        std::ofstream f(path);
        f << "NAME : synthetic-n" << (n + 1) << "-k" << V << "\n";
        f << "TYPE : CVRP\nDIMENSION : " << (n + 1) << "\nEDGE_WEIGHT_TYPE : EUC_2D\nCAPACITY : " << cap << "\n";
        f << "NODE_COORD_SECTION\n" << std::setprecision(9);
        for (int i = 0; i <= n; ++i) f << (i + 1) << " " << x[i] << " " << y[i] << "\n";
        f << "DEMAND_SECTION\n";
        for (int i = 0; i <= n; ++i) f << (i + 1) << " " << d[i] << "\n";
        f << "DEPOT_SECTION\n1\n-1\nEOF\n";
    }
    try {
        auto config = MultiObjectiveVRPConfig<float>::load_from_file(path);
        MultiObjectiveVRPConfig<float>::configure_for_size(config.get(), config->get_num_customers());
        const MultiObjectiveVRPConfig<float>* vrp = config.get();
        config->population_size = pop;
        config->elite_size = pop / 5;
        config->mutant_size = pop / 6;
        config->max_generations = gens;
        config->seed = 7;
        Solver<float> solver(std::move(config), false);
        solver.run();
        const auto front = solver.get_pareto_front();
        std::printf("{\"vehicles\": %d, \"capacity\": %d, \"front\": [", vrp->get_num_vehicles(),
                    vrp->get_vehicle_capacity());
        for (size_t i = 0; i < front.size(); ++i)
            std::printf("%s[%.9g, %.9g]", i ? ", " : "", (double)front[i].objectives[0], (double)front[i].objectives[1]);
        const auto routes = vrp->routes_of(solver.get_best_permutation());
        std::printf("], \"routes\": %zu}\n", routes.size());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
