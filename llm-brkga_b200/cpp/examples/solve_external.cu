// solve_external.cu -- a config written the way the reference's LLM solver writes them
// (a BRKGAConfig subclass with a host fitness_function and, optionally, its own
// evaluate_population_gpu kernel; llm_solver/core/execution_manager.py builds a main like
// the one below around such a config), run unchanged on the drop-in header.
//
// Problem: single-machine weighted completion time.  n jobs with processing times p and
// weights w; the keys order the jobs (ascending, ties to the lower job); fitness =
// sum over jobs of w_j * C_j with C_j the job's completion time, minimised.  The
// two-objective modes add a second weight vector and minimise both sums (NSGA-II).
//
// Usage: solve_external <host|gpu|host2|gpu2> [n] [seed] [generations]
// Prints the generated main's lines, then one JSON line: the best fitness, the config's
// own fitness of the best keys, and the first and last entries of the fitness history;
// in the two-objective modes the Pareto front's size and its objective pairs.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>

#include "../brkga_b200.hpp"

// one thread per row: the row's jobs in key order (stable insertion sort), then the same
// float sums as the host fitness, rounded the same way (no contraction into FMA)
__global__ void weighted_completion_kernel(const float* keys, float* fitness, int rows, int n, const float* p,
                                           const float* w, const float* w2) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const float* k = keys + (size_t)r * n;
    int order[64];
    for (int i = 0; i < n; ++i) {
        int j = i;
        while (j > 0 && k[order[j - 1]] > k[i]) {
            order[j] = order[j - 1];
            --j;
        }
        order[j] = i;
    }
    float c = 0.0f, total = 0.0f, total2 = 0.0f;
    for (int q = 0; q < n; ++q) {
        const int job = order[q];
        c = __fadd_rn(c, p[job]);
        total = __fadd_rn(total, __fmul_rn(w[job], c));
        if (w2) total2 = __fadd_rn(total2, __fmul_rn(w2[job], c));
    }
    if (w2) {
        fitness[2 * r] = total;
        fitness[2 * r + 1] = total2;
    } else {
        fitness[r] = total;
    }
}

template <typename T>
class WeightedCompletionConfig : public BRKGAConfig<T> {
public:
    std::vector<T> p, w, w2;
    bool use_gpu = false;
    float* d_p = nullptr;
    float* d_w = nullptr;
    float* d_w2 = nullptr;

    WeightedCompletionConfig(std::vector<T> proc, std::vector<T> weight, std::vector<T> weight2, bool gpu)
        : BRKGAConfig<T>(std::vector<int>{(int)proc.size()}, weight2.empty() ? 1 : 2), p(std::move(proc)),
          w(std::move(weight)), w2(std::move(weight2)), use_gpu(gpu) {
        this->population_size = 256;
        this->elite_size = 51;
        this->mutant_size = 25;
        this->elite_prob = 0.7;
        this->max_generations = 200;
        this->comparator = [](T a, T b) { return a < b; };
        this->fitness_function = [this](const Individual<T>& ind) { return weighted_completion(ind.get_chromosome(), w); };
        if (!w2.empty()) {
            this->objective_functions[0] = [this](const Individual<T>& ind) {
                return weighted_completion(ind.get_chromosome(), w);
            };
            this->objective_functions[1] = [this](const Individual<T>& ind) {
                return weighted_completion(ind.get_chromosome(), w2);
            };
        }
        if (use_gpu) {
            upload(p, &d_p);
            upload(w, &d_w);
            if (!w2.empty()) upload(w2, &d_w2);
        }
    }
    ~WeightedCompletionConfig() override {
        if (d_p) cudaFree(d_p);
        if (d_w) cudaFree(d_w);
        if (d_w2) cudaFree(d_w2);
    }
    static void upload(const std::vector<T>& v, float** d) {
        cudaMalloc(d, v.size() * sizeof(float));
        cudaMemcpy(*d, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice);
    }

    static std::unique_ptr<WeightedCompletionConfig<T>> create_default(int n, unsigned seed, bool gpu, bool two) {
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> up(1.0f, 100.0f), uw(1.0f, 10.0f);
        std::vector<T> proc(n), weight(n), weight2;
        for (int i = 0; i < n; ++i) {
            proc[i] = up(rng);
            weight[i] = uw(rng);
        }
        if (two)
            for (int i = 0; i < n; ++i) weight2.push_back(uw(rng));
        return std::make_unique<WeightedCompletionConfig<T>>(proc, weight, weight2, gpu);
    }

    T weighted_completion(const std::vector<T>& keys, const std::vector<T>& weights) const {
        std::vector<int> order(keys.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
        float c = 0.0f, total = 0.0f;
        for (int job : order) {
            c = c + p[job];
            const float prod = weights[job] * c;
            total = total + prod;
        }
        return total;
    }

    bool has_gpu_evaluation() const override { return use_gpu; }
    void evaluate_population_gpu(T* d_population, T* d_fitness, int pop_size, int chrom_len) override {
        weighted_completion_kernel<<<(pop_size + 127) / 128, 128>>>(d_population, d_fitness, pop_size, chrom_len,
                                                                   d_p, d_w, d_w2);
        cudaDeviceSynchronize();
    }
    void print_solution(const Individual<T>& ind) override {
        std::cout << "Weighted completion time: " << weighted_completion(ind.get_chromosome(), w) << std::endl;
    }
};

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "host";
    const bool gpu = mode == "gpu" || mode == "gpu2";
    const bool two = mode == "host2" || mode == "gpu2";
    const int n = argc > 2 ? std::atoi(argv[2]) : 40;
    const unsigned seed = argc > 3 ? (unsigned)std::atoi(argv[3]) : 1u;
    const int gens = argc > 4 ? std::atoi(argv[4]) : 200;
    if (n < 1 || n > 64) {
        std::fprintf(stderr, "n must lie in [1, 64]\n");
        return 2;
    }
    try {
        std::cout << "Creating configuration..." << std::endl;
        auto config = WeightedCompletionConfig<float>::create_default(n, seed, gpu, two);
        config->max_generations = gens;
        std::cout << "Creating BRKGA solver..." << std::endl;
        Solver<float> solver(std::move(config), true, 50);
        const char* quick_test_env = std::getenv("QUICK_TEST");
        if (quick_test_env) {
            auto* config_ptr = solver.get_config();
            if (config_ptr) config_ptr->max_generations = std::atoi(quick_test_env);
        }
        std::cout << "Running optimization..." << std::endl;
        const auto t0 = std::chrono::steady_clock::now();
        solver.run();
        const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (two) {
            // the generated main's multi-objective branch: the Pareto front
            auto pareto = solver.get_pareto_front();
            std::cout << "Pareto front size: " << pareto.size() << std::endl;
            std::printf("{\"seconds\": %.6f, \"front\": %zu, \"points\": [", seconds, pareto.size());
            for (size_t i = 0; i < pareto.size(); ++i)
                std::printf("%s[%.9g, %.9g]", i ? ", " : "", (double)pareto[i].objectives[0],
                            (double)pareto[i].objectives[1]);
            std::printf("]}\n");
            return 0;
        }
        const auto& best = solver.get_best_individual();
        std::cout << "Best fitness: " << best.fitness << std::endl;
        auto* config_ptr = solver.get_config();
        if (config_ptr) config_ptr->print_solution(best);
        const auto& hist = solver.get_fitness_history();
        const float again = config_ptr->fitness_function(best);
        std::printf("{\"seconds\": %.6f, \"best\": %.9g, \"check\": %.9g, \"history\": %zu, \"first\": %.9g, "
                    "\"last\": %.9g}\n",
                    seconds, (double)best.fitness, (double)again, hist.size(), (double)hist.front(), (double)hist.back());
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
