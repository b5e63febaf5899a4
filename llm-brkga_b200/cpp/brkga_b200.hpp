// brkga_b200.hpp -- drop-in C++ host interface with the reference's class names and
// signatures (hsaseendran/llm-brkga: core/individual.hpp, core/config.hpp,
// configs/tsp_config.hpp, configs/knapsack_config.hpp, configs/multi_tsp_config.hpp,
// core/solver.hpp), running on the B200 engine through the C ABI (include/brkga_b200.h).
//
// A program written against the reference switches by including this header instead of
// "core/solver.hpp" + "configs/*.hpp" and linking libbrkga_b200.so.  Errors the reference
// prints and swallows are thrown here as std::runtime_error with the library's message.
//
// Scope: the problem configs the engine implements on the GPU (TSP from a matrix or from
// TSPLIB coordinates, knapsack, bi-objective TSP, TSPJ, job scheduling, continuous
// functions, MO-VRP), and single-objective configs that bring their own fitness -- a host
// fitness_function or their own evaluate_population_gpu kernel, as LLM-written configs do.
// Those run on the engine's external-fitness path: keys, crossover, mutants and the elite
// partition on the device, the config's fitness between them.
#ifndef BRKGA_B200_HPP
#define BRKGA_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/brkga_b200.h"

namespace brkga_b200_detail {
inline void check(int32_t code, const char* what) {
    if (code != BRKGA_OK) {
        char buf[512];
        brkga_last_error(buf, sizeof(buf));
        throw std::runtime_error(std::string(what) + ": " + buf);
    }
}
}  // namespace brkga_b200_detail

// core/individual.hpp:9-226
template <typename T>
class Individual {
public:
    std::vector<std::vector<T>> chromosomes;
    T fitness;
    bool evaluated;
    std::vector<T> objectives;
    int rank;
    T crowding_distance;

    explicit Individual(int length = 0)
        : chromosomes(1, std::vector<T>(length)), fitness(T(0)), evaluated(false), rank(-1), crowding_distance(0) {}
    Individual(const std::vector<int>& lens, int num_objectives = 0)
        : fitness(T(0)), evaluated(false), rank(-1), crowding_distance(0) {
        for (int l : lens) chromosomes.emplace_back(l);
        if (num_objectives > 0) objectives.assign(num_objectives, T(0));
    }
    std::vector<T>& get_chromosome() { return chromosomes[0]; }
    const std::vector<T>& get_chromosome() const { return chromosomes[0]; }
    std::vector<T>& chromosome() { return chromosomes[0]; }
    const std::vector<T>& chromosome() const { return chromosomes[0]; }
    std::vector<T>& get_component(int i) { return chromosomes[i]; }
    const std::vector<T>& get_component(int i) const { return chromosomes[i]; }
    int size() const { return chromosomes.empty() ? 0 : (int)chromosomes[0].size(); }
    int num_components() const { return (int)chromosomes.size(); }
    T get_fitness() const { return fitness; }
    bool is_evaluated() const { return evaluated; }
    bool is_multi_objective() const { return !objectives.empty(); }
    T& operator[](int i) { return chromosomes[0][i]; }
    const T& operator[](int i) const { return chromosomes[0][i]; }
    // minimisation dominance, core/individual.hpp:99-114
    bool dominates(const Individual& o) const {
        if (objectives.empty() || objectives.size() != o.objectives.size()) return false;
        bool better = false;
        for (size_t i = 0; i < objectives.size(); ++i) {
            if (objectives[i] > o.objectives[i]) return false;
            if (objectives[i] < o.objectives[i]) better = true;
        }
        return better;
    }
    std::vector<T> flatten() const {
        std::vector<T> f;
        for (const auto& c : chromosomes) f.insert(f.end(), c.begin(), c.end());
        return f;
    }
};

// core/config.hpp:14-229
template <typename T>
class BRKGAConfig {
public:
    std::vector<int> component_lengths;
    int num_components;
    int population_size;
    int elite_size;
    int mutant_size;
    double elite_prob;
    int max_generations;
    int threads_per_block;
    int blocks_per_grid;
    std::function<T(const Individual<T>&)> fitness_function;
    std::function<std::vector<std::vector<T>>(const Individual<T>&)> decoder;
    std::function<bool(T, T)> comparator;
    int num_objectives;
    std::vector<std::function<T(const Individual<T>&)>> objective_functions;
    // engine extras (not in the reference): Philox seed, islands, device
    uint64_t seed = 1;
    int num_islands = 1;
    int migration_interval = 0;
    int num_migrants = 0;
    int device = 0;
    // random 2-opt local search for configs that have one (TSPJ); the reference runs it in
    // its multi-GPU island loop every 2 generations on 100 elites with 5 moves
    // (core/solver.hpp:166, 459-461); 0 = off
    int local_search_interval = 0;
    int local_search_individuals = 100;
    int local_search_moves = 5;
    // NSGA-II (two objectives): fresh random offspring per generation.  The reference's
    // NSGA-II ignores mutant_size (core/solver.hpp:1019-1032), so the default is 0 whatever
    // mutant_size holds (MultiObjectiveVRPConfig::configure_for_size sets it to P / 6).
    int nsga2_random_offspring = 0;

    explicit BRKGAConfig(int chrom_len) : BRKGAConfig(std::vector<int>{chrom_len}) {}
    explicit BRKGAConfig(const std::vector<int>& lens, int n_objectives = 1)
        : component_lengths(lens), num_components((int)lens.size()), population_size(100), elite_size(20),
          mutant_size(10), elite_prob(0.7), max_generations(1000), threads_per_block(256), blocks_per_grid(32),
          num_objectives(n_objectives) {
        objective_functions.resize(n_objectives > 1 ? n_objectives : 0);
    }
    virtual ~BRKGAConfig() = default;

    // the device instance this config evaluates on (nullptr: no GPU evaluation)
    virtual brkga_problem* problem_handle() { return nullptr; }

    virtual bool has_gpu_evaluation() const { return false; }
    // core/config.hpp:50-53: d_population [pop_size][chrom_len], d_fitness [pop_size]
    virtual void evaluate_population_gpu(T* d_population, T* d_fitness, int pop_size, int chrom_len) {
        brkga_problem* pb = problem_handle();
        if (!pb) return;
        brkga_b200_detail::check(
            brkga_evaluate_population_sync(pb, d_population, d_fitness, pop_size, chrom_len), "evaluate_population_gpu");
    }
    virtual bool has_local_search() const { return false; }
    virtual void print_solution(const Individual<T>& ind) {
        std::cout << "Best fitness: " << ind.fitness << std::endl;
    }
    virtual bool validate_solution(const Individual<T>&) { return true; }
    // core/config.hpp:159-179
    virtual bool is_valid() const {
        bool ok = !component_lengths.empty() &&
                  std::all_of(component_lengths.begin(), component_lengths.end(), [](int l) { return l > 0; }) &&
                  population_size > 0 && elite_prob >= 0.0 && elite_prob <= 1.0 && max_generations > 0 &&
                  num_objectives > 0;
        if (!ok) return false;
        if (num_objectives == 1) return elite_size > 0 && mutant_size >= 0 && elite_size + mutant_size <= population_size;
        return true;
    }
    int get_total_chromosome_length() const {
        int t = 0;
        for (int l : component_lengths) t += l;
        return t;
    }
    int chromosome_length() const { return get_total_chromosome_length(); }
    int get_offspring_size() const { return population_size - elite_size - mutant_size; }
    void update_cuda_grid_size() { blocks_per_grid = (population_size + threads_per_block - 1) / threads_per_block; }
    bool is_multi_objective() const { return num_objectives > 1; }
};

// a config backed by a device instance
template <typename T>
class DeviceProblemConfig : public BRKGAConfig<T> {
public:
    using BRKGAConfig<T>::BRKGAConfig;
    ~DeviceProblemConfig() override {
        if (pb_) brkga_problem_destroy(pb_);
    }
    brkga_problem* problem_handle() override { return pb_; }
    bool has_gpu_evaluation() const override { return pb_ != nullptr; }

protected:
    void create(const brkga_problem_desc& d) {
        brkga_b200_detail::check(brkga_problem_create(&d, this->device, &pb_), "problem upload");
    }
    brkga_problem* pb_ = nullptr;
};

// configs/tsp_config.hpp:24-381
template <typename T>
class TSPConfig : public DeviceProblemConfig<T> {
public:
    // TSPConfig(distances, name): explicit N x N matrix
    TSPConfig(const std::vector<std::vector<T>>& distances, const std::string& name = "TSP")
        : DeviceProblemConfig<T>((int)distances.size()), num_cities_((int)distances.size()), name_(name) {
        std::vector<float> flat((size_t)num_cities_ * num_cities_);
        for (int i = 0; i < num_cities_; ++i)
            for (int j = 0; j < num_cities_; ++j) flat[(size_t)i * num_cities_ + j] = (float)distances[i][j];
        brkga_problem_desc d{};
        d.kind = BRKGA_TSP_MATRIX;
        d.n = num_cities_;
        d.matrix = flat.data();
        this->create(d);
        setup();
    }
    // engine-native: Euclidean distances from [n][2] coordinates, computed on the device
    // exactly as the reference builds its matrix (configs/tsp_config.hpp:361-370)
    static std::unique_ptr<TSPConfig<T>> from_coordinates(const std::vector<std::pair<T, T>>& xy,
                                                          const std::string& name = "TSP") {
        return std::unique_ptr<TSPConfig<T>>(new TSPConfig<T>(xy, name, 0));
    }
    // configs/tsp_config.hpp:260-265, 301-380 (TSPLIB NODE_COORD_SECTION)
    static std::unique_ptr<TSPConfig<T>> load_from_file(const std::string& filename) {
        std::ifstream f(filename);
        if (!f) throw std::runtime_error("File does not exist: " + filename);
        std::string line, name;
        int n = 0;
        bool reading = false;
        std::vector<std::pair<T, T>> xy;
        while (std::getline(f, line)) {
            if (line.empty()) continue;
            if (line.find("NAME") != std::string::npos && line.find(':') != std::string::npos) {
                name = line.substr(line.find(':') + 1);
                name.erase(0, name.find_first_not_of(" \t"));
                name.erase(name.find_last_not_of(" \t\r") + 1);
            } else if (line.find("DIMENSION") != std::string::npos) {
                std::istringstream is(line);
                std::string tok;
                while (is >> tok)
                    if (std::isdigit((unsigned char)tok[0])) {
                        n = std::stoi(tok);
                        break;
                    }
                xy.assign(n, {T(0), T(0)});
            } else if (line.find("NODE_COORD_SECTION") != std::string::npos) {
                reading = true;
            } else if (line.find("EOF") != std::string::npos) {
                break;
            } else if (reading) {
                std::istringstream is(line);
                int id;
                T x, y;
                if (is >> id >> x >> y && id > 0 && id <= n) xy[id - 1] = {x, y};
            }
        }
        if (xy.empty()) throw std::runtime_error("No coordinates found in TSPLIB file");
        if (name.empty()) name = filename;
        return from_coordinates(xy, name);
    }
    // configs/tsp_config.hpp:267-286
    static void configure_for_size(TSPConfig<T>* c, int n) {
        if (n <= 20) {
            c->population_size = 200, c->elite_size = 40, c->mutant_size = 20, c->max_generations = 100;
        } else if (n <= 50) {
            c->population_size = 1000, c->elite_size = 800, c->mutant_size = 400, c->max_generations = 2000;
        } else {
            c->population_size = 8000, c->elite_size = 1600, c->mutant_size = 800, c->max_generations = 5000;
        }
        c->elite_prob = 0.7;
        c->update_cuda_grid_size();
    }
    int get_num_cities() const { return num_cities_; }
    const std::string& get_instance_name() const { return name_; }
    bool is_gpu_available() const { return this->pb_ != nullptr; }

private:
    TSPConfig(const std::vector<std::pair<T, T>>& xy, const std::string& name, int)
        : DeviceProblemConfig<T>((int)xy.size()), num_cities_((int)xy.size()), name_(name) {
        std::vector<float> flat(2 * xy.size());
        for (size_t i = 0; i < xy.size(); ++i) {
            flat[2 * i] = (float)xy[i].first;
            flat[2 * i + 1] = (float)xy[i].second;
        }
        brkga_problem_desc d{};
        d.kind = BRKGA_TSP_COORDS;
        d.n = num_cities_;
        d.coords = flat.data();
        this->create(d);
        setup();
    }
    void setup() {
        this->comparator = [](T a, T b) { return a < b; };
        this->update_cuda_grid_size();
    }
    int num_cities_;
    std::string name_;
};

// configs/knapsack_config.hpp:11-62 (threshold decode, penalty x1000, maximise); greedy
// key-order decoding is the engine's addition (greedy = true)
template <typename T>
class KnapsackConfig : public DeviceProblemConfig<T> {
public:
    KnapsackConfig(const std::vector<T>& w, const std::vector<T>& v, T cap, const std::string& name = "Knapsack",
                   bool greedy = false)
        : DeviceProblemConfig<T>((int)w.size()), weights_(w), values_(v), capacity_(cap), name_(name) {
        if (w.size() != v.size()) throw std::invalid_argument("Weights and values must have same size");
        std::vector<int32_t> wi(w.size()), vi(v.size());
        for (size_t i = 0; i < w.size(); ++i) {
            if (w[i] != std::floor(w[i]) || v[i] != std::floor(v[i]))
                throw std::invalid_argument("the GPU knapsack takes integer weights and values");
            wi[i] = (int32_t)w[i];
            vi[i] = (int32_t)v[i];
        }
        brkga_problem_desc d{};
        d.kind = greedy ? BRKGA_KNAP_GREEDY : BRKGA_KNAP_THRESHOLD;
        d.n = (int)w.size();
        d.weights = wi.data();
        d.values = vi.data();
        d.capacity = (float)cap;
        this->create(d);
        this->comparator = [](T a, T b) { return a > b; };
        this->update_cuda_grid_size();
    }
    // configs/knapsack_config.hpp:307-331
    static void configure_for_size(KnapsackConfig<T>* c, int n) {
        if (n <= 50) {
            c->population_size = 200, c->elite_size = 40, c->mutant_size = 20, c->max_generations = 300;
        } else if (n <= 100) {
            c->population_size = 400, c->elite_size = 80, c->mutant_size = 40, c->max_generations = 500;
        } else if (n <= 500) {
            c->population_size = 800, c->elite_size = 160, c->mutant_size = 80, c->max_generations = 1000;
        } else {
            c->population_size = 1200, c->elite_size = 240, c->mutant_size = 120, c->max_generations = 1500;
        }
        c->elite_prob = 0.7;
        c->update_cuda_grid_size();
    }
    const std::vector<T>& get_weights() const { return weights_; }
    const std::vector<T>& get_values() const { return values_; }
    T get_capacity() const { return capacity_; }

    // configs/knapsack_config.hpp:180-304: ".csv" files hold "weight,value[,capacity]" rows
    // (the first row with a numeric third field gives the capacity, else half the total
    // weight); other files hold "num_items capacity" and then "weight value" lines; '#'
    // lines are comments
    static std::unique_ptr<KnapsackConfig<T>> load_from_file(const std::string& filename, bool greedy = false) {
        std::ifstream f(filename);
        if (!f.good()) throw std::runtime_error("File does not exist: " + filename);
        const size_t slash = filename.find_last_of('/');
        std::string name = (slash == std::string::npos) ? filename : filename.substr(slash + 1);
        const size_t dot = name.find_last_of('.');
        const std::string ext = (dot == std::string::npos) ? "" : name.substr(dot + 1);
        if (dot != std::string::npos) name = name.substr(0, dot);
        std::vector<T> w, v;
        T cap = 0;
        std::string line;
        if (ext == "csv") {
            bool have_cap = false;
            while (std::getline(f, line)) {
                if (line.empty() || line[0] == '#') continue;
                std::vector<std::string> fields;
                std::stringstream ss(line);
                std::string cell;
                while (std::getline(ss, cell, ',')) {
                    const size_t a = cell.find_first_not_of(" \t\r\n");
                    fields.push_back(a == std::string::npos ? std::string()
                                                            : cell.substr(a, cell.find_last_not_of(" \t\r\n") - a + 1));
                }
                if (fields.size() < 2) continue;
                if (!have_cap && fields.size() >= 3) {
                    try {
                        cap = (T)std::stod(fields[2]);
                        have_cap = true;
                    } catch (...) {
                    }
                }
                try {
                    const T wi = (T)std::stod(fields[0]), vi = (T)std::stod(fields[1]);
                    w.push_back(wi);
                    v.push_back(vi);
                } catch (...) {
                }
            }
            if (w.empty()) throw std::runtime_error("No valid items found in CSV file");
            if (!have_cap) {
                T total = 0;
                for (T x : w) total += x;
                cap = total * (T)0.5;
            }
        } else {
            bool items = false;
            int count = 0;
            while (std::getline(f, line)) {
                if (line.empty() || line[0] == '#') continue;
                std::istringstream is(line);
                if (!items) {
                    if (is >> count >> cap) items = true;
                } else {
                    T wi, vi;
                    if (is >> wi >> vi) {
                        w.push_back(wi);
                        v.push_back(vi);
                    }
                }
            }
            if (w.empty()) throw std::runtime_error("No items found in file");
        }
        return std::make_unique<KnapsackConfig<T>>(w, v, cap, name, greedy);
    }
    // configs/knapsack_config.hpp:157-178 draws real weights and values; the device
    // knapsack sums integers, so this draws integers in [1, max] (std::mt19937(seed))
    static std::unique_ptr<KnapsackConfig<T>> create_random(int num_items, T max_weight = 50, T max_value = 100,
                                                           T capacity_ratio = 0.5,
                                                           const std::string& name = "Random_Knapsack",
                                                           unsigned seed = 1, bool greedy = false) {
        std::mt19937 rng(seed);
        std::uniform_int_distribution<int> dw(1, (int)max_weight), dv(1, (int)max_value);
        std::vector<T> w(num_items), v(num_items);
        T total = 0;
        for (int i = 0; i < num_items; ++i) {
            w[i] = (T)dw(rng);
            v[i] = (T)dv(rng);
            total += w[i];
        }
        return std::make_unique<KnapsackConfig<T>>(w, v, total * capacity_ratio, name + "_" + std::to_string(num_items),
                                                   greedy);
    }

private:
    std::vector<T> weights_, values_;
    T capacity_;
    std::string name_;
};

// configs/multi_tsp_config.hpp:16-296 (depot 0, two objectives)
template <typename T>
class MultiTSPConfig : public DeviceProblemConfig<T> {
public:
    MultiTSPConfig(const std::vector<std::vector<T>>& distances, const std::vector<std::vector<T>>& times,
                   const std::string& name = "MultiTSP")
        : DeviceProblemConfig<T>(std::vector<int>{(int)distances.size() - 1}, 2), name_(name) {
        const int dim = (int)distances.size();
        std::vector<float> a((size_t)dim * dim), b((size_t)dim * dim);
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < dim; ++j) {
                a[(size_t)i * dim + j] = (float)distances[i][j];
                b[(size_t)i * dim + j] = (float)times[i][j];
            }
        brkga_problem_desc d{};
        d.kind = BRKGA_BITSP_MATRIX;
        d.n = dim - 1;
        d.matrix = a.data();
        d.matrix2 = b.data();
        this->create(d);
        // core/config.hpp defaults as MultiTSPConfig sets them (multi_tsp_config.hpp:34-39)
        this->population_size = 100;
        this->elite_size = 0;
        this->mutant_size = 0;
        this->max_generations = 500;
        this->elite_prob = 0.7;
        this->update_cuda_grid_size();
    }
    int get_num_cities() const { return this->component_lengths[0]; }

private:
    std::string name_;
};

// configs/job_scheduling_gpu_config.hpp:16-197: gene i puts job i on machine
// (int)(key * machines); fitness = makespan (largest machine load), minimised
// configs/multi_objective_vrp_config.hpp:21-449: a capacitated VRP with two objectives (total
// distance plus the overload and fleet penalties; the longest route).  Decode and objectives
// run on the device (BRKGA_MOVRP); runs take the NSGA-II path.
template <typename T>
class MultiObjectiveVRPConfig : public DeviceProblemConfig<T> {
public:
    struct Customer {
        int id;
        T x, y;
        int demand;
    };
    // nodes[0] is the depot; vehicles is the fleet the reference reads from the name ("-k<V>")
    MultiObjectiveVRPConfig(const std::vector<Customer>& nodes, int vehicle_capacity, int vehicles,
                            const std::string& name = "MO-VRP")
        : DeviceProblemConfig<T>(std::vector<int>{(int)nodes.size() - 1}, 2), customers_(nodes),
          capacity_(vehicle_capacity), vehicles_(vehicles), name_(name) {
        if (nodes.size() < 2) throw std::invalid_argument("MO-VRP needs a depot and at least one customer");
        std::vector<float> xy(2 * nodes.size());
        std::vector<int32_t> dem(nodes.size());
        for (size_t i = 0; i < nodes.size(); ++i) {
            xy[2 * i] = (float)nodes[i].x;
            xy[2 * i + 1] = (float)nodes[i].y;
            dem[i] = nodes[i].demand;
        }
        brkga_problem_desc d{};
        d.kind = BRKGA_MOVRP;
        d.n = (int)nodes.size() - 1;
        d.coords = xy.data();
        d.demands = dem.data();
        d.vehicle_capacity = vehicle_capacity;
        d.vehicles = vehicles;
        this->create(d);
        this->update_cuda_grid_size();
    }

    // configs/multi_objective_vrp_config.hpp:78-165: "NAME : <name>", "DIMENSION : <depot +
    // customers>", "CAPACITY : <c>", then NODE_COORD_SECTION (id x y, ids from 1, the depot
    // first) and DEMAND_SECTION (id demand); the fleet is the number after "-k" in the name,
    // else max(3, customers / 6)
    static std::unique_ptr<MultiObjectiveVRPConfig<T>> load_from_file(const std::string& filename) {
        std::ifstream f(filename);
        if (!f.is_open()) throw std::runtime_error("Cannot open VRP file: " + filename);
        auto value_after_colon = [](const std::string& line) {
            const size_t c = line.find(':');
            std::string v = (c == std::string::npos) ? line : line.substr(c + 1);
            v.erase(0, v.find_first_not_of(" \t"));
            v.erase(v.find_last_not_of(" \t\r") + 1);
            return v;
        };
        std::string line, name;
        int dim = 0, capacity = 0;
        bool coords = false;
        while (std::getline(f, line)) {
            if (line.find("NODE_COORD_SECTION") != std::string::npos) {
                coords = true;
                break;
            }
            if (line.find("NAME") != std::string::npos && line.find(':') != std::string::npos)
                name = value_after_colon(line);
            else if (line.find("DIMENSION") != std::string::npos)
                dim = std::stoi(value_after_colon(line));
            else if (line.find("CAPACITY") != std::string::npos)
                capacity = std::stoi(value_after_colon(line));
        }
        if (!coords || dim < 2) throw std::runtime_error("VRP file without NODE_COORD_SECTION: " + filename);
        std::vector<Customer> nodes(dim, Customer{0, T(0), T(0), 0});
        for (int i = 0; i < dim; ++i) {
            int id;
            T x, y;
            if (!(f >> id >> x >> y) || id < 1 || id > dim) throw std::runtime_error("bad coordinate line in " + filename);
            nodes[id - 1] = Customer{id - 1, x, y, 0};
        }
        bool demands = false;
        while (std::getline(f, line))
            if (line.find("DEMAND_SECTION") != std::string::npos) {
                demands = true;
                break;
            }
        if (demands)
            for (int i = 0; i < dim; ++i) {
                int id, dem;
                if (!(f >> id >> dem) || id < 1 || id > dim) throw std::runtime_error("bad demand line in " + filename);
                nodes[id - 1].demand = dem;
            }
        const size_t k = name.find("-k");
        const int vehicles = (k != std::string::npos) ? std::stoi(name.substr(k + 2)) : std::max(3, (dim - 1) / 6);
        return std::make_unique<MultiObjectiveVRPConfig<T>>(nodes, capacity, vehicles, name);
    }
    // configs/multi_objective_vrp_config.hpp:190-211
    static void configure_for_size(MultiObjectiveVRPConfig<T>* c, int num_customers) {
        if (num_customers <= 50) {
            c->population_size = 1000, c->max_generations = 1500;
        } else if (num_customers <= 100) {
            c->population_size = 1500, c->max_generations = 2000;
        } else {
            c->population_size = 2000, c->max_generations = 2500;
        }
        c->elite_size = c->population_size / 5;
        c->mutant_size = c->population_size / 6;
        c->elite_prob = 0.10;
        c->update_cuda_grid_size();
    }
    int get_num_customers() const { return (int)customers_.size() - 1; }
    int get_num_vehicles() const { return vehicles_; }
    int get_vehicle_capacity() const { return capacity_; }
    const std::vector<Customer>& get_customers() const { return customers_; }
    const std::string& get_instance_name() const { return name_; }
    // the routes (customers 1..n in visiting order) of a device-decoded order such as
    // Solver::get_best_permutation() -- the split of decode_routes (:236-264), for reports
    std::vector<std::vector<int>> routes_of(const std::vector<int>& perm) const {
        std::vector<std::vector<int>> routes;
        std::vector<int> cur;
        int load = 0;
        for (int g : perm) {
            const int c = g + 1, dem = customers_[c].demand;
            if (load + dem > capacity_ && !cur.empty()) {
                routes.push_back(cur);
                cur.clear();
                load = 0;
            }
            cur.push_back(c);
            load += dem;
        }
        if (!cur.empty()) routes.push_back(cur);
        return routes;
    }

private:
    std::vector<Customer> customers_;
    int capacity_, vehicles_;
    std::string name_;
};

template <typename T>
class JobSchedulingGPUConfig : public DeviceProblemConfig<T> {
public:
    JobSchedulingGPUConfig(const std::vector<T>& jobs, int machines, const std::string& name = "JobScheduling_GPU")
        : DeviceProblemConfig<T>((int)jobs.size()), job_times_(jobs), machines_(machines), name_(name) {
        if (machines <= 0) throw std::invalid_argument("Number of machines must be positive");
        std::vector<float> jt(jobs.begin(), jobs.end());
        brkga_problem_desc d{};
        d.kind = BRKGA_JOBSCHED;
        d.n = (int)jobs.size();
        d.job_times = jt.data();
        d.machines = machines;
        this->create(d);
        this->comparator = [](T a, T b) { return a < b; };
        this->threads_per_block = 256;
        this->update_cuda_grid_size();
    }
    // configs/job_scheduling_gpu_config.hpp:216-229
    static std::unique_ptr<JobSchedulingGPUConfig<T>> create_test_instance(int num_jobs = 50, int num_machines = 5) {
        std::vector<T> jobs;
        for (int i = 0; i < num_jobs; ++i) jobs.push_back((T)(10 + (i % 40)));
        return std::make_unique<JobSchedulingGPUConfig<T>>(
            jobs, num_machines, "Test_GPU_J" + std::to_string(num_jobs) + "_M" + std::to_string(num_machines));
    }
    bool is_gpu_available() const { return this->pb_ != nullptr; }
    int get_num_machines() const { return machines_; }

private:
    std::vector<T> job_times_;
    int machines_;
    std::string name_;
};

// configs/continuous_opt_gpu_config.hpp:20-240: x = key * (upper - lower) + lower
enum class OptimizationFunction { SPHERE, RASTRIGIN, ROSENBROCK };

template <typename T>
class ContinuousOptGPUConfig : public DeviceProblemConfig<T> {
public:
    ContinuousOptGPUConfig(int num_vars, T lower, T upper, OptimizationFunction func = OptimizationFunction::SPHERE,
                           const std::string& name = "ContinuousOpt_GPU")
        : DeviceProblemConfig<T>(num_vars), lower_(lower), upper_(upper), func_(func), name_(name) {
        brkga_problem_desc d{};
        d.kind = BRKGA_CONTINUOUS;
        d.n = num_vars;
        d.function = func == OptimizationFunction::RASTRIGIN    ? BRKGA_FN_RASTRIGIN
                     : func == OptimizationFunction::ROSENBROCK ? BRKGA_FN_ROSENBROCK
                                                                : BRKGA_FN_SPHERE;
        d.lower = (float)lower;
        d.upper = (float)upper;
        this->create(d);
        this->comparator = [](T a, T b) { return a < b; };
        this->threads_per_block = 256;
        this->update_cuda_grid_size();
    }
    // configs/continuous_opt_gpu_config.hpp:216-237
    static std::unique_ptr<ContinuousOptGPUConfig<T>> create_sphere(int num_vars = 30) {
        return std::make_unique<ContinuousOptGPUConfig<T>>(num_vars, (T)-5.12, (T)5.12, OptimizationFunction::SPHERE,
                                                           "Sphere_GPU_" + std::to_string(num_vars));
    }
    static std::unique_ptr<ContinuousOptGPUConfig<T>> create_rastrigin(int num_vars = 30) {
        return std::make_unique<ContinuousOptGPUConfig<T>>(num_vars, (T)-5.12, (T)5.12,
                                                           OptimizationFunction::RASTRIGIN,
                                                           "Rastrigin_GPU_" + std::to_string(num_vars));
    }
    static std::unique_ptr<ContinuousOptGPUConfig<T>> create_rosenbrock(int num_vars = 30) {
        return std::make_unique<ContinuousOptGPUConfig<T>>(num_vars, (T)-5.0, (T)10.0,
                                                           OptimizationFunction::ROSENBROCK,
                                                           "Rosenbrock_GPU_" + std::to_string(num_vars));
    }
    // the decision variables of a chromosome
    std::vector<T> decode(const Individual<T>& ind) const {
        std::vector<T> x;
        for (T g : ind.chromosomes[0]) x.push_back(g * (upper_ - lower_) + lower_);
        return x;
    }
    bool is_gpu_available() const { return this->pb_ != nullptr; }

private:
    T lower_, upper_;
    OptimizationFunction func_;
    std::string name_;
};

// configs/tspj_config.hpp:24-983: a tour over the depot (node 0) and c cities plus an
// assignment of c job types to the tour positions; chromosome = c city keys then c job
// keys; fitness = makespan (max of the tour length and the latest arrival + job time)
template <typename T>
class TSPJConfig : public DeviceProblemConfig<T> {
public:
    TSPJConfig(const std::vector<std::vector<T>>& travel, const std::vector<std::vector<T>>& jobs,
               const std::string& name = "TSPJ")
        : DeviceProblemConfig<T>(std::vector<int>{(int)travel.size() - 1, (int)travel.size() - 1}),
          num_cities_((int)travel.size() - 1), name_(name) {
        const int dim = (int)travel.size();
        if (dim < 2 || (int)jobs.size() != dim) throw std::invalid_argument("TSPJ needs two (c+1) x (c+1) matrices");
        std::vector<float> a((size_t)dim * dim), b((size_t)dim * dim);
        for (int i = 0; i < dim; ++i) {
            if ((int)travel[i].size() != dim || (int)jobs[i].size() != dim)
                throw std::invalid_argument("TSPJ matrices must be square and of equal size");
            for (int j = 0; j < dim; ++j) {
                a[(size_t)i * dim + j] = (float)travel[i][j];
                b[(size_t)i * dim + j] = (float)jobs[i][j];
            }
        }
        brkga_problem_desc d{};
        d.kind = BRKGA_TSPJ;
        d.n = num_cities_;
        d.matrix = a.data();
        d.matrix2 = b.data();
        this->create(d);
        this->comparator = [](T x, T y) { return x < y; };
        this->threads_per_block = 256;
        this->update_cuda_grid_size();
    }
    bool has_local_search() const override { return true; }

    // configs/tspj_config.hpp:727-770: <name>_TT.csv / <name>_JT.csv, or
    // <name>_cost_table_by_coordinates.csv / <name>_tasktime_table.csv, given either file
    static std::unique_ptr<TSPJConfig<T>> load_from_file(const std::string& filename) {
        const size_t slash = filename.find_last_of('/');
        const std::string dir = (slash == std::string::npos) ? "." : filename.substr(0, slash);
        std::string base = (slash == std::string::npos) ? filename : filename.substr(slash + 1);
        const size_t dot = base.find_last_of('.');
        if (dot != std::string::npos) base = base.substr(0, dot);
        std::string tt, jt, name;
        auto cut = [&](const std::string& tag) { return base.substr(0, base.find(tag)); };
        if (base.find("_TT") != std::string::npos) {
            name = cut("_TT"), tt = filename, jt = dir + "/" + name + "_JT.csv";
        } else if (base.find("_JT") != std::string::npos) {
            name = cut("_JT"), jt = filename, tt = dir + "/" + name + "_TT.csv";
        } else if (base.find("_cost_table_by_coordinates") != std::string::npos) {
            name = cut("_cost_table_by_coordinates"), tt = filename, jt = dir + "/" + name + "_tasktime_table.csv";
        } else if (base.find("_tasktime_table") != std::string::npos) {
            name = cut("_tasktime_table"), jt = filename,
            tt = dir + "/" + name + "_cost_table_by_coordinates.csv";
        } else {
            throw std::runtime_error(
                "TSPJ CSV files must be named with '_TT'/'_JT' or '_cost_table_by_coordinates'/'_tasktime_table' suffix");
        }
        if (!std::ifstream(tt).good()) throw std::runtime_error("Travel times file not found: " + tt);
        if (!std::ifstream(jt).good()) throw std::runtime_error("Job times file not found: " + jt);
        return std::make_unique<TSPJConfig<T>>(load_csv_matrix(tt), load_csv_matrix(jt), name);
    }
    // configs/tspj_config.hpp:803-825
    static void configure_for_size(TSPJConfig<T>* c, int n) {
        if (n <= 10) {
            c->population_size = 300, c->elite_size = 60, c->mutant_size = 30, c->max_generations = 500;
        } else if (n <= 20) {
            c->population_size = 600, c->elite_size = 120, c->mutant_size = 60, c->max_generations = 1000;
        } else if (n <= 50) {
            c->population_size = 1000, c->elite_size = 200, c->mutant_size = 100, c->max_generations = 2000;
        } else {
            c->population_size = 2000, c->elite_size = 350, c->mutant_size = 200, c->max_generations = 30000;
        }
        c->elite_prob = 0.75;
        c->update_cuda_grid_size();
    }
    int get_num_cities() const { return num_cities_; }
    int get_num_jobs() const { return num_cities_; }
    const std::string& get_instance_name() const { return name_; }

private:
    // comma-separated rows; '#' lines and empty lines skipped; unparsable cells read as 0
    // (configs/tspj_config.hpp:773-800)
    static std::vector<std::vector<T>> load_csv_matrix(const std::string& path) {
        std::ifstream f(path);
        std::vector<std::vector<T>> m;
        std::string line;
        while (std::getline(f, line)) {
            if (line.empty() || line[0] == '#') continue;
            std::vector<T> row;
            std::stringstream ss(line);
            std::string cell;
            while (std::getline(ss, cell, ',')) {
                const size_t a = cell.find_first_not_of(" \t\r\n");
                if (a == std::string::npos) continue;
                cell = cell.substr(a, cell.find_last_not_of(" \t\r\n") - a + 1);
                try {
                    row.push_back((T)std::stod(cell));
                } catch (const std::exception&) {
                    row.push_back(T(0));
                }
            }
            if (!row.empty()) m.push_back(row);
        }
        return m;
    }
    int num_cities_;
    std::string name_;
};

// core/solver.hpp:44-1726: device-resident population, one CUDA graph per chunk of
// generations; run / initialize / evolve_generation / get_best_individual /
// get_pareto_front / get_fitness_history / get_config / export_pareto_front
template <typename T>
class Solver {
public:
    Solver(std::unique_ptr<BRKGAConfig<T>> cfg, bool verbose = true, int print_freq = 50)
        : config_(std::move(cfg)), verbose_(verbose), print_freq_(print_freq) {
        if (!config_->is_valid()) throw std::runtime_error("Invalid configuration");
        n_ = config_->get_total_chromosome_length();
        brkga_problem* pb = config_->problem_handle();
        if (!pb) {
            // a config with its own fitness: the engine's external-fitness path
            const bool mo = config_->num_objectives > 1;
            if (config_->num_objectives > 2)
                throw std::runtime_error("external-fitness configs have one or two objectives");
            if (!config_->has_gpu_evaluation()) {
                if (!mo && !config_->fitness_function) throw std::runtime_error("Fitness function not set");
                if (mo && ((int)config_->objective_functions.size() < 2 || !config_->objective_functions[0] ||
                           !config_->objective_functions[1]))
                    throw std::runtime_error("Multi-objective mode but no objective functions defined");
            }
            brkga_problem_desc d{};
            d.kind = BRKGA_EXTERNAL;
            d.n = n_;
            d.num_objectives = mo ? 2 : 1;
            // the reference's comparator says which fitness is better (core/config.hpp:36);
            // objectives are minimised (Individual::dominates)
            d.maximize = (!mo && config_->comparator && config_->comparator(T(1), T(0))) ? 1 : 0;
            brkga_b200_detail::check(brkga_problem_create(&d, config_->device, &ext_pb_), "Solver");
            pb = ext_pb_;
        }
        brkga_params p;
        brkga_params_default(&p);
        p.population_size = config_->population_size;
        p.elite_size = config_->elite_size;
        p.mutant_size = config_->num_objectives > 1 ? config_->nsga2_random_offspring : config_->mutant_size;
        p.elite_prob = config_->elite_prob;
        p.max_generations = config_->max_generations;
        p.seed = config_->seed;
        p.num_islands = config_->num_islands;
        p.migration_interval = config_->migration_interval;
        p.num_migrants = config_->num_migrants;
        p.device = config_->device;
        if (config_->has_local_search()) {
            p.local_search_interval = config_->local_search_interval;
            p.local_search_individuals = config_->local_search_individuals;
            p.local_search_moves = config_->local_search_moves;
        }
        const int32_t rc = brkga_create(pb, &p, &e_);
        if (rc != BRKGA_OK) {
            char buf[512];
            brkga_last_error(buf, sizeof(buf));
            if (ext_pb_) brkga_problem_destroy(ext_pb_);
            ext_pb_ = nullptr;
            throw std::runtime_error(std::string("Solver: ") + buf);
        }
        best_ = Individual<T>(config_->component_lengths, config_->num_objectives > 1 ? config_->num_objectives : 0);
    }
    ~Solver() {
        if (e_) brkga_destroy(e_);
        if (ext_pb_) brkga_problem_destroy(ext_pb_);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    void initialize() {
        brkga_b200_detail::check(brkga_initialize(e_), "initialize");
        if (ext_pb_) external_generation();  // the initial population, evaluated by the config
        initialized_ = true;
    }
    void evolve_generation() { evolve(1); }
    void evolve(int generations) {
        if (!ext_pb_) {
            brkga_b200_detail::check(brkga_evolve(e_, generations), "evolve");
            return;
        }
        if (!initialized_) initialize();
        for (int g = 0; g < generations; ++g) {
            external_generation();
            if (verbose_ && print_freq_ > 0 && brkga_generation(e_) % print_freq_ == 0)
                std::cout << "Generation " << brkga_generation(e_) << ": best fitness " << std::setprecision(6)
                          << get_best_individual().fitness << std::endl;
        }
    }
    // Solver::run (core/solver.hpp:1517-1556): initialize, then config->max_generations
    // generations (read now, so a caller may change it after construction)
    void run() {
        initialize();
        evolve(config_->max_generations);
        brkga_b200_detail::check(brkga_synchronize(e_), "run");
        if (verbose_) {
            const auto& b = get_best_individual();
            std::cout << "Evolution completed: " << brkga_generation(e_) << " generations, best fitness "
                      << std::setprecision(6) << b.fitness << std::endl;
        }
    }
    const Individual<T>& get_best_individual() {
        std::vector<float> k(n_), f(2);
        brkga_b200_detail::check(brkga_get_best(e_, k.data(), nullptr, f.data()), "get_best_individual");
        size_t off = 0;  // the flat key row, component by component (core/solver.hpp:300-312)
        for (size_t c = 0; c < best_.chromosomes.size(); ++c) {
            const size_t len = (size_t)config_->component_lengths[c];
            best_.chromosomes[c].assign(k.begin() + off, k.begin() + off + len);
            off += len;
        }
        best_.fitness = f[0];
        if (config_->num_objectives > 1) best_.objectives = {(T)f[0], (T)f[1]};
        best_.evaluated = true;
        return best_;
    }
    // the decoded tour / selection order of the best individual
    std::vector<int> get_best_permutation() {
        std::vector<int32_t> p(n_);
        brkga_b200_detail::check(brkga_get_best(e_, nullptr, p.data(), nullptr), "get_best_permutation");
        return std::vector<int>(p.begin(), p.end());
    }
    std::vector<Individual<T>> get_pareto_front() {
        std::vector<Individual<T>> out;
        if (config_->num_objectives < 2) return out;
        const int cap = config_->population_size;
        std::vector<float> obj((size_t)cap * 2), keys((size_t)cap * n_);
        int32_t cnt = 0;
        brkga_b200_detail::check(brkga_get_pareto_front(e_, obj.data(), keys.data(), cap, &cnt), "get_pareto_front");
        for (int i = 0; i < std::min<int>(cnt, cap); ++i) {
            Individual<T> ind(config_->component_lengths, 2);
            ind.chromosomes[0].assign(keys.begin() + (size_t)i * n_, keys.begin() + (size_t)(i + 1) * n_);
            ind.objectives = {(T)obj[2 * i], (T)obj[2 * i + 1]};
            ind.fitness = ind.objectives[0];
            ind.rank = 0;
            ind.evaluated = true;
            out.push_back(ind);
        }
        return out;
    }
    const std::vector<T>& get_fitness_history() {
        const int len = brkga_generation(e_) + 1;
        std::vector<float> h(len);
        int32_t got = 0;
        brkga_b200_detail::check(brkga_get_fitness_history(e_, h.data(), len, &got), "get_fitness_history");
        history_.assign(h.begin(), h.begin() + got);
        return history_;
    }
    BRKGAConfig<T>* get_config() { return config_.get(); }
    void export_pareto_front(const std::string& filename) {
        auto front = get_pareto_front();
        std::ofstream f(filename);
        f << "# Pareto Front\n# Objectives: " << config_->num_objectives << "\n# Solutions: " << front.size() << "\n";
        for (const auto& ind : front) f << ind.objectives[0] << " " << ind.objectives[1] << "\n";
    }

private:
    // one generation (the initial population first) with the config's own fitness: its
    // evaluate_population_gpu on dense device rows, or its fitness_function /
    // objective_functions on each row (Population::evaluate_all, core/population.hpp:523-527,
    // 567-595, 626-652); BRKGA elite rows keep their fitness.  An NSGA-II generation whose
    // diversity pass replaced rows asks for those too (BRKGA_ERR_NOT_READY).
    void external_generation() {
        const bool gpu = config_->has_gpu_evaluation();
        const int m = config_->num_objectives > 1 ? 2 : 1;
        for (;;) {
            float* dk = nullptr;
            float* df = nullptr;
            int32_t ld = 0, first = 0, count = 0;
            brkga_b200_detail::check(brkga_external_begin(e_, gpu ? 1 : 0, &dk, &df, &ld, &first, &count),
                                     "evolve_generation");
            if (gpu) {
                if (count > 0) config_->evaluate_population_gpu(reinterpret_cast<T*>(dk), reinterpret_cast<T*>(df), count, n_);
            } else {
                rows_.resize((size_t)count * n_);
                fit_.resize((size_t)count * m);
                brkga_b200_detail::check(brkga_external_get_rows(e_, rows_.data()), "evolve_generation");
                Individual<T> ind(config_->component_lengths, m > 1 ? m : 0);
                for (int i = 0; i < count; ++i) {
                    size_t off = (size_t)i * n_;
                    for (size_t c = 0; c < ind.chromosomes.size(); ++c) {
                        const size_t len = (size_t)config_->component_lengths[c];
                        ind.chromosomes[c].assign(rows_.begin() + off, rows_.begin() + off + len);
                        off += len;
                    }
                    ind.evaluated = false;
                    if (m == 1)
                        fit_[i] = (float)config_->fitness_function(ind);
                    else
                        for (int o = 0; o < m; ++o) fit_[(size_t)i * m + o] = (float)config_->objective_functions[o](ind);
                }
                brkga_b200_detail::check(brkga_external_set_fitness(e_, fit_.data()), "evolve_generation");
            }
            const int32_t rc = brkga_external_commit(e_);
            if (rc == BRKGA_OK) return;
            if (rc != BRKGA_ERR_NOT_READY) brkga_b200_detail::check(rc, "evolve_generation");
        }
    }

    std::unique_ptr<BRKGAConfig<T>> config_;
    bool verbose_;
    int print_freq_;
    brkga_problem* ext_pb_ = nullptr;  // the external-fitness problem this Solver made
    bool initialized_ = false;
    std::vector<float> rows_, fit_;
    brkga_engine* e_ = nullptr;
    int n_ = 0;
    Individual<T> best_;
    std::vector<T> history_;
};

#endif  // BRKGA_B200_HPP
