"""Python front end of libbrkga_b200.so (the C ABI in include/brkga_b200.h).

The classes mirror the reference's solver surface (hsaseendran/llm-brkga,
brkga/core/solver.hpp): ``Solver.run / initialize / evolve_generation /
get_best_individual / get_fitness_history / get_pareto_front``, problem configs built
like ``TSPConfig``, ``KnapsackConfig`` and ``MultiTSPConfig``.  Everything below is a
ctypes binding: every operation runs in the CUDA library; there is no Python or CPU
implementation of the hot path, and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libbrkga_b200.so")
REPO_DIR = os.path.dirname(PKG_DIR)
HEADER_PATH = os.path.join(REPO_DIR, "include", "brkga_b200.h")

TSP_COORDS, TSP_MATRIX, KNAP_THRESHOLD, KNAP_GREEDY, BITSP_COORDS, BITSP_MATRIX, TSPJ = 1, 2, 3, 4, 5, 6, 7
JOBSCHED, CONTINUOUS = 8, 9
MOVRP = 10
EXTERNAL = 11
SPHERE, RASTRIGIN, ROSENBROCK = 0, 1, 2

STATUS = {0: "OK", -1: "INVALID", -2: "OOM", -3: "CUDA", -4: "TIMEOUT", -5: "CANCELLED",
          -6: "UNSUPPORTED", -7: "BUSY", -8: "NOT_READY"}


class BrkgaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class ProblemDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n", C.c_int32), ("coords", C.c_void_p), ("coords2", C.c_void_p),
                ("matrix", C.c_void_p), ("matrix2", C.c_void_p), ("weights", C.c_void_p),
                ("values", C.c_void_p), ("capacity", C.c_float), ("job_times", C.c_void_p),
                ("machines", C.c_int32), ("function", C.c_int32), ("lower", C.c_float), ("upper", C.c_float),
                ("demands", C.c_void_p), ("vehicle_capacity", C.c_int32), ("vehicles", C.c_int32),
                ("maximize", C.c_int32), ("num_objectives", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("population_size", C.c_int32), ("elite_size", C.c_int32), ("mutant_size", C.c_int32),
                ("elite_prob", C.c_double), ("max_generations", C.c_int32), ("seed", C.c_uint64),
                ("num_islands", C.c_int32), ("migration_interval", C.c_int32), ("num_migrants", C.c_int32),
                ("device", C.c_int32), ("diversity_interval", C.c_int32), ("mutation_rate", C.c_double),
                ("local_search_interval", C.c_int32), ("local_search_individuals", C.c_int32),
                ("local_search_moves", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_active", C.c_int32), ("memory_budget", C.c_int64),
                ("generations_per_tick", C.c_int32)]


def build() -> None:
    """Compile the CUDA library for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.check_call(["make", "-s", "-C", PKG_DIR, "-j8"])


_lib = None
_vp, _i32, _i64, _u32, _u64, _f, _d = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_float, C.c_double


def lib():
    """Load libbrkga_b200.so.  Raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not found: build it first (make -C {PKG_DIR})")
    L = C.CDLL(LIB_PATH)
    sig = {
        "brkga_abi_version": (_i32, []),
        "brkga_last_error": (_i32, [C.c_char_p, C.c_size_t]),
        "brkga_params_default": (None, [C.POINTER(Params)]),
        "brkga_problem_create": (_i32, [C.POINTER(ProblemDesc), _i32, C.POINTER(_vp)]),
        "brkga_problem_destroy": (_i32, [_vp]),
        "brkga_problem_num_objectives": (_i32, [_vp]),
        "brkga_problem_maximize": (_i32, [_vp]),
        "brkga_evaluate_population": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
        "brkga_evaluate_population_sync": (_i32, [_vp, _vp, _vp, _i32, _i32]),
        "brkga_sort_fitness": (_i32, [_vp, _i32, _i32, _i32, _vp, _vp]),
        "brkga_generation_step": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _d, _i32, _u64, _u32,
                                         _i32, _vp]),
        "brkga_init_population": (_i32, [_vp, _vp, _vp, _i32, _i32, _u64, _i32, _vp]),
        "brkga_local_search": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _u64, _u32, _i32, _vp]),
        "brkga_pareto_rank": (_i32, [_vp, _i32, _i32, _vp, _vp]),
        "brkga_pareto_rank_bitmatrix": (_i32, [_vp, _i32, _i32, _vp, _vp]),
        "brkga_pareto_rank_noalloc": (_i32, [_vp, _i32, _i32, _vp, _vp]),
        "brkga_crowding": (_i32, [_vp, _vp, _i32, _i32, _vp, _vp]),
        "brkga_create": (_i32, [_vp, C.POINTER(Params), C.POINTER(_vp)]),
        "brkga_destroy": (_i32, [_vp]),
        "brkga_initialize": (_i32, [_vp]),
        "brkga_evolve": (_i32, [_vp, _i32]),
        "brkga_synchronize": (_i32, [_vp]),
        "brkga_run": (_i32, [_vp]),
        "brkga_generation": (_i32, [_vp]),
        "brkga_get_stream": (_i32, [_vp, C.POINTER(_vp)]),
        "brkga_engine_info": (_i32, [_vp, _vp, _i32]),
        "brkga_get_best": (_i32, [_vp, _vp, _vp, _vp]),
        "brkga_get_fitness_history": (_i32, [_vp, _vp, _i32, C.POINTER(_i32)]),
        "brkga_get_population": (_i32, [_vp, _vp, _vp]),
        "brkga_set_population": (_i32, [_vp, _vp]),
        "brkga_get_pareto_front": (_i32, [_vp, _vp, _vp, _i32, C.POINTER(_i32)]),
        "brkga_external_begin": (_i32, [_vp, _i32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_i32),
                                        C.POINTER(_i32), C.POINTER(_i32)]),
        "brkga_external_get_rows": (_i32, [_vp, _vp]),
        "brkga_external_set_fitness": (_i32, [_vp, _vp]),
        "brkga_external_commit": (_i32, [_vp]),
        "brkga_batch_create": (_i32, [C.POINTER(_vp), C.POINTER(Params), _i32, C.POINTER(_vp)]),
        "brkga_batch_destroy": (_i32, [_vp]),
        "brkga_batch_evolve": (_i32, [_vp, _i32]),
        "brkga_batch_synchronize": (_i32, [_vp]),
        "brkga_batch_get_best": (_i32, [_vp, _vp]),
        "brkga_batch_get_best_keys": (_i32, [_vp, _i32, _vp, _vp]),
        "brkga_server_create": (_i32, [C.POINTER(ServerConfig), C.POINTER(_vp)]),
        "brkga_server_destroy": (_i32, [_vp]),
        "brkga_server_submit": (_i32, [_vp, C.POINTER(ProblemDesc), C.POINTER(Params), _i32, C.POINTER(_i64)]),
        "brkga_server_step": (_i32, [_vp]),
        "brkga_server_poll": (_i32, [_vp, _i64, _vp, C.POINTER(_i32), C.POINTER(_d)]),
        "brkga_server_cancel": (_i32, [_vp, _i64]),
        "brkga_server_stats": (_i32, [_vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().brkga_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(code):
    if code != 0:
        raise BrkgaError(code, last_error())
    return code


def _ptr(a):
    return None if a is None else a.ctypes.data


def _dptr(t):
    """device pointer of a torch tensor (or an int address)"""
    if t is None:
        return None
    return t if isinstance(t, int) else t.data_ptr()


def _stream(s):
    if s is None:
        return None
    return s if isinstance(s, int) else s.cuda_stream


# ---------------------------------------------------------------------------------------
# problems
# ---------------------------------------------------------------------------------------
class Problem:
    """Device-resident instance (TSPConfig / KnapsackConfig / MultiTSPConfig data)."""

    def __init__(self, kind, n, coords=None, coords2=None, matrix=None, matrix2=None, weights=None, values=None,
                 capacity=0.0, device=0, job_times=None, machines=0, function=0, lower=0.0, upper=0.0,
                 demands=None, vehicle_capacity=0, vehicles=0, maximize=False, num_objectives=1):
        keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        d = ProblemDesc(kind, n, arr(coords, np.float32), arr(coords2, np.float32), arr(matrix, np.float32),
                        arr(matrix2, np.float32), arr(weights, np.int32), arr(values, np.int32), float(capacity),
                        arr(job_times, np.float32), int(machines), int(function), float(lower), float(upper),
                        arr(demands, np.int32), int(vehicle_capacity), int(vehicles), int(bool(maximize)),
                        int(num_objectives))
        h = C.c_void_p()
        check(lib().brkga_problem_create(C.byref(d), device, C.byref(h)))
        # n is the chromosome length (genes); a TSPJ instance of c cities has 2c genes
        self.h, self.kind, self.device = h, kind, device
        self.n = 2 * n if kind == TSPJ else n
        self.cities = n
        self.capacity = capacity

    @property
    def num_objectives(self):
        return lib().brkga_problem_num_objectives(self.h)

    @property
    def maximize(self):
        return bool(lib().brkga_problem_maximize(self.h))

    def close(self):
        if self.h:
            lib().brkga_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # drop-in for BRKGAConfig::evaluate_population_gpu (device buffers)
    def evaluate_population(self, d_pop, d_fit, pop_size, chrom_len=None, ld=None, d_perm=None, stream=None):
        chrom_len = self.n if chrom_len is None else chrom_len
        check(lib().brkga_evaluate_population(self.h, _dptr(d_pop), _dptr(d_fit), pop_size, chrom_len,
                                              ld or chrom_len, _dptr(d_perm), _stream(stream)))


def tsp(coords, device=0):
    coords = np.asarray(coords, np.float32)
    return Problem(TSP_COORDS, coords.shape[0], coords=coords, device=device)


def tsp_matrix(matrix, device=0):
    matrix = np.asarray(matrix, np.float32)
    return Problem(TSP_MATRIX, matrix.shape[0], matrix=matrix, device=device)


def knapsack(weights, values, capacity, greedy=True, device=0):
    w = np.asarray(weights, np.int32)
    return Problem(KNAP_GREEDY if greedy else KNAP_THRESHOLD, w.shape[0], weights=w, values=values,
                   capacity=capacity, device=device)


def bitsp(coords, coords2, device=0):
    """bi-objective TSP: two coordinate sets of n+1 points, point 0 the depot"""
    coords = np.asarray(coords, np.float32)
    return Problem(BITSP_COORDS, coords.shape[0] - 1, coords=coords, coords2=coords2, device=device)


def bitsp_matrix(matrix, matrix2, device=0):
    matrix = np.asarray(matrix, np.float32)
    return Problem(BITSP_MATRIX, matrix.shape[0] - 1, matrix=matrix, matrix2=matrix2, device=device)


def tspj(travel, jobs, device=0):
    """TSPJ (TSPJConfig): travel times and job durations over the depot and c cities,
    both [c+1][c+1]; chromosomes hold 2c keys (city keys, then job keys)"""
    travel = np.asarray(travel, np.float32)
    return Problem(TSPJ, travel.shape[0] - 1, matrix=travel, matrix2=jobs, device=device)


def jobsched(job_times, machines, device=0):
    """job scheduling (JobSchedulingGPUConfig): gene i puts job i on machine
    floor(key * machines); fitness = makespan"""
    jt = np.asarray(job_times, np.float32)
    return Problem(JOBSCHED, jt.shape[0], job_times=jt, machines=machines, device=device)


def movrp(coords, demands, vehicle_capacity, vehicles, device=0):
    """bi-objective capacitated VRP (MultiObjectiveVRPConfig): coords and demands of the
    depot (point 0) and n customers; objectives total distance and longest route"""
    coords = np.asarray(coords, np.float32)
    return Problem(MOVRP, coords.shape[0] - 1, coords=coords, demands=demands, vehicle_capacity=vehicle_capacity,
                   vehicles=vehicles, device=device)


def external(n, maximize=False, num_objectives=1, device=0):
    """A problem whose fitness the caller computes (a BRKGAConfig with its own
    fitness_function / objective_functions, core/config.hpp:33-53): n keys per row; one
    objective (BRKGA) or two (NSGA-II, minimised)."""
    return Problem(EXTERNAL, n, device=device, maximize=maximize, num_objectives=num_objectives)


def movrp_routes(perm, demands, vehicle_capacity):
    """the routes (customers 1..n in visiting order, as MultiObjectiveVRPConfig::decode_routes
    lists them) of a row the device decoded, e.g. the permutation of get_best_individual:
    report formatting only, the objectives come from the device"""
    routes, cur, load = [], [], 0
    for g in np.asarray(perm):
        c = int(g) + 1
        d = int(demands[c])
        if load + d > vehicle_capacity and cur:
            routes.append(cur)
            cur, load = [], 0
        cur.append(c)
        load += d
    if cur:
        routes.append(cur)
    return routes


def continuous(n, lower, upper, function=SPHERE, device=0):
    """continuous optimisation (ContinuousOptGPUConfig): sphere, Rastrigin or Rosenbrock
    over n variables x = key * (upper - lower) + lower"""
    return Problem(CONTINUOUS, n, function=function, lower=lower, upper=upper, device=device)


def params(population_size=100, elite_size=20, mutant_size=10, elite_prob=0.7, max_generations=1000, seed=1,
           num_islands=1, migration_interval=0, num_migrants=0, device=0, diversity_interval=25,
           mutation_rate=0.0, local_search_interval=0, local_search_individuals=100, local_search_moves=5):
    return Params(population_size, elite_size, mutant_size, elite_prob, max_generations, seed, num_islands,
                  migration_interval, num_migrants, device, diversity_interval, mutation_rate,
                  local_search_interval, local_search_individuals, local_search_moves)


# ---------------------------------------------------------------------------------------
# solver (Solver<T>, core/solver.hpp)
# ---------------------------------------------------------------------------------------
class Solver:
    def __init__(self, problem: Problem, prm: Params):
        self.problem, self.prm = problem, prm
        h = C.c_void_p()
        check(lib().brkga_create(problem.h, C.byref(prm), C.byref(h)))
        self.h = h
        self.n = problem.n
        self.m = problem.num_objectives
        self._ext_count = 0  # rows pending an external fitness (set by external_begin)

    def close(self):
        if getattr(self, "h", None):
            lib().brkga_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initialize(self):
        check(lib().brkga_initialize(self.h))

    def evolve(self, generations=1):
        check(lib().brkga_evolve(self.h, generations))

    def evolve_generation(self):
        self.evolve(1)

    def synchronize(self):
        check(lib().brkga_synchronize(self.h))

    def run(self):
        check(lib().brkga_run(self.h))

    @property
    def generation(self):
        return lib().brkga_generation(self.h)

    @property
    def info(self):
        """(threads per row CTA, float4 groups per thread, grid, coordinates staged)"""
        out = np.zeros(4, np.int32)
        check(lib().brkga_engine_info(self.h, _ptr(out), 4))
        return tuple(int(x) for x in out)

    @property
    def stream(self):
        """the engine's cudaStream_t as an integer handle"""
        s = C.c_void_p()
        check(lib().brkga_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def get_best_individual(self):
        keys = np.zeros(self.n, np.float32)
        fit = np.zeros(2, np.float32)
        if self.problem.kind == EXTERNAL:  # not decoded by the engine
            check(lib().brkga_get_best(self.h, _ptr(keys), None, _ptr(fit)))
            return keys, None, (fit[0] if self.m == 1 else fit[:2].copy())
        perm = np.zeros(self.n, np.int32)
        check(lib().brkga_get_best(self.h, _ptr(keys), _ptr(perm), _ptr(fit)))
        return keys, perm, (fit[0] if self.m == 1 else fit[:2].copy())

    # external fitness (Problem of kind EXTERNAL): the engine builds and ranks the rows, the
    # caller evaluates the pending rows between begin and commit
    def external_begin(self, dense=False):
        """(address of the first pending row's keys, address of its fitness, row stride in
        floats, its row index, number of pending rows)"""
        k, f, ld, first, cnt = C.c_void_p(), C.c_void_p(), C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().brkga_external_begin(self.h, int(bool(dense)), C.byref(k), C.byref(f), C.byref(ld),
                                         C.byref(first), C.byref(cnt)))
        self._ext_count = cnt.value
        return k.value, f.value, ld.value, first.value, cnt.value

    def external_rows(self):
        keys = np.zeros((self._ext_count, self.n), np.float32)
        check(lib().brkga_external_get_rows(self.h, _ptr(keys)))
        return keys

    def external_set_fitness(self, fitness):
        fitness = np.ascontiguousarray(fitness, np.float32)
        want = (self._ext_count,) if self.m == 1 else (self._ext_count, self.m)
        if fitness.shape != want:
            raise ValueError(f"need fitness of shape {want}")
        check(lib().brkga_external_set_fitness(self.h, _ptr(fitness)))

    def external_commit(self):
        """True when the generation is complete; False when an NSGA-II diversity pass left
        refill rows that need fitness (call external_begin again)"""
        rc = lib().brkga_external_commit(self.h)
        if rc == -8:
            return False
        check(rc)
        return True

    def external_step(self, fitness_of_rows):
        """one generation (the initial population on the first call): fitness_of_rows maps
        keys [rows][n] (numpy) to their fitness [rows] (or [rows][2])"""
        while True:
            self.external_begin()
            self.external_set_fitness(fitness_of_rows(self.external_rows()))
            if self.external_commit():
                return

    def get_fitness_history(self):
        cap = self.generation + 1
        out = np.zeros(cap, np.float32)
        ln = C.c_int32()
        check(lib().brkga_get_fitness_history(self.h, _ptr(out), cap, C.byref(ln)))
        return out[: ln.value]

    def rows(self):
        return self.prm.population_size if self.m > 1 else \
            (self.prm.population_size // max(1, self.prm.num_islands)) * max(1, self.prm.num_islands)

    def get_population(self):
        r = self.rows()
        keys = np.zeros((r, self.n), np.float32)
        fit = np.zeros((r, self.m), np.float32)
        check(lib().brkga_get_population(self.h, _ptr(keys), _ptr(fit)))
        return keys, (fit[:, 0].copy() if self.m == 1 else fit)

    def set_population(self, keys):
        keys = np.ascontiguousarray(keys, np.float32)
        check(lib().brkga_set_population(self.h, _ptr(keys)))

    def get_pareto_front(self):
        cap = self.prm.population_size
        obj = np.zeros((cap, 2), np.float32)
        keys = np.zeros((cap, self.n), np.float32)
        cnt = C.c_int32()
        check(lib().brkga_get_pareto_front(self.h, _ptr(obj), _ptr(keys), cap, C.byref(cnt)))
        c = min(cnt.value, cap)
        return obj[:c], keys[:c]


# ---------------------------------------------------------------------------------------
# operators on device buffers (torch tensors or raw addresses)
# ---------------------------------------------------------------------------------------
def sort_fitness(d_fit, P, segments, maximize, d_sorted, stream=None):
    check(lib().brkga_sort_fitness(_dptr(d_fit), P, segments, int(bool(maximize)), _dptr(d_sorted),
                                   _stream(stream)))


def generation_step(problem, d_pop, d_fit, d_sorted, d_next, d_next_fit, P, E, M, rho, ld, seed, generation,
                    island=0, stream=None):
    check(lib().brkga_generation_step(problem.h, _dptr(d_pop), _dptr(d_fit), _dptr(d_sorted), _dptr(d_next),
                                      _dptr(d_next_fit), P, E, M, rho, ld, seed, generation, island,
                                      _stream(stream)))


def local_search(problem, d_pop, d_fit, num_to_improve, num_moves, seed, generation, ld=0, island=0, stream=None):
    """TSPJ random 2-opt on rows [0, num_to_improve) (brkga_local_search)"""
    check(lib().brkga_local_search(problem.h, _dptr(d_pop), _dptr(d_fit), num_to_improve, problem.n, ld,
                                   num_moves, seed, generation, island, _stream(stream)))


def init_population(problem, d_pop, d_fit, P, ld, seed, island=0, stream=None):
    check(lib().brkga_init_population(problem.h, _dptr(d_pop), _dptr(d_fit), P, ld, seed, island,
                                      _stream(stream)))


def pareto_rank(d_obj, N, m, d_rank, stream=None, bitmatrix=False):
    fn = lib().brkga_pareto_rank_bitmatrix if bitmatrix else lib().brkga_pareto_rank
    check(fn(_dptr(d_obj), N, m, _dptr(d_rank), _stream(stream)))


def crowding(d_obj, d_rank, N, m, d_cd, stream=None):
    check(lib().brkga_crowding(_dptr(d_obj), _dptr(d_rank), N, m, _dptr(d_cd), _stream(stream)))


def header_functions(path=HEADER_PATH):
    """names of the functions include/brkga_b200.h declares"""
    import re
    txt = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|void)\s+(brkga_\w+)\s*\(", txt, re.M)))


@dataclass
class Instance:
    """synthetic instance generator output"""
    coords: np.ndarray = None
    coords2: np.ndarray = None
    weights: np.ndarray = None
    values: np.ndarray = None
    capacity: float = 0.0


# ---------------------------------------------------------------------------------------
# batched solving and serving
# ---------------------------------------------------------------------------------------
class Batch:
    """many independent instances advanced together (brkga_batch_*)"""

    def __init__(self, problems, prms):
        self.problems, self.prms = list(problems), list(prms)
        arr = (C.c_void_p * len(problems))(*[p.h for p in problems])
        parr = (Params * len(prms))(*prms)
        h = C.c_void_p()
        check(lib().brkga_batch_create(arr, parr, len(problems), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().brkga_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def evolve(self, generations):
        check(lib().brkga_batch_evolve(self.h, generations))

    def synchronize(self):
        check(lib().brkga_batch_synchronize(self.h))

    def best(self):
        out = np.zeros((len(self.problems), 2), np.float32)
        check(lib().brkga_batch_get_best(self.h, _ptr(out)))
        return out

    def best_keys(self, index):
        keys = np.zeros(self.problems[index].n, np.float32)
        fit = np.zeros(2, np.float32)
        check(lib().brkga_batch_get_best_keys(self.h, index, _ptr(keys), _ptr(fit)))
        return keys, fit


class Server:
    """continuous batching of solve requests (brkga_server_*)"""

    def __init__(self, device=0, max_active=256, memory_budget=0, generations_per_tick=25):
        cfg = ServerConfig(device, max_active, memory_budget, generations_per_tick)
        h = C.c_void_p()
        check(lib().brkga_server_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().brkga_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, kind, n, prm, stall=0, coords=None, coords2=None, matrix=None, matrix2=None, weights=None,
               values=None, capacity=0.0, job_times=None, machines=0, function=0, lower=0.0, upper=0.0,
               demands=None, vehicle_capacity=0, vehicles=0):
        keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        d = ProblemDesc(kind, n, arr(coords, np.float32), arr(coords2, np.float32), arr(matrix, np.float32),
                        arr(matrix2, np.float32), arr(weights, np.int32), arr(values, np.int32), float(capacity),
                        arr(job_times, np.float32), int(machines), int(function), float(lower), float(upper),
                        arr(demands, np.int32), int(vehicle_capacity), int(vehicles))
        rid = C.c_int64()
        check(lib().brkga_server_submit(self.h, C.byref(d), C.byref(prm), stall, C.byref(rid)))
        return rid.value

    def step(self):
        check(lib().brkga_server_step(self.h))

    def poll(self, rid):
        """None while pending, else (status, best[2], generations, latency seconds)"""
        best = np.zeros(2, np.float32)
        gens = C.c_int32()
        lat = C.c_double()
        code = lib().brkga_server_poll(self.h, rid, _ptr(best), C.byref(gens), C.byref(lat))
        if code == -8:
            return None
        return code, best, gens.value, lat.value

    def cancel(self, rid):
        check(lib().brkga_server_cancel(self.h, rid))

    def stats(self):
        q, a, f = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().brkga_server_stats(self.h, C.byref(q), C.byref(a), C.byref(f)))
        return q.value, a.value, f.value
