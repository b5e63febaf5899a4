"""ctypes front end of the CPU oracle (oracle/liboracle.so) and of the reference
harness (oracle/_ref/libref.so).

TEST INFRASTRUCTURE ONLY: the checker.  Imported by tests/, ``__graft_entry__.smoke()``
and bench.py's cpu_baseline / reference legs; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref.so")

TSP_COORDS, TSP_MATRIX, KNAP_THRESHOLD, KNAP_GREEDY, BITSP_COORDS, BITSP_MATRIX, TSPJ = 1, 2, 3, 4, 5, 6, 7
JOBSCHED, CONTINUOUS = 8, 9
MOVRP = 10

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


class Problem(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("n", C.c_int32),
        ("xy", C.c_void_p), ("xy2", C.c_void_p), ("mat", C.c_void_p), ("mat2", C.c_void_p),
        ("w", C.c_void_p), ("v", C.c_void_p), ("cap", C.c_float),
        ("jt", C.c_void_p), ("machines", C.c_int32), ("function", C.c_int32), ("lo", C.c_float), ("hi", C.c_float),
        ("vcap", C.c_int32),
    ]


class Params(C.Structure):
    _fields_ = [("P", C.c_int32), ("E", C.c_int32), ("M", C.c_int32), ("rho", C.c_double),
                ("seed", C.c_uint64), ("island", C.c_int32)]


class NsgaParams(C.Structure):
    _fields_ = [("P", C.c_int32), ("Mn", C.c_int32), ("rho", C.c_double), ("mut_rate", C.c_double),
                ("seed", C.c_uint64), ("diversity_interval", C.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_draw.restype = C.c_uint32
        L.orc_draw.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int]
        L.orc_u24.restype = C.c_float
        L.orc_u24.argtypes = [C.c_uint32]
        L.orc_prob_threshold.restype = C.c_uint32
        L.orc_prob_threshold.argtypes = [C.c_double]
        L.orc_okey.restype = C.c_uint32
        L.orc_okey.argtypes = [C.c_float]
        L.orc_decode_rows.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _i32p]
        L.orc_canon_sum.restype = C.c_float
        L.orc_canon_sum.argtypes = [_f32p, C.c_int]
        L.orc_eval_perm.argtypes = [C.POINTER(Problem), _i32p, _f32p, _f32p]
        L.orc_decode_problem.argtypes = [C.POINTER(Problem), _f32p, _i32p]
        L.orc_movrp_values.argtypes = [_f32p, C.c_int, _f32p]
        L.orc_movrp_routes.restype = C.c_int
        L.orc_movrp_routes.argtypes = [C.POINTER(Problem), _i32p, _i32p]
        L.orc_continuous_f64.restype = C.c_double
        L.orc_continuous_f64.argtypes = [C.POINTER(Problem), _f32p]
        L.orc_local_search.argtypes = [C.POINTER(Problem), _f32p, _f32p, _i32p, C.c_int, C.c_int, C.c_int,
                                       C.c_uint64, C.c_uint32, C.c_int]
        L.orc_eval_perm_f64.argtypes = [C.POINTER(Problem), _i32p, _f64p]
        L.orc_tsp_len_seq.restype = C.c_float
        L.orc_tsp_len_seq.argtypes = [C.POINTER(Problem), _i32p]
        L.orc_evaluate.argtypes = [C.POINTER(Problem), _f32p, C.c_int, C.c_int, _f32p]
        L.orc_sort_fitness.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        L.orc_generation_core.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _i32p,
                                          _i32p, _i32p, _u8p, _f32p, _f32p, _f32p]
        L.orc_brkga_generation.argtypes = [C.POINTER(Problem), C.POINTER(Params), C.c_uint32, _f32p, _f32p,
                                           _i32p, C.c_int, _f32p, _f32p]
        L.orc_brkga_init.argtypes = [C.POINTER(Problem), C.POINTER(Params), C.c_int, _f32p, _f32p]
        L.orc_migrate.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _i32p]
        L.orc_brkga_run.argtypes = [C.POINTER(Problem), C.POINTER(Params), C.c_int, C.c_int, _f32p, _f32p,
                                    _i32p, _f32p]
        L.orc_pareto_ranks.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        L.orc_pareto_ranks_strict.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        L.orc_crowding_f32.argtypes = [_f32p, _i32p, C.c_int, C.c_int, _f32p]
        L.orc_crowding_f64.argtypes = [_f32p, _i32p, C.c_int, C.c_int, _f64p]
        L.orc_crowding_strict_f32.argtypes = [_f32p, _i32p, C.c_int, C.c_int, _f32p]
        L.orc_nsga2_select.restype = C.c_int
        L.orc_nsga2_select.argtypes = [_i32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, _i32p]
        L.orc_nsga2_offspring_core.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _i32p, _f32p, _i32p, _u8p,
                                               _u8p, _f32p, _f32p]
        L.orc_nsga2_offspring.argtypes = [C.POINTER(NsgaParams), C.c_uint32, C.c_int, C.c_int, _f32p, _i32p,
                                          _f32p, _f32p]
        L.orc_nsga2_generation.argtypes = [C.POINTER(Problem), C.POINTER(NsgaParams), C.c_uint32, C.c_int,
                                           _f32p, _f32p, _i32p, _f32p]
        L.orc_nsga2_init.argtypes = [C.POINTER(Problem), C.POINTER(NsgaParams), C.c_int, _f32p, _f32p, _i32p,
                                     _f32p]
        L.orc_nsga2_diversity.restype = C.c_int
        L.orc_nsga2_diversity.argtypes = [C.POINTER(Problem), C.POINTER(NsgaParams), C.c_uint32, C.c_int,
                                          _f32p, _f32p, _i32p, _f32p]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------------------
# problem construction (keeps numpy buffers alive on the returned object)
# ---------------------------------------------------------------------------------------
class OracleProblem:
    def __init__(self, kind, n, xy=None, xy2=None, mat=None, mat2=None, w=None, v=None, cap=0.0, jt=None,
                 machines=0, function=0, lo=0.0, hi=0.0, vcap=0):
        self.kind, self.n = kind, n
        self._keep = []

        def ptr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data

        self.s = Problem(kind, n, ptr(xy, np.float32), ptr(xy2, np.float32), ptr(mat, np.float32),
                         ptr(mat2, np.float32), ptr(w, np.int32), ptr(v, np.int32), float(cap),
                         ptr(jt, np.float32), int(machines), int(function), float(lo), float(hi), int(vcap))

    @property
    def m(self):
        return 2 if self.kind in (BITSP_COORDS, BITSP_MATRIX, MOVRP) else 1

    @property
    def maximize(self):
        return self.kind in (KNAP_THRESHOLD, KNAP_GREEDY)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def decode(keys, n=None, ld=None):
    keys = np.ascontiguousarray(keys, dtype=np.float32)
    if keys.ndim == 1:
        keys = keys[None, :]
    rows = keys.shape[0]
    ld = ld or keys.shape[1]
    n = n or ld
    perm = np.empty((rows, n), np.int32)
    lib().orc_decode_rows(keys, rows, n, ld, perm)
    return perm


def evaluate(pb: OracleProblem, keys, ld=None):
    keys = np.ascontiguousarray(keys, dtype=np.float32)
    rows = keys.shape[0]
    ld = ld or keys.shape[1]
    fit = np.empty((rows, pb.m), np.float32)
    lib().orc_evaluate(C.byref(pb.s), keys, rows, ld, fit)
    return fit[:, 0].copy() if pb.m == 1 else fit


def local_search(pb: OracleProblem, pop, fit, rows, count, ld, moves, seed, gen, island=0):
    """TSPJ random 2-opt on rows[:count] (in place)"""
    lib().orc_local_search(C.byref(pb.s), pop, fit, np.ascontiguousarray(rows, np.int32), count, ld, moves,
                           seed, gen, island)


def continuous_f64(pb: OracleProblem, keys):
    keys = np.ascontiguousarray(np.atleast_2d(keys)[:, :pb.n], dtype=np.float32)
    return np.array([lib().orc_continuous_f64(C.byref(pb.s), np.ascontiguousarray(r)) for r in keys])


def decode_problem(pb: OracleProblem, keys):
    """the problem's own decode of each row (TSPJ: city order, then job order offset by c)"""
    keys = np.ascontiguousarray(np.atleast_2d(keys), dtype=np.float32)
    out = np.zeros((keys.shape[0], pb.n), np.int32)
    for r in range(keys.shape[0]):
        row = np.ascontiguousarray(keys[r, :pb.n])
        p = np.zeros(pb.n, np.int32)
        lib().orc_decode_problem(C.byref(pb.s), row, p)
        out[r] = p
    return out


def eval_f64(pb: OracleProblem, perm):
    out = np.empty(2, np.float64)
    lib().orc_eval_perm_f64(C.byref(pb.s), np.ascontiguousarray(perm, np.int32), out)
    return out[: pb.m]


def sort_fitness(fit, maximize=False):
    fit = np.ascontiguousarray(fit, np.float32)
    out = np.empty(fit.shape[0], np.int32)
    lib().orc_sort_fitness(fit, fit.shape[0], int(bool(maximize)), out)
    return out


def params(P, E, M, rho, seed, island=0):
    return Params(P, E, M, rho, seed, island)


def brkga_init(pb, pr, ld):
    pop = np.zeros((pr.P, ld), np.float32)
    fit = np.zeros(pr.P, np.float32)
    lib().orc_brkga_init(C.byref(pb.s), C.byref(pr), ld, pop, fit)
    return pop, fit


def brkga_generation(pb, pr, g, pop, fit, sorted_idx, ld):
    newpop = np.zeros_like(pop)
    newfit = np.zeros_like(fit)
    lib().orc_brkga_generation(C.byref(pb.s), C.byref(pr), g, pop, fit, np.ascontiguousarray(sorted_idx, np.int32),
                               ld, newpop, newfit)
    return newpop, newfit


def brkga_run(pb, pr, G, ld):
    pop = np.zeros((pr.P, ld), np.float32)
    fit = np.zeros(pr.P, np.float32)
    srt = np.zeros(pr.P, np.int32)
    hist = np.zeros(G + 1, np.float32)
    lib().orc_brkga_run(C.byref(pb.s), C.byref(pr), G, ld, pop, fit, srt, hist)
    return pop, fit, srt, hist


def migrate(k, Pi, m, n, ld, maximize, pop, fit, srt):
    lib().orc_migrate(k, Pi, m, n, ld, int(bool(maximize)), pop, fit, srt)


def pareto_ranks(obj, strict=False):
    """the reference's ranks (default) or textbook ranks (strict=True)"""
    obj = np.ascontiguousarray(obj, np.float32)
    N, m = obj.shape
    r = np.empty(N, np.int32)
    (lib().orc_pareto_ranks_strict if strict else lib().orc_pareto_ranks)(obj, N, m, r)
    return r


def crowding(obj, rank, f64=False, strict=False):
    obj = np.ascontiguousarray(obj, np.float32)
    N, m = obj.shape
    if strict:
        out = np.empty(N, np.float32)
        lib().orc_crowding_strict_f32(obj, np.ascontiguousarray(rank, np.int32), N, m, out)
    elif f64:
        out = np.empty(N, np.float64)
        lib().orc_crowding_f64(obj, np.ascontiguousarray(rank, np.int32), N, m, out)
    else:
        out = np.empty(N, np.float32)
        lib().orc_crowding_f32(obj, np.ascontiguousarray(rank, np.int32), N, m, out)
    return out


def nsga2_select(rank, cd, obj, P):
    rank = np.ascontiguousarray(rank, np.int32)
    obj = np.ascontiguousarray(obj, np.float32)
    sel = np.empty(P, np.int32)
    got = lib().orc_nsga2_select(rank, np.ascontiguousarray(cd, np.float32), obj, rank.shape[0], obj.shape[1], P,
                                 sel)
    return sel[:got]


def nsga2_params(P, Mn, rho, mut_rate, seed, diversity_interval=25):
    return NsgaParams(P, Mn, rho, mut_rate, seed, diversity_interval)


def nsga2_init(pb, pr, ld):
    pop = np.zeros((pr.P, ld), np.float32)
    obj = np.zeros((pr.P, 2), np.float32)
    rank = np.zeros(pr.P, np.int32)
    cd = np.zeros(pr.P, np.float32)
    lib().orc_nsga2_init(C.byref(pb.s), C.byref(pr), ld, pop, obj, rank, cd)
    return pop, obj, rank, cd


def nsga2_generation(pb, pr, g, ld, pop, obj, rank, cd):
    lib().orc_nsga2_generation(C.byref(pb.s), C.byref(pr), g, ld, pop, obj, rank, cd)


def nsga2_offspring(pr, g, n, ld, pop, rank, cd):
    off = np.zeros((pr.P, ld), np.float32)
    lib().orc_nsga2_offspring(C.byref(pr), g, n, ld, pop, np.ascontiguousarray(rank, np.int32),
                              np.ascontiguousarray(cd, np.float32), off)
    return off


# ---------------------------------------------------------------------------------------
# reference harness
# ---------------------------------------------------------------------------------------
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    """Load the reference harness.  The reference must not see a GPU (its CPU path is
    the one pinned and timed), so CUDA_VISIBLE_DEVICES must be empty in this process
    before its first CUDA call."""
    global _ref
    if _ref is None:
        if os.environ.get("CUDA_VISIBLE_DEVICES", None) != "":
            raise RuntimeError("load the reference harness only with CUDA_VISIBLE_DEVICES=''")
        R = C.CDLL(REF_PATH)
        R.ref_tsp_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _f32p, C.c_int, _f32p, C.c_void_p]
        R.ref_knap_eval.argtypes = [_f32p, _f32p, C.c_float, C.c_int, _f32p, C.c_int, _f32p]
        R.ref_bitsp_eval.argtypes = [_f32p, _f32p, C.c_int, _f32p, C.c_int, _f32p]
        R.ref_tspj_eval.argtypes = [_f32p, _f32p, C.c_int, _f32p, C.c_int, _f32p, C.c_void_p]
        R.ref_job_eval.argtypes = [_f32p, C.c_int, C.c_int, _f32p, C.c_int, _f32p]
        R.ref_movrp_eval.argtypes = [_f32p, _i32p, C.c_int, C.c_int, C.c_int, _f32p, C.c_int, _f32p, C.c_void_p]
        R.ref_cont_eval.argtypes = [C.c_int, C.c_float, C.c_float, C.c_int, _f32p, C.c_int, _f32p]
        R.ref_pareto.argtypes = [_f32p, C.c_int, _i32p, _f32p]
        R.ref_nsga2_select.argtypes = [_f32p, C.c_int, C.c_int, _i32p]
        R.ref_solver_create_wct.restype = C.c_void_p
        R.ref_solver_create_wct.argtypes = [C.c_int, C.c_uint, C.c_int, C.c_int, C.c_int, C.c_double]
        R.ref_brkga_generation.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint32,
                                           _f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _u8p, _f32p]
        R.ref_nsga2_offspring.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_double, C.c_uint32, _f32p, _i32p,
                                          _f32p, _f32p, _i32p, _u8p, _u8p, _f32p]
        R.ref_generation_seconds.restype = C.c_double
        R.ref_generation_seconds.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint32,
                                             _f32p, _f32p]
        R.ref_population_sort_seconds.restype = C.c_double
        R.ref_population_sort_seconds.argtypes = [_f32p, C.c_int, C.c_int, C.c_int]
        R.ref_solver_create.restype = C.c_void_p
        R.ref_solver_create_movrp.restype = C.c_void_p
        R.ref_solver_create_movrp.argtypes = [_f32p, _i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        R.ref_solver_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_float, C.c_int, C.c_int, C.c_int, C.c_double]
        R.ref_solver_mode.restype = C.c_char_p
        R.ref_solver_mode.argtypes = [C.c_void_p]
        R.ref_solver_evolve.restype = C.c_double
        R.ref_solver_evolve.argtypes = [C.c_void_p, C.c_int]
        R.ref_solver_best.restype = C.c_double
        R.ref_solver_best.argtypes = [C.c_void_p]
        R.ref_solver_destroy.argtypes = [C.c_void_p]
        _ref = R
    return _ref


def coords_matrix(xy):
    """The reference's float distance matrix from coordinates (configs/tsp_config.hpp:359-371)."""
    xy = np.asarray(xy, np.float32)
    dx = xy[:, None, 0] - xy[None, :, 0]
    dy = xy[:, None, 1] - xy[None, :, 1]
    return np.sqrt(dx * dx + dy * dy).astype(np.float32)


def movrp_values(keys):
    """MultiObjectiveVRPConfig's biased sort values of one chromosome"""
    keys = np.ascontiguousarray(keys, dtype=np.float32)
    out = np.empty_like(keys)
    lib().orc_movrp_values(keys, keys.shape[0], out)
    return out


def movrp_routes(pb: OracleProblem, perm):
    """route index of each sorted position, and the route count"""
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    route_of = np.zeros(pb.n, np.int32)
    count = lib().orc_movrp_routes(C.byref(pb.s), perm, route_of)
    return route_of, count
