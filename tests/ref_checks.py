"""Cases that run the reference's own code (oracle/_ref/libref.so) and the comparisons
that pin the oracle to it.  Every function here must run in a process with
CUDA_VISIBLE_DEVICES="" (the reference then takes its CPU path); tests call them
through ``python tests/ref_checks.py <check>`` in a child process.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(os.path.dirname(HERE), "oracle"), HERE]

import instances as I  # noqa: E402
import oracle as O  # noqa: E402


# ---------------------------------------------------------------------------------------
# reference runs
# ---------------------------------------------------------------------------------------
def ref_tsp_case(n, rows, seed, scale=1.0, key_fn=None):
    R = O.ref()
    xy = I.tsp_coords(n, seed, scale)
    keys = (key_fn or I.keys)(rows, n, seed + 1)
    fit = np.zeros(rows, np.float32)
    perm = np.zeros((rows, n), np.int32)
    assert R.ref_tsp_eval(xy.ctypes.data, None, n, keys, rows, fit, perm.ctypes.data) == 0
    return dict(xy=xy, keys=keys, fit=fit, perm=perm)


def ref_tsp_matrix_case(n, rows, seed):
    R = O.ref()
    rng = np.random.default_rng(seed)
    mat = (rng.random((n, n)) * 100).astype(np.float32)
    np.fill_diagonal(mat, 0)
    keys = I.keys(rows, n, seed + 1)
    fit = np.zeros(rows, np.float32)
    perm = np.zeros((rows, n), np.int32)
    assert R.ref_tsp_eval(None, mat.ctypes.data, n, keys, rows, fit, perm.ctypes.data) == 0
    return dict(mat=mat, keys=keys, fit=fit, perm=perm)


def ref_knap_case(n, rows, seed):
    R = O.ref()
    w, v, cap = I.knap_items(n, seed)
    keys = I.keys(rows, n, seed + 1)
    keys[0, :] = 0.9  # everything selected: over capacity, penalty path
    keys[1, :] = 0.5  # nothing selected (strictly greater than 0.5)
    fit = np.zeros(rows, np.float32)
    assert R.ref_knap_eval(w.astype(np.float32), v.astype(np.float32), float(cap), n, keys, rows, fit) == 0
    return dict(w=w, v=v, cap=np.float32(cap), keys=keys, fit=fit)


def ref_bitsp_case(n, rows, seed):
    R = O.ref()
    a, b = I.tsp_coords(n + 1, seed), I.tsp_coords(n + 1, seed + 1)
    ma, mb = O.coords_matrix(a), O.coords_matrix(b)
    keys = I.keys(rows, n, seed + 2)
    obj = np.zeros((rows, 2), np.float32)
    assert R.ref_bitsp_eval(ma, mb, n + 1, keys, rows, obj) == 0
    return dict(xy=a, xy2=b, keys=keys, obj=obj)


def pareto_points(N, seed, dup):
    rng = np.random.default_rng(seed)
    obj = rng.random((N, 2), dtype=np.float32)
    if dup:
        obj = (np.round(obj * 12) / 12).astype(np.float32)
    return np.ascontiguousarray(obj)


def ref_pareto_case(N, seed, dup):
    R = O.ref()
    obj = pareto_points(N, seed, dup)
    rank = np.zeros(N, np.int32)
    cd = np.zeros(N, np.float32)
    assert R.ref_pareto(obj, N, rank, cd) == 0
    return dict(obj=obj, rank=rank, cd=cd)


def ref_select_case(N, P, seed):
    R = O.ref()
    obj = pareto_points(N, seed, False)
    sel = np.zeros(P, np.int32)
    assert R.ref_nsga2_select(obj, N, P, sel) == P
    return dict(obj=obj, sel=sel, P=np.int32(P))


def ref_generation_case(n, P, E, M, rho, seed):
    """one reference generation from a sorted population, plus the draws it consumed"""
    R = O.ref()
    xy = I.tsp_coords(n, seed)
    keys = I.keys(P, n, seed + 1)
    pb = O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    fit = np.array([O.lib().orc_tsp_len_seq(O.C.byref(pb.s), p) for p in O.decode(keys)], np.float32)
    order = np.argsort(fit, kind="stable")
    keys, fit = np.ascontiguousarray(keys[order]), np.ascontiguousarray(fit[order])
    off = P - E - M
    out_keys = np.zeros((P, n), np.float32)
    out_fit = np.zeros(P, np.float32)
    ep = np.zeros(max(off, 1), np.int32)
    npar = np.zeros(max(off, 1), np.int32)
    coin = np.zeros((max(off, 1), n), np.uint8)
    mut = np.zeros((max(M, 1), n), np.float32)
    assert R.ref_brkga_generation(xy, n, P, E, M, rho, seed, keys, fit, out_keys, out_fit, ep, npar, coin, mut) == 0
    return dict(xy=xy, keys=keys, fit=fit, out_keys=out_keys, out_fit=out_fit, ep=ep, np=npar, coin=coin, mut=mut,
                shape=np.array([n, P, E, M], np.int32), rho=np.float64(rho))


def ref_nsga_offspring_case(n, P, rho, seed):
    R = O.ref()
    a, b = I.tsp_coords(n + 1, seed), I.tsp_coords(n + 1, seed + 1)
    ma, mb = O.coords_matrix(a), O.coords_matrix(b)
    keys = I.keys(P, n, seed + 2)
    rng = np.random.default_rng(seed + 3)
    rank = rng.integers(0, 4, P).astype(np.int32)
    cd = rng.random(P, dtype=np.float32)
    cd[::5] = np.inf
    out = np.zeros((P, n), np.float32)
    picks = np.zeros((P, 4), np.int32)
    coin = np.zeros((P, n), np.uint8)
    mflag = np.zeros((P, n), np.uint8)
    mkey = np.zeros((P, n), np.float32)
    assert R.ref_nsga2_offspring(ma, mb, n + 1, P, rho, seed, keys, rank, cd, out, picks, coin, mflag, mkey) == 0
    return dict(keys=keys, rank=rank, cd=cd, out=out, picks=picks, coin=coin, mflag=mflag, mkey=mkey,
                shape=np.array([n, P], np.int32))


# ---------------------------------------------------------------------------------------
# comparisons of the oracle with a reference case (used on golden files and live)
# ---------------------------------------------------------------------------------------
def check_tsp(d, matrix=False):
    n = d["keys"].shape[1]
    pb = O.OracleProblem(O.TSP_MATRIX, n, mat=d["mat"]) if matrix else O.OracleProblem(O.TSP_COORDS, n, xy=d["xy"])
    perm = O.decode(d["keys"])
    np.testing.assert_array_equal(perm, d["perm"])
    seq = np.array([O.lib().orc_tsp_len_seq(O.C.byref(pb.s), p) for p in perm], np.float32)
    np.testing.assert_array_equal(seq, d["fit"])  # the reference's own FP32 order, bit for bit
    canon = O.evaluate(pb, d["keys"])
    den = np.maximum(np.abs(d["fit"]), 1e-30)
    assert np.max(np.abs(canon - d["fit"]) / den) <= 1e-5
    f64 = np.array([O.eval_f64(pb, p)[0] for p in perm])
    assert np.max(np.abs(f64 - d["fit"]) / np.maximum(f64, 1e-30)) <= 1e-5


def check_knap(d):
    n = d["keys"].shape[1]
    pb = O.OracleProblem(O.KNAP_THRESHOLD, n, w=d["w"], v=d["v"], cap=float(d["cap"]))
    np.testing.assert_array_equal(O.evaluate(pb, d["keys"]), d["fit"])


def check_bitsp(d):
    n = d["keys"].shape[1]
    pb = O.OracleProblem(O.BITSP_COORDS, n, xy=d["xy"], xy2=d["xy2"])
    got = O.evaluate(pb, d["keys"])
    assert np.max(np.abs(got - d["obj"]) / d["obj"]) <= 1e-5
    for r, p in enumerate(O.decode(d["keys"])):
        f64 = O.eval_f64(pb, p)
        assert np.max(np.abs(f64 - d["obj"][r]) / f64) <= 1e-5


def ref_tspj_case(c, rows, seed, key_fn=None):
    R = O.ref()
    travel, jobs = I.tspj_instance(c, seed)
    keys = (key_fn or I.keys)(rows, 2 * c, seed + 1)
    fit = np.zeros(rows, np.float32)
    perm = np.zeros((rows, 2 * c), np.int32)
    assert R.ref_tspj_eval(travel, jobs, c + 1, keys, rows, fit, perm.ctypes.data) == 0
    return dict(travel=travel, jobs=jobs, keys=keys, fit=fit, perm=perm)


def check_tspj(d):
    # the reference sums in sequence and so does the oracle: bit-exact makespans
    c = d["keys"].shape[1] // 2
    pb = O.OracleProblem(O.TSPJ, 2 * c, mat=d["travel"], mat2=d["jobs"])
    perm = O.decode_problem(pb, d["keys"])
    ref = d["perm"].copy()
    ref[:, :c] -= 1       # reference cities 1..c -> key indices 0..c-1
    ref[:, c:] += c - 1   # reference job types 1..c -> key indices c..2c-1
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(O.evaluate(pb, d["keys"]).view(np.uint32), d["fit"].view(np.uint32))
    f64 = np.array([O.eval_f64(pb, p)[0] for p in perm])
    assert np.max(np.abs(f64 - d["fit"]) / np.maximum(f64, 1e-30)) <= 1e-5


def ref_job_case(n, machines, rows, seed):
    R = O.ref()
    rng = np.random.default_rng(seed)
    jt = (1.0 + rng.random(n) * 99.0).astype(np.float32)
    keys = I.keys(rows, n, seed + 1)
    fit = np.zeros(rows, np.float32)
    assert R.ref_job_eval(jt, n, machines, keys, rows, fit) == 0
    return dict(jt=jt, machines=np.int32(machines), keys=keys, fit=fit)


def check_job(d):
    n = d["keys"].shape[1]
    pb = O.OracleProblem(O.JOBSCHED, n, jt=d["jt"], machines=int(d["machines"]))
    np.testing.assert_array_equal(O.evaluate(pb, d["keys"]).view(np.uint32), d["fit"].view(np.uint32))


def ref_movrp_case(n, rows, seed, vehicles=None, overload=False, key_fn=None):
    R = O.ref()
    xy, dem, cap, V = I.movrp_instance(n, seed, vehicles, overload)
    keys = (key_fn or I.keys)(rows, n, seed + 1)
    obj = np.zeros((rows, 2), np.float32)
    perm = np.zeros((rows, n), np.int32)
    assert R.ref_movrp_eval(xy, dem, n, cap, V, keys, rows, obj, perm.ctypes.data) == 0
    return dict(xy=xy, dem=dem, cap=np.int32(cap), vehicles=np.int32(V), keys=keys, obj=obj, perm=perm)


def movrp_problem(d):
    n = d["keys"].shape[1]
    return O.OracleProblem(O.MOVRP, n, xy=d["xy"], w=d["dem"], machines=int(d["vehicles"]), vcap=int(d["cap"]))


def check_movrp(d):
    pb = movrp_problem(d)
    np.testing.assert_array_equal(O.decode_problem(pb, d["keys"]) + 1, d["perm"])
    np.testing.assert_array_equal(O.evaluate(pb, d["keys"]).view(np.uint32), d["obj"].view(np.uint32))


CONT_BOUNDS = {0: (-5.12, 5.12), 1: (-5.12, 5.12), 2: (-5.0, 10.0)}  # create_sphere/_rastrigin/_rosenbrock


def ref_cont_case(function, n, rows, seed):
    R = O.ref()
    lo, hi = CONT_BOUNDS[function]
    keys = I.keys(rows, n, seed)
    fit = np.zeros(rows, np.float32)
    assert R.ref_cont_eval(function, lo, hi, n, keys, rows, fit) == 0
    return dict(function=np.int32(function), lo=np.float32(lo), hi=np.float32(hi), keys=keys, fit=fit)


def check_cont(d):
    n = d["keys"].shape[1]
    pb = O.OracleProblem(O.CONTINUOUS, n, function=int(d["function"]), lo=float(d["lo"]), hi=float(d["hi"]))
    # the oracle adds in the reference's order with the same libm: bit-exact
    np.testing.assert_array_equal(O.evaluate(pb, d["keys"]).view(np.uint32), d["fit"].view(np.uint32))


def check_pareto(d, crowd=True):
    rank = O.pareto_ranks(d["obj"])
    np.testing.assert_array_equal(rank, d["rank"])
    if crowd:
        cd = O.crowding(d["obj"], rank)
        fin = np.isfinite(d["cd"])
        np.testing.assert_array_equal(np.isfinite(cd), fin)
        # with no ties in either objective the reference's order is the oracle's order
        if len(np.unique(d["obj"][:, 0])) == len(d["obj"]) and len(np.unique(d["obj"][:, 1])) == len(d["obj"]):
            np.testing.assert_array_equal(cd, d["cd"])
        assert np.all(np.abs(cd[fin] - d["cd"][fin]) <= 1e-5 * np.maximum(1, np.abs(d["cd"][fin])))


def check_select(d):
    obj, P = d["obj"], int(d["P"])
    rank = O.pareto_ranks(obj)
    cd = O.crowding(obj, rank)
    sel = O.nsga2_select(rank, cd, obj, P)
    assert sorted(sel.tolist()) == sorted(d["sel"].tolist())


def check_generation(d):
    n, P, E, M = (int(x) for x in d["shape"])
    pb = O.OracleProblem(O.TSP_COORDS, n, xy=d["xy"])
    srt = np.arange(P, dtype=np.int32)  # the input is given in rank order
    newpop = np.zeros((P, n), np.float32)
    newfit = np.zeros(P, np.float32)
    off = P - E - M
    O.lib().orc_generation_core(P, E, M, n, n, d["keys"], d["fit"], srt, d["ep"][:max(off, 1)],
                                d["np"][:max(off, 1)], np.ascontiguousarray(d["coin"]),
                                np.ascontiguousarray(d["mut"]), newpop, newfit)
    seq = np.array([O.lib().orc_tsp_len_seq(O.C.byref(pb.s), p) for p in O.decode(newpop)], np.float32)
    seq[:E] = newfit[:E]
    order = np.argsort(seq, kind="stable")
    np.testing.assert_array_equal(newpop[order], d["out_keys"])
    np.testing.assert_array_equal(seq[order], d["out_fit"])


def check_nsga_offspring(d):
    n, P = (int(x) for x in d["shape"])
    out = np.zeros((P, n), np.float32)
    O.lib().orc_nsga2_offspring_core(P, n, n, d["keys"], d["rank"], d["cd"], np.ascontiguousarray(d["picks"]),
                                     np.ascontiguousarray(d["coin"]), np.ascontiguousarray(d["mflag"]),
                                     np.ascontiguousarray(d["mkey"]), out)
    np.testing.assert_array_equal(out, d["out"])


LIVE = {
    "tsp": lambda: [check_tsp(ref_tsp_case(n, 8, 10 + n)) for n in (1, 2, 5, 52, 129, 1000)],
    "tsp_ties": lambda: [check_tsp(ref_tsp_case(n, 8, 20 + n, key_fn=I.tied_keys)) for n in (5, 60, 500)],
    "tsp_wild": lambda: [check_tsp(ref_tsp_case(n, 8, 30 + n, key_fn=I.wild_keys)) for n in (7, 300)],
    "tsp_matrix": lambda: check_tsp(ref_tsp_matrix_case(40, 8, 3), matrix=True),
    "knap": lambda: [check_knap(ref_knap_case(n, 8, n)) for n in (1, 50, 5000)],
    "bitsp": lambda: [check_bitsp(ref_bitsp_case(n, 8, n)) for n in (1, 20, 300)],
    "tspj": lambda: [check_tspj(ref_tspj_case(c, 8, 40 + c)) for c in (1, 2, 5, 52, 300)],
    "tspj_ties": lambda: [check_tspj(ref_tspj_case(c, 8, 50 + c, key_fn=I.tied_keys)) for c in (6, 100)],
    "jobsched": lambda: [check_job(ref_job_case(n, M, 8, n + M)) for (n, M) in ((1, 1), (50, 5), (300, 32), (1000, 70))],
    "continuous": lambda: [check_cont(ref_cont_case(f, n, 8, 7 * f + n)) for f in (0, 1, 2) for n in (1, 2, 30, 500)],
    "movrp": lambda: [check_movrp(ref_movrp_case(n, 8, 60 + n, V, ov))
                      for (n, V, ov) in ((1, None, False), (2, 1, False), (31, 5, False), (31, 2, False),
                                         (100, None, True), (1000, None, False))],
    "movrp_ties": lambda: [check_movrp(ref_movrp_case(n, 8, 70 + n, key_fn=I.tied_keys)) for n in (8, 200)],
    "pareto": lambda: [check_pareto(ref_pareto_case(N, N, False)) for N in (1, 2, 3, 500, 4096)],
    "pareto_dup": lambda: [check_pareto(ref_pareto_case(N, N, True), crowd=False) for N in (64, 2048)],
    "select": lambda: [check_select(ref_select_case(N, N // 2, N)) for N in (40, 1000)],
    "generation": lambda: [check_generation(ref_generation_case(n, P, E, M, 0.7, s))
                           for (n, P, E, M, s) in ((52, 256, 51, 25, 1), (10, 30, 6, 0, 2), (33, 64, 1, 63, 3),
                                                   (200, 500, 75, 75, 4))],
    "nsga_offspring": lambda: [check_nsga_offspring(ref_nsga_offspring_case(n, P, 0.7, s))
                               for (n, P, s) in ((15, 24, 1), (100, 64, 2), (1, 8, 3))],
}

if __name__ == "__main__":
    assert os.environ.get("CUDA_VISIBLE_DEVICES") == "", "run with CUDA_VISIBLE_DEVICES="
    LIVE[sys.argv[1]]()
    print("ok", sys.argv[1])
