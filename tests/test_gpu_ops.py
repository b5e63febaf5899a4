"""Operator parity on the GPU: every kernel through the C ABI against the CPU oracle on
the same seeded inputs.  Integer and index results (permutations, ranks, elite orders,
knapsack fitness, children's keys) must be bit-exact; FP32 tour lengths are compared bit
for bit with the oracle's canonical FP32 order and within 1e-5 relative of FP64."""
import numpy as np
import pytest

import instances as I
import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL_F64 = 1e-5  # FP32 tour length vs the FP64 restatement


def B():
    import brkga_b200
    return brkga_b200


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def eval_gpu(pb, keys, cuda, ld=None):
    import torch
    rows, width = keys.shape
    n = pb.n
    d_keys = dev(keys, cuda)
    d_fit = torch.zeros(rows * pb.num_objectives, dtype=torch.float32, device=cuda)
    d_perm = torch.zeros(rows * n, dtype=torch.int32, device=cuda)
    pb.evaluate_population(d_keys, d_fit, rows, n, ld=ld or width, d_perm=d_perm)
    fit = host(d_fit).reshape(rows, pb.num_objectives)
    return (fit[:, 0] if pb.num_objectives == 1 else fit), host(d_perm).reshape(rows, n)


def check_tsp(pb_gpu, pb_orc, keys, cuda, ld=None):
    fit, perm = eval_gpu(pb_gpu, keys, cuda, ld)
    n = pb_gpu.n
    kk = keys[:, :n]
    ref_perm = O.decode(kk)
    np.testing.assert_array_equal(perm, ref_perm)
    ref_fit = O.evaluate(pb_orc, kk)
    np.testing.assert_array_equal(fit.view(np.uint32), ref_fit.view(np.uint32))
    for r in range(min(8, keys.shape[0])):
        f64 = O.eval_f64(pb_orc, ref_perm[r])
        rel = np.abs(np.atleast_1d(fit[r]).astype(np.float64) - f64) / np.maximum(np.abs(f64), 1e-30)
        assert rel.max() <= REL_TOL_F64, (r, rel)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 31, 52, 100, 128, 129, 257, 1000, 1001, 2048, 4096, 5000, 8192])
def test_tsp_decode_fitness(cuda, n):
    xy = I.tsp_coords(n, seed=n)
    rows = 64 if n <= 2048 else 16
    keys = I.keys(rows, n, seed=100 + n)
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda)


@pytest.mark.parametrize("n", [5, 52, 1000])
def test_tsp_ties_and_wild_keys(cuda, n):
    xy = I.tsp_coords(n, seed=7)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    check_tsp(pb, po, I.tied_keys(32, n, seed=1), cuda)
    check_tsp(pb, po, I.tied_keys(8, n, seed=2, levels=1), cuda)  # every key equal
    check_tsp(pb, po, I.wild_keys(32, n, seed=3), cuda)


@pytest.mark.parametrize("n", [7, 1000, 5000, 12000])
def test_decode_degenerate_keys(cuda, n):
    """keys that crowd the value-range buckets (all equal, outside [0,1), NaN-heavy, few tie
    levels) take the bounded fallback sort; the order is still (key, index)"""
    xy = I.tsp_coords(n, seed=3)
    keys = I.degenerate_keys(n, seed=n)
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda)
    w, v, cap = I.knap_items(n, seed=4)
    fit, perm = eval_gpu(B().knapsack(w, v, cap, greedy=True), keys, cuda)
    np.testing.assert_array_equal(perm, O.decode(keys))
    np.testing.assert_array_equal(fit, O.evaluate(O.OracleProblem(O.KNAP_GREEDY, n, w=w, v=v, cap=cap), keys))


@pytest.mark.parametrize("c", [3, 500, 2000])
def test_tspj_degenerate_keys(cuda, c):
    """two key segments (cities, jobs) with crowded buckets: each segment sorted on its own"""
    travel, jobs = I.tspj_instance(c, seed=c)
    keys = I.degenerate_keys(2 * c, seed=c + 1)
    po = O.OracleProblem(O.TSPJ, 2 * c, mat=travel, mat2=jobs)
    fit, perm = eval_gpu(B().tspj(travel, jobs), keys, cuda)
    np.testing.assert_array_equal(perm, O.decode_problem(po, keys))
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


@pytest.mark.parametrize("n", [3, 53, 999])
def test_tsp_unaligned_dense_rows(cuda, n):
    # the reference's dense [pop][chrom_len] layout: rows not 16-byte aligned
    xy = I.tsp_coords(n, seed=11)
    keys = I.keys(40, n, seed=12)
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda, ld=n)


@pytest.mark.parametrize("n", [1, 5, 52, 300])
def test_tsp_matrix(cuda, n):
    xy = I.tsp_coords(n, seed=21, scale=1000.0)
    mat = O.coords_matrix(xy)
    mat[0, n - 1] += 1.0  # asymmetric entry: orientation matters
    keys = I.keys(32, n, seed=22)
    check_tsp(B().tsp_matrix(mat), O.OracleProblem(O.TSP_MATRIX, n, mat=mat), keys, cuda)


@pytest.mark.parametrize("n", [1, 10, 300, 500])
def test_bitsp(cuda, n):
    a, b = I.tsp_coords(n + 1, seed=31), I.tsp_coords(n + 1, seed=32)
    keys = I.keys(48, n, seed=33)
    check_tsp(B().bitsp(a, b), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=b), keys, cuda)
    ma, mb = O.coords_matrix(a), O.coords_matrix(b)
    check_tsp(B().bitsp_matrix(ma, mb), O.OracleProblem(O.BITSP_MATRIX, n, mat=ma, mat2=mb), keys, cuda)


@pytest.mark.parametrize("n", [1, 10, 500, 5000, 10000])
@pytest.mark.parametrize("greedy", [False, True])
def test_knapsack(cuda, n, greedy):
    w, v, cap = I.knap_items(n, seed=n)
    pb = B().knapsack(w, v, cap, greedy=greedy)
    po = O.OracleProblem(O.KNAP_GREEDY if greedy else O.KNAP_THRESHOLD, n, w=w, v=v, cap=cap)
    keys = I.keys(32 if n <= 5000 else 8, n, seed=41)
    fit, _ = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


def test_knapsack_greedy_zero_weights_and_tiny_capacity(cuda):
    n = 700
    w, v, _ = I.knap_items(n, seed=5)
    w[::7] = 0
    for cap in (0.0, 3.5, 120.0):
        pb = B().knapsack(w, v, cap, greedy=True)
        po = O.OracleProblem(O.KNAP_GREEDY, n, w=w, v=v, cap=cap)
        keys = I.keys(16, n, seed=6)
        fit, _ = eval_gpu(pb, keys, cuda)
        np.testing.assert_array_equal(fit, O.evaluate(po, keys))


@pytest.mark.parametrize("P", [1, 2, 3, 100, 256, 2048, 4096, 16384])
@pytest.mark.parametrize("maximize", [False, True])
def test_sort_fitness(cuda, P, maximize):
    import torch
    rng = np.random.default_rng(P)
    segs = 3
    fit = rng.random(P * segs, dtype=np.float32)
    fit[::5] = np.round(fit[::5] * 4) / 4  # ties
    d_sorted = torch.zeros(P * segs, dtype=torch.int32, device=cuda)
    B().sort_fitness(dev(fit, cuda), P, segs, maximize, d_sorted)
    got = host(d_sorted).reshape(segs, P)
    for s in range(segs):
        np.testing.assert_array_equal(got[s], O.sort_fitness(fit[s * P:(s + 1) * P], maximize))


def run_gen(cuda, pb, po, P, E, M, rho, seed, g, island=0):
    import torch
    n = pb.n
    ld = (n + 3) // 4 * 4
    pr = O.params(P, E, M, rho, seed, island)
    pop, fit = O.brkga_init(po, pr, ld)
    srt = O.sort_fitness(fit, po.maximize)
    ref_pop, ref_fit = O.brkga_generation(po, pr, g, pop, fit, srt, ld)
    d_next = torch.zeros(P * ld, dtype=torch.float32, device=cuda)
    d_nfit = torch.zeros(P, dtype=torch.float32, device=cuda)
    B().generation_step(pb, dev(pop, cuda), dev(fit, cuda), dev(srt, cuda), d_next, d_nfit, P, E, M, rho, ld,
                        seed, g, island)
    np.testing.assert_array_equal(host(d_next).reshape(P, ld), ref_pop)
    np.testing.assert_array_equal(host(d_nfit).view(np.uint32), ref_fit.view(np.uint32))


@pytest.mark.parametrize("n,P,E,M", [(52, 256, 51, 25), (1000, 2048, 307, 307), (7, 10, 1, 0), (13, 9, 3, 6)])
def test_generation_step(cuda, n, P, E, M):
    xy = I.tsp_coords(n, seed=1)
    run_gen(cuda, B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), P, E, M, 0.7, 1234, 5, island=2)


def test_generation_step_knapsack(cuda):
    n = 600
    w, v, cap = I.knap_items(n, seed=3)
    run_gen(cuda, B().knapsack(w, v, cap), O.OracleProblem(O.KNAP_GREEDY, n, w=w, v=v, cap=cap), 128, 20, 20, 0.7,
            99, 3)


@pytest.mark.parametrize("rho", [0.0, 1.0])
def test_generation_step_extreme_rho(cuda, rho):
    n = 40
    xy = I.tsp_coords(n, seed=4)
    run_gen(cuda, B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), 64, 10, 6, rho, 5, 1)


def test_init_population(cuda):
    import torch
    n, P = 77, 100
    ld = 80
    xy = I.tsp_coords(n, seed=9)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    d_pop = torch.zeros(P * ld, dtype=torch.float32, device=cuda)
    d_fit = torch.zeros(P, dtype=torch.float32, device=cuda)
    B().init_population(pb, d_pop, d_fit, P, ld, 42, 1)
    ref_pop, ref_fit = O.brkga_init(po, O.params(P, 1, 0, 0.7, 42, 1), ld)
    np.testing.assert_array_equal(host(d_pop).reshape(P, ld), ref_pop)
    np.testing.assert_array_equal(host(d_fit), ref_fit)


def pareto_points(N, seed, dup=False):
    rng = np.random.default_rng(seed)
    obj = rng.random((N, 2), dtype=np.float32)
    if dup:
        obj = np.round(obj * 16) / 16  # ties and exact duplicates
        obj = obj.astype(np.float32)
    return obj


@pytest.mark.parametrize("N", [1, 2, 3, 100, 1000, 4096, 8192])
@pytest.mark.parametrize("dup", [False, True])
def test_pareto_rank_and_crowding(cuda, N, dup):
    import torch
    obj = pareto_points(N, seed=N, dup=dup)
    d_obj = dev(obj, cuda)
    d_rank = torch.zeros(N, dtype=torch.int32, device=cuda)
    B().pareto_rank(d_obj, N, 2, d_rank)
    ref_rank = O.pareto_ranks(obj)
    np.testing.assert_array_equal(host(d_rank), ref_rank)
    d_rank2 = torch.zeros(N, dtype=torch.int32, device=cuda)
    B().pareto_rank(d_obj, N, 2, d_rank2, bitmatrix=True)
    np.testing.assert_array_equal(host(d_rank2), ref_rank)
    if N > 4096:
        return  # the crowding kernel's limit; ranks above are still checked
    d_cd = torch.zeros(N, dtype=torch.float32, device=cuda)
    B().crowding(d_obj, dev(ref_rank, cuda), N, 2, d_cd)
    np.testing.assert_array_equal(host(d_cd).view(np.uint32), O.crowding(obj, ref_rank).view(np.uint32))
    cd64 = O.crowding(obj, ref_rank, f64=True)
    fin = np.isfinite(cd64)
    got = host(d_cd)
    assert np.array_equal(np.isfinite(got), fin)
    assert np.all(np.abs(got[fin] - cd64[fin]) <= 1e-5 * np.maximum(1.0, np.abs(cd64[fin])))


@pytest.mark.parametrize("m", [1, 3])
def test_pareto_rank_bitmatrix_any_m(cuda, m):
    import torch
    rng = np.random.default_rng(m)
    N = 700
    obj = (np.round(rng.random((N, m)) * 10) / 10).astype(np.float32)
    d_rank = torch.zeros(N, dtype=torch.int32, device=cuda)
    B().pareto_rank(dev(obj, cuda), N, m, d_rank)
    np.testing.assert_array_equal(host(d_rank), O.pareto_ranks(obj))
