"""Chromosomes longer than the shared-memory row kernel takes (a row's counters,
composites and permutation above 227 KB: n above about 13,900 genes with coordinates).
Those rows are decoded by the kernel that keeps its sort scratch in global memory; its
permutations, fitness values and children must equal the oracle's bit for bit, like
the shared-memory kernel's, and it must take over exactly where the other stops fitting."""
import numpy as np
import pytest

import instances as I
import oracle as O
from test_gpu_engine import oracle_islands
from test_gpu_ops import B, check_tsp, dev, eval_gpu, host, run_gen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [13000, 14500, 20000, 65537])
def test_tsp_decode_fitness_large(cuda, n):
    # 13000 still fits in shared memory; the others take the global-memory kernel
    xy = I.tsp_coords(n, seed=n)
    keys = I.keys(6, n, seed=n + 1)
    keys[0, ::7] = keys[0, 3]  # ties broken by index
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda)


@pytest.mark.parametrize("n", [20000, 65537])
def test_decode_degenerate_keys_large(cuda, n):
    """the global-memory kernel's fallback sort on keys that crowd its buckets"""
    xy = I.tsp_coords(n, seed=5)
    keys = I.degenerate_keys(n, seed=n)
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda)


def test_tspj_degenerate_keys_large(cuda):
    """two key segments of 8200 cities and jobs (beyond shared memory) with crowded buckets;
    travel and job times are plain uniform tables, 8201 x 8201 each"""
    c = 8200
    rng = np.random.default_rng(7)
    travel = rng.random((c + 1, c + 1), dtype=np.float32) * np.float32(100.0)
    jobs = rng.random((c + 1, c + 1), dtype=np.float32) * np.float32(100.0)
    keys = I.degenerate_keys(2 * c, seed=8)[[0, 3, 6, 8, 9]]
    po = O.OracleProblem(O.TSPJ, 2 * c, mat=travel, mat2=jobs)
    fit, perm = eval_gpu(B().tspj(travel, jobs), keys, cuda)
    np.testing.assert_array_equal(perm, O.decode_problem(po, keys))
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


def test_tsp_unaligned_rows_large(cuda):
    n, ld = 20001, 20003  # odd stride: scalar loads of the given keys
    xy = I.tsp_coords(n, seed=3)
    keys = np.zeros((4, ld), np.float32)
    keys[:, :n] = I.keys(4, n, seed=4)
    check_tsp(B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), keys, cuda, ld=ld)


@pytest.mark.parametrize("greedy", [True, False])
def test_knapsack_large(cuda, greedy):
    n = 30000
    w, v, cap = I.knap_items(n, seed=5)
    pb = B().knapsack(w, v, cap, greedy=greedy)
    po = O.OracleProblem(O.KNAP_GREEDY if greedy else O.KNAP_THRESHOLD, n, w=w, v=v, cap=cap)
    keys = I.keys(5, n, seed=6)
    fit, perm = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(fit, O.evaluate(po, keys))
    if greedy:
        np.testing.assert_array_equal(perm, O.decode(keys))


def test_bitsp_large(cuda):
    n = 16000
    a, c = I.tsp_coords(n + 1, seed=7), I.tsp_coords(n + 1, seed=8)
    pb, po = B().bitsp(a, c), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=c)
    keys = I.keys(3, n, seed=9)
    fit, perm = eval_gpu(pb, keys, cuda)
    np.testing.assert_array_equal(perm, O.decode(keys))
    np.testing.assert_array_equal(fit.view(np.uint32), O.evaluate(po, keys).view(np.uint32))


def test_generation_step_large(cuda):
    n = 18000
    xy = I.tsp_coords(n, seed=10)
    run_gen(cuda, B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy), 24, 5, 3, 0.7, 77, 4)


def test_engine_large_bit_exact(cuda):
    n, P, E, M, G = 15000, 24, 5, 3, 3
    xy = I.tsp_coords(n, seed=11)
    pb, po = B().tsp(xy), O.OracleProblem(O.TSP_COORDS, n, xy=xy)
    s = B().Solver(pb, B().params(P, E, M, 0.7, G, seed=13))
    assert s.info[0] == 0  # the global-memory row kernel
    s.run()
    keys, fit = s.get_population()
    rk, rf, rh = oracle_islands(po, P, E, M, 0.7, 13, 1, 0, 0, G, (n + 3) // 4 * 4)
    np.testing.assert_array_equal(keys, rk)
    np.testing.assert_array_equal(fit, rf)
    np.testing.assert_array_equal(s.get_fitness_history(), rh)
    bk, bp, bf = s.get_best_individual()
    np.testing.assert_array_equal(bp, O.decode(rk[0])[0])
    s.close()


def test_engine_nsga2_large_bit_exact(cuda):
    n, P, G = 14000, 16, 3
    a, c = I.tsp_coords(n + 1, seed=12), I.tsp_coords(n + 1, seed=13)
    pb, po = B().bitsp(a, c), O.OracleProblem(O.BITSP_COORDS, n, xy=a, xy2=c)
    s = B().Solver(pb, B().params(P, 0, 2, 0.7, G, seed=21, diversity_interval=25))
    s.initialize()
    ld = (n + 3) // 4 * 4
    pr = O.nsga2_params(P, 2, 0.7, 5.0 / n, 21, 25)
    pop, obj, rank, cd = O.nsga2_init(po, pr, ld)
    for g in range(1, G + 1):
        s.evolve(1)
        O.nsga2_generation(po, pr, g, ld, pop, obj, rank, cd)
        gk, go = s.get_population()
        np.testing.assert_array_equal(gk, pop[:, :n], err_msg=f"generation {g}")
        np.testing.assert_array_equal(go, obj, err_msg=f"generation {g}")
    s.close()


def test_batch_rejects_rows_beyond_shared_memory(cuda):
    n = 20000
    pb = B().tsp(I.tsp_coords(n, seed=14))
    with pytest.raises(B().BrkgaError) as ei:
        B().Batch([pb], [B().params(16, 3, 2, 0.7, 5, seed=1)])
    assert ei.value.code == -6
    assert "brkga_create" in str(ei.value)
